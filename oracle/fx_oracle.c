/*
 * CPU restatement of the per-block Godunov MHD update (TEST INFRASTRUCTURE).
 *
 * Plain C99, compiled with -ffp-contract=off by oracle/Makefile into
 * oracle/_ref/libfxoracle.so.  Only tests/ (and the smoke check) load it, as a
 * checker; nothing in the product links it.  Each function restates the
 * reference routine it cites (paths relative to the reference project) with
 * the same double operations in the same order, so it agrees with the
 * reference bit for bit; the tests pin it against golden vectors generated
 * from the reference (tests/golden/) and against the compiled reference
 * itself (oracle/_ref/libprjref_*.so).
 *
 * Besides the pointwise kernels it holds a complete RK2 step for a single
 * block whose six sides are physical outflow boundaries (the whole ghost
 * fill then reduces to the physical-boundary bands), in the reference's
 * per-block layout: W[v][stage][cell] (WIDX), Bf[d][stage][face] (FACE_IDX).
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>

#define BS 16
#define NG 2
#define PBS (BS + 2 * NG)
#define NCELLS (PBS * PBS * PBS)
#define NFACES ((PBS + 1) * PBS * PBS)
#define NEDGES ((PBS + 1) * (PBS + 1) * PBS)
#define PLANE (2 * NCELLS)

/* ---- layout (src/prj_defs.h:392-453) ------------------------------------ */

static int lidx(int i, int j, int k)
{
    return ((i + NG) * PBS + (j + NG)) * PBS + (k + NG);
}

static int face_idx(int d, int i, int j, int k)
{
    if (d == 0) return (i + NG) * PBS * PBS + (j + NG) * PBS + (k + NG);
    if (d == 1) return (i + NG) * (PBS + 1) * PBS + (j + NG) * PBS + (k + NG);
    return (i + NG) * PBS * (PBS + 1) + (j + NG) * (PBS + 1) + (k + NG);
}

static int edge_idx(int d, int i, int j, int k)
{
    if (d == 0) return (i + NG) * (PBS + 1) * (PBS + 1) + (j + NG) * (PBS + 1) + (k + NG);
    if (d == 1) return (i + NG) * PBS * (PBS + 1) + (j + NG) * (PBS + 1) + (k + NG);
    return (i + NG) * (PBS + 1) * PBS + (j + NG) * PBS + (k + NG);
}

static double dmin(double a, double b) { return a < b ? a : b; }
static double dmax(double a, double b) { return a > b ? a : b; }

/* ---- pointwise kernels ---------------------------------------------------- */

/* src/prj_reconstruct.h:355-375 */
double fxo_mc_slope(double qm, double q0, double qp)
{
    double sl = q0 - qm;
    double sr = qp - q0;
    double c0 = 2.0 * sl;
    double c1 = sl + 0.5 * (sr - sl);
    double c2 = 2.0 * sr;
    double mn = c0 < c1 ? c0 : c1;
    double mx = c0 > c1 ? c0 : c1;
    double slope;

    mn = mn < c2 ? mn : c2;
    mx = mx > c2 ? mx : c2;
    slope = sl > 0.0 ? mn : mx;
    return (sl * sr > 0.0) ? slope : 0.0;
}

/* problems/prj_problem_ideal_eos.h:24-32: out = T, p, gamma */
void fxo_eos_rey(double g, double rho, double eint, double *out)
{
    out[0] = (g - 1.0) * eint / 0.95655684e18;
    out[1] = (g - 1.0) * rho * eint;
    out[2] = g;
}

/* problems/prj_problem_ideal_eos.h:8-22 (eint and pressure from T) */
void fxo_eos_rty(double g, double rho, double T, double *eint, double *p)
{
    *eint = 0.95655684e18 * T / (g - 1.0);
    *p = rho * 0.95655684e18 * T;
}

/* src/prj_eos.c:2112-2151 */
void fxo_prim2cons(int nv, const double *w, double *u)
{
    double rho = w[0], v1 = w[1], v2 = w[2], v3 = w[3], eint = w[4];

    u[0] = rho;
    u[1] = rho * v1;
    u[2] = rho * v2;
    u[3] = rho * v3;
    if (nv == 9) {
        double b1 = w[6], b2 = w[7], b3 = w[8];
        u[4] = rho * eint + 0.5 * rho * (v1 * v1 + v2 * v2 + v3 * v3) + 0.5 * (b1 * b1 + b2 * b2 + b3 * b3);
        u[5] = rho * w[5];
        u[6] = b1;
        u[7] = b2;
        u[8] = b3;
    } else {
        u[4] = rho * eint + 0.5 * rho * (v1 * v1 + v2 * v2 + v3 * v3);
        u[5] = rho * w[5];
    }
}

/* src/prj_eos.c:2153-2220 */
void fxo_cons2prim(int nv, const double *u, double *w)
{
    double rho = u[0], v1, v2, v3, kinetic;
    int v;

    if (rho == 0.0) {
        for (v = 0; v < nv; ++v) w[v] = 0.0;
        return;
    }
    v1 = u[1] / rho;
    v2 = u[2] / rho;
    v3 = u[3] / rho;
    kinetic = 0.5 * (v1 * v1 + v2 * v2 + v3 * v3);
    w[0] = rho;
    w[1] = v1;
    w[2] = v2;
    w[3] = v3;
    if (nv == 9) {
        double magnetic = 0.5 * (u[6] * u[6] + u[7] * u[7] + u[8] * u[8]) / rho;
        w[4] = u[4] / rho - kinetic - magnetic;
        w[5] = u[5] / rho;
        w[6] = u[6];
        w[7] = u[7];
        w[8] = u[8];
    } else {
        w[4] = u[4] / rho - kinetic;
        w[5] = u[5] / rho;
    }
}

/* ---- HLLD, src/prj_riemann.c:81-440 -------------------------------------- */

typedef struct {
    double rho, vx, vy, vz, bx, by, bz, p, gamma, ye, e, pt;
    double U[9], F[9];
} hstate;

typedef struct {
    double rho, vx, vy, vz, bx, by, bz, ye, e;
    double U[9];
} hstar;

static int g_fail;

static void fill_u(double rho, double vx, double vy, double vz, double bx, double by, double bz,
    double ye, double e, double *U)
{
    U[0] = rho;
    U[1] = rho * vx;
    U[2] = rho * vy;
    U[3] = rho * vz;
    U[4] = e;
    U[5] = rho * ye;
    U[6] = bx;
    U[7] = by;
    U[8] = bz;
}

static void fill_f(const hstate *s, double *F)
{
    double b2 = s->bx * s->bx + s->by * s->by + s->bz * s->bz;
    double pt = s->p + 0.5 * b2;
    double vdotb = s->vx * s->bx + s->vy * s->by + s->vz * s->bz;

    F[0] = s->rho * s->vx;
    F[1] = s->rho * s->vx * s->vx + pt - s->bx * s->bx;
    F[2] = s->rho * s->vx * s->vy - s->bx * s->by;
    F[3] = s->rho * s->vx * s->vz - s->bx * s->bz;
    F[4] = (s->e + pt) * s->vx - s->bx * vdotb;
    F[5] = s->rho * s->ye * s->vx;
    F[6] = 0.0;
    F[7] = s->by * s->vx - s->bx * s->vy;
    F[8] = s->bz * s->vx - s->bx * s->vz;
}

static void state_from_prim(const double *W, double p, double gamma, double bn, hstate *s)
{
    double kinetic, magnetic;

    s->rho = W[0];
    s->vx = W[1];
    s->vy = W[2];
    s->vz = W[3];
    s->bx = bn;
    s->by = W[7];
    s->bz = W[8];
    s->p = p;
    s->gamma = gamma;
    s->ye = W[5];
    if (s->rho <= 0.0 || s->p <= 0.0 || s->gamma <= 0.0) g_fail = 1;
    kinetic = 0.5 * s->rho * (s->vx * s->vx + s->vy * s->vy + s->vz * s->vz);
    magnetic = 0.5 * (s->bx * s->bx + s->by * s->by + s->bz * s->bz);
    s->e = s->rho * W[4] + kinetic + magnetic;
    s->pt = s->p + magnetic;
    fill_u(s->rho, s->vx, s->vy, s->vz, s->bx, s->by, s->bz, s->ye, s->e, s->U);
    fill_f(s, s->F);
}

static double fast_speed(const hstate *s)
{
    double a2 = s->gamma * s->p / s->rho;
    double bx2_rho = s->bx * s->bx / s->rho;
    double b2_rho = (s->bx * s->bx + s->by * s->by + s->bz * s->bz) / s->rho;
    double disc = (a2 + b2_rho) * (a2 + b2_rho) - 4.0 * a2 * bx2_rho;
    double cf2;

    if (disc < 0.0) {
        if (disc < -1.0e-12 * (a2 + b2_rho) * (a2 + b2_rho)) g_fail = 1;
        disc = 0.0;
    }
    cf2 = 0.5 * (a2 + b2_rho + sqrt(disc));
    if (cf2 < 0.0 || !isfinite(cf2)) g_fail = 1;
    return sqrt(cf2);
}

static void outer_star(const hstate *s, double S, double SM, double pt_star, hstar *st)
{
    double alpha = S - s->vx;
    double smdiff = S - SM;
    double denom, vdotb, vsb;

    if (fabs(smdiff) <= 1.0e-14 * (fabs(S) + fabs(SM) + 1.0)) g_fail = 1;
    st->rho = s->rho * alpha / smdiff;
    if (st->rho <= 0.0 || !isfinite(st->rho)) g_fail = 1;
    st->vx = SM;
    st->bx = s->bx;
    st->ye = s->ye;
    denom = s->rho * alpha * smdiff - s->bx * s->bx;
    if (fabs(denom) < 1.0e-8 * pt_star) {
        st->vy = s->vy;
        st->vz = s->vz;
        st->by = s->by;
        st->bz = s->bz;
    } else {
        double f = (SM - s->vx) / denom;
        double mag = (s->rho * alpha * alpha - s->bx * s->bx) / denom;
        st->vy = s->vy - s->bx * s->by * f;
        st->vz = s->vz - s->bx * s->bz * f;
        st->by = s->by * mag;
        st->bz = s->bz * mag;
    }
    vdotb = s->vx * s->bx + s->vy * s->by + s->vz * s->bz;
    vsb = st->vx * st->bx + st->vy * st->by + st->vz * st->bz;
    st->e = (alpha * s->e - s->pt * s->vx + pt_star * SM + s->bx * (vdotb - vsb)) / smdiff;
    fill_u(st->rho, st->vx, st->vy, st->vz, st->bx, st->by, st->bz, st->ye, st->e, st->U);
}

static void double_star(const hstar *l, const hstar *r, double bx, int right_side, hstar *ss)
{
    double sl = sqrt(l->rho), sr = sqrt(r->rho);
    double inv, sgn, vy, vz, by, bz, vbss;

    if (sl + sr <= 0.0) g_fail = 1;
    inv = 1.0 / (sl + sr);
    sgn = bx < 0.0 ? -1.0 : 1.0;
    vy = (sl * l->vy + sr * r->vy + (r->by - l->by) * sgn) * inv;
    vz = (sl * l->vz + sr * r->vz + (r->bz - l->bz) * sgn) * inv;
    by = (sl * r->by + sr * l->by + sl * sr * (r->vy - l->vy) * sgn) * inv;
    bz = (sl * r->bz + sr * l->bz + sl * sr * (r->vz - l->vz) * sgn) * inv;
    vbss = (right_side ? r->vx : l->vx) * bx + vy * by + vz * bz;
    if (!right_side) {
        double vbl = l->vx * bx + l->vy * l->by + l->vz * l->bz;
        *ss = *l;
        ss->e = l->e - sl * sgn * (vbl - vbss);
    } else {
        double vbr = r->vx * bx + r->vy * r->by + r->vz * r->bz;
        *ss = *r;
        ss->e = r->e + sr * sgn * (vbr - vbss);
    }
    ss->vy = vy;
    ss->vz = vz;
    ss->by = by;
    ss->bz = bz;
    fill_u(ss->rho, ss->vx, ss->vy, ss->vz, ss->bx, ss->by, ss->bz, ss->ye, ss->e, ss->U);
}

static void face_out(double vx, double vy, double vz, double bx, double by, double bz, double *out)
{
    out[9] = vx;
    out[10] = vy;
    out[11] = vz;
    out[12] = bz * vx - bx * vz;
    out[13] = bx * vy - by * vx;
}

/* out[0..8] flux, [9..11] v_face, [12] Bv1, [13] Bv2; returns 1 on a
 * reference fail path */
int fxo_hlld(const double *WL, const double *WR, double pL, double pR, double gL, double gR,
    double bn, double *out)
{
    hstate L, R;
    hstar Ls, Rs, ss;
    double cfL, cfR, SL, SR, denom, SM, ptl, ptr, pt;
    int v, bn_small;

    g_fail = 0;
    state_from_prim(WL, pL, gL, bn, &L);
    state_from_prim(WR, pR, gR, bn, &R);
    cfL = fast_speed(&L);
    cfR = fast_speed(&R);
    SL = dmin(L.vx - cfL, R.vx - cfR);
    SR = dmax(L.vx + cfL, R.vx + cfR);
    if (!(SL < SR)) g_fail = 1;
    if (0.0 <= SL) {
        for (v = 0; v < 9; ++v) out[v] = L.F[v];
        face_out(L.vx, L.vy, L.vz, L.bx, L.by, L.bz, out);
        return g_fail;
    }
    if (SR <= 0.0) {
        for (v = 0; v < 9; ++v) out[v] = R.F[v];
        face_out(R.vx, R.vy, R.vz, R.bx, R.by, R.bz, out);
        return g_fail;
    }
    denom = R.rho * (SR - R.vx) - L.rho * (SL - L.vx);
    if (fabs(denom) <= 1.0e-14 * (fabs(R.rho * (SR - R.vx)) + fabs(L.rho * (SL - L.vx)) + 1.0)) g_fail = 1;
    SM = (R.rho * R.vx * (SR - R.vx) - L.rho * L.vx * (SL - L.vx) + (L.pt - R.pt)) / denom;
    ptl = L.pt + L.rho * (SL - L.vx) * (SM - L.vx);
    ptr = R.pt + R.rho * (SR - R.vx) * (SM - R.vx);
    pt = 0.5 * (ptl + ptr);
    if (pt <= 0.0 || !isfinite(pt)) {
        double inv = 1.0 / (SR - SL);
        double Uh[9];

        for (v = 0; v < 9; ++v) {
            out[v] = (SR * L.F[v] - SL * R.F[v] + SL * SR * (R.U[v] - L.U[v])) * inv;
            Uh[v] = (SR * R.U[v] - SL * L.U[v] + L.F[v] - R.F[v]) * inv;
        }
        face_out(Uh[1] / Uh[0], Uh[2] / Uh[0], Uh[3] / Uh[0], Uh[6], Uh[7], Uh[8], out);
        return g_fail;
    }
    bn_small = (0.5 * bn * bn < 1.0e-8 * pt);
    if (0.0 <= SM) {
        double SLs;

        outer_star(&L, SL, SM, pt, &Ls);
        SLs = SM - fabs(bn) / sqrt(Ls.rho);
        if (0.0 <= SLs || bn_small) {
            for (v = 0; v < 9; ++v) out[v] = L.F[v] + SL * (Ls.U[v] - L.U[v]);
            face_out(Ls.vx, Ls.vy, Ls.vz, Ls.bx, Ls.by, Ls.bz, out);
        } else {
            outer_star(&R, SR, SM, pt, &Rs);
            double_star(&Ls, &Rs, bn, 0, &ss);
            for (v = 0; v < 9; ++v) out[v] = L.F[v] + SL * (Ls.U[v] - L.U[v]) + SLs * (ss.U[v] - Ls.U[v]);
            face_out(ss.vx, ss.vy, ss.vz, ss.bx, ss.by, ss.bz, out);
        }
    } else {
        double SRs;

        outer_star(&R, SR, SM, pt, &Rs);
        SRs = SM + fabs(bn) / sqrt(Rs.rho);
        if (SRs <= 0.0 || bn_small) {
            for (v = 0; v < 9; ++v) out[v] = R.F[v] + SR * (Rs.U[v] - R.U[v]);
            face_out(Rs.vx, Rs.vy, Rs.vz, Rs.bx, Rs.by, Rs.bz, out);
        } else {
            outer_star(&L, SL, SM, pt, &Ls);
            double_star(&Ls, &Rs, bn, 1, &ss);
            for (v = 0; v < 9; ++v) out[v] = R.F[v] + SR * (Rs.U[v] - R.U[v]) + SRs * (ss.U[v] - Rs.U[v]);
            face_out(ss.vx, ss.vy, ss.vz, ss.bx, ss.by, ss.bz, out);
        }
    }
    return g_fail;
}

/* ---- HLLC, src/prj_riemann.c:8-17, 1433-1599 (hydro build) --------------- */

static void hllc_state(const double *W, double p, double g, double *U, double *F, double *cs)
{
    double rho = W[0], v1 = W[1], v2 = W[2], v3 = W[3], eint = W[4];
    double etot = rho * eint + 0.5 * rho * (v1 * v1 + v2 * v2 + v3 * v3);

    U[0] = rho;
    U[1] = rho * v1;
    U[2] = rho * v2;
    U[3] = rho * v3;
    U[4] = etot;
    U[5] = rho * W[5];
    *cs = sqrt(g * p / rho);
    F[0] = rho * v1;
    F[1] = rho * v1 * v1 + p;
    F[2] = rho * v1 * v2;
    F[3] = rho * v1 * v3;
    F[4] = (etot + p) * v1;
    F[5] = rho * W[5] * v1;
}

/* out[0..5] flux, [6..8] v_face */
void fxo_hllc(const double *WL, const double *WR, double pL, double pR, double gL, double gR,
    double du, double dv, double dw, double *out)
{
    double UL[6], UR[6], FL[6], FR[6], Us[6];
    double csL, csR, SL, SR, cfmax, th, SM, rs, eor;
    int v;

    hllc_state(WL, pL, gL, UL, FL, &csL);
    hllc_state(WR, pR, gR, UR, FR, &csR);
    SL = dmin(WL[1] - csL, WR[1] - csR);
    SR = dmax(WL[1] + csL, WR[1] + csR);
    cfmax = dmax(csL, csR);
    th = (-dmin(du, 0.0) + cfmax) / (-dmin(dmin(dv, dw), 0.0) + cfmax);
    th *= th;
    th = dmin(1.0, th * th);
    SM = (th * (pR - pL) + UL[1] * (SL - WL[1]) - UR[1] * (SR - WR[1])) /
        (UL[0] * (SL - WL[1]) - UR[0] * (SR - WR[1]));
    if (0.0 <= SL) {
        for (v = 0; v < 6; ++v) out[v] = FL[v];
        out[6] = WL[1];
        out[7] = WL[2];
        out[8] = WL[3];
        return;
    }
    if (SR <= 0.0) {
        for (v = 0; v < 6; ++v) out[v] = FR[v];
        out[6] = WR[1];
        out[7] = WR[2];
        out[8] = WR[3];
        return;
    }
    out[6] = SM;
    if (0.0 <= SM) {
        out[7] = WL[2];
        out[8] = WL[3];
        for (v = 0; v < 6; ++v) Us[v] = UL[v];
        rs = UL[0] * (SL - WL[1]) / (SL - SM);
        Us[0] = rs;
        Us[1] = rs * SM;
        Us[2] = rs * WL[2];
        Us[3] = rs * WL[3];
        eor = UL[4] / UL[0] + (SM - WL[1]) * (SM + pL / (UL[0] * (SL - WL[1])));
        Us[4] = rs * eor;
        Us[5] = rs * WL[5];
        for (v = 0; v < 6; ++v) out[v] = FL[v] + SL * (Us[v] - UL[v]);
    } else {
        out[7] = WR[2];
        out[8] = WR[3];
        for (v = 0; v < 6; ++v) Us[v] = UR[v];
        rs = UR[0] * (SR - WR[1]) / (SR - SM);
        Us[0] = rs;
        Us[1] = rs * SM;
        Us[2] = rs * WR[2];
        Us[3] = rs * WR[3];
        eor = UR[4] / UR[0] + (SM - WR[1]) * (SM + pR / (UR[0] * (SR - WR[1])));
        Us[4] = rs * eor;
        Us[5] = rs * WR[5];
        for (v = 0; v < 6; ++v) out[v] = FR[v] + SR * (Us[v] - UR[v]);
    }
}

/* ---- upwind corner EMF, src/prj_mhd.c:660-680 ----------------------------- */
double fxo_emf_upwind(const double *f, const double *c, const double *vn)
{
    double emf = 0.25 * (f[0] + f[1] + f[2] + f[3]);

    if (vn[0] > 0.0) emf += 0.25 * (f[3] - c[3]);
    else if (vn[0] < 0.0) emf += 0.25 * (f[1] - c[0]);
    else emf += 0.125 * (f[3] - c[3] + f[1] - c[0]);
    if (vn[1] > 0.0) emf += 0.25 * (f[2] - c[1]);
    else if (vn[1] < 0.0) emf += 0.25 * (f[0] - c[0]);
    else emf += 0.125 * (f[2] - c[1] + f[0] - c[0]);
    if (vn[2] > 0.0) emf += 0.25 * (f[3] - c[2]);
    else if (vn[2] < 0.0) emf += 0.25 * (f[1] - c[1]);
    else emf += 0.125 * (f[3] - c[2] + f[1] - c[1]);
    if (vn[3] > 0.0) emf += 0.25 * (f[2] - c[2]);
    else if (vn[3] < 0.0) emf += 0.25 * (f[0] - c[3]);
    else emf += 0.125 * (f[2] - c[2] + f[0] - c[3]);
    return emf;
}

/* ---- one block, all sides outflow: a full RK2 step ------------------------ */

typedef struct {
    int nv;
    double gamma;
    double dx[3];
    double *W;            /* nv x 2 x NCELLS */
    double *Bf;           /* 3 x 2 x NFACES (MHD) */
    double *flux[3];      /* [v][cell] untiled, face (i,j,k) at LIDX */
    double *vn[3];        /* normal face velocity at LIDX */
    double *bv1[3];
    double *bv2[3];
    double *emf[3];
    int *fid[3];
} blk;

static double *Wv(blk *b, int v, int slot) { return b->W + (size_t)v * PLANE + (size_t)slot * NCELLS; }
static double *Bfd(blk *b, int d, int slot) { return b->Bf + ((size_t)d * 2 + slot) * NFACES; }

static int gmap(int dir, int lv)
{
    if (lv >= 1 && lv <= 3) return 1 + (dir + lv - 1) % 3;
    if (lv >= 6) return 6 + (dir + lv - 6) % 3;
    return lv;
}

/* prj_flux_update for one block (src/prj_flux.c:2149-2521) */
static void flux_update(blk *b, int wslot)
{
    const int mhd = b->nv == 9;
    int dir;

    for (dir = 0; dir < 3; ++dir) {
        const int s = dir == 0 ? PBS * PBS : dir == 1 ? PBS : 1;
        int lo[3], hi[3], i, j, k, a;

        for (a = 0; a < 3; ++a) {
            lo[a] = a == dir ? 0 : (mhd ? -1 : 0);
            hi[a] = a == dir ? BS : (mhd ? BS : BS - 1);
        }
        for (i = lo[0]; i <= hi[0]; ++i) {
            for (j = lo[1]; j <= hi[1]; ++j) {
                for (k = lo[2]; k <= hi[2]; ++k) {
                    const int cR = lidx(i, j, k), cL = cR - s;
                    double WL[9], WR[9], q[4], p[4], out[14];
                    double pL, pR;
                    int lv, n;

                    for (lv = 0; lv < b->nv; ++lv) {
                        const double *src = Wv(b, gmap(dir, lv), wslot);

                        q[0] = src[cL - s]; q[1] = src[cL]; q[2] = src[cR]; q[3] = src[cR + s];
                        WL[lv] = q[1] + 0.5 * fxo_mc_slope(q[0], q[1], q[2]);
                        WR[lv] = q[2] - 0.5 * fxo_mc_slope(q[1], q[2], q[3]);
                    }
                    for (n = 0; n < 4; ++n) {
                        const int c = cL - s + n * s;
                        p[n] = (b->gamma - 1.0) * Wv(b, 0, wslot)[c] * Wv(b, 4, wslot)[c];
                    }
                    pL = p[1] + 0.5 * fxo_mc_slope(p[0], p[1], p[2]);
                    pR = p[2] - 0.5 * fxo_mc_slope(p[1], p[2], p[3]);
                    if (mhd) {
                        double bn = Bfd(b, dir, wslot)[face_idx(dir, i, j, k)];

                        WL[6] = bn;
                        WR[6] = bn;
                        fxo_hlld(WL, WR, pL, pR, b->gamma, b->gamma, bn, out);
                        b->bv1[dir][cR] = out[12];
                        b->bv2[dir][cR] = out[13];
                    } else {
                        const int da = (dir + 1) % 3, db = (dir + 2) % 3;
                        const int sa = da == 0 ? PBS * PBS : da == 1 ? PBS : 1;
                        const int sb = db == 0 ? PBS * PBS : db == 1 ? PBS : 1;
                        const double *un = Wv(b, 1 + dir, wslot);
                        const double *ua = Wv(b, 1 + da, wslot);
                        const double *ub = Wv(b, 1 + db, wslot);
                        double du = un[cR] - un[cL];
                        double dv = dmin(dmin(ua[cL] - ua[cL - sa], ua[cL + sa] - ua[cL]),
                            dmin(ua[cR] - ua[cR - sa], ua[cR + sa] - ua[cR]));
                        double dw = dmin(dmin(ub[cL] - ub[cL - sb], ub[cL + sb] - ub[cL]),
                            dmin(ub[cR] - ub[cR - sb], ub[cR + sb] - ub[cR]));
                        double h[9];

                        fxo_hllc(WL, WR, pL, pR, b->gamma, b->gamma, du, dv, dw, h);
                        for (lv = 0; lv < 6; ++lv) out[lv] = h[lv];
                        out[9] = h[6];
                    }
                    for (lv = 0; lv < b->nv; ++lv) {
                        b->flux[dir][(size_t)gmap(dir, lv) * NCELLS + cR] = out[lv];
                    }
                    b->vn[dir][cR] = out[9];
                }
            }
        }
    }
}

/* prj_timeint_mhd_update_emf (src/prj_timeint.c:292-413), eta = 0 */
static void update_emf(blk *b, int wslot)
{
    int dir;

    for (dir = 0; dir < 3; ++dir) {
        const int up = (dir + 1) % 3, right = (dir + 2) % 3;
        const int su = up == 0 ? PBS * PBS : up == 1 ? PBS : 1;
        const int sr = right == 0 ? PBS * PBS : right == 1 ? PBS : 1;
        int e[3];

        for (e[0] = 0; e[0] <= (dir == 0 ? BS - 1 : BS); ++e[0]) {
            for (e[1] = 0; e[1] <= (dir == 1 ? BS - 1 : BS); ++e[1]) {
                for (e[2] = 0; e[2] <= (dir == 2 ? BS - 1 : BS); ++e[2]) {
                    const int c0 = lidx(e[0], e[1], e[2]);
                    const int cells[4] = {c0, c0 - su, c0 - su - sr, c0 - sr};
                    double f[4], c[4], vn[4];
                    int n;

                    f[0] = b->bv1[right][c0];
                    f[1] = b->bv2[up][c0];
                    f[2] = b->bv1[right][c0 - su];
                    f[3] = b->bv2[up][c0 - sr];
                    for (n = 0; n < 4; ++n) {
                        const int cc = cells[n];
                        c[n] = Wv(b, 6 + up, wslot)[cc] * Wv(b, 1 + right, wslot)[cc] -
                            Wv(b, 6 + right, wslot)[cc] * Wv(b, 1 + up, wslot)[cc];
                    }
                    vn[0] = b->vn[right][c0];
                    vn[1] = b->vn[up][c0];
                    vn[2] = b->vn[right][c0 - su];
                    vn[3] = b->vn[up][c0 - sr];
                    b->emf[dir][edge_idx(dir, e[0], e[1], e[2])] = fxo_emf_upwind(f, c, vn);
                }
            }
        }
    }
}

/* prj_timeint_mhd_update_bf (src/prj_timeint.c:415-495) */
static void update_bf(blk *b, int stage, double dt)
{
    const int src = stage == 1 ? 0 : 1, dst = stage == 1 ? 1 : 0;
    const double *e1 = b->emf[0], *e2 = b->emf[1], *e3 = b->emf[2];
    int d, i, j, k;

    for (d = 0; d < 3; ++d) {
        for (i = 0; i <= (d == 0 ? BS : BS - 1); ++i) {
            for (j = 0; j <= (d == 1 ? BS : BS - 1); ++j) {
                for (k = 0; k <= (d == 2 ? BS : BS - 1); ++k) {
                    const int f = face_idx(d, i, j, k);
                    double v = Bfd(b, d, src)[f];

                    if (d == 0) {
                        v += -dt * (e3[edge_idx(2, i, j + 1, k)] - e3[edge_idx(2, i, j, k)]) / b->dx[1];
                        v += dt * (e2[edge_idx(1, i, j, k + 1)] - e2[edge_idx(1, i, j, k)]) / b->dx[2];
                    } else if (d == 1) {
                        v += -dt * (e1[edge_idx(0, i, j, k + 1)] - e1[edge_idx(0, i, j, k)]) / b->dx[2];
                        v += dt * (e3[edge_idx(2, i + 1, j, k)] - e3[edge_idx(2, i, j, k)]) / b->dx[0];
                    } else {
                        v += -dt * (e2[edge_idx(1, i + 1, j, k)] - e2[edge_idx(1, i, j, k)]) / b->dx[0];
                        v += dt * (e1[edge_idx(0, i, j + 1, k)] - e1[edge_idx(0, i, j, k)]) / b->dx[1];
                    }
                    if (stage == 2) v = 0.5 * Bfd(b, d, 0)[f] + 0.5 * v;
                    Bfd(b, d, dst)[f] = v;
                }
            }
        }
    }
}

/* per-cell stage updates (src/prj_timeint.c:1255-1349, 1562-1654), no sources */
static void update_cells(blk *b, int stage, double dt, double *dt_src)
{
    const double area[3] = {b->dx[1] * b->dx[2], b->dx[0] * b->dx[2], b->dx[0] * b->dx[1]};
    const double vol = b->dx[0] * b->dx[1] * b->dx[2];
    const int nv = b->nv;
    int i, j, k, v;

    for (i = 0; i < BS; ++i) {
        for (j = 0; j < BS; ++j) {
            for (k = 0; k < BS; ++k) {
                const int c = lidx(i, j, k);
                double w[9], u[9], un[9], div[9], ds;

                for (v = 0; v < nv; ++v) {
                    div[v] = -(area[0] * (b->flux[0][(size_t)v * NCELLS + c + PBS * PBS] - b->flux[0][(size_t)v * NCELLS + c]) +
                        area[1] * (b->flux[1][(size_t)v * NCELLS + c + PBS] - b->flux[1][(size_t)v * NCELLS + c]) +
                        area[2] * (b->flux[2][(size_t)v * NCELLS + c + 1] - b->flux[2][(size_t)v * NCELLS + c])) / vol;
                }
                for (v = 0; v < nv; ++v) w[v] = Wv(b, v, 0)[c];
                fxo_prim2cons(nv, w, u);
                ds = 0.02 * u[4] / (fabs(0.0) + 1.0e-50);
                if (ds < *dt_src) *dt_src = ds;
                if (stage == 1) {
                    for (v = 0; v < nv; ++v) un[v] = u[v] + dt * (0.0 + div[v]);
                } else {
                    double u1[9];

                    for (v = 0; v < nv; ++v) w[v] = Wv(b, v, 1)[c];
                    fxo_prim2cons(nv, w, u1);
                    for (v = 0; v < nv; ++v) un[v] = 0.5 * u[v] + 0.5 * (u1[v] + dt * (0.0 + div[v]));
                }
                if (nv == 9) {
                    const int s = stage == 1 ? 1 : 0;
                    un[6] = 0.5 * (Bfd(b, 0, s)[face_idx(0, i, j, k)] + Bfd(b, 0, s)[face_idx(0, i + 1, j, k)]);
                    un[7] = 0.5 * (Bfd(b, 1, s)[face_idx(1, i, j, k)] + Bfd(b, 1, s)[face_idx(1, i, j + 1, k)]);
                    un[8] = 0.5 * (Bfd(b, 2, s)[face_idx(2, i, j, k)] + Bfd(b, 2, s)[face_idx(2, i, j, k + 1)]);
                }
                fxo_cons2prim(nv, un, w);
                for (v = 0; v < nv; ++v) Wv(b, v, stage == 1 ? 1 : 0)[c] = w[v];
            }
        }
    }
}

/* outflow band of prj_boundary_apply_axis_band (src/prj_boundary.c:413-480) */
static void band(blk *b, int slot, int axis, int side, int edge_corner)
{
    const int a1 = (axis + 1) % 3, a2 = (axis + 2) % 3;
    const int nlo = side == 0 ? -NG : BS, nhi = side == 0 ? 0 : BS + NG;
    const int tlo = edge_corner ? -NG : 0, thi = edge_corner ? BS + NG : BS;
    const int nvg = b->nv;
    int a, t1, t2, v;

    for (a = nlo; a < nhi; ++a) {
        const int sa = side == 0 ? -a - 1 : 2 * BS - 1 - a;
        for (t1 = tlo; t1 < thi; ++t1) {
            for (t2 = tlo; t2 < thi; ++t2) {
                int idx[3], src[3];

                if (edge_corner && t1 >= 0 && t1 < BS && t2 >= 0 && t2 < BS) continue;
                idx[axis] = a; idx[a1] = t1; idx[a2] = t2;
                src[axis] = sa; src[a1] = t1; src[a2] = t2;
                for (v = 0; v < nvg; ++v) {
                    double *q = Wv(b, v, slot);
                    q[lidx(idx[0], idx[1], idx[2])] = q[lidx(src[0], src[1], src[2])];
                }
            }
        }
    }
}

static int face_ok(int dir, const int idx[3])
{
    int d;
    for (d = 0; d < 3; ++d) {
        int hi = dir == d ? BS + NG : BS + NG - 1;
        if (idx[d] < -NG || idx[d] > hi) return 0;
    }
    return 1;
}

/* prj_boundary_apply_bf_axis with face fidelity (src/prj_boundary.c:599-625, 883-933) */
static void bf_band(blk *b, int slot, int axis, int side)
{
    int dir, i, j, k;

    for (dir = 0; dir < 3; ++dir) {
        const int max_axis = dir == axis ? BS : BS - 1;
        for (i = -NG; i < BS + NG; ++i) {
            for (j = -NG; j < BS + NG; ++j) {
                for (k = -NG; k < BS + NG; ++k) {
                    int idx[3] = {i, j, k}, src[3] = {i, j, k};
                    int sf, df, fid;

                    if (side == 0) {
                        if (idx[axis] >= 0) continue;
                        src[axis] = 0;
                    } else {
                        if (idx[axis] <= max_axis) continue;
                        src[axis] = max_axis;
                    }
                    if (!face_ok(dir, src)) continue;
                    sf = face_idx(dir, src[0], src[1], src[2]);
                    fid = b->fid[dir][sf];
                    if (fid == 0) continue;
                    df = face_idx(dir, i, j, k);
                    if (fid < b->fid[dir][df]) continue;
                    Bfd(b, dir, slot)[df] = Bfd(b, dir, slot)[sf];
                    if (fid > b->fid[dir][df]) b->fid[dir][df] = fid;
                }
            }
        }
    }
}

/* prj_boundary_fill_ghosts_and_bf for a block whose six sides are physical */
static void ghost_fill(blk *b, int slot)
{
    int pass, axis, side, d, i, j, k;

    for (axis = 0; axis < 3; ++axis)
        for (side = 0; side < 2; ++side) band(b, slot, axis, side, 0);
    if (b->nv == 9) {
        for (d = 0; d < 3; ++d) {
            memset(b->fid[d], 0, NFACES * sizeof(int));
            for (i = 0; i <= (d == 0 ? BS : BS - 1); ++i)
                for (j = 0; j <= (d == 1 ? BS : BS - 1); ++j)
                    for (k = 0; k <= (d == 2 ? BS : BS - 1); ++k) b->fid[d][face_idx(d, i, j, k)] = 2;
        }
        for (pass = 0; pass < 3; ++pass)
            for (axis = 0; axis < 3; ++axis)
                for (side = 0; side < 2; ++side) bf_band(b, slot, axis, side);
    }
    for (pass = 0; pass < 3; ++pass)
        for (axis = 0; axis < 3; ++axis)
            for (side = 0; side < 2; ++side) band(b, slot, axis, side, 1);
    if (b->nv == 9) {
        for (pass = 0; pass < 3; ++pass)
            for (axis = 0; axis < 3; ++axis)
                for (side = 0; side < 2; ++side) bf_band(b, slot, axis, side);
        /* prj_mhd_bf2bc_impl over all 20^3 cells (src/prj_mhd.c:555-603) */
        for (i = -NG; i < BS + NG; ++i) {
            for (j = -NG; j < BS + NG; ++j) {
                for (k = -NG; k < BS + NG; ++k) {
                    const int c = lidx(i, j, k);
                    Wv(b, 6, slot)[c] = 0.5 * (Bfd(b, 0, slot)[face_idx(0, i, j, k)] + Bfd(b, 0, slot)[face_idx(0, i + 1, j, k)]);
                    Wv(b, 7, slot)[c] = 0.5 * (Bfd(b, 1, slot)[face_idx(1, i, j, k)] + Bfd(b, 1, slot)[face_idx(1, i, j + 1, k)]);
                    Wv(b, 8, slot)[c] = 0.5 * (Bfd(b, 2, slot)[face_idx(2, i, j, k)] + Bfd(b, 2, slot)[face_idx(2, i, j, k + 1)]);
                }
            }
        }
    }
}

/* prj_timeint_calc_dt for one block (src/prj_timeint.c:2144-2256) */
double fxo_calc_dt(int nv, double gamma, const double *dx, const double *W, double cfl)
{
    double dt_min = 1.0e99;
    int i, j, k;

    (void)nv;
    for (i = 0; i < BS; ++i) {
        for (j = 0; j < BS; ++j) {
            for (k = 0; k < BS; ++k) {
                const int c = lidx(i, j, k);
                double rho = W[0 * PLANE + c];
                double p = (gamma - 1.0) * rho * W[4 * PLANE + c];
                double cs = sqrt(gamma * p / rho);
                double denom = (fabs(W[1 * PLANE + c]) + cs) / dx[0] + (fabs(W[2 * PLANE + c]) + cs) / dx[1] +
                    (fabs(W[3 * PLANE + c]) + cs) / dx[2];
                double dt = cfl / denom;
                if (dt < dt_min) dt_min = dt;
            }
        }
    }
    return dt_min;
}

/* One RK2 step (prj_timeint_step, src/prj_timeint.c:3221-3227) of one block
 * with outflow boundaries on all six sides.  Returns dt_src. */
double fxo_step_block(int nv, double gamma, const double *dx, double *W, double *Bf, double dt)
{
    blk b;
    double dt_src = 1.0e100;
    int d, stage;

    memset(&b, 0, sizeof(b));
    b.nv = nv;
    b.gamma = gamma;
    b.dx[0] = dx[0];
    b.dx[1] = dx[1];
    b.dx[2] = dx[2];
    b.W = W;
    b.Bf = Bf;
    for (d = 0; d < 3; ++d) {
        b.flux[d] = calloc((size_t)nv * NCELLS, sizeof(double));
        b.vn[d] = calloc(NCELLS, sizeof(double));
        b.bv1[d] = calloc(NCELLS, sizeof(double));
        b.bv2[d] = calloc(NCELLS, sizeof(double));
        b.emf[d] = calloc(NEDGES, sizeof(double));
        b.fid[d] = calloc(NFACES, sizeof(int));
    }
    for (stage = 1; stage <= 2; ++stage) {
        const int src = stage == 1 ? 0 : 1;
        flux_update(&b, src);
        if (nv == 9) {
            update_emf(&b, src);
            update_bf(&b, stage, dt);
        }
        update_cells(&b, stage, dt, &dt_src);
        ghost_fill(&b, stage == 1 ? 1 : 0);
    }
    for (d = 0; d < 3; ++d) {
        free(b.flux[d]);
        free(b.vn[d]);
        free(b.bv1[d]);
        free(b.bv2[d]);
        free(b.emf[d]);
        free(b.fid[d]);
    }
    return dt_src;
}

/* ---- dynamic AMR: pass 1 of prj_amr_tag (src/prj_amr.c:1611-1705) ------- */

/* one refinement criterion, the amr_* arrays of prj_mesh (src/prj_types.h:482-490) */
typedef struct fxo_amr_crit {
    int set;
    int estimator;   /* 0 Loehner, 1 velocity, 2 pressure scale height, 3 fractional jump */
    int lohner_var;  /* 0 density, 1 pressure, 2 temperature */
    int jump_var;    /* 0 density, 1 pressure */
    double refine_thresh;
    double derefine_thresh;
    double lohner_eps;
} fxo_amr_crit;

typedef struct tagblk {
    int nv;
    double gamma;
    const double *W;      /* slot 0 is read */
    const double *grav;   /* 3 x 8000 or NULL */
    const double *dx;
} tagblk;

/* storage index clamp of prj_amr_clamp_storage_index (src/prj_amr.c:713-722) */
static int clampi(int i)
{
    if (i < -NG) return -NG;
    if (i >= BS + NG) return BS + NG - 1;
    return i;
}

static double t_prim(const tagblk *t, int v, int i, int j, int k)
{
    return t->W[(size_t)v * PLANE + lidx(clampi(i), clampi(j), clampi(k))];
}

/* eosvar pressure / temperature / gamma of the ideal gas at a cell (what
 * prj_eos_fill_mesh leaves there) */
static double t_gas_p(const tagblk *t, int i, int j, int k)
{
    int c = lidx(i, j, k);
    return (t->gamma - 1.0) * t->W[c] * t->W[(size_t)4 * PLANE + c];
}

/* prj_amr_total_pressure_non_gr_at (src/prj_amr.c:805-819); unclamped */
static double t_ptot(const tagblk *t, int i, int j, int k)
{
    double p = t_gas_p(t, i, j, k);
    if (t->nv == 9) {
        int c = lidx(i, j, k);
        double b1 = t->W[(size_t)6 * PLANE + c];
        double b2 = t->W[(size_t)7 * PLANE + c];
        double b3 = t->W[(size_t)8 * PLANE + c];
        p += 0.5 * (b1 * b1 + b2 * b2 + b3 * b3);
    }
    return p;
}

/* prj_loehner_cell_value (src/prj_amr.c:930-942): density and total
 * pressure clamp the index, temperature does not */
static double t_lohner_value(const tagblk *t, int var, int i, int j, int k)
{
    if (var == 0) return t_prim(t, 0, i, j, k);
    if (var == 2) {
        int c = lidx(i, j, k);
        return (t->gamma - 1.0) * t->W[(size_t)4 * PLANE + c] / 0.95655684e18;
    }
    return t_ptot(t, clampi(i), clampi(j), clampi(k));
}

/* prj_loehner_cell_indicator (src/prj_amr.c:944-1005) */
static double t_lohner(const tagblk *t, int var, double eps, int i, int j, int k)
{
    double u0 = t_lohner_value(t, var, i, j, k);
    double uxm = t_lohner_value(t, var, i - 1, j, k);
    double uxp = t_lohner_value(t, var, i + 1, j, k);
    double uym = t_lohner_value(t, var, i, j - 1, k);
    double uyp = t_lohner_value(t, var, i, j + 1, k);
    double uzm = t_lohner_value(t, var, i, j, k - 1);
    double uzp = t_lohner_value(t, var, i, j, k + 1);
    double num_x = uxp - 2.0 * u0 + uxm;
    double num_y = uyp - 2.0 * u0 + uym;
    double num_z = uzp - 2.0 * u0 + uzm;
    double num_xy = 0.25 * (t_lohner_value(t, var, i + 1, j + 1, k) - t_lohner_value(t, var, i + 1, j - 1, k) -
        t_lohner_value(t, var, i - 1, j + 1, k) + t_lohner_value(t, var, i - 1, j - 1, k));
    double num_xz = 0.25 * (t_lohner_value(t, var, i + 1, j, k + 1) - t_lohner_value(t, var, i + 1, j, k - 1) -
        t_lohner_value(t, var, i - 1, j, k + 1) + t_lohner_value(t, var, i - 1, j, k - 1));
    double num_yz = 0.25 * (t_lohner_value(t, var, i, j + 1, k + 1) - t_lohner_value(t, var, i, j + 1, k - 1) -
        t_lohner_value(t, var, i, j - 1, k + 1) + t_lohner_value(t, var, i, j - 1, k - 1));
    double den_x = fabs(uxp - u0) + fabs(u0 - uxm) + eps * (fabs(uxp) + 2.0 * fabs(u0) + fabs(uxm));
    double den_y = fabs(uyp - u0) + fabs(u0 - uym) + eps * (fabs(uyp) + 2.0 * fabs(u0) + fabs(uym));
    double den_z = fabs(uzp - u0) + fabs(u0 - uzm) + eps * (fabs(uzp) + 2.0 * fabs(u0) + fabs(uzm));
    double numerator = num_x * num_x + num_y * num_y + num_z * num_z +
        2.0 * (num_xy * num_xy + num_xz * num_xz + num_yz * num_yz);
    double denominator = den_x * den_x + den_y * den_y + den_z * den_z + 1.0e-14;
    return sqrt(numerator / denominator);
}

/* prj_block_sound_speed_at (src/prj_amr.c:840-862) */
static double t_sound_speed(const tagblk *t, int i, int j, int k)
{
    double rho = t_prim(t, 0, i, j, k);
    double eint = t_prim(t, 4, i, j, k);
    double p;
    if (rho <= 0.0 || eint < 0.0) return 0.0;
    p = t_ptot(t, clampi(i), clampi(j), clampi(k));
    if (p <= 0.0 || t->gamma <= 0.0) return 0.0;
    return sqrt(t->gamma * p / rho);
}

/* prj_velocity_cell_indicator (src/prj_amr.c:1007-1038) */
static double t_velocity(const tagblk *t, int i, int j, int k)
{
    double v1 = t_prim(t, 1, i, j, k);
    double v2 = t_prim(t, 2, i, j, k);
    double v3 = t_prim(t, 3, i, j, k);
    double cs = t_sound_speed(t, i, j, k);
    double m = 0.0;
    int axis, side;
    for (axis = 0; axis < 3; ++axis) {
        for (side = -1; side <= 1; side += 2) {
            int di = axis == 0 ? side : 0;
            int dj = axis == 1 ? side : 0;
            int dk = axis == 2 ? side : 0;
            double dv1 = v1 - t_prim(t, 1, i + di, j + dj, k + dk);
            double dv2 = v2 - t_prim(t, 2, i + di, j + dj, k + dk);
            double dv3 = v3 - t_prim(t, 3, i + di, j + dj, k + dk);
            double dv = sqrt(dv1 * dv1 + dv2 * dv2 + dv3 * dv3) / (cs + 1.0e-14);
            m = dmax(m, dv);
        }
    }
    return m;
}

/* prj_pressure_scale_height_cell_indicator, non-GR branch (src/prj_amr.c:1065-1144) */
static double t_scale_height(const tagblk *t, int i, int j, int k)
{
    int c = lidx(i, j, k);
    double rho, p, g1, g2, g3, accel, cs, hp;
    if (t->grav == 0) return 0.0;
    rho = t_prim(t, 0, i, j, k);
    p = t_ptot(t, i, j, k);
    g1 = t->grav[c];
    g2 = t->grav[NCELLS + c];
    g3 = t->grav[2 * NCELLS + c];
    accel = sqrt(g1 * g1 + g2 * g2 + g3 * g3);
    cs = t->dx[0];
    if (t->dx[1] > cs) cs = t->dx[1];
    if (t->dx[2] > cs) cs = t->dx[2];
    if (rho <= 0.0 || p <= 0.0 || accel <= 0.0) return 0.0;
    hp = p / (rho * accel);
    if (hp <= 0.0) return 0.0;
    return cs / hp;
}

/* prj_fractional_jump_cell_indicator (src/prj_amr.c:1146-1202); unclamped */
static double t_jump_value(const tagblk *t, int var, int i, int j, int k)
{
    if (var == 1) return t_ptot(t, i, j, k);
    return t->W[lidx(i, j, k)];
}

static double t_jump(const tagblk *t, int var, int i, int j, int k)
{
    double q0 = t_jump_value(t, var, i, j, k);
    double m = 0.0;
    int di, dj, dk;
    if (q0 <= 0.0) return 0.0;
    for (di = -1; di <= 1; ++di) {
        for (dj = -1; dj <= 1; ++dj) {
            for (dk = -1; dk <= 1; ++dk) {
                double q, den;
                if (di == 0 && dj == 0 && dk == 0) continue;
                q = t_jump_value(t, var, i + di, j + dj, k + dk);
                if (q <= 0.0) continue;
                den = q0 < q ? q0 : q;
                m = dmax(m, fabs(q0 - q) / (den + 1.0e-14));
            }
        }
    }
    return m;
}

/* prj_amr_cell_indicator_for_estimator (src/prj_amr.c:1204-1221) */
static double t_indicator(const tagblk *t, const fxo_amr_crit *c, int i, int j, int k)
{
    if (c->estimator == 3) return t_jump(t, c->jump_var, i, j, k);
    if (c->estimator == 2) return t_scale_height(t, i, j, k);
    if (c->estimator == 1) return t_velocity(t, i, j, k);
    return t_lohner(t, c->lohner_var, c->lohner_eps, i, j, k);
}

/* prj_amr_refine_boundary_mask_for_cell (src/prj_amr.c:120-144), buffer 2 */
static unsigned t_cell_mask(int i, int j, int k)
{
    unsigned m = 0u;
    if (i < 2) m |= 1u;
    if (i >= BS - 2) m |= 2u;
    if (j < 2) m |= 4u;
    if (j >= BS - 2) m |= 8u;
    if (k < 2) m |= 16u;
    if (k >= BS - 2) m |= 32u;
    return m;
}

/* Pass 1 of prj_amr_tag for one active block: out[0] refine vote (0/1),
 * out[1] derefine vote (0/-1), out[2] boundary side mask. */
void fxo_amr_vote(int nv, double gamma, const double *W, const double *grav, const double *dx,
    int has_parent, const fxo_amr_crit *crit, int ncrit, double reach_density, int *out)
{
    tagblk t;
    int refine = 0;
    int derefine = has_parent ? 1 : 0;
    int has_refine = 0, has_derefine = 0;
    unsigned mask = 0u;
    int i, j, k, n;

    t.nv = nv;
    t.gamma = gamma;
    t.W = W;
    t.grav = grav;
    t.dx = dx;
    for (i = 0; i < BS; ++i) {
        for (j = 0; j < BS; ++j) {
            for (k = 0; k < BS; ++k) {
                unsigned cm = t_cell_mask(i, j, k);
                double sum = 0.0;
                if (refine != 0 && cm == 0u) continue;
                if (reach_density > 0.0 && W[lidx(i, j, k)] > reach_density) {
                    has_refine = 1;
                    refine = 1;
                    derefine = 0;
                    mask |= cm;
                }
                for (n = 0; n < ncrit; ++n) {
                    if (crit[n].set == 0 || crit[n].refine_thresh <= 0.0) continue;
                    has_refine = 1;
                    sum += t_indicator(&t, &crit[n], i, j, k) / crit[n].refine_thresh;
                }
                if (sum > 1.0) {
                    refine = 1;
                    mask |= cm;
                }
            }
        }
    }
    if (derefine != 0) {
        for (i = -1; i <= BS && derefine != 0; ++i) {
            for (j = -1; j <= BS && derefine != 0; ++j) {
                for (k = -1; k <= BS; ++k) {
                    double sum = 0.0;
                    for (n = 0; n < ncrit; ++n) {
                        if (crit[n].set == 0 || crit[n].derefine_thresh <= 0.0) continue;
                        has_derefine = 1;
                        sum += t_indicator(&t, &crit[n], i, j, k) / crit[n].derefine_thresh;
                    }
                    if (sum >= 1.0) {
                        derefine = 0;
                        break;
                    }
                }
            }
        }
    }
    if (has_refine == 0) refine = 0;
    if (has_derefine == 0) derefine = 0;
    out[0] = refine ? 1 : 0;
    out[1] = derefine ? -1 : 0;
    out[2] = (int)mask;
}

/* ---- WENO-Z3 face value (src/prj_reconstruct.h:383-423) ----------------- */
double fxo_weno3_face(double qm, double q0, double qp, double target)
{
    const double eps = 1.0e-40;
    double p0 = q0 + target * (q0 - qm);
    double p1 = q0 + target * (qp - q0);
    double dl = q0 - qm;
    double dr = qp - q0;
    double beta0 = dl * dl;
    double beta1 = dr * dr;
    double tau3 = beta0 - beta1;
    double g0, g1, a0, a1;
    if (tau3 < 0.0) tau3 = -tau3;
    if (target > 0.0) {
        g0 = 1.0 / 3.0;
        g1 = 2.0 / 3.0;
    } else {
        g0 = 2.0 / 3.0;
        g1 = 1.0 / 3.0;
    }
    a0 = g0 * (1.0 + tau3 / (eps + beta0));
    a1 = g1 * (1.0 + tau3 / (eps + beta1));
    return (a0 * p0 + a1 * p1) / (a0 + a1);
}
