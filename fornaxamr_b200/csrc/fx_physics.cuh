/*
 * Device-side pointwise physics of the per-block Godunov MHD update.
 *
 * Every function here evaluates the same IEEE-754 double operations, in the
 * same association order, as the reference routine it cites; the library is
 * compiled with --fmad=false so no multiply-add is contracted.  With correctly
 * rounded division and square root (CUDA's default for double) the results
 * are bit-identical to the reference's CPU path built with -ffp-contract=off.
 * Comments give the C association explicitly where it matters, e.g.
 * "a * b * c" is (a*b)*c.
 *
 * The pointwise functions are host-callable too (FX_HD), so the adjoint's
 * building blocks can be checked against finite differences on the host.
 *
 * Failures the reference turns into exit(1) (non-positive density, invalid
 * wave ordering, ...) are reported through fx_fail(): the first failing
 * thread records a code and its position in the device error word and the
 * kernel continues with whatever values result, so no launch ever traps.
 */
#ifndef FX_PHYSICS_CUH
#define FX_PHYSICS_CUH

#include <cmath>

#include "fx_layout.h"

/* error codes (first error wins); the host maps them to the reference's
 * fail-fast messages */
enum fx_err_code {
    FX_OK = 0,
    FX_ERR_HLLD_RHO = 1,       /* prj_riemann.c:159-161 non-positive density */
    FX_ERR_HLLD_P = 2,         /* prj_riemann.c:162-164 non-positive gas pressure */
    FX_ERR_HLLD_GAMMA = 3,     /* prj_riemann.c:165-167 */
    FX_ERR_HLLD_DISC = 4,      /* prj_riemann.c:128-130 negative fast-speed discriminant */
    FX_ERR_HLLD_CF = 5,        /* prj_riemann.c:134-136 invalid fast speed */
    FX_ERR_HLLD_ORDER = 6,     /* prj_riemann.c:361-363 invalid fast-wave ordering */
    FX_ERR_HLLD_DENOM = 7,     /* prj_riemann.c:380-384 degenerate contact-speed denominator */
    FX_ERR_HLLD_OUTER = 8,     /* prj_riemann.c:198-200 outer wave coincides with contact */
    FX_ERR_HLLD_STARRHO = 9,   /* prj_riemann.c:203-205 invalid star density */
    FX_ERR_HLLD_DSTAR = 10,    /* prj_riemann.c:250-252 invalid double-star weights */
    FX_ERR_EMF_NONFINITE = 11, /* prj_timeint.c:171-176, prj_mhd.c:650-654 */
    FX_ERR_BF_NONFINITE = 12,  /* prj_timeint.c:441-443 non-finite updated magnetic field */
    FX_ERR_EOS_ZERO_RHO = 13,  /* prj_eos.c:248-250 zero density in eos fill */
    FX_ERR_ETA = 14,           /* prj_timeint.c:255-257, 279-281 */
    FX_ERR_B_NONFINITE = 15,   /* prj_timeint.c:506-508, prj_mhd.c:593-595 */
    FX_ERR_TIMEOUT = 16,       /* a bounded device wait gave up */
    FX_ERR_AMR_NONFINITE = 17  /* prj_amr.c:1892-1896, 2186-2189 non-finite field in a remesh */
};

struct FxErr {
    int code;
    int block;
    int index;
    int aux;
};

FX_HD void fx_fail(FxErr *err, int code, int block, int index)
{
#ifdef __CUDA_ARCH__
    if (err != nullptr && atomicCAS(&err->code, 0, code) == 0) {
        err->block = block;
        err->index = index;
    }
#else
    /* host evaluation (checks of the adjoint building blocks) */
    if (err != nullptr && err->code == 0) {
        err->code = code;
        err->block = block;
        err->index = index;
    }
#endif
}

FX_HD double fx_min(double a, double b) { return a < b ? a : b; }
FX_HD double fx_max(double a, double b) { return a > b ? a : b; }

/* the face solver's divisions (correctly rounded, as in the reference) */
FX_HD double fx_div(double a, double b) { return a / b; }

/* A thread-local record of the first failure, with fx_fail's
 * first-error-wins rule: the face kernel collects a face's checks here (a
 * predicated store each, so the checks do not split the solver into short
 * basic blocks) and reports the record once the face is done. */
struct FxErrLocal {
    int code = 0;
    int block = 0;
    int index = 0;
};

FX_HD void fx_fail(FxErrLocal *err, int code, int block, int index)
{
    const bool first = err->code == 0;
    err->code = first ? code : err->code;
    err->block = first ? block : err->block;
    err->index = first ? index : err->index;
}

/* ------------------------------------------------------------------------ */
/* Branch policies.  The solvers below take their data-dependent decisions  */
/* (limiter candidate, wave-speed argument, fan region, upwind direction)   */
/* through a policy: FxBrFree evaluates each comparison (the solver as the   */
/* reference runs it), FxBrRecord evaluates and records them in one 64-bit   */
/* word per face or edge, and FxBrReplay takes them from such a word -- the */
/* discrete map with its branches frozen at the recorded state, the map the */
/* discrete adjoint differentiates -- counting the decisions whose           */
/* comparison now comes out otherwise.                                       */
/* ------------------------------------------------------------------------ */
struct FxBrFree {
    FX_HD bool bit(int, bool c) { return c; }
    FX_HD unsigned field(int, unsigned c) { return c; }
};

struct FxBrRecord {
    unsigned long long w = 0;
    FX_HD bool bit(int k, bool c)
    {
        if (c) w |= 1ULL << k;
        return c;
    }
    FX_HD unsigned field(int k, unsigned c)
    {
        w |= (unsigned long long)c << k;
        return c;
    }
};

struct FxBrReplay {
    unsigned long long w = 0;
    unsigned flips = 0;
    FX_HD bool bit(int k, bool c)
    {
        const bool f = ((w >> k) & 1ULL) != 0;
        flips += f != c ? 1u : 0u;
        return f;
    }
    FX_HD unsigned field(int k, unsigned c)
    {
        const unsigned f = (unsigned)(w >> k) & 3u;
        flips += f != c ? 1u : 0u;
        return f;
    }
};

/* bit positions of a face's word: MC candidates 2 bits per slope at
 * 4 q + 2 s (q: the reconstructed quantity, 0-8; s: 0 the left cell's
 * slope, 1 the right cell's), then the HLLD decisions */
enum FxBrBit {
    FX_BR_DISC_L = 36, FX_BR_DISC_R = 37, FX_BR_SL = 38, FX_BR_SR = 39, FX_BR_SUPER_L = 40,
    FX_BR_SUPER_R = 41, FX_BR_HLL = 42, FX_BR_BNSMALL = 43, FX_BR_LEFT = 44, FX_BR_DEGEN_N = 45,
    FX_BR_SINGLE = 46, FX_BR_DEGEN_F = 47, FX_BR_BNEG = 48
};

/* ------------------------------------------------------------------------ */
/* MC limited slope, src/prj_reconstruct.h:355-375 (branchless form).        */
/* ------------------------------------------------------------------------ */
FX_HD double fx_mc_slope(double qm, double q0, double qp)
{
    const double sl = q0 - qm;
    const double sr = qp - q0;
    const double c0 = 2.0 * sl;
    const double c1 = sl + 0.5 * (sr - sl);
    const double c2 = 2.0 * sr;
    double mn = c0 < c1 ? c0 : c1;
    double mx = c0 > c1 ? c0 : c1;
    mn = mn < c2 ? mn : c2;
    mx = mx > c2 ? mx : c2;
    const double slope = sl > 0.0 ? mn : mx;
    return (sl * sr > 0.0) ? slope : 0.0;
}

/* fx_mc_slope with its selection through a policy: candidate 0, 1, 2 (c0,
 * c1, c2) or 3 (zero slope) in the 2-bit field at bit k; the selected
 * candidate is the same double fx_mc_slope returns */
template <class BR>
FX_HD double fx_mc_slope_br(double qm, double q0, double qp, BR &br, int k)
{
    const double sl = q0 - qm;
    const double sr = qp - q0;
    const double c0 = 2.0 * sl;
    const double c1 = sl + 0.5 * (sr - sl);
    const double c2 = 2.0 * sr;
    unsigned reg = 3u;
    if (sl * sr > 0.0) {
        if (sl > 0.0) {
            const double m = c0 < c1 ? c0 : c1;
            reg = m < c2 ? (c0 < c1 ? 0u : 1u) : 2u;
        } else {
            const double m = c0 > c1 ? c0 : c1;
            reg = m > c2 ? (c0 > c1 ? 0u : 1u) : 2u;
        }
    }
    reg = br.field(k, reg);
    return reg == 0u ? c0 : reg == 1u ? c1 : reg == 2u ? c2 : 0.0;
}

/* ------------------------------------------------------------------------ */
/* Ideal gas (problems/prj_problem_ideal_eos.h:24-32 through the USER branch */
/* of prj_eos_rey, src/prj_eos.c:772-788).                                   */
/* ------------------------------------------------------------------------ */
FX_HD double fx_pressure(double g, double rho, double eint)
{
    return (g - 1.0) * rho * eint;            /* ((g-1)*rho)*eint */
}

FX_HD double fx_temperature(double g, double eint)
{
    return (g - 1.0) * eint / FX_IDEAL_ENERGY_SCALE;
}

/* WENO-Z3 face value of prj_reconstruct_weno3_face (src/prj_reconstruct.h:383-423):
 * target +0.5 gives the i+1/2 (left) state of cell (qm, q0, qp), -0.5 the
 * i-1/2 (right) state; Z weights alpha_k = gamma_k (1 + tau3 / (eps + beta_k)) */
FX_HD double fx_weno3_face(double qm, double q0, double qp, double target)
{
    const double eps = 1.0e-40;
    const double p0 = q0 + target * (q0 - qm);
    const double p1 = q0 + target * (qp - q0);
    const double dl = q0 - qm;
    const double dr = qp - q0;
    const double beta0 = dl * dl;
    const double beta1 = dr * dr;
    double tau3 = beta0 - beta1;
    if (tau3 < 0.0) {
        tau3 = -tau3;
    }
    const double gamma0 = target > 0.0 ? 1.0 / 3.0 : 2.0 / 3.0;
    const double gamma1 = target > 0.0 ? 2.0 / 3.0 : 1.0 / 3.0;
    const double alpha0 = gamma0 * (1.0 + tau3 / (eps + beta0));
    const double alpha1 = gamma1 * (1.0 + tau3 / (eps + beta1));
    const double sum = alpha0 + alpha1;
    return (alpha0 * p0 + alpha1 * p1) / sum;
}

/* WENO-Z7 (src/prj_reconstruct.h:425-521): the i+1/2 face value of the cell
 * at q[3] from q[0..6].  Smoothness indicators are quadratic forms over
 * four consecutive cells, evaluated term by term in the order (0,0), (0,1),
 * (0,2), (0,3), (1,1), (1,2), (1,3), (2,2), (2,3), (3,3) as ((c q_a) q_b),
 * accumulated left to right and divided by 240; a term with a negative
 * coefficient subtracts (|c| q_a) q_b, which is the same double.  The i-1/2
 * face is the same formula on the mirrored stencil. */
FX_HD double fx_weno7_beta(const double c[10], double q0, double q1, double q2, double q3)
{
    const double q[4] = {q0, q1, q2, q3};
    double acc = c[0] * q[0] * q[0];
    int t = 1;
#pragma unroll
    for (int a = 0; a < 4; ++a) {
#pragma unroll
        for (int b = a; b < 4; ++b) {
            if (a == 0 && b == 0) continue;
            acc = acc + c[t] * q[a] * q[b];
            ++t;
        }
    }
    return acc / 240.0;
}

FX_HD double fx_weno7_plus(double q0, double q1, double q2, double q3, double q4, double q5, double q6)
{
    /* Balsara-Shu seventh-order smoothness coefficients, one row per
     * sub-stencil, terms in the order above */
    const double C0[10] = {547.0, -3882.0, 4642.0, -1854.0, 7043.0, -17246.0, 7042.0, 11003.0, -9402.0, 2107.0};
    const double C1[10] = {267.0, -1642.0, 1602.0, -494.0, 2843.0, -5966.0, 1922.0, 3443.0, -2522.0, 547.0};
    const double C2[10] = {547.0, -2522.0, 1922.0, -494.0, 3443.0, -5966.0, 1602.0, 2843.0, -1642.0, 267.0};
    const double C3[10] = {2107.0, -9402.0, 7042.0, -1854.0, 11003.0, -17246.0, 4642.0, 7043.0, -3882.0, 547.0};
    const double eps = 1.0e-40;
    /* third-order candidates of the four sub-stencils */
    const double p0 = (-3.0 * q0 + 13.0 * q1 - 23.0 * q2 + 25.0 * q3) / 12.0;
    const double p1 = (q1 - 5.0 * q2 + 13.0 * q3 + 3.0 * q4) / 12.0;
    const double p2 = (-q2 + 7.0 * q3 + 7.0 * q4 - q5) / 12.0;
    const double p3 = (3.0 * q3 + 13.0 * q4 - 5.0 * q5 + q6) / 12.0;
    const double b0 = fx_weno7_beta(C0, q0, q1, q2, q3);
    const double b1 = fx_weno7_beta(C1, q1, q2, q3, q4);
    const double b2 = fx_weno7_beta(C2, q2, q3, q4, q5);
    const double b3 = fx_weno7_beta(C3, q3, q4, q5, q6);
    /* global indicator tau7 and Z weights with the linear weights 1/35,
     * 12/35, 18/35, 4/35 */
    double tau7 = b0 - b3 + 3.0 * (b1 - b2);
    if (tau7 < 0.0) {
        tau7 = -tau7;
    }
    const double r0 = tau7 / (eps + b0);
    const double r1 = tau7 / (eps + b1);
    const double r2 = tau7 / (eps + b2);
    const double r3 = tau7 / (eps + b3);
    const double a0 = (1.0 / 35.0) * (1.0 + r0 * r0);
    const double a1 = (12.0 / 35.0) * (1.0 + r1 * r1);
    const double a2 = (18.0 / 35.0) * (1.0 + r2 * r2);
    const double a3 = (4.0 / 35.0) * (1.0 + r3 * r3);
    const double sum = a0 + a1 + a2 + a3;
    return (a0 * p0 + a1 * p1 + a2 * p2 + a3 * p3) / sum;
}

/* minmod slope of prj_reconstruct_minmod_slope (src/prj_reconstruct.h:46-62) */
FX_HD double fx_minmod_slope(double qm, double q0, double qp)
{
    const double sl = q0 - qm;
    const double sr = qp - q0;
    if (sl * sr <= 0.0) {
        return 0.0;
    }
    return fabs(sl) < fabs(sr) ? sl : sr;
}

/* Barth-Jespersen limited prolongation (use_BJ), the stencil read through
 * q(di, dj, dk) / q(di, dj) with offsets in {-1, 0, 1}:
 * prj_reconstruct_cell_for_prolongate_bj and _face_for_prolongate_bj
 * (src/prj_reconstruct.h:145-195, 248-290).  The central-difference
 * gradient is scaled by the largest alpha in [0, 1] that keeps the eight
 * fine sub-cell (four sub-face) values at offsets +-1/4 inside the range of
 * the stencil's neighbours; the minimum / maximum and the alpha reduction run
 * in the reference's loop order (a < b ? a : b, so the order decides which
 * of +0.0 and -0.0 survives a tie). */
FX_HD double fx_bj_min(double a, double b) { return a < b ? a : b; }
FX_HD double fx_bj_max(double a, double b) { return a > b ? a : b; }
FX_HD double fx_bj_clamp01(double x) { return x < 0.0 ? 0.0 : (x > 1.0 ? 1.0 : x); }

/* alpha update of one sub-cell value base + delta */
FX_HD double fx_bj_alpha(double alpha, double base, double delta, double qmin, double qmax)
{
    const double q = base + delta;
    if (q > qmax) {
        const double a = delta != 0.0 ? (qmax - base) / delta : 0.0;
        return fx_bj_min(alpha, fx_bj_clamp01(a));
    }
    if (q < qmin) {
        const double a = delta != 0.0 ? (qmin - base) / delta : 0.0;
        return fx_bj_min(alpha, fx_bj_clamp01(a));
    }
    return alpha;
}

template <class Q>
FX_HD double fx_bj_cell(const Q &q, double tx, double ty, double tz)
{
    const double base = q(0, 0, 0);
    const double g0 = 0.5 * (q(1, 0, 0) - q(-1, 0, 0));
    const double g1 = 0.5 * (q(0, 1, 0) - q(0, -1, 0));
    const double g2 = 0.5 * (q(0, 0, 1) - q(0, 0, -1));
    double qmin = q(-1, -1, -1);
    double qmax = qmin;
#pragma unroll 1
    for (int n = 0; n < 27; ++n) {
        if (n == 13) continue;
        const double v = q(n / 9 - 1, (n / 3) % 3 - 1, n % 3 - 1);
        qmin = fx_bj_min(qmin, v);
        qmax = fx_bj_max(qmax, v);
    }
    double alpha = 1.0;
#pragma unroll
    for (int s = 0; s < 8; ++s) {
        const double o0 = (s & 4) ? 0.25 : -0.25;
        const double o1 = (s & 2) ? 0.25 : -0.25;
        const double o2 = (s & 1) ? 0.25 : -0.25;
        const double delta = g0 * o0 + g1 * o1 + g2 * o2;
        alpha = fx_bj_alpha(alpha, base, delta, qmin, qmax);
    }
    return base + alpha * (g0 * tx + g1 * ty + g2 * tz);
}

template <class Q>
FX_HD double fx_bj_face(const Q &q, double t0, double t1)
{
    const double base = q(0, 0);
    const double g0 = 0.5 * (q(1, 0) - q(-1, 0));
    const double g1 = 0.5 * (q(0, 1) - q(0, -1));
    double qmin = q(-1, -1);
    double qmax = qmin;
#pragma unroll
    for (int n = 0; n < 9; ++n) {
        if (n == 4) continue;
        const double v = q(n / 3 - 1, n % 3 - 1);
        qmin = fx_bj_min(qmin, v);
        qmax = fx_bj_max(qmax, v);
    }
    double alpha = 1.0;
#pragma unroll
    for (int s = 0; s < 4; ++s) {
        const double o0 = (s & 2) ? 0.25 : -0.25;
        const double o1 = (s & 1) ? 0.25 : -0.25;
        const double delta = g0 * o0 + g1 * o1;
        alpha = fx_bj_alpha(alpha, base, delta, qmin, qmax);
    }
    return base + alpha * (g0 * t0 + g1 * t1);
}

/* prj_eos_prim2cons, src/prj_eos.c:2112-2151 */
template <bool MHD>
FX_HD void fx_prim2cons(const double *w, double *u)
{
    const double rho = w[FX_RHO];
    const double v1 = w[FX_V1];
    const double v2 = w[FX_V2];
    const double v3 = w[FX_V3];
    const double eint = w[FX_EINT];
    u[FX_RHO] = rho;
    u[FX_V1] = rho * v1;
    u[FX_V2] = rho * v2;
    u[FX_V3] = rho * v3;
    if (MHD) {
        const double b1 = w[FX_B1];
        const double b2 = w[FX_B2];
        const double b3 = w[FX_B3];
        u[FX_ETOT] = rho * eint + 0.5 * rho * (v1 * v1 + v2 * v2 + v3 * v3) +
            0.5 * (b1 * b1 + b2 * b2 + b3 * b3);
        u[FX_YE] = rho * w[FX_YE];
        u[FX_B1] = b1;
        u[FX_B2] = b2;
        u[FX_B3] = b3;
    } else {
        u[FX_ETOT] = rho * eint + 0.5 * rho * (v1 * v1 + v2 * v2 + v3 * v3);
        u[FX_YE] = rho * w[FX_YE];
    }
}

/* prj_eos_cons2prim, src/prj_eos.c:2153-2220 (no floors) */
template <bool MHD>
FX_HD void fx_cons2prim(const double *u, double *w)
{
    const double rho = u[FX_RHO];
    if (rho == 0.0) {
        for (int v = 0; v < (MHD ? 9 : 6); ++v) {
            w[v] = 0.0;
        }
        return;
    }
    const double v1 = u[FX_V1] / rho;
    const double v2 = u[FX_V2] / rho;
    const double v3 = u[FX_V3] / rho;
    const double kinetic = 0.5 * (v1 * v1 + v2 * v2 + v3 * v3);
    w[FX_RHO] = rho;
    w[FX_V1] = v1;
    w[FX_V2] = v2;
    w[FX_V3] = v3;
    if (MHD) {
        const double magnetic = 0.5 * (u[FX_B1] * u[FX_B1] + u[FX_B2] * u[FX_B2] +
            u[FX_B3] * u[FX_B3]) / rho;
        w[FX_EINT] = u[FX_ETOT] / rho - kinetic - magnetic;
        w[FX_YE] = u[FX_YE] / rho;
        w[FX_B1] = u[FX_B1];
        w[FX_B2] = u[FX_B2];
        w[FX_B3] = u[FX_B3];
    } else {
        w[FX_EINT] = u[FX_ETOT] / rho - kinetic;
        w[FX_YE] = u[FX_YE] / rho;
    }
}

/* ------------------------------------------------------------------------ */
/* HLLD (Miyoshi & Kusano 2005) as in src/prj_riemann.c:81-440.              */
/* ------------------------------------------------------------------------ */
#define FX_HLLD_SMALL 1.0e-8

struct FxHlldState {
    double rho, vx, vy, vz, bx, by, bz, p, gamma, ye, e, pt;
};

struct FxHlldStar {
    double rho, vx, vy, vz, bx, by, bz, ye, e;
};

/* prj_hlld_fill_conserved, src/prj_riemann.c:81-94 (component v) */
FX_HD double fx_hlld_u(const FxHlldStar &s, int v)
{
    switch (v) {
    case 0: return s.rho;
    case 1: return s.rho * s.vx;
    case 2: return s.rho * s.vy;
    case 3: return s.rho * s.vz;
    case 4: return s.e;
    case 5: return s.rho * s.ye;
    case 6: return s.bx;
    case 7: return s.by;
    default: return s.bz;
    }
}

FX_HD double fx_hlld_state_u(const FxHlldState &s, int v)
{
    switch (v) {
    case 0: return s.rho;
    case 1: return s.rho * s.vx;
    case 2: return s.rho * s.vy;
    case 3: return s.rho * s.vz;
    case 4: return s.e;
    case 5: return s.rho * s.ye;
    case 6: return s.bx;
    case 7: return s.by;
    default: return s.bz;
    }
}

/* prj_hlld_fill_flux, src/prj_riemann.c:96-115 (component v) */
FX_HD double fx_hlld_state_f(const FxHlldState &s, int v)
{
    const double b2 = s.bx * s.bx + s.by * s.by + s.bz * s.bz;
    const double pt = s.p + 0.5 * b2;
    switch (v) {
    case 0: return s.rho * s.vx;
    case 1: return s.rho * s.vx * s.vx + pt - s.bx * s.bx;
    case 2: return s.rho * s.vx * s.vy - s.bx * s.by;
    case 3: return s.rho * s.vx * s.vz - s.bx * s.bz;
    case 4: {
        const double vdotb = s.vx * s.bx + s.vy * s.by + s.vz * s.bz;
        return (s.e + pt) * s.vx - s.bx * vdotb;
    }
    case 5: return s.rho * s.ye * s.vx;
    case 6: return 0.0;
    case 7: return s.by * s.vx - s.bx * s.vy;
    default: return s.bz * s.vx - s.bx * s.vz;
    }
}

/* prj_hlld_state_from_prim, src/prj_riemann.c:142-178; w is the local
 * (direction-rotated) primitive vector, the normal field is bn. */
template <class E>
FX_HD void fx_hlld_state_e(const double *w, double p, double gamma, double bn,
    FxHlldState &s, E *err, int blk, int idx)
{
    s.rho = w[FX_RHO];
    s.vx = w[FX_V1];
    s.vy = w[FX_V2];
    s.vz = w[FX_V3];
    s.bx = bn;
    s.by = w[FX_B2];
    s.bz = w[FX_B3];
    s.p = p;
    s.gamma = gamma;
    s.ye = w[FX_YE];
    if (s.rho <= 0.0) fx_fail(err, FX_ERR_HLLD_RHO, blk, idx);
    if (s.p <= 0.0) fx_fail(err, FX_ERR_HLLD_P, blk, idx);
    if (s.gamma <= 0.0) fx_fail(err, FX_ERR_HLLD_GAMMA, blk, idx);
    const double kinetic = 0.5 * s.rho * (s.vx * s.vx + s.vy * s.vy + s.vz * s.vz);
    const double magnetic = 0.5 * (s.bx * s.bx + s.by * s.by + s.bz * s.bz);
    s.e = s.rho * w[FX_EINT] + kinetic + magnetic;
    s.pt = s.p + magnetic;
}

FX_HD void fx_hlld_state(const double *w, double p, double gamma, double bn,
    FxHlldState &s, FxErr *err, int blk, int idx)
{
    fx_hlld_state_e(w, p, gamma, bn, s, err, blk, idx);
}

/* prj_hlld_fast_speed, src/prj_riemann.c:117-140; the clamp of a negative
 * discriminant is decision bit k */
template <class BR, class E = FxErr>
FX_HD double fx_hlld_fast_speed_br(const FxHlldState &s, E *err, int blk, int idx, BR &br, int k)
{
    const double a2 = fx_div(s.gamma * s.p, s.rho);
    const double bx2_rho = fx_div(s.bx * s.bx, s.rho);
    const double b2_rho = fx_div(s.bx * s.bx + s.by * s.by + s.bz * s.bz, s.rho);
    double disc = (a2 + b2_rho) * (a2 + b2_rho) - 4.0 * a2 * bx2_rho;
    if (br.bit(k, disc < 0.0)) {
        if (disc < -1.0e-12 * (a2 + b2_rho) * (a2 + b2_rho)) {
            fx_fail(err, FX_ERR_HLLD_DISC, blk, idx);
        }
        disc = 0.0;
    }
    const double cf2 = 0.5 * (a2 + b2_rho + sqrt(disc));
    if (cf2 < 0.0 || !isfinite(cf2)) {
        fx_fail(err, FX_ERR_HLLD_CF, blk, idx);
    }
    return sqrt(cf2);
}

FX_HD double fx_hlld_fast_speed(const FxHlldState &s, FxErr *err, int blk, int idx)
{
    FxBrFree br;
    return fx_hlld_fast_speed_br(s, err, blk, idx, br, 0);
}

/* prj_hlld_outer_star, src/prj_riemann.c:185-232; the degenerate-denominator
 * branch is decision bit k */
template <class BR, class E = FxErr>
FX_HD void fx_hlld_outer_star_br(const FxHlldState &s, double S, double SM,
    double pt_star, FxHlldStar &st, E *err, int blk, int idx, BR &br, int k)
{
    const double alpha = S - s.vx;
    const double smdiff = S - SM;
    if (fabs(smdiff) <= 1.0e-14 * (fabs(S) + fabs(SM) + 1.0)) {
        fx_fail(err, FX_ERR_HLLD_OUTER, blk, idx);
    }
    st.rho = fx_div(s.rho * alpha, smdiff);
    if (st.rho <= 0.0 || !isfinite(st.rho)) {
        fx_fail(err, FX_ERR_HLLD_STARRHO, blk, idx);
    }
    st.vx = SM;
    st.bx = s.bx;
    st.ye = s.ye;
    const double denom = s.rho * alpha * smdiff - s.bx * s.bx;
    if (br.bit(k, fabs(denom) < FX_HLLD_SMALL * pt_star)) {
        st.vy = s.vy;
        st.vz = s.vz;
        st.by = s.by;
        st.bz = s.bz;
    } else {
        const double sm_diff_vx_over_denom = fx_div(SM - s.vx, denom);
        const double mag_factor = fx_div(s.rho * alpha * alpha - s.bx * s.bx, denom);
        st.vy = s.vy - s.bx * s.by * sm_diff_vx_over_denom;
        st.vz = s.vz - s.bx * s.bz * sm_diff_vx_over_denom;
        st.by = s.by * mag_factor;
        st.bz = s.bz * mag_factor;
    }
    const double vdotb = s.vx * s.bx + s.vy * s.by + s.vz * s.bz;
    const double vstar_dotbstar = st.vx * st.bx + st.vy * st.by + st.vz * st.bz;
    st.e = fx_div(alpha * s.e - s.pt * s.vx + pt_star * SM + s.bx * (vdotb - vstar_dotbstar), smdiff);
}

FX_HD void fx_hlld_outer_star(const FxHlldState &s, double S, double SM,
    double pt_star, FxHlldStar &st, FxErr *err, int blk, int idx)
{
    FxBrFree br;
    fx_hlld_outer_star_br(s, S, SM, pt_star, st, err, blk, idx, br, 0);
}

/* prj_hlld_double_star_one, src/prj_riemann.c:234-282 */
FX_HD void fx_hlld_double_star(const FxHlldStar &left, const FxHlldStar &right,
    double bx, bool right_side, FxHlldStar &ss, FxErr *err, int blk, int idx)
{
    const double sqrt_l = sqrt(left.rho);
    const double sqrt_r = sqrt(right.rho);
    if (sqrt_l + sqrt_r <= 0.0) {
        fx_fail(err, FX_ERR_HLLD_DSTAR, blk, idx);
    }
    const double inv_sum = 1.0 / (sqrt_l + sqrt_r);
    const double sign_bx = bx < 0.0 ? -1.0 : 1.0;
    const double vy_ss = (sqrt_l * left.vy + sqrt_r * right.vy +
        (right.by - left.by) * sign_bx) * inv_sum;
    const double vz_ss = (sqrt_l * left.vz + sqrt_r * right.vz +
        (right.bz - left.bz) * sign_bx) * inv_sum;
    const double by_ss = (sqrt_l * right.by + sqrt_r * left.by +
        sqrt_l * sqrt_r * (right.vy - left.vy) * sign_bx) * inv_sum;
    const double bz_ss = (sqrt_l * right.bz + sqrt_r * left.bz +
        sqrt_l * sqrt_r * (right.vz - left.vz) * sign_bx) * inv_sum;
    const double vbdot_ss = (right_side ? right.vx : left.vx) * bx + vy_ss * by_ss + vz_ss * bz_ss;
    if (!right_side) {
        const double vbdot_l = left.vx * bx + left.vy * left.by + left.vz * left.bz;
        ss = left;
        ss.e = left.e - sqrt_l * sign_bx * (vbdot_l - vbdot_ss);
    } else {
        const double vbdot_r = right.vx * bx + right.vy * right.by + right.vz * right.bz;
        ss = right;
        ss.e = right.e + sqrt_r * sign_bx * (vbdot_r - vbdot_ss);
    }
    ss.vy = vy_ss;
    ss.vz = vz_ss;
    ss.by = by_ss;
    ss.bz = bz_ss;
}

/* Face outputs of the MHD solver: local-frame flux (9), face velocity (3)
 * and the two face EMF products (prj_hlld_face_outputs,
 * src/prj_riemann.c:305-319). */
struct FxFaceOut {
    double F[9];
    double v[3];
    double bv1;
    double bv2;
};

FX_HD void fx_face_outputs(double vx, double vy, double vz,
    double bx, double by, double bz, FxFaceOut &o)
{
    o.v[0] = vx;
    o.v[1] = vy;
    o.v[2] = vz;
    o.bv1 = bz * vx - bx * vz;
    o.bv2 = bx * vy - by * vx;
}

/* prj_riemann_hlld, src/prj_riemann.c:321-440 */
static __device__ __noinline__ void fx_riemann_hlld(const double *WL, const double *WR,
    double pL, double pR, double gL, double gR, double bn, FxFaceOut &o,
    FxErr *err, int blk, int idx)
{
    FxHlldState L, R;
    fx_hlld_state(WL, pL, gL, bn, L, err, blk, idx);
    fx_hlld_state(WR, pR, gR, bn, R, err, blk, idx);
    const double cfL = fx_hlld_fast_speed(L, err, blk, idx);
    const double cfR = fx_hlld_fast_speed(R, err, blk, idx);
    const double SL = fx_min(L.vx - cfL, R.vx - cfR);
    const double SR = fx_max(L.vx + cfL, R.vx + cfR);
    if (!(SL < SR)) {
        fx_fail(err, FX_ERR_HLLD_ORDER, blk, idx);
    }
    if (0.0 <= SL) {
        for (int v = 0; v < 9; ++v) o.F[v] = fx_hlld_state_f(L, v);
        fx_face_outputs(L.vx, L.vy, L.vz, L.bx, L.by, L.bz, o);
        return;
    }
    if (SR <= 0.0) {
        for (int v = 0; v < 9; ++v) o.F[v] = fx_hlld_state_f(R, v);
        fx_face_outputs(R.vx, R.vy, R.vz, R.bx, R.by, R.bz, o);
        return;
    }
    const double denom = R.rho * (SR - R.vx) - L.rho * (SL - L.vx);
    if (fabs(denom) <= 1.0e-14 *
        (fabs(R.rho * (SR - R.vx)) + fabs(L.rho * (SL - L.vx)) + 1.0)) {
        fx_fail(err, FX_ERR_HLLD_DENOM, blk, idx);
    }
    const double SM = (R.rho * R.vx * (SR - R.vx) -
        L.rho * L.vx * (SL - L.vx) + (L.pt - R.pt)) / denom;
    const double pt_star_l = L.pt + L.rho * (SL - L.vx) * (SM - L.vx);
    const double pt_star_r = R.pt + R.rho * (SR - R.vx) * (SM - R.vx);
    const double pt_star = 0.5 * (pt_star_l + pt_star_r);
    if (pt_star <= 0.0 || !isfinite(pt_star)) {
        /* HLL fallback, src/prj_riemann.c:392-409 */
        const double inv = 1.0 / (SR - SL);
        double Uh[9];
        for (int v = 0; v < 9; ++v) {
            const double lf = fx_hlld_state_f(L, v);
            const double rf = fx_hlld_state_f(R, v);
            const double lu = fx_hlld_state_u(L, v);
            const double ru = fx_hlld_state_u(R, v);
            o.F[v] = (SR * lf - SL * rf + SL * SR * (ru - lu)) * inv;
            Uh[v] = (SR * ru - SL * lu + lf - rf) * inv;
        }
        const double rho = Uh[0];
        fx_face_outputs(Uh[1] / rho, Uh[2] / rho, Uh[3] / rho, Uh[6], Uh[7], Uh[8], o);
        return;
    }
    const bool bn_small = (0.5 * bn * bn < FX_HLLD_SMALL * pt_star);
    FxHlldStar Ls, Rs, ss;
    if (0.0 <= SM) {
        fx_hlld_outer_star(L, SL, SM, pt_star, Ls, err, blk, idx);
        const double SLs = SM - fabs(bn) / sqrt(Ls.rho);
        if (0.0 <= SLs || bn_small) {
            for (int v = 0; v < 9; ++v) {
                o.F[v] = fx_hlld_state_f(L, v) + SL * (fx_hlld_u(Ls, v) - fx_hlld_state_u(L, v));
            }
            fx_face_outputs(Ls.vx, Ls.vy, Ls.vz, Ls.bx, Ls.by, Ls.bz, o);
        } else {
            fx_hlld_outer_star(R, SR, SM, pt_star, Rs, err, blk, idx);
            fx_hlld_double_star(Ls, Rs, bn, false, ss, err, blk, idx);
            for (int v = 0; v < 9; ++v) {
                const double us = fx_hlld_u(Ls, v);
                o.F[v] = fx_hlld_state_f(L, v) + SL * (us - fx_hlld_state_u(L, v)) +
                    SLs * (fx_hlld_u(ss, v) - us);
            }
            fx_face_outputs(ss.vx, ss.vy, ss.vz, ss.bx, ss.by, ss.bz, o);
        }
    } else {
        fx_hlld_outer_star(R, SR, SM, pt_star, Rs, err, blk, idx);
        const double SRs = SM + fabs(bn) / sqrt(Rs.rho);
        if (SRs <= 0.0 || bn_small) {
            for (int v = 0; v < 9; ++v) {
                o.F[v] = fx_hlld_state_f(R, v) + SR * (fx_hlld_u(Rs, v) - fx_hlld_state_u(R, v));
            }
            fx_face_outputs(Rs.vx, Rs.vy, Rs.vz, Rs.bx, Rs.by, Rs.bz, o);
        } else {
            fx_hlld_outer_star(L, SL, SM, pt_star, Ls, err, blk, idx);
            fx_hlld_double_star(Ls, Rs, bn, true, ss, err, blk, idx);
            for (int v = 0; v < 9; ++v) {
                const double us = fx_hlld_u(Rs, v);
                o.F[v] = fx_hlld_state_f(R, v) + SR * (us - fx_hlld_state_u(R, v)) +
                    SRs * (fx_hlld_u(ss, v) - us);
            }
            fx_face_outputs(ss.vx, ss.vy, ss.vz, ss.bx, ss.by, ss.bz, o);
        }
    }
}

/* Same solver with the left and right star branches folded into one code
 * path.  With `left` = (0 <= SM), the reference's two branches
 * (src/prj_riemann.c:413-438) are the same sequence of operations applied to
 * the near state N = left ? L : R and the far state F = left ? R : L:
 *   Ns = outer_star(N, S_N); a = |bn|/sqrt(Ns.rho); S_Ns = SM -/+ a;
 *   single star if (left ? 0 <= S_Ns : S_Ns <= 0) || bn_small;
 *   else Fs = outer_star(F, S_F) and the double star of (Ls, Rs), whose
 *   energy update e = Ns.e -/+ sqrt(Ns.rho) sign(bn) (vb_Ns - vb_ss) uses the
 *   near star in both branches (its normal velocity is SM on either side).
 * Selecting operands and choosing between x - t and x + t are exact, so the
 * result is bit-identical to fx_riemann_hlld; warps whose faces straddle
 * SM = 0 no longer execute both branches. */
template <class BR, class E = FxErr>
FX_HD void fx_riemann_hlld_folded_br(const double *WL, const double *WR,
    double pL, double pR, double gL, double gR, double bn, FxFaceOut &o,
    E *err, int blk, int idx, BR &br)
{
    FxHlldState L, R;
    fx_hlld_state_e(WL, pL, gL, bn, L, err, blk, idx);
    fx_hlld_state_e(WR, pR, gR, bn, R, err, blk, idx);
    const double cfL = fx_hlld_fast_speed_br(L, err, blk, idx, br, FX_BR_DISC_L);
    const double cfR = fx_hlld_fast_speed_br(R, err, blk, idx, br, FX_BR_DISC_R);
    const double aL = L.vx - cfL, aR = R.vx - cfR;
    const double bL = L.vx + cfL, bR = R.vx + cfR;
    const double SL = br.bit(FX_BR_SL, aL < aR) ? aL : aR;   /* fx_min */
    const double SR = br.bit(FX_BR_SR, bL > bR) ? bL : bR;   /* fx_max */
    if (!(SL < SR)) {
        fx_fail(err, FX_ERR_HLLD_ORDER, blk, idx);
    }
    const bool super_l = br.bit(FX_BR_SUPER_L, 0.0 <= SL);
    if (super_l || br.bit(FX_BR_SUPER_R, SR <= 0.0)) {
        const FxHlldState &X = super_l ? L : R;
#pragma unroll
        for (int v = 0; v < 9; ++v) o.F[v] = fx_hlld_state_f(X, v);
        fx_face_outputs(X.vx, X.vy, X.vz, X.bx, X.by, X.bz, o);
        return;
    }
    const double denom = R.rho * (SR - R.vx) - L.rho * (SL - L.vx);
    if (fabs(denom) <= 1.0e-14 *
        (fabs(R.rho * (SR - R.vx)) + fabs(L.rho * (SL - L.vx)) + 1.0)) {
        fx_fail(err, FX_ERR_HLLD_DENOM, blk, idx);
    }
    const double SM = fx_div(R.rho * R.vx * (SR - R.vx) -
        L.rho * L.vx * (SL - L.vx) + (L.pt - R.pt), denom);
    const double pt_star_l = L.pt + L.rho * (SL - L.vx) * (SM - L.vx);
    const double pt_star_r = R.pt + R.rho * (SR - R.vx) * (SM - R.vx);
    const double pt_star = 0.5 * (pt_star_l + pt_star_r);
    if (br.bit(FX_BR_HLL, pt_star <= 0.0 || !isfinite(pt_star))) {
        const double inv = fx_div(1.0, SR - SL);
        double Uh[9];
#pragma unroll
        for (int v = 0; v < 9; ++v) {
            const double lf = fx_hlld_state_f(L, v);
            const double rf = fx_hlld_state_f(R, v);
            const double lu = fx_hlld_state_u(L, v);
            const double ru = fx_hlld_state_u(R, v);
            o.F[v] = (SR * lf - SL * rf + SL * SR * (ru - lu)) * inv;
            Uh[v] = (SR * ru - SL * lu + lf - rf) * inv;
        }
        const double rho = Uh[0];
        fx_face_outputs(fx_div(Uh[1], rho), fx_div(Uh[2], rho), fx_div(Uh[3], rho), Uh[6], Uh[7], Uh[8], o);
        return;
    }
    const bool bn_small = br.bit(FX_BR_BNSMALL, 0.5 * bn * bn < FX_HLLD_SMALL * pt_star);
    const bool left = br.bit(FX_BR_LEFT, 0.0 <= SM);
    const FxHlldState N = left ? L : R;
    const double SN = left ? SL : SR;
    FxHlldStar Ns;
    fx_hlld_outer_star_br(N, SN, SM, pt_star, Ns, err, blk, idx, br, FX_BR_DEGEN_N);
    const double sqN = sqrt(Ns.rho);
    const double a = fx_div(fabs(bn), sqN);
    const double SNs = left ? SM - a : SM + a;
    const bool single = br.bit(FX_BR_SINGLE, (left ? (0.0 <= SNs) : (SNs <= 0.0)) || bn_small);
    if (single) {
#pragma unroll
        for (int v = 0; v < 9; ++v) {
            o.F[v] = fx_hlld_state_f(N, v) + SN * (fx_hlld_u(Ns, v) - fx_hlld_state_u(N, v));
        }
        fx_face_outputs(Ns.vx, Ns.vy, Ns.vz, Ns.bx, Ns.by, Ns.bz, o);
        return;
    }
    const FxHlldState Fr = left ? R : L;
    const double SF = left ? SR : SL;
    FxHlldStar Fs;
    fx_hlld_outer_star_br(Fr, SF, SM, pt_star, Fs, err, blk, idx, br, FX_BR_DEGEN_F);
    const FxHlldStar Ls = left ? Ns : Fs;
    const FxHlldStar Rs = left ? Fs : Ns;
    /* prj_hlld_double_star_one, src/prj_riemann.c:234-282 */
    /* sqrt(Ls.rho), sqrt(Rs.rho): the near star's was taken above */
    const double sqF = sqrt(Fs.rho);
    const double sqrt_l = left ? sqN : sqF;
    const double sqrt_r = left ? sqF : sqN;
    if (sqrt_l + sqrt_r <= 0.0) {
        fx_fail(err, FX_ERR_HLLD_DSTAR, blk, idx);
    }
    const double inv_sum = fx_div(1.0, sqrt_l + sqrt_r);
    const double sign_bx = br.bit(FX_BR_BNEG, bn < 0.0) ? -1.0 : 1.0;
    FxHlldStar ss = Ns;
    ss.vy = (sqrt_l * Ls.vy + sqrt_r * Rs.vy + (Rs.by - Ls.by) * sign_bx) * inv_sum;
    ss.vz = (sqrt_l * Ls.vz + sqrt_r * Rs.vz + (Rs.bz - Ls.bz) * sign_bx) * inv_sum;
    ss.by = (sqrt_l * Rs.by + sqrt_r * Ls.by + sqrt_l * sqrt_r * (Rs.vy - Ls.vy) * sign_bx) * inv_sum;
    ss.bz = (sqrt_l * Rs.bz + sqrt_r * Ls.bz + sqrt_l * sqrt_r * (Rs.vz - Ls.vz) * sign_bx) * inv_sum;
    const double vbdot_ss = Ns.vx * bn + ss.vy * ss.by + ss.vz * ss.bz;
    const double vbdot_n = Ns.vx * bn + Ns.vy * Ns.by + Ns.vz * Ns.bz;
    const double t = (left ? sqrt_l : sqrt_r) * sign_bx * (vbdot_n - vbdot_ss);
    ss.e = left ? Ns.e - t : Ns.e + t;
#pragma unroll
    for (int v = 0; v < 9; ++v) {
        const double us = fx_hlld_u(Ns, v);
        o.F[v] = fx_hlld_state_f(N, v) + SN * (us - fx_hlld_state_u(N, v)) +
            SNs * (fx_hlld_u(ss, v) - us);
    }
    fx_face_outputs(ss.vx, ss.vy, ss.vz, ss.bx, ss.by, ss.bz, o);
}

FX_HD void fx_riemann_hlld_folded(const double *WL, const double *WR,
    double pL, double pR, double gL, double gR, double bn, FxFaceOut &o,
    FxErr *err, int blk, int idx)
{
    FxBrFree br;
    fx_riemann_hlld_folded_br(WL, WR, pL, pR, gL, gR, bn, o, err, blk, idx, br);
}

/* ------------------------------------------------------------------------ */
/* HLLC for the hydro build, src/prj_riemann.c:1433-1599 and the theta       */
/* pressure-jump limiter of src/prj_riemann.c:8-17.                          */
/* ------------------------------------------------------------------------ */
FX_HD double fx_theta_limiter(double cfmax, double du, double dv, double dw)
{
    double theta_r = (-fx_min(du, 0.0) + cfmax) / (-fx_min(fx_min(dv, dw), 0.0) + cfmax);
    theta_r *= theta_r;
    return fx_min(1.0, theta_r * theta_r);
}

/* prj_riemann_state, src/prj_riemann.c:1433-1492 (hydro: 6 components) */
FX_HD void fx_hllc_state(const double *W, double p, double gamma,
    double *U, double *F, double &cs)
{
    const double rho = W[FX_RHO];
    const double v1 = W[FX_V1];
    const double v2 = W[FX_V2];
    const double v3 = W[FX_V3];
    const double eint = W[FX_EINT];
    const double etot = rho * eint + 0.5 * rho * (v1 * v1 + v2 * v2 + v3 * v3);
    U[0] = rho;
    U[1] = rho * v1;
    U[2] = rho * v2;
    U[3] = rho * v3;
    U[4] = etot;
    U[5] = rho * W[FX_YE];
    cs = sqrt(gamma * p / rho);
    F[0] = rho * v1;
    F[1] = rho * v1 * v1 + p;
    F[2] = rho * v1 * v2;
    F[3] = rho * v1 * v3;
    F[4] = (etot + p) * v1;
    F[5] = rho * W[FX_YE] * v1;
}

/* prj_riemann_hllc, src/prj_riemann.c:1494-1599; F[6], vface[3] out */
static __device__ __noinline__ void fx_riemann_hllc(const double *WL, const double *WR,
    double pL, double pR, double gL, double gR, double du, double dv, double dw,
    double *flux, double *v_face)
{
    double UL[6], UR[6], FL[6], FR[6], Ustar[6];
    double csL, csR;
    fx_hllc_state(WL, pL, gL, UL, FL, csL);
    fx_hllc_state(WR, pR, gR, UR, FR, csR);
    const double SL = fx_min(WL[FX_V1] - csL, WR[FX_V1] - csR);
    const double SR = fx_max(WL[FX_V1] + csL, WR[FX_V1] + csR);
    const double cfmax = fx_max(csL, csR);
    const double theta = fx_theta_limiter(cfmax, du, dv, dw);
    const double SM = (theta * (pR - pL) +
        UL[1] * (SL - WL[FX_V1]) -
        UR[1] * (SR - WR[FX_V1])) /
        (UL[0] * (SL - WL[FX_V1]) -
            UR[0] * (SR - WR[FX_V1]));
    if (0.0 <= SL) {
        for (int v = 0; v < 6; ++v) flux[v] = FL[v];
        v_face[0] = WL[FX_V1];
        v_face[1] = WL[FX_V2];
        v_face[2] = WL[FX_V3];
        return;
    }
    if (SR <= 0.0) {
        for (int v = 0; v < 6; ++v) flux[v] = FR[v];
        v_face[0] = WR[FX_V1];
        v_face[1] = WR[FX_V2];
        v_face[2] = WR[FX_V3];
        return;
    }
    v_face[0] = SM;
    if (0.0 <= SM) {
        v_face[1] = WL[FX_V2];
        v_face[2] = WL[FX_V3];
        for (int v = 0; v < 6; ++v) Ustar[v] = UL[v];
        const double rho_star = UL[0] * (SL - WL[FX_V1]) / (SL - SM);
        Ustar[0] = rho_star;
        Ustar[1] = rho_star * SM;
        Ustar[2] = rho_star * WL[FX_V2];
        Ustar[3] = rho_star * WL[FX_V3];
        const double e_over_rho = UL[4] / UL[0] +
            (SM - WL[FX_V1]) * (SM + pL / (UL[0] * (SL - WL[FX_V1])));
        Ustar[4] = rho_star * e_over_rho;
        Ustar[5] = rho_star * WL[FX_YE];
        for (int v = 0; v < 6; ++v) flux[v] = FL[v] + SL * (Ustar[v] - UL[v]);
    } else {
        v_face[1] = WR[FX_V2];
        v_face[2] = WR[FX_V3];
        for (int v = 0; v < 6; ++v) Ustar[v] = UR[v];
        const double rho_star = UR[0] * (SR - WR[FX_V1]) / (SR - SM);
        Ustar[0] = rho_star;
        Ustar[1] = rho_star * SM;
        Ustar[2] = rho_star * WR[FX_V2];
        Ustar[3] = rho_star * WR[FX_V3];
        const double e_over_rho = UR[4] / UR[0] +
            (SM - WR[FX_V1]) * (SM + pR / (UR[0] * (SR - WR[FX_V1])));
        Ustar[4] = rho_star * e_over_rho;
        Ustar[5] = rho_star * WR[FX_YE];
        for (int v = 0; v < 6; ++v) flux[v] = FR[v] + SR * (Ustar[v] - UR[v]);
    }
}

/* ------------------------------------------------------------------------ */
/* Upwind corner EMF, src/prj_mhd.c:627-718 (eta term separate).            */
/* ------------------------------------------------------------------------ */
/* the upwind direction of face n (0: vn > 0, 1: vn < 0, 2: vn == 0) is the
 * 2-bit decision field at bit 2 n of an edge's word */
template <class BR>
FX_HD double fx_emf_upwind_br(const double f[4], const double c[4], const double vn[4], BR &br)
{
    unsigned u[4];
#pragma unroll
    for (int n = 0; n < 4; ++n) {
        u[n] = br.field(2 * n, vn[n] > 0.0 ? 0u : vn[n] < 0.0 ? 1u : 2u);
    }
    double emf = 0.25 * (f[0] + f[1] + f[2] + f[3]);
    if (u[0] == 0u) {
        emf += 0.25 * (f[3] - c[3]);
    } else if (u[0] == 1u) {
        emf += 0.25 * (f[1] - c[0]);
    } else {
        emf += 0.125 * (f[3] - c[3] + f[1] - c[0]);
    }
    if (u[1] == 0u) {
        emf += 0.25 * (f[2] - c[1]);
    } else if (u[1] == 1u) {
        emf += 0.25 * (f[0] - c[0]);
    } else {
        emf += 0.125 * (f[2] - c[1] + f[0] - c[0]);
    }
    if (u[2] == 0u) {
        emf += 0.25 * (f[3] - c[2]);
    } else if (u[2] == 1u) {
        emf += 0.25 * (f[1] - c[1]);
    } else {
        emf += 0.125 * (f[3] - c[2] + f[1] - c[1]);
    }
    if (u[3] == 0u) {
        emf += 0.25 * (f[2] - c[2]);
    } else if (u[3] == 1u) {
        emf += 0.25 * (f[0] - c[3]);
    } else {
        emf += 0.125 * (f[2] - c[2] + f[0] - c[3]);
    }
    return emf;
}

FX_HD double fx_emf_upwind(const double f[4], const double c[4], const double vn[4])
{
    FxBrFree br;
    return fx_emf_upwind_br(f, c, vn, br);
}

/* artificial CT resistivity of one cell, src/prj_timeint.c:222-262 */
#define FX_ETA_BOOST 1.0e12
#define FX_ETA_RHO_FLOOR 1.0e13
#define FX_ETA_YE_THR 0.25

FX_HD double fx_cell_eta(double rho, double ye)
{
    /* max(0, log(x)) is exactly +0 for x <= 1 (log(1) = +0, log(x < 1) < 0),
     * and 1e12 * 0 * f = +0 for any finite f >= 0: the logarithms are only
     * evaluated for dense cells, with the reference's arithmetic. */
    const double xr = rho / FX_ETA_RHO_FLOOR;
    if (!(isfinite(rho) && rho > 0.0) || !(xr > 1.0)) {
        return 0.0;
    }
    double rho_factor = fx_max(0.0, log(xr));
    double ye_factor = 0.0;
    if (isfinite(ye) && ye > 0.0) {
        ye_factor = fx_max(0.0, log(ye / FX_ETA_YE_THR));
    }
    return FX_ETA_BOOST * rho_factor * ye_factor;
}

#endif
