/*
 * Discrete adjoint (reverse mode) of the pointwise pieces of the MHD update:
 * vector-Jacobian products of the MC reconstruction, the folded HLLD solver,
 * the face outputs, the upwind edge EMF and the primitive <-> conserved maps.
 *
 * Each *_vjp function recomputes the forward values it needs from its
 * inputs (nothing is stored between the forward and the reverse pass beyond
 * the stage inputs), takes the adjoints of the outputs and ACCUMULATES the
 * adjoints of the inputs.  Branches (limiter selections, Riemann fan
 * regions, upwind directions) are taken as in the forward evaluation and
 * held fixed: the result is the derivative of the piecewise-smooth map on
 * the piece the forward evaluation lies on.  Non-smooth points (a limiter
 * exactly at a switch, |bn| at 0) take the one-sided derivative of the
 * branch the forward code selects.
 *
 * All functions are host-callable (FX_HD) so they can be checked against
 * finite differences of the forward functions on the host.
 */
#ifndef FX_ADJOINT_CUH
#define FX_ADJOINT_CUH

#include "fx_physics.cuh"

/* ------------------------------------------------------------------------ */
/* MC slope (fx_mc_slope): d slope / d (qm, q0, qp) times gb, accumulated     */
/* ------------------------------------------------------------------------ */
FX_HD void fxa_mc_vjp(double qm, double q0, double qp, double gb, double &qmb, double &q0b, double &qpb)
{
    const double sl = q0 - qm;
    const double sr = qp - q0;
    if (!(sl * sr > 0.0) || gb == 0.0) {
        return;
    }
    const double c0 = 2.0 * sl;
    const double c1 = sl + 0.5 * (sr - sl);
    const double c2 = 2.0 * sr;
    int pick;
    if (sl > 0.0) {
        const int m = c0 < c1 ? 0 : 1;
        const double mv = m == 0 ? c0 : c1;
        pick = mv < c2 ? m : 2;
    } else {
        const int m = c0 > c1 ? 0 : 1;
        const double mv = m == 0 ? c0 : c1;
        pick = mv > c2 ? m : 2;
    }
    double slb = 0.0, srb = 0.0;
    if (pick == 0) {
        slb = 2.0 * gb;
    } else if (pick == 1) {
        slb = 0.5 * gb;
        srb = 0.5 * gb;
    } else {
        srb = 2.0 * gb;
    }
    qmb -= slb;
    q0b += slb - srb;
    qpb += srb;
}

/* ------------------------------------------------------------------------ */
/* HLLD pieces                                                               */
/* ------------------------------------------------------------------------ */

/* adjoint of an FxHlldState (gamma is a constant here) */
struct FxaS {
    double rho, vx, vy, vz, bx, by, bz, p, ye, e, pt;
};

/* adjoint of an FxHlldStar */
struct FxaSt {
    double rho, vx, vy, vz, bx, by, bz, ye, e;
};

FX_HD void fxa_clear(FxaS &a)
{
    a.rho = a.vx = a.vy = a.vz = a.bx = a.by = a.bz = a.p = a.ye = a.e = a.pt = 0.0;
}

FX_HD void fxa_clear(FxaSt &a)
{
    a.rho = a.vx = a.vy = a.vz = a.bx = a.by = a.bz = a.ye = a.e = 0.0;
}

/* fx_hlld_state: w (local primitives), p, bn -> state; w index 6 is unused
 * (the normal field is bn) */
FX_HD void fxa_state_vjp(const double *w, const FxaS &sb, double *wb, double &pb, double &bnb, double bn)
{
    const double rho = w[FX_RHO];
    const double vx = w[FX_V1];
    const double vy = w[FX_V2];
    const double vz = w[FX_V3];
    const double by = w[FX_B2];
    const double bz = w[FX_B3];
    /* e = rho eint + 0.5 rho |v|^2 + 0.5 |b|^2, pt = p + 0.5 |b|^2 */
    wb[FX_RHO] += sb.rho + sb.e * (w[FX_EINT] + 0.5 * (vx * vx + vy * vy + vz * vz));
    wb[FX_EINT] += sb.e * rho;
    wb[FX_V1] += sb.vx + sb.e * rho * vx;
    wb[FX_V2] += sb.vy + sb.e * rho * vy;
    wb[FX_V3] += sb.vz + sb.e * rho * vz;
    const double magb = sb.e + sb.pt;
    bnb += sb.bx + magb * bn;
    wb[FX_B2] += sb.by + magb * by;
    wb[FX_B3] += sb.bz + magb * bz;
    wb[FX_YE] += sb.ye;
    pb += sb.p + sb.pt;
}

/* fx_hlld_fast_speed */
FX_HD void fxa_fast_speed_vjp(const FxHlldState &s, double cfb, FxaS &sb)
{
    if (cfb == 0.0) {
        return;
    }
    const double a2 = s.gamma * s.p / s.rho;
    const double bx2r = s.bx * s.bx / s.rho;
    const double b2r = (s.bx * s.bx + s.by * s.by + s.bz * s.bz) / s.rho;
    const double s1 = a2 + b2r;
    double disc = s1 * s1 - 4.0 * a2 * bx2r;
    const bool clamped = disc < 0.0;
    if (clamped) {
        disc = 0.0;
    }
    const double sq = sqrt(disc);
    const double cf = sqrt(0.5 * (s1 + sq));
    const double cf2b = cfb * 0.5 / cf;
    double s1b = 0.5 * cf2b;
    const double sqb = 0.5 * cf2b;
    const double discb = (!clamped && sq > 0.0) ? sqb * 0.5 / sq : 0.0;
    s1b += discb * 2.0 * s1;
    double a2b = -4.0 * bx2r * discb;
    const double bx2rb = -4.0 * a2 * discb;
    a2b += s1b;
    const double b2rb = s1b;
    sb.p += a2b * s.gamma / s.rho;
    sb.rho -= a2b * a2 / s.rho;
    sb.rho -= b2rb * b2r / s.rho;
    sb.bx += b2rb * 2.0 * s.bx / s.rho;
    sb.by += b2rb * 2.0 * s.by / s.rho;
    sb.bz += b2rb * 2.0 * s.bz / s.rho;
    sb.bx += bx2rb * 2.0 * s.bx / s.rho;
    sb.rho -= bx2rb * bx2r / s.rho;
}

/* fx_hlld_state_f, all nine components */
FX_HD void fxa_flux_vjp(const FxHlldState &s, const double *Fb, FxaS &sb)
{
    const double rho = s.rho, vx = s.vx, vy = s.vy, vz = s.vz;
    const double bx = s.bx, by = s.by, bz = s.bz;
    const double pt = s.p + 0.5 * (bx * bx + by * by + bz * bz);
    const double vdotb = vx * bx + vy * by + vz * bz;
    sb.rho += Fb[0] * vx + Fb[1] * vx * vx + Fb[2] * vx * vy + Fb[3] * vx * vz + Fb[5] * s.ye * vx;
    sb.vx += Fb[0] * rho + Fb[1] * 2.0 * rho * vx + Fb[2] * rho * vy + Fb[3] * rho * vz +
        Fb[4] * ((s.e + pt) - bx * bx) + Fb[5] * rho * s.ye + Fb[7] * by + Fb[8] * bz;
    sb.vy += Fb[2] * rho * vx - Fb[4] * bx * by - Fb[7] * bx;
    sb.vz += Fb[3] * rho * vx - Fb[4] * bx * bz - Fb[8] * bx;
    sb.e += Fb[4] * vx;
    const double ptb = Fb[1] + Fb[4] * vx;
    sb.p += ptb;
    sb.bx += -2.0 * bx * Fb[1] - by * Fb[2] - bz * Fb[3] + Fb[4] * (-vdotb - bx * vx) - Fb[7] * vy -
        Fb[8] * vz + ptb * bx;
    sb.by += -bx * Fb[2] - Fb[4] * bx * vy + Fb[7] * vx + ptb * by;
    sb.bz += -bx * Fb[3] - Fb[4] * bx * vz + Fb[8] * vx + ptb * bz;
    sb.ye += Fb[5] * rho * vx;
}

/* one component of fx_hlld_state_f: sb += w * d f_v / d s */
FX_HD void fxa_flux_vjp_comp(const FxHlldState &s, int v, double w, FxaS &sb)
{
    double Fb[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    Fb[v] = w;
    fxa_flux_vjp(s, Fb, sb);
}

/* fx_hlld_state_u: sb += (du/ds)^T (scale * Fb) */
FX_HD void fxa_u_vjp(const FxHlldState &s, const double *Fb, double scale, FxaS &sb)
{
    sb.rho += scale * (Fb[0] + Fb[1] * s.vx + Fb[2] * s.vy + Fb[3] * s.vz + Fb[5] * s.ye);
    sb.vx += scale * Fb[1] * s.rho;
    sb.vy += scale * Fb[2] * s.rho;
    sb.vz += scale * Fb[3] * s.rho;
    sb.e += scale * Fb[4];
    sb.ye += scale * Fb[5] * s.rho;
    sb.bx += scale * Fb[6];
    sb.by += scale * Fb[7];
    sb.bz += scale * Fb[8];
}

/* one component of fx_hlld_state_u: sb += w * d u_v / d s */
FX_HD void fxa_u_vjp_comp(const FxHlldState &s, int v, double w, FxaS &sb)
{
    switch (v) {
    case 0: sb.rho += w; break;
    case 1: sb.rho += w * s.vx; sb.vx += w * s.rho; break;
    case 2: sb.rho += w * s.vy; sb.vy += w * s.rho; break;
    case 3: sb.rho += w * s.vz; sb.vz += w * s.rho; break;
    case 4: sb.e += w; break;
    case 5: sb.rho += w * s.ye; sb.ye += w * s.rho; break;
    case 6: sb.bx += w; break;
    case 7: sb.by += w; break;
    default: sb.bz += w; break;
    }
}

/* fx_hlld_u of a star state: sb += (du/ds)^T (scale * Fb) */
FX_HD void fxa_ustar_vjp(const FxHlldStar &s, const double *Fb, double scale, FxaSt &sb)
{
    sb.rho += scale * (Fb[0] + Fb[1] * s.vx + Fb[2] * s.vy + Fb[3] * s.vz + Fb[5] * s.ye);
    sb.vx += scale * Fb[1] * s.rho;
    sb.vy += scale * Fb[2] * s.rho;
    sb.vz += scale * Fb[3] * s.rho;
    sb.e += scale * Fb[4];
    sb.ye += scale * Fb[5] * s.rho;
    sb.bx += scale * Fb[6];
    sb.by += scale * Fb[7];
    sb.bz += scale * Fb[8];
}

/* sum_v Fb[v] u_v for a state and a star state */
FX_HD double fxa_u_dot(const FxHlldState &s, const double *Fb)
{
    return Fb[0] * s.rho + Fb[1] * s.rho * s.vx + Fb[2] * s.rho * s.vy + Fb[3] * s.rho * s.vz + Fb[4] * s.e +
        Fb[5] * s.rho * s.ye + Fb[6] * s.bx + Fb[7] * s.by + Fb[8] * s.bz;
}

FX_HD double fxa_ustar_dot(const FxHlldStar &s, const double *Fb)
{
    return Fb[0] * s.rho + Fb[1] * s.rho * s.vx + Fb[2] * s.rho * s.vy + Fb[3] * s.rho * s.vz + Fb[4] * s.e +
        Fb[5] * s.rho * s.ye + Fb[6] * s.bx + Fb[7] * s.by + Fb[8] * s.bz;
}

/* fx_face_outputs: v = (vx, vy, vz), bv1 = bz vx - bx vz, bv2 = bx vy - by vx.
 * ob = (v[3], bv1, bv2) adjoints; writes the adjoints of the six inputs. */
FX_HD void fxa_outputs_vjp(double vx, double vy, double vz, double bx, double by, double bz,
    const double *ob, double *xb)
{
    const double bv1b = ob[3];
    const double bv2b = ob[4];
    xb[0] = ob[0] + bv1b * bz - bv2b * by;
    xb[1] = ob[1] + bv2b * bx;
    xb[2] = ob[2] - bv1b * bx;
    xb[3] = -bv1b * vz + bv2b * vy;
    xb[4] = -bv2b * vx;
    xb[5] = bv1b * vx;
}

/* fx_hlld_outer_star: (s, S, SM, pt_star) -> st */
FX_HD void fxa_outer_star_vjp(const FxHlldState &s, double S, double SM, double pts, const FxaSt &stb,
    FxaS &sb, double &Sb, double &SMb, double &ptsb)
{
    const double alpha = S - s.vx;
    const double sd = S - SM;
    const double rhos = s.rho * alpha / sd;
    const double den = s.rho * alpha * sd - s.bx * s.bx;
    const bool copied = fabs(den) < FX_HLLD_SMALL * pts;
    double q = 0.0, mf = 0.0, vys, vzs, bys, bzs;
    if (copied) {
        vys = s.vy;
        vzs = s.vz;
        bys = s.by;
        bzs = s.bz;
    } else {
        q = (SM - s.vx) / den;
        mf = (s.rho * alpha * alpha - s.bx * s.bx) / den;
        vys = s.vy - s.bx * s.by * q;
        vzs = s.vz - s.bx * s.bz * q;
        bys = s.by * mf;
        bzs = s.bz * mf;
    }
    const double vdotb = s.vx * s.bx + s.vy * s.by + s.vz * s.bz;
    const double vsb = SM * s.bx + vys * bys + vzs * bzs;
    const double num = alpha * s.e - s.pt * s.vx + pts * SM + s.bx * (vdotb - vsb);
    const double es = num / sd;

    const double numb = stb.e / sd;
    double sdb = -stb.e * es / sd;
    double alphab = numb * s.e;
    sb.e += numb * alpha;
    sb.pt -= numb * s.vx;
    sb.vx -= numb * s.pt;
    ptsb += numb * SM;
    SMb += numb * pts;
    sb.bx += numb * (vdotb - vsb);
    const double vdotbb = numb * s.bx;
    const double vsbb = -numb * s.bx;
    SMb += vsbb * s.bx;
    sb.bx += vsbb * SM;
    const double vysb = stb.vy + vsbb * bys;
    const double bysb = stb.by + vsbb * vys;
    const double vzsb = stb.vz + vsbb * bzs;
    const double bzsb = stb.bz + vsbb * vzs;
    sb.vx += vdotbb * s.bx;
    sb.bx += vdotbb * s.vx;
    sb.vy += vdotbb * s.by;
    sb.by += vdotbb * s.vy;
    sb.vz += vdotbb * s.bz;
    sb.bz += vdotbb * s.vz;
    if (copied) {
        sb.vy += vysb;
        sb.vz += vzsb;
        sb.by += bysb;
        sb.bz += bzsb;
    } else {
        sb.vy += vysb;
        sb.bx -= vysb * s.by * q;
        sb.by -= vysb * s.bx * q;
        double qb = -vysb * s.bx * s.by;
        sb.vz += vzsb;
        sb.bx -= vzsb * s.bz * q;
        sb.bz -= vzsb * s.bx * q;
        qb -= vzsb * s.bx * s.bz;
        sb.by += bysb * mf;
        double mfb = bysb * s.by;
        sb.bz += bzsb * mf;
        mfb += bzsb * s.bz;
        SMb += qb / den;
        sb.vx -= qb / den;
        double denb = -qb * q / den;
        sb.rho += mfb * alpha * alpha / den;
        alphab += mfb * 2.0 * s.rho * alpha / den;
        sb.bx -= mfb * 2.0 * s.bx / den;
        denb -= mfb * mf / den;
        sb.rho += denb * alpha * sd;
        alphab += denb * s.rho * sd;
        sdb += denb * s.rho * alpha;
        sb.bx -= denb * 2.0 * s.bx;
    }
    SMb += stb.vx;
    sb.bx += stb.bx;
    sb.ye += stb.ye;
    sb.rho += stb.rho * alpha / sd;
    alphab += stb.rho * s.rho / sd;
    sdb -= stb.rho * rhos / sd;
    Sb += alphab;
    sb.vx -= alphab;
    Sb += sdb;
    SMb -= sdb;
}

FX_HD void fxa_add(FxaS &a, const FxaS &b)
{
    a.rho += b.rho; a.vx += b.vx; a.vy += b.vy; a.vz += b.vz; a.bx += b.bx; a.by += b.by;
    a.bz += b.bz; a.p += b.p; a.ye += b.ye; a.e += b.e; a.pt += b.pt;
}

/* Reverse mode of fx_riemann_hlld_folded.  ob[14] = adjoints of F[9], v[3],
 * bv1, bv2; accumulates WLb[9], WRb[9] (index 6 untouched: the normal field
 * enters through bn), pLb, pRb, bnb.  gamma is the same on both sides. */
FX_HD void fxa_hlld_vjp(const double *WL, const double *WR, double pL, double pR, double g, double bn,
    const double *ob, double *WLb, double *WRb, double &pLb, double &pRb, double &bnb)
{
    FxHlldState L, R;
    fx_hlld_state(WL, pL, g, bn, L, nullptr, 0, 0);
    fx_hlld_state(WR, pR, g, bn, R, nullptr, 0, 0);
    const double cfL = fx_hlld_fast_speed(L, nullptr, 0, 0);
    const double cfR = fx_hlld_fast_speed(R, nullptr, 0, 0);
    const double aL = L.vx - cfL, aR = R.vx - cfR;
    const double bL = L.vx + cfL, bR = R.vx + cfR;
    const double SL = fx_min(aL, aR);
    const double SR = fx_max(bL, bR);
    FxaS Lb, Rb;
    fxa_clear(Lb);
    fxa_clear(Rb);
    double SLb = 0.0, SRb = 0.0;
    const double *Fb = ob;
    const double *outb = ob + 9; /* v[3], bv1, bv2 */
    double xb[6];

    if (0.0 <= SL || SR <= 0.0) {
        const bool isL = 0.0 <= SL;
        const FxHlldState &X = isL ? L : R;
        FxaS &Xb = isL ? Lb : Rb;
        fxa_flux_vjp(X, Fb, Xb);
        fxa_outputs_vjp(X.vx, X.vy, X.vz, X.bx, X.by, X.bz, outb, xb);
        Xb.vx += xb[0]; Xb.vy += xb[1]; Xb.vz += xb[2]; Xb.bx += xb[3]; Xb.by += xb[4]; Xb.bz += xb[5];
    } else {
        const double denom = R.rho * (SR - R.vx) - L.rho * (SL - L.vx);
        const double smnum = R.rho * R.vx * (SR - R.vx) - L.rho * L.vx * (SL - L.vx) + (L.pt - R.pt);
        const double SM = smnum / denom;
        const double ptl = L.pt + L.rho * (SL - L.vx) * (SM - L.vx);
        const double ptr = R.pt + R.rho * (SR - R.vx) * (SM - R.vx);
        const double pts = 0.5 * (ptl + ptr);
        double SMb = 0.0, ptsb = 0.0;
        if (pts <= 0.0 || !isfinite(pts)) {
            /* HLL fallback: Uh_v = (SR ru - SL lu + lf - rf) / (SR - SL),
             * F_v = (SR lf - SL rf + SL SR (ru - lu)) / (SR - SL) */
            const double inv = 1.0 / (SR - SL);
            double Uh[9];
            for (int v = 0; v < 9; ++v) {
                Uh[v] = (SR * fx_hlld_state_u(R, v) - SL * fx_hlld_state_u(L, v) + fx_hlld_state_f(L, v) -
                    fx_hlld_state_f(R, v)) * inv;
            }
            const double rho = Uh[0];
            const double vx = Uh[1] / rho, vy = Uh[2] / rho, vz = Uh[3] / rho;
            fxa_outputs_vjp(vx, vy, vz, Uh[6], Uh[7], Uh[8], outb, xb);
            double Uhb[9];
            for (int v = 0; v < 9; ++v) Uhb[v] = 0.0;
            Uhb[1] += xb[0] / rho;
            Uhb[2] += xb[1] / rho;
            Uhb[3] += xb[2] / rho;
            Uhb[0] -= (xb[0] * vx + xb[1] * vy + xb[2] * vz) / rho;
            Uhb[6] += xb[3];
            Uhb[7] += xb[4];
            Uhb[8] += xb[5];
            double invb = 0.0;
            for (int v = 0; v < 9; ++v) {
                const double lf = fx_hlld_state_f(L, v), rf = fx_hlld_state_f(R, v);
                const double lu = fx_hlld_state_u(L, v), ru = fx_hlld_state_u(R, v);
                const double fb = Fb[v];
                const double du = ru - lu;
                SRb += fb * (lf + SL * du) * inv + Uhb[v] * ru * inv;
                SLb += fb * (-rf + SR * du) * inv - Uhb[v] * lu * inv;
                invb += fb * (SR * lf - SL * rf + SL * SR * du) + Uhb[v] * (SR * ru - SL * lu + lf - rf);
                fxa_flux_vjp_comp(L, v, fb * SR * inv + Uhb[v] * inv, Lb);
                fxa_flux_vjp_comp(R, v, -fb * SL * inv - Uhb[v] * inv, Rb);
                fxa_u_vjp_comp(R, v, fb * SL * SR * inv + Uhb[v] * SR * inv, Rb);
                fxa_u_vjp_comp(L, v, -fb * SL * SR * inv - Uhb[v] * SL * inv, Lb);
            }
            SRb -= invb * inv * inv;
            SLb += invb * inv * inv;
        } else {
            const bool bn_small = (0.5 * bn * bn < FX_HLLD_SMALL * pts);
            const bool left = (0.0 <= SM);
            const FxHlldState &N = left ? L : R;
            FxaS &Nb = left ? Lb : Rb;
            const double SN = left ? SL : SR;
            double SNb = 0.0;
            FxHlldStar Ns;
            fx_hlld_outer_star(N, SN, SM, pts, Ns, nullptr, 0, 0);
            const double sqn_ns = sqrt(Ns.rho);
            const double a = fabs(bn) / sqn_ns;
            const double SNs = left ? SM - a : SM + a;
            const bool single = (left ? (0.0 <= SNs) : (SNs <= 0.0)) || bn_small;
            FxaSt Nsb;
            fxa_clear(Nsb);
            const double dN = fxa_u_dot(N, Fb);
            const double dNs = fxa_ustar_dot(Ns, Fb);
            if (single) {
                /* F = f(N) + SN (u(Ns) - u(N)) */
                SNb += dNs - dN;
                fxa_outputs_vjp(Ns.vx, Ns.vy, Ns.vz, Ns.bx, Ns.by, Ns.bz, outb, xb);
                Nsb.vx += xb[0]; Nsb.vy += xb[1]; Nsb.vz += xb[2]; Nsb.bx += xb[3]; Nsb.by += xb[4]; Nsb.bz += xb[5];
                fxa_ustar_vjp(Ns, Fb, SN, Nsb);
            } else {
                const FxHlldState &Fr = left ? R : L;
                FxaS &Frb = left ? Rb : Lb;
                const double SF = left ? SR : SL;
                double SFb = 0.0;
                FxHlldStar Fs;
                fx_hlld_outer_star(Fr, SF, SM, pts, Fs, nullptr, 0, 0);
                const FxHlldStar &Ls = left ? Ns : Fs;
                const FxHlldStar &Rs = left ? Fs : Ns;
                const double sql = sqrt(Ls.rho);
                const double sqr = sqrt(Rs.rho);
                const double inv = 1.0 / (sql + sqr);
                const double sgn = bn < 0.0 ? -1.0 : 1.0;
                FxHlldStar ss = Ns;
                const double Avy = sql * Ls.vy + sqr * Rs.vy + (Rs.by - Ls.by) * sgn;
                const double Avz = sql * Ls.vz + sqr * Rs.vz + (Rs.bz - Ls.bz) * sgn;
                const double Aby = sql * Rs.by + sqr * Ls.by + sql * sqr * (Rs.vy - Ls.vy) * sgn;
                const double Abz = sql * Rs.bz + sqr * Ls.bz + sql * sqr * (Rs.vz - Ls.vz) * sgn;
                ss.vy = Avy * inv;
                ss.vz = Avz * inv;
                ss.by = Aby * inv;
                ss.bz = Abz * inv;
                const double vbss = Ns.vx * bn + ss.vy * ss.by + ss.vz * ss.bz;
                const double vbn = Ns.vx * bn + Ns.vy * Ns.by + Ns.vz * Ns.bz;
                const double sqn = left ? sql : sqr;
                const double t = sqn * sgn * (vbn - vbss);
                ss.e = left ? Ns.e - t : Ns.e + t;
                /* F = f(N) + SN (u(Ns) - u(N)) + SNs (u(ss) - u(Ns)) */
                const double dss = fxa_ustar_dot(ss, Fb);
                SNb += dNs - dN;
                const double SNsb = dss - dNs;
                FxaSt ssb;
                fxa_clear(ssb);
                fxa_outputs_vjp(ss.vx, ss.vy, ss.vz, ss.bx, ss.by, ss.bz, outb, xb);
                ssb.vx += xb[0]; ssb.vy += xb[1]; ssb.vz += xb[2]; ssb.bx += xb[3]; ssb.by += xb[4]; ssb.bz += xb[5];
                fxa_ustar_vjp(ss, Fb, SNs, ssb);
                fxa_ustar_vjp(Ns, Fb, SN - SNs, Nsb);
                /* SNs = SM -/+ a, a = |bn| / sqrt(Ns.rho) */
                SMb += SNsb;
                const double ab = left ? -SNsb : SNsb;
                if (bn != 0.0) {
                    bnb += ab * sgn / sqn_ns;
                }
                Nsb.rho -= ab * 0.5 * a / Ns.rho;
                /* ss.e = Ns.e -/+ t */
                Nsb.e += ssb.e;
                const double tb = left ? -ssb.e : ssb.e;
                double sqnb = tb * sgn * (vbn - vbss);
                const double vbnb = tb * sqn * sgn;
                const double vbssb = -tb * sqn * sgn;
                Nsb.vx += vbnb * bn;
                bnb += vbnb * Ns.vx;
                Nsb.vy += vbnb * Ns.by;
                Nsb.by += vbnb * Ns.vy;
                Nsb.vz += vbnb * Ns.bz;
                Nsb.bz += vbnb * Ns.vz;
                Nsb.vx += vbssb * bn;
                bnb += vbssb * Ns.vx;
                ssb.vy += vbssb * ss.by;
                ssb.by += vbssb * ss.vy;
                ssb.vz += vbssb * ss.bz;
                ssb.bz += vbssb * ss.vz;
                /* ss copies rho, vx, bx, ye (and e before the update) from Ns */
                Nsb.rho += ssb.rho;
                Nsb.vx += ssb.vx;
                Nsb.bx += ssb.bx;
                Nsb.ye += ssb.ye;
                /* transverse double-star components */
                FxaSt Lsb, Rsb;
                fxa_clear(Lsb);
                fxa_clear(Rsb);
                double sqlb = 0.0, sqrb = 0.0, invb = 0.0;
                const double Avyb = ssb.vy * inv;
                invb += ssb.vy * Avy;
                sqlb += Avyb * Ls.vy;
                Lsb.vy += Avyb * sql;
                sqrb += Avyb * Rs.vy;
                Rsb.vy += Avyb * sqr;
                Rsb.by += Avyb * sgn;
                Lsb.by -= Avyb * sgn;
                const double Avzb = ssb.vz * inv;
                invb += ssb.vz * Avz;
                sqlb += Avzb * Ls.vz;
                Lsb.vz += Avzb * sql;
                sqrb += Avzb * Rs.vz;
                Rsb.vz += Avzb * sqr;
                Rsb.bz += Avzb * sgn;
                Lsb.bz -= Avzb * sgn;
                const double Abyb = ssb.by * inv;
                invb += ssb.by * Aby;
                sqlb += Abyb * (Rs.by + sqr * (Rs.vy - Ls.vy) * sgn);
                Rsb.by += Abyb * sql;
                sqrb += Abyb * (Ls.by + sql * (Rs.vy - Ls.vy) * sgn);
                Lsb.by += Abyb * sqr;
                Rsb.vy += Abyb * sql * sqr * sgn;
                Lsb.vy -= Abyb * sql * sqr * sgn;
                const double Abzb = ssb.bz * inv;
                invb += ssb.bz * Abz;
                sqlb += Abzb * (Rs.bz + sqr * (Rs.vz - Ls.vz) * sgn);
                Rsb.bz += Abzb * sql;
                sqrb += Abzb * (Ls.bz + sql * (Rs.vz - Ls.vz) * sgn);
                Lsb.bz += Abzb * sqr;
                Rsb.vz += Abzb * sql * sqr * sgn;
                Lsb.vz -= Abzb * sql * sqr * sgn;
                sqlb -= invb * inv * inv;
                sqrb -= invb * inv * inv;
                if (left) {
                    sqlb += sqnb;
                } else {
                    sqrb += sqnb;
                }
                Lsb.rho += sqlb * 0.5 / sql;
                Rsb.rho += sqrb * 0.5 / sqr;
                FxaSt &nsb_part = left ? Lsb : Rsb;
                FxaSt &fsb = left ? Rsb : Lsb;
                Nsb.rho += nsb_part.rho; Nsb.vx += nsb_part.vx; Nsb.vy += nsb_part.vy; Nsb.vz += nsb_part.vz;
                Nsb.bx += nsb_part.bx; Nsb.by += nsb_part.by; Nsb.bz += nsb_part.bz; Nsb.ye += nsb_part.ye;
                Nsb.e += nsb_part.e;
                fxa_outer_star_vjp(Fr, SF, SM, pts, fsb, Frb, SFb, SMb, ptsb);
                if (left) {
                    SRb += SFb;
                } else {
                    SLb += SFb;
                }
            }
            fxa_flux_vjp(N, Fb, Nb);
            fxa_u_vjp(N, Fb, -SN, Nb);
            fxa_outer_star_vjp(N, SN, SM, pts, Nsb, Nb, SNb, SMb, ptsb);
            if (left) {
                SLb += SNb;
            } else {
                SRb += SNb;
            }
            (void)bn_small;
        }
        /* pts = 0.5 (ptl + ptr) */
        const double ptlb = 0.5 * ptsb;
        const double ptrb = 0.5 * ptsb;
        Lb.pt += ptlb;
        Lb.rho += ptlb * (SL - L.vx) * (SM - L.vx);
        SLb += ptlb * L.rho * (SM - L.vx);
        SMb += ptlb * L.rho * (SL - L.vx);
        Lb.vx -= ptlb * L.rho * ((SM - L.vx) + (SL - L.vx));
        Rb.pt += ptrb;
        Rb.rho += ptrb * (SR - R.vx) * (SM - R.vx);
        SRb += ptrb * R.rho * (SM - R.vx);
        SMb += ptrb * R.rho * (SR - R.vx);
        Rb.vx -= ptrb * R.rho * ((SM - R.vx) + (SR - R.vx));
        /* SM = smnum / denom */
        const double smnb = SMb / denom;
        const double denb = -SMb * SM / denom;
        Rb.rho += smnb * R.vx * (SR - R.vx);
        Rb.vx += smnb * R.rho * (SR - 2.0 * R.vx);
        SRb += smnb * R.rho * R.vx;
        Lb.rho -= smnb * L.vx * (SL - L.vx);
        Lb.vx -= smnb * L.rho * (SL - 2.0 * L.vx);
        SLb -= smnb * L.rho * L.vx;
        Lb.pt += smnb;
        Rb.pt -= smnb;
        Rb.rho += denb * (SR - R.vx);
        SRb += denb * R.rho;
        Rb.vx -= denb * R.rho;
        Lb.rho -= denb * (SL - L.vx);
        SLb -= denb * L.rho;
        Lb.vx += denb * L.rho;
    }
    /* SL = min(L.vx - cfL, R.vx - cfR), SR = max(L.vx + cfL, R.vx + cfR) */
    double cfLb = 0.0, cfRb = 0.0;
    if (aL < aR) {
        Lb.vx += SLb;
        cfLb -= SLb;
    } else {
        Rb.vx += SLb;
        cfRb -= SLb;
    }
    if (bL > bR) {
        Lb.vx += SRb;
        cfLb += SRb;
    } else {
        Rb.vx += SRb;
        cfRb += SRb;
    }
    fxa_fast_speed_vjp(L, cfLb, Lb);
    fxa_fast_speed_vjp(R, cfRb, Rb);
    fxa_state_vjp(WL, Lb, WLb, pLb, bnb, bn);
    fxa_state_vjp(WR, Rb, WRb, pRb, bnb, bn);
}

/* ------------------------------------------------------------------------ */
/* One face: MC reconstruction of the 4-cell stencil + HLLD                  */
/* ------------------------------------------------------------------------ */

#ifdef __CUDACC__
#define FXA_MEMBER __host__ __device__ __forceinline__
#else
#define FXA_MEMBER inline
#endif

/* The stencil of one face: cells n = 0..3 (L-1, L, R, R+1) along the sweep,
 * local-frame primitives lv = 0 rho, 1-3 velocity (normal first), 4 eint,
 * 5 ye, 7-8 transverse field (6 unused).  LD(n, lv) loads a value,
 * ACC(n, lv, x) accumulates an adjoint; the kernel reads and atomically
 * updates the block arrays, the host check uses plain arrays.  Pressures
 * are the cells' (g-1) rho eint, reconstructed like the other variables
 * (the k_flux evaluation). */
template <class LD>
FX_HD void fxa_face_states_t(const LD &ld, double g, double bn, double *WL, double *WR, double &pL, double &pR)
{
    const int lvs[8] = {0, 1, 2, 3, 4, 5, 7, 8};
#pragma unroll
    for (int q = 0; q < 8; ++q) {
        const int lv = lvs[q];
        const double a = ld(0, lv), b = ld(1, lv), c = ld(2, lv), d = ld(3, lv);
        WL[lv] = b + 0.5 * fx_mc_slope(a, b, c);
        WR[lv] = c - 0.5 * fx_mc_slope(b, c, d);
    }
    WL[FX_B1] = bn;
    WR[FX_B1] = bn;
    double p4[4];
#pragma unroll
    for (int n = 0; n < 4; ++n) {
        p4[n] = fx_pressure(g, ld(n, FX_RHO), ld(n, FX_EINT));
    }
    pL = p4[1] + 0.5 * fx_mc_slope(p4[0], p4[1], p4[2]);
    pR = p4[2] - 0.5 * fx_mc_slope(p4[1], p4[2], p4[3]);
}

/* ob[14]: adjoints of F[9], v[3], bv1, bv2; accumulates the stencil
 * adjoints through acc and the face-normal field's into bnb */
template <class LD, class ACC>
FX_HD void fxa_face_vjp_t(const LD &ld, const ACC &acc, double g, double bn, const double *ob, double &bnb)
{
    double WL[9], WR[9], pL, pR;
    fxa_face_states_t(ld, g, bn, WL, WR, pL, pR);
    double WLb[9], WRb[9];
    for (int v = 0; v < 9; ++v) {
        WLb[v] = 0.0;
        WRb[v] = 0.0;
    }
    double pLb = 0.0, pRb = 0.0;
    fxa_hlld_vjp(WL, WR, pL, pR, g, bn, ob, WLb, WRb, pLb, pRb, bnb);
    const int lvs[8] = {0, 1, 2, 3, 4, 5, 7, 8};
#pragma unroll
    for (int q = 0; q < 8; ++q) {
        const int lv = lvs[q];
        const double a = ld(0, lv), b = ld(1, lv), c = ld(2, lv), d = ld(3, lv);
        /* WL = b + 0.5 mc(a, b, c); WR = c - 0.5 mc(b, c, d) */
        double ab = 0.0, bb = WLb[lv], cb = WRb[lv], db = 0.0;
        fxa_mc_vjp(a, b, c, 0.5 * WLb[lv], ab, bb, cb);
        fxa_mc_vjp(b, c, d, -0.5 * WRb[lv], bb, cb, db);
        acc(0, lv, ab);
        acc(1, lv, bb);
        acc(2, lv, cb);
        acc(3, lv, db);
    }
    double rho4[4], e4[4], p4[4], p4b[4] = {0.0, 0.0, 0.0, 0.0};
    for (int n = 0; n < 4; ++n) {
        rho4[n] = ld(n, FX_RHO);
        e4[n] = ld(n, FX_EINT);
        p4[n] = fx_pressure(g, rho4[n], e4[n]);
    }
    p4b[1] += pLb;
    fxa_mc_vjp(p4[0], p4[1], p4[2], 0.5 * pLb, p4b[0], p4b[1], p4b[2]);
    p4b[2] += pRb;
    fxa_mc_vjp(p4[1], p4[2], p4[3], -0.5 * pRb, p4b[1], p4b[2], p4b[3]);
    for (int n = 0; n < 4; ++n) {
        acc(n, FX_RHO, p4b[n] * (g - 1.0) * e4[n]);
        acc(n, FX_EINT, p4b[n] * (g - 1.0) * rho4[n]);
    }
}

struct FxaArrayLoad {
    const double *w;
    FXA_MEMBER double operator()(int n, int lv) const { return w[n * 9 + lv]; }
};

struct FxaArrayAcc {
    double *wb;
    FXA_MEMBER void operator()(int n, int lv, double x) const { wb[n * 9 + lv] += x; }
};

/* array forms (w4[n * 9 + lv]) used by the host checks */
FX_HD void fxa_face_eval(const double *w4, double g, double bn, FxFaceOut &o)
{
    double WL[9], WR[9], pL, pR;
    fxa_face_states_t(FxaArrayLoad{w4}, g, bn, WL, WR, pL, pR);
    fx_riemann_hlld_folded(WL, WR, pL, pR, g, g, bn, o, nullptr, 0, 0);
}

FX_HD void fxa_face_vjp(const double *w4, double g, double bn, const double *ob, double *w4b, double &bnb)
{
    fxa_face_vjp_t(FxaArrayLoad{w4}, FxaArrayAcc{w4b}, g, bn, ob, bnb);
}

/* ------------------------------------------------------------------------ */
/* Upwind edge EMF (fx_emf_upwind): d emf / d (f[4], c[4]) times eb          */
/* ------------------------------------------------------------------------ */
FX_HD void fxa_emf_upwind_vjp(const double *vn, double eb, double *fb, double *cb)
{
    fb[0] += 0.25 * eb;
    fb[1] += 0.25 * eb;
    fb[2] += 0.25 * eb;
    fb[3] += 0.25 * eb;
    /* (face index, cell index) pairs of the four upwind terms for vn > 0
     * and vn < 0 (an exact zero averages the two) */
    const int pf[4][2] = {{3, 1}, {2, 0}, {3, 1}, {2, 0}};
    const int pc[4][2] = {{3, 0}, {1, 0}, {2, 1}, {2, 3}};
    for (int n = 0; n < 4; ++n) {
        const double w_pos = vn[n] > 0.0 ? 0.25 : (vn[n] < 0.0 ? 0.0 : 0.125);
        const double w_neg = vn[n] < 0.0 ? 0.25 : (vn[n] > 0.0 ? 0.0 : 0.125);
        fb[pf[n][0]] += w_pos * eb;
        cb[pc[n][0]] -= w_pos * eb;
        fb[pf[n][1]] += w_neg * eb;
        cb[pc[n][1]] -= w_neg * eb;
    }
}

/* ------------------------------------------------------------------------ */
/* prim <-> cons (MHD, 9 variables)                                          */
/* ------------------------------------------------------------------------ */

/* u = prim2cons(w): accumulates wb += (du/dw)^T ub.  The field components
 * of u are copies of w's; pass ub[6..8] = 0 where the caller replaces them. */
FX_HD void fxa_prim2cons_vjp(const double *w, const double *ub, double *wb)
{
    const double rho = w[FX_RHO], v1 = w[FX_V1], v2 = w[FX_V2], v3 = w[FX_V3];
    const double eint = w[FX_EINT];
    const double v2sum = v1 * v1 + v2 * v2 + v3 * v3;
    wb[FX_RHO] += ub[FX_RHO] + ub[FX_V1] * v1 + ub[FX_V2] * v2 + ub[FX_V3] * v3 +
        ub[FX_ETOT] * (eint + 0.5 * v2sum) + ub[FX_YE] * w[FX_YE];
    wb[FX_V1] += ub[FX_V1] * rho + ub[FX_ETOT] * rho * v1;
    wb[FX_V2] += ub[FX_V2] * rho + ub[FX_ETOT] * rho * v2;
    wb[FX_V3] += ub[FX_V3] * rho + ub[FX_ETOT] * rho * v3;
    wb[FX_EINT] += ub[FX_ETOT] * rho;
    wb[FX_YE] += ub[FX_YE] * rho;
    wb[FX_B1] += ub[FX_ETOT] * w[FX_B1] + ub[FX_B1];
    wb[FX_B2] += ub[FX_ETOT] * w[FX_B2] + ub[FX_B2];
    wb[FX_B3] += ub[FX_ETOT] * w[FX_B3] + ub[FX_B3];
}

/* w = cons2prim(u): writes ub = (dw/du)^T wb (rho > 0) */
FX_HD void fxa_cons2prim_vjp(const double *u, const double *wb, double *ub)
{
    const double rho = u[FX_RHO];
    const double v1 = u[FX_V1] / rho, v2 = u[FX_V2] / rho, v3 = u[FX_V3] / rho;
    const double b1 = u[FX_B1], b2 = u[FX_B2], b3 = u[FX_B3];
    const double mag = 0.5 * (b1 * b1 + b2 * b2 + b3 * b3) / rho;
    const double eb = wb[FX_EINT];
    /* eint = E/rho - 0.5 |v|^2 - mag, v = m / rho */
    const double v1b = wb[FX_V1] - eb * v1;
    const double v2b = wb[FX_V2] - eb * v2;
    const double v3b = wb[FX_V3] - eb * v3;
    ub[FX_V1] = v1b / rho;
    ub[FX_V2] = v2b / rho;
    ub[FX_V3] = v3b / rho;
    ub[FX_ETOT] = eb / rho;
    ub[FX_YE] = wb[FX_YE] / rho;
    ub[FX_B1] = wb[FX_B1] - eb * b1 / rho;
    ub[FX_B2] = wb[FX_B2] - eb * b2 / rho;
    ub[FX_B3] = wb[FX_B3] - eb * b3 / rho;
    ub[FX_RHO] = wb[FX_RHO] - (v1b * v1 + v2b * v2 + v3b * v3) / rho +
        eb * (-u[FX_ETOT] / (rho * rho) + mag / rho) - wb[FX_YE] * u[FX_YE] / (rho * rho);
}

#endif
