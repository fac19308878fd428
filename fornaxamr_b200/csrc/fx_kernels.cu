/*
 * Per-phase kernels of the RK2 Godunov MHD update, one thread per face, edge
 * or cell.  Every kernel takes a block list: the plain (drop-in) form passes
 * one block per launch, as the reference's per-block loops do; the batched
 * form passes every block of the mesh in one launch.
 *
 * Phase                       reference
 * face fluxes (k_flux)        prj_flux_update, src/prj_flux.c:2149-2521
 * edge EMFs (k_emf)           prj_timeint_mhd_update_emf, src/prj_timeint.c:292-413
 * CT face update (k_bf_update) prj_timeint_mhd_update_bf, src/prj_timeint.c:415-495
 * cell update (k_cell_update) src/prj_timeint.c:1255-1349 and 1562-1654,
 *                             src terms src/prj_src.c:32-139, 717-768
 * eos fill (k_eos_fill)       prj_eos_fill_block/_active_cells, src/prj_eos.c:1087-1162
 * dt (k_calc_dt)              prj_timeint_calc_dt, src/prj_timeint.c:2144-2256
 * ghost programs              prj_boundary_fill_ghosts_and_bf, src/prj_boundary.c:1150-1241
 * bf2bc                       prj_mhd_bf2bc_impl, src/prj_mhd.c:555-603: ghost cells in
 *                             the ghost programs, active cells in k_cell_field_active
 */
#include <cuda_runtime.h>

#include <type_traits>

#include "../../include/fornax_b200.h"
#include "fx_kernels.h"
#include "fx_physics.cuh"

namespace {

constexpr int kPlane = FX_NSTAGES * FX_NCELLS; /* stride between variables of W */

__device__ __forceinline__ int fx_axis_stride(int dir)
{
    return dir == 0 ? FX_PBS * FX_PBS : dir == 1 ? FX_PBS : 1;
}

/* local (sweep-rotated) variable -> global variable, prj_flux_build_var_map
 * (src/prj_flux.c:274-349): the sweep-normal velocity and field go to slot 1
 * and 6 of the local vector. */
__device__ __forceinline__ int fx_gmap(int dir, int lv)
{
    if (lv >= 1 && lv <= 3) {
        return 1 + (dir + lv - 1) % 3;
    }
    if (lv >= 6) {
        return 6 + (dir + lv - 6) % 3;
    }
    return lv;
}

__device__ __forceinline__ unsigned long long fx_double_key(double d)
{
    unsigned long long bits = (unsigned long long)__double_as_longlong(d);
    return (bits >> 63) ? ~bits : (bits | 0x8000000000000000ULL);
}

/* ------------------------------------------------------------------------ */
/* Face fluxes                                                               */
/* ------------------------------------------------------------------------ */
/* FULL: store every component the reference stores (the drop-in form);
 * otherwise only what later phases read (hydro flux components, the normal
 * face velocity, Bv1/Bv2).  blockIdx.z is the sweep direction.  TPB/MINB
 * set the launch shape (threads per CTA, resident CTAs per SM the register
 * allocation must allow); the autotuner picks among the compiled shapes. */
/* left state of the face from cells (qm, q0, q1), right state from (q0,
 * q1, q2): MC slopes (the reference's fast path, prj_flux_recon_var_mc:
 * q +- 0.5 slope) or WENO-Z3 face values (its per-face path,
 * src/prj_flux.c:440-475) */
/* cells of a face's stencil along the sweep: 4 (cL - 1 .. cR + 1) for MC
 * and WENO-Z3, 8 (cL - 3 .. cR + 3) for WENO-Z7; q[n] is cell cL + n - NS/2 + 1 */
template <int RECON>
struct FxStencil {
    static constexpr int NS = RECON == FX_RECON_WENO7 ? 8 : 4;
};

template <int RECON>
__device__ __forceinline__ void fx_recon_pair(const double (&q)[FxStencil<RECON>::NS], double &wl, double &wr)
{
    if constexpr (RECON == FX_RECON_WENO7) {
        /* left state: cells cL-3 .. cL+3 at +1/2; right state: cells cR-3 ..
         * cR+3 at -1/2, i.e. the mirrored stencil cR+3 .. cR-3 at +1/2 */
        wl = fx_weno7_plus(q[0], q[1], q[2], q[3], q[4], q[5], q[6]);
        wr = fx_weno7_plus(q[7], q[6], q[5], q[4], q[3], q[2], q[1]);
    } else if constexpr (RECON == FX_RECON_WENO3) {
        wl = fx_weno3_face(q[0], q[1], q[2], 0.5);
        wr = fx_weno3_face(q[1], q[2], q[3], -0.5);
    } else {
        wl = q[1] + 0.5 * fx_mc_slope(q[0], q[1], q[2]);
        wr = q[2] - 0.5 * fx_mc_slope(q[1], q[2], q[3]);
    }
}

/* MC face values of a 4-cell stencil with the limiter's selections through
 * a branch policy: bits 4 q + 0 and 4 q + 2 of the face's word */
template <class BR>
__device__ __forceinline__ void fx_recon_pair_br(const double (&q)[4], double &wl, double &wr, BR &br, int q4)
{
    wl = q[1] + 0.5 * fx_mc_slope_br(q[0], q[1], q[2], br, q4);
    wr = q[2] - 0.5 * fx_mc_slope_br(q[1], q[2], q[3], br, q4 + 2);
}

/* a stencil value of the face kernel: through the read-only data path for
 * the 4-cell stencils (MC, WENO-Z3), a plain load for WENO-Z7's 8 cells */
template <int RECON>
__device__ __forceinline__ double fx_stencil_load(const double *p)
{
    if constexpr (RECON == FX_RECON_WENO7) {
        return *p;
    } else {
        return __ldg(p);
    }
}

/* BRM: 0 the solver as it stands; 1 record / 2 replay every face's
 * decisions in D.br_words (FxBrRecord / FxBrReplay; MHD, MC and the plain
 * form only), the branch-frozen map the adjoint checks use */
template <bool MHD, bool FULL, int TPB, int MINB, int RECON, int BRM = 0>
__global__ void __launch_bounds__(TPB, MINB) k_flux(FxDev D, const int *__restrict__ blist,
    int wslot, int bfslot)
{
    static_assert(BRM == 0 || (MHD && FULL && RECON == FX_RECON_MC), "decision record / replay: MHD, MC, plain");
    using Br = typename std::conditional<BRM == 1, FxBrRecord,
        typename std::conditional<BRM == 2, FxBrReplay, FxBrFree>::type>::type;
    Br br;
    if (D.ctl->skip) {
        return;
    }
    /* gamma is uniform for the ideal gas: its MC slope is exactly 0, so the
     * MC face values equal g bit for bit; the WENO weights of a constant
     * stencil are evaluated as the reference does (their sum need not be 1).
     * Those face values depend on g alone, so one thread of the CTA
     * evaluates them for all (before any thread leaves). */
    __shared__ double s_gface[2];
    if constexpr (RECON != FX_RECON_MC) {
        if (threadIdx.x == 0) {
            double gS[FxStencil<RECON>::NS];
#pragma unroll
            for (int n = 0; n < FxStencil<RECON>::NS; ++n) {
                gS[n] = D.gamma;
            }
            fx_recon_pair<RECON>(gS, s_gface[0], s_gface[1]);
        }
        __syncthreads();
    }
    /* grid (face chunk, direction, block): the three sweeps of a block are
     * scheduled back to back, so its stencil cells are re-read from L2 */
    const int dir = blockIdx.y;
    const int b = blist[blockIdx.z];
    /* MHD carries one transverse ghost layer of faces for the CT EMFs
     * (src/prj_flux.c:2241-2251); hydro transverse faces are [0, 15]. */
    constexpr int T = MHD ? FX_BS + 2 : FX_BS;
    constexpr int TLO = MHD ? -1 : 0;
    constexpr int NF = (FX_BS + 1) * T * T;
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= NF) {
        return;
    }
    /* this face's decision word (record / replay) */
    const size_t bri = D.br_off + ((size_t)b * 3 + dir) * NF + t;
    if constexpr (BRM == 2) {
        br.w = D.br_words[bri];
    }
    const int e2 = dir == 2 ? FX_BS + 1 : T;
    const int e1 = dir == 1 ? FX_BS + 1 : T;
    const int k = (dir == 2 ? 0 : TLO) + t % e2;
    t /= e2;
    const int j = (dir == 1 ? 0 : TLO) + t % e1;
    const int i = (dir == 0 ? 0 : TLO) + t / e1;
    const int s = fx_axis_stride(dir);
    const int cR = fx_lidx(i, j, k);
    const int cL = cR - s;
    const int nv = MHD ? 9 : 6;
    const double *Wb = D.W + (size_t)b * FX_W_COUNT(nv) + (size_t)wslot * FX_NCELLS;
    const double g = D.gamma;

    double WL[9];
    double WR[9];
    /* density and internal energy at the stencil cells also give the
     * reconstructed pressure (eosvar p = (g-1) rho e of each cell).  The
     * MC and WENO-Z3 stencils come through the read-only data path
     * (fx_stencil_load): this launch does not write W (on the 128^3 state
     * 0.628 -> 0.623 ms at 64 x 8, 0.699 -> 0.665 ms at 256 x 3; the normal
     * field that way, and the EMF, CT, fill and cell kernels, measured no
     * faster; WENO-Z7's 8-cell stencils 4.60 ms with plain loads against
     * 4.75 ms). */
    constexpr int NS = FxStencil<RECON>::NS;
    const int c0 = cL - (NS / 2 - 1) * s;   /* first stencil cell */
    double rhoS[NS], eintS[NS];
    {
        const double *qr = Wb + (size_t)FX_RHO * kPlane + c0;
        const double *qe = Wb + (size_t)FX_EINT * kPlane + c0;
#pragma unroll
        for (int n = 0; n < NS; ++n) {
            rhoS[n] = fx_stencil_load<RECON>(qr + n * s);
            eintS[n] = fx_stencil_load<RECON>(qe + n * s);
        }
    }
    if constexpr (BRM == 0) {
        fx_recon_pair<RECON>(rhoS, WL[FX_RHO], WR[FX_RHO]);
        fx_recon_pair<RECON>(eintS, WL[FX_EINT], WR[FX_EINT]);
    } else {
        fx_recon_pair_br(rhoS, WL[FX_RHO], WR[FX_RHO], br, 4 * FX_RHO);
        fx_recon_pair_br(eintS, WL[FX_EINT], WR[FX_EINT], br, 4 * FX_EINT);
    }
#pragma unroll
    for (int lv = 1; lv < nv; ++lv) {
        if (lv == FX_EINT || (MHD && lv == FX_B1)) {
            continue;
        }
        const double *q = Wb + (size_t)fx_gmap(dir, lv) * kPlane + c0;
        double qs[NS];
#pragma unroll
        for (int n = 0; n < NS; ++n) {
            qs[n] = fx_stencil_load<RECON>(q + n * s);
        }
        if constexpr (BRM == 0) {
            fx_recon_pair<RECON>(qs, WL[lv], WR[lv]);
        } else {
            fx_recon_pair_br(qs, WL[lv], WR[lv], br, 4 * lv);
        }
    }
    double pS[NS];
#pragma unroll
    for (int n = 0; n < NS; ++n) {
        pS[n] = fx_pressure(g, rhoS[n], eintS[n]);
    }
    double pL, pR;
    if constexpr (BRM == 0) {
        fx_recon_pair<RECON>(pS, pL, pR);
    } else {
        /* the pressure takes the normal field's (unreconstructed) bits */
        fx_recon_pair_br(pS, pL, pR, br, 4 * FX_B1);
    }
    double gL = g, gR = g;
    if constexpr (RECON != FX_RECON_MC) {
        gL = s_gface[0];
        gR = s_gface[1];
    }
    const size_t fbase = (size_t)b * FX_FLUX_COUNT(nv) + (size_t)dir * nv * FX_NCELLS;
    const size_t vbase = (size_t)b * FX_VR_COUNT + (size_t)dir * 3 * FX_NCELLS;
    if (MHD) {
        const double bn = D.Bf[(size_t)b * FX_BF_COUNT + ((size_t)dir * FX_NSTAGES + bfslot) * FX_NFACES +
            fx_face_idx(dir, i, j, k)];
        WL[FX_B1] = bn;
        WR[FX_B1] = bn;
        FxFaceOut o;
        if constexpr (BRM == 0) {
            FxErrLocal le;
            FxBrFree bf;
            fx_riemann_hlld_folded_br(WL, WR, pL, pR, gL, gR, bn, o, &le, b, cR, bf);
            if (le.code != 0) {
                fx_fail(D.err, le.code, le.block, le.index);
            }
        } else {
            fx_riemann_hlld_folded_br(WL, WR, pL, pR, gL, gR, bn, o, D.err, b, cR, br);
            if constexpr (BRM == 1) {
                D.br_words[bri] = br.w;
            } else if (br.flips) {
                atomicAdd(D.br_flips, (unsigned long long)br.flips);
            }
        }
#pragma unroll
        for (int lv = 0; lv < (FULL ? 9 : 6); ++lv) {
            D.flux[fbase + fx_bidx(9, fx_gmap(dir, lv), i, j, k)] = o.F[lv];
        }
#pragma unroll
        for (int m = 0; m < (FULL ? 3 : 1); ++m) {
            D.vr[vbase + fx_bidx(3, (dir + m) % 3, i, j, k)] = o.v[m];
        }
        const size_t bvi = (size_t)b * FX_BV_COUNT + (size_t)dir * FX_NCELLS + cR;
        D.bv1[bvi] = o.bv1;
        D.bv2[bvi] = o.bv2;
    } else {
        /* transverse velocity deltas of the theta limiter,
         * prj_flux_velocity_deltas (src/prj_flux.c:1967-2036) */
        const int da = (dir + 1) % 3;
        const int db = (dir + 2) % 3;
        const int sa = fx_axis_stride(da);
        const int sb = fx_axis_stride(db);
        const double *un = Wb + (size_t)(1 + dir) * kPlane;
        const double *ua = Wb + (size_t)(1 + da) * kPlane;
        const double *ub = Wb + (size_t)(1 + db) * kPlane;
        const double du = un[cR] - un[cL];
        const double dv = fx_min(fx_min(ua[cL] - ua[cL - sa], ua[cL + sa] - ua[cL]),
            fx_min(ua[cR] - ua[cR - sa], ua[cR + sa] - ua[cR]));
        const double dw = fx_min(fx_min(ub[cL] - ub[cL - sb], ub[cL + sb] - ub[cL]),
            fx_min(ub[cR] - ub[cR - sb], ub[cR + sb] - ub[cR]));
        double F[6];
        double v[3];
        fx_riemann_hllc(WL, WR, pL, pR, gL, gR, du, dv, dw, F, v);
#pragma unroll
        for (int lv = 0; lv < 6; ++lv) {
            D.flux[fbase + fx_bidx(6, fx_gmap(dir, lv), i, j, k)] = F[lv];
        }
#pragma unroll
        for (int m = 0; m < (FULL ? 3 : 1); ++m) {
            D.vr[vbase + fx_bidx(3, (dir + m) % 3, i, j, k)] = v[m];
        }
    }
}

/* ------------------------------------------------------------------------ */
/* Edge EMFs                                                                 */
/* ------------------------------------------------------------------------ */
/* The per-block launches of the plain form: one thread per edge, so a
 * single block still fills the device; the cell EMF components and eta of
 * an edge's four cells are evaluated per edge (same arithmetic). */
__device__ __forceinline__ double fx_cell_emf(const double *Wb, int dir, int c)
{
    const int a = (dir + 1) % 3;
    const int bb = (dir + 2) % 3;
    const double bA = Wb[(size_t)(FX_B1 + a) * kPlane + c];
    const double bB = Wb[(size_t)(FX_B1 + bb) * kPlane + c];
    const double vA = Wb[(size_t)(FX_V1 + a) * kPlane + c];
    const double vB = Wb[(size_t)(FX_V1 + bb) * kPlane + c];
    return bA * vB - bB * vA;
}

__global__ void __launch_bounds__(128) k_emf_edges(FxDev D, const int *__restrict__ blist, int wslot, int bfslot)
{
    if (D.ctl->skip) {
        return;
    }
    const int b = blist[blockIdx.y];
    constexpr int NE = FX_BS * (FX_BS + 1) * (FX_BS + 1);
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= 3 * NE) {
        return;
    }
    const int dir = t / NE;
    t -= dir * NE;
    const int te = t; /* edge index within the direction */
    const int x2 = dir == 2 ? FX_BS : FX_BS + 1;
    const int x1 = dir == 1 ? FX_BS : FX_BS + 1;
    int e[3];
    e[2] = t % x2;
    t /= x2;
    e[1] = t % x1;
    e[0] = t / x1;
    const int up = (dir + 1) % 3;
    const int right = (dir + 2) % 3;
    const int su = fx_axis_stride(up);
    const int sr = fx_axis_stride(right);
    const int c0 = fx_lidx(e[0], e[1], e[2]);   /* cell0 = e; face0 = face1 = e */
    const int c1 = c0 - su;                      /* cell1 = e - up */
    const int c2 = c0 - su - sr;                 /* cell2 = e - up - right */
    const int c3 = c0 - sr;                      /* cell3 = e - right */
    const double *Wb = D.W + (size_t)b * FX_W_COUNT(9) + (size_t)wslot * FX_NCELLS;
    const double *bv1r = D.bv1 + (size_t)b * FX_BV_COUNT + (size_t)right * FX_NCELLS;
    const double *bv2u = D.bv2 + (size_t)b * FX_BV_COUNT + (size_t)up * FX_NCELLS;
    const double *vrr = D.vr + (size_t)b * FX_VR_COUNT + (size_t)right * 3 * FX_NCELLS;
    const double *vru = D.vr + (size_t)b * FX_VR_COUNT + (size_t)up * 3 * FX_NCELLS;
    double f[4], c[4], vn[4];
    /* face0 = e (right-normal), face1 = e (up-normal), face2 = e - up
     * (right-normal), face3 = e - right (up-normal) */
    f[0] = bv1r[c0];
    f[1] = bv2u[c0];
    f[2] = bv1r[c1];
    f[3] = bv2u[c3];
    c[0] = fx_cell_emf(Wb, dir, c0);
    c[1] = fx_cell_emf(Wb, dir, c1);
    c[2] = fx_cell_emf(Wb, dir, c2);
    c[3] = fx_cell_emf(Wb, dir, c3);
    vn[0] = vrr[fx_bidx_cell(3, right, c0)];
    vn[1] = vru[fx_bidx_cell(3, up, c0)];
    vn[2] = vrr[fx_bidx_cell(3, right, c1)];
    vn[3] = vru[fx_bidx_cell(3, up, c3)];
    const int eidx = fx_edge_idx(dir, e[0], e[1], e[2]);
    for (int n = 0; n < 4; ++n) {
        if (!isfinite(f[n]) || !isfinite(c[n]) || !isfinite(vn[n])) {
            fx_fail(D.err, FX_ERR_EMF_NONFINITE, b, eidx);
        }
    }
    /* edge resistivity: run-time eta plus the maximum artificial eta of the
     * four incident cells (src/prj_timeint.c:265-290) */
    double eta_cells = 0.0;
    {
        const int cells[4] = {c0, c1, c2, c3};
        for (int n = 0; n < 4; ++n) {
            const double ce = fx_cell_eta(Wb[(size_t)FX_RHO * kPlane + cells[n]],
                Wb[(size_t)FX_YE * kPlane + cells[n]]);
            if (!isfinite(ce) || ce < 0.0) {
                fx_fail(D.err, FX_ERR_ETA, b, eidx);
            }
            if (ce > eta_cells) {
                eta_cells = ce;
            }
        }
    }
    const double eta = D.mhd_eta + eta_cells;
    double emf;
    if (D.br_mode == 0) {
        emf = fx_emf_upwind(f, c, vn);
    } else {
        /* this edge's decision word (record / replay) */
        const size_t bri = D.br_eoff + ((size_t)b * 3 + dir) * NE + te;
        if (D.br_mode == 1) {
            FxBrRecord br;
            emf = fx_emf_upwind_br(f, c, vn, br);
            D.br_edges[bri] = br.w;
        } else {
            FxBrReplay br;
            br.w = D.br_edges[bri];
            emf = fx_emf_upwind_br(f, c, vn, br);
            if (br.flips) {
                atomicAdd(D.br_flips, (unsigned long long)br.flips);
            }
        }
    }
    if (eta != 0.0) {
        /* resistive term, src/prj_mhd.c:682-709 */
        const double *bf = D.Bf + (size_t)b * FX_BF_COUNT;
        const double *b1 = bf + (size_t)(0 * FX_NSTAGES + bfslot) * FX_NFACES;
        const double *b2 = bf + (size_t)(1 * FX_NSTAGES + bfslot) * FX_NFACES;
        const double *b3 = bf + (size_t)(2 * FX_NSTAGES + bfslot) * FX_NFACES;
        const FxBlockDev &B = D.blk[b];
        const int i = e[0], j = e[1], k = e[2];
        double curl_b;
        if (dir == 0) {
            curl_b = (b3[fx_face_idx(2, i, j, k)] - b3[fx_face_idx(2, i, j - 1, k)]) / B.dx[1] -
                (b2[fx_face_idx(1, i, j, k)] - b2[fx_face_idx(1, i, j, k - 1)]) / B.dx[2];
        } else if (dir == 1) {
            curl_b = (b1[fx_face_idx(0, i, j, k)] - b1[fx_face_idx(0, i, j, k - 1)]) / B.dx[2] -
                (b3[fx_face_idx(2, i, j, k)] - b3[fx_face_idx(2, i - 1, j, k)]) / B.dx[0];
        } else {
            curl_b = (b2[fx_face_idx(1, i, j, k)] - b2[fx_face_idx(1, i - 1, j, k)]) / B.dx[0] -
                (b1[fx_face_idx(0, i, j, k)] - b1[fx_face_idx(0, i, j - 1, k)]) / B.dx[1];
        }
        emf += eta * curl_b;
    }
    if (!isfinite(emf)) {
        fx_fail(D.err, FX_ERR_EMF_NONFINITE, b, eidx);
    }
    D.emf[(size_t)b * FX_EMF_COUNT + (size_t)dir * FX_NEDGES + eidx] = emf;
}

/* One CTA per (block, chunk of edge layers along i).  For each layer i the
 * CTA first evaluates, once per cell of plane i (j, k in [-1, 16]), the
 * three cell-centred EMF components and the artificial eta (the reference
 * precomputes the same per-cell grids, src/prj_timeint.c:313-338 and
 * prj_timeint_mhd_fill_eta_mask), keeping planes i - 1 and i in shared
 * memory; then its threads sweep the layer's edges of all three directions
 * (an edge along x at layer i reads plane i only, edges along y and z read
 * planes i - 1 and i).  The face EMFs and normal velocities of an edge come
 * straight from global memory (each is read by two edges, coalesced along
 * k).  Arithmetic of prj_timeint_mhd_update_emf (src/prj_timeint.c:292-413). */
/* edge layers per CTA: measured flat between 1 and 17 layers (0.178-0.189
 * ms for 512 blocks), 2 the fastest */
constexpr int kEmfChunk = 2;
constexpr int kEmfChunks = (FX_BS + 1 + kEmfChunk - 1) / kEmfChunk;

__global__ void __launch_bounds__(256, 5) k_emf(FxDev D, const int *__restrict__ blist, int wslot, int bfslot)
{
    if (D.ctl->skip) {
        return;
    }
    constexpr int P2 = FX_PBS * FX_PBS;          /* cells per plane */
    /* [plane parity][E1, E2, E3, eta][in-plane cell] */
    __shared__ double cq[2][4][P2];
    const int b = blist[blockIdx.y];
    const int l0 = blockIdx.x * kEmfChunk;
    const int l1 = min(l0 + kEmfChunk, FX_BS + 1);
    const double *Wb = D.W + (size_t)b * FX_W_COUNT(9) + (size_t)wslot * FX_NCELLS;

    /* cell quantities of plane i into buffer (i + 2) & 1 */
    auto cells = [&](int i) {
        double (*q)[P2] = cq[(i + 2) & 1];
        for (int t = threadIdx.x; t < (FX_BS + 2) * (FX_BS + 2); t += blockDim.x) {
            const int jj = t / (FX_BS + 2);
            const int kk = t - jj * (FX_BS + 2);
            const int c = fx_lidx(i, jj - 1, kk - 1);
            const double b1 = Wb[(size_t)FX_B1 * kPlane + c];
            const double b2 = Wb[(size_t)FX_B2 * kPlane + c];
            const double b3 = Wb[(size_t)FX_B3 * kPlane + c];
            const double v1 = Wb[(size_t)FX_V1 * kPlane + c];
            const double v2 = Wb[(size_t)FX_V2 * kPlane + c];
            const double v3 = Wb[(size_t)FX_V3 * kPlane + c];
            /* prj_timeint_mhd_cell_emf_all, src/prj_timeint.c:171-176 */
            const double e1 = b2 * v3 - b3 * v2;
            const double e2 = b3 * v1 - b1 * v3;
            const double e3 = b1 * v2 - b2 * v1;
            if (!isfinite(e1) || !isfinite(e2) || !isfinite(e3)) {
                fx_fail(D.err, FX_ERR_EMF_NONFINITE, b, c);
            }
            const double eta = fx_cell_eta(Wb[(size_t)FX_RHO * kPlane + c], Wb[(size_t)FX_YE * kPlane + c]);
            if (!isfinite(eta) || eta < 0.0) {
                fx_fail(D.err, FX_ERR_ETA, b, c);
            }
            const int pc = (jj - 1 + FX_NG) * FX_PBS + (kk - 1 + FX_NG);
            q[0][pc] = e1;
            q[1][pc] = e2;
            q[2][pc] = e3;
            q[3][pc] = eta;
        }
    };

    constexpr int N0 = (FX_BS + 1) * (FX_BS + 1);   /* x edges of a layer (i < 16) */
    constexpr int N1 = FX_BS * (FX_BS + 1);         /* y edges */
    constexpr int N2 = (FX_BS + 1) * FX_BS;         /* z edges */
    cells(l0 - 1);
    for (int i0 = l0; i0 < l1; ++i0) {
        cells(i0);
        __syncthreads();
        const int cur = (i0 + 2) & 1;   /* buffer of plane i0; plane i0 - 1 in 1 - cur */
        const int n0 = i0 < FX_BS ? N0 : 0;
        const int ntot = n0 + N1 + N2;
        for (int t = threadIdx.x; t < ntot; t += blockDim.x) {
            int dir, u = t;
            if (u < n0) {
                dir = 0;
            } else if ((u -= n0) < N1) {
                dir = 1;
            } else {
                u -= N1;
                dir = 2;
            }
            /* k runs over 17 edges for x and y edges, 16 for z edges:
             * constant divisors */
            int j, k;
            if (dir == 2) {
                j = u / FX_BS;
                k = u - j * FX_BS;
            } else {
                j = u / (FX_BS + 1);
                k = u - j * (FX_BS + 1);
            }
            const int up = (dir + 1) % 3;
            const int right = (dir + 2) % 3;
            /* the four cells: c0 = e, c1 = e - up, c2 = e - up - right,
             * c3 = e - right; buffer and in-plane index */
            const int pc = (j + FX_NG) * FX_PBS + (k + FX_NG);
            int cb[4], ci[4];
            if (dir == 0) {
                cb[0] = cur; ci[0] = pc;
                cb[1] = cur; ci[1] = pc - FX_PBS;
                cb[2] = cur; ci[2] = pc - FX_PBS - 1;
                cb[3] = cur; ci[3] = pc - 1;
            } else if (dir == 1) {
                cb[0] = cur; ci[0] = pc;
                cb[1] = cur; ci[1] = pc - 1;
                cb[2] = 1 - cur; ci[2] = pc - 1;
                cb[3] = 1 - cur; ci[3] = pc;
            } else {
                cb[0] = cur; ci[0] = pc;
                cb[1] = 1 - cur; ci[1] = pc;
                cb[2] = 1 - cur; ci[2] = pc - FX_PBS;
                cb[3] = cur; ci[3] = pc - FX_PBS;
            }
            double c[4];
            /* edge resistivity: run-time eta plus the maximum artificial eta
             * of the four incident cells (src/prj_timeint.c:265-290) */
            double eta_cells = 0.0;
#pragma unroll
            for (int n = 0; n < 4; ++n) {
                c[n] = cq[cb[n]][dir][ci[n]];
                const double ce = cq[cb[n]][3][ci[n]];
                if (ce > eta_cells) {
                    eta_cells = ce;
                }
            }
            const int c0 = fx_lidx(i0, j, k);
            const int c1 = c0 - fx_axis_stride(up);
            const int c3 = c0 - fx_axis_stride(right);
            const double *bv1r = D.bv1 + (size_t)b * FX_BV_COUNT + (size_t)right * FX_NCELLS;
            const double *bv2u = D.bv2 + (size_t)b * FX_BV_COUNT + (size_t)up * FX_NCELLS;
            const double *vrr = D.vr + (size_t)b * FX_VR_COUNT + (size_t)right * 3 * FX_NCELLS;
            const double *vru = D.vr + (size_t)b * FX_VR_COUNT + (size_t)up * 3 * FX_NCELLS;
            double f[4], vn[4];
            f[0] = bv1r[c0];
            f[1] = bv2u[c0];
            f[2] = bv1r[c1];
            f[3] = bv2u[c3];
            vn[0] = vrr[fx_bidx_cell(3, right, c0)];
            vn[1] = vru[fx_bidx_cell(3, up, c0)];
            vn[2] = vrr[fx_bidx_cell(3, right, c1)];
            vn[3] = vru[fx_bidx_cell(3, up, c3)];
            const int eidx = fx_edge_idx(dir, i0, j, k);
            for (int n = 0; n < 4; ++n) {
                if (!isfinite(f[n]) || !isfinite(vn[n])) {
                    fx_fail(D.err, FX_ERR_EMF_NONFINITE, b, eidx);
                }
            }
            const double eta = D.mhd_eta + eta_cells;
            double emf = fx_emf_upwind(f, c, vn);
            if (eta != 0.0) {
                /* resistive term, src/prj_mhd.c:682-709 */
                const double *bf = D.Bf + (size_t)b * FX_BF_COUNT;
                const double *b1 = bf + (size_t)(0 * FX_NSTAGES + bfslot) * FX_NFACES;
                const double *b2 = bf + (size_t)(1 * FX_NSTAGES + bfslot) * FX_NFACES;
                const double *b3 = bf + (size_t)(2 * FX_NSTAGES + bfslot) * FX_NFACES;
                const FxBlockDev &B = D.blk[b];
                const int i = i0;
                double curl_b;
                if (dir == 0) {
                    curl_b = (b3[fx_face_idx(2, i, j, k)] - b3[fx_face_idx(2, i, j - 1, k)]) / B.dx[1] -
                        (b2[fx_face_idx(1, i, j, k)] - b2[fx_face_idx(1, i, j, k - 1)]) / B.dx[2];
                } else if (dir == 1) {
                    curl_b = (b1[fx_face_idx(0, i, j, k)] - b1[fx_face_idx(0, i, j, k - 1)]) / B.dx[2] -
                        (b3[fx_face_idx(2, i, j, k)] - b3[fx_face_idx(2, i - 1, j, k)]) / B.dx[0];
                } else {
                    curl_b = (b2[fx_face_idx(1, i, j, k)] - b2[fx_face_idx(1, i - 1, j, k)]) / B.dx[0] -
                        (b1[fx_face_idx(0, i, j, k)] - b1[fx_face_idx(0, i, j - 1, k)]) / B.dx[1];
                }
                emf += eta * curl_b;
            }
            if (!isfinite(emf)) {
                fx_fail(D.err, FX_ERR_EMF_NONFINITE, b, eidx);
            }
            D.emf[(size_t)b * FX_EMF_COUNT + (size_t)dir * FX_NEDGES + eidx] = emf;
        }
        __syncthreads(); /* plane i0 - 1's buffer takes plane i0 + 1 next */
    }
}

/* ------------------------------------------------------------------------ */
/* CT face update                                                            */
/* ------------------------------------------------------------------------ */
/* one face of direction DIR (compile-time, so the index arithmetic divides
 * by constants); grid (face chunk, direction, block) */
template <int DIR>
__device__ __forceinline__ void fx_bf_face(const FxDev &D, int b, int t, int stage, double dt)
{
    constexpr int x2 = DIR == 2 ? FX_BS + 1 : FX_BS;
    constexpr int x1 = DIR == 1 ? FX_BS + 1 : FX_BS;
    const int k = t % x2;
    t /= x2;
    const int j = t % x1;
    const int i = t / x1;
    const int src_slot = stage == 2 ? 1 : 0;
    const int dst_slot = stage == 1 ? 1 : 0;
    double *bf = D.Bf + (size_t)b * FX_BF_COUNT;
    const double *e = D.emf + (size_t)b * FX_EMF_COUNT;
    const double *e1 = e;
    const double *e2 = e + FX_NEDGES;
    const double *e3 = e + 2 * FX_NEDGES;
    const FxBlockDev &B = D.blk[b];
    const int f = fx_face_idx(DIR, i, j, k);
    double value = bf[((size_t)DIR * FX_NSTAGES + src_slot) * FX_NFACES + f];
    if (DIR == 0) {
        value += -dt * (e3[fx_edge_idx(2, i, j + 1, k)] - e3[fx_edge_idx(2, i, j, k)]) / B.dx[1];
        value += dt * (e2[fx_edge_idx(1, i, j, k + 1)] - e2[fx_edge_idx(1, i, j, k)]) / B.dx[2];
    } else if (DIR == 1) {
        value += -dt * (e1[fx_edge_idx(0, i, j, k + 1)] - e1[fx_edge_idx(0, i, j, k)]) / B.dx[2];
        value += dt * (e3[fx_edge_idx(2, i + 1, j, k)] - e3[fx_edge_idx(2, i, j, k)]) / B.dx[0];
    } else {
        value += -dt * (e2[fx_edge_idx(1, i + 1, j, k)] - e2[fx_edge_idx(1, i, j, k)]) / B.dx[0];
        value += dt * (e1[fx_edge_idx(0, i, j + 1, k)] - e1[fx_edge_idx(0, i, j, k)]) / B.dx[1];
    }
    if (!isfinite(value)) {
        fx_fail(D.err, FX_ERR_BF_NONFINITE, b, f);
    }
    if (stage == 2) {
        value = 0.5 * bf[((size_t)DIR * FX_NSTAGES + 0) * FX_NFACES + f] + 0.5 * value;
    }
    bf[((size_t)DIR * FX_NSTAGES + dst_slot) * FX_NFACES + f] = value;
}

__global__ void __launch_bounds__(128) k_bf_update(FxDev D, const int *__restrict__ blist, int stage)
{
    if (D.ctl->skip) {
        return;
    }
    constexpr int NF = (FX_BS + 1) * FX_BS * FX_BS;
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= NF) {
        return;
    }
    const double dt = D.ctl->dt_stage;
    const int b = blist[blockIdx.z];
    switch (blockIdx.y) {
    case 0: fx_bf_face<0>(D, b, t, stage, dt); break;
    case 1: fx_bf_face<1>(D, b, t, stage, dt); break;
    default: fx_bf_face<2>(D, b, t, stage, dt); break;
    }
}

/* ------------------------------------------------------------------------ */
/* Cell update (flux divergence + sources + RK2 combine + cons2prim)         */
/* ------------------------------------------------------------------------ */
/* STAGE 1 / 2: the RK2 stages; STAGE 0: the stage-1 arithmetic written in
 * place to slot 0 with the field of Bf slot 0 (an eSSPRK substep,
 * prj_timeint_eSSPRK_step, src/prj_timeint.c:2484-2508) */
template <bool MHD, int STAGE>
__global__ void __launch_bounds__(128) k_cell_update(FxDev D, const int *__restrict__ blist,
    int gravity, int store_rhs)
{
    if (D.ctl->skip) {
        return;
    }
    const double dt = D.ctl->dt_stage;
    const int b = blist[blockIdx.y];
    constexpr int nv = MHD ? 9 : 6;
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= FX_BS * FX_BS * FX_BS) {
        return;
    }
    const int k = t % FX_BS;
    const int j = (t / FX_BS) % FX_BS;
    const int i = t / (FX_BS * FX_BS);
    const int c = fx_lidx(i, j, k);
    const FxBlockDev &B = D.blk[b];
    const double *W = D.W + (size_t)b * FX_W_COUNT(nv);
    const double *fx = D.flux + (size_t)b * FX_FLUX_COUNT(nv);
    const double *fy = fx + (size_t)nv * FX_NCELLS;
    const double *fz = fy + (size_t)nv * FX_NCELLS;

    /* prj_flux_div, src/prj_flux.c:2523-2533 (hydro components; the B
     * components are replaced by the face average below) */
    double fluxdiv[6];
#pragma unroll
    for (int v = 0; v < 6; ++v) {
        fluxdiv[v] = -(B.area[0] * (fx[fx_bidx(nv, v, i + 1, j, k)] - fx[fx_bidx(nv, v, i, j, k)]) +
            B.area[1] * (fy[fx_bidx(nv, v, i, j + 1, k)] - fy[fx_bidx(nv, v, i, j, k)]) +
            B.area[2] * (fz[fx_bidx(nv, v, i, j, k + 1)] - fz[fx_bidx(nv, v, i, j, k)])) / B.vol;
    }

    double w[9];
    double u[9];
#pragma unroll
    for (int v = 0; v < nv; ++v) {
        w[v] = W[(size_t)v * kPlane + c];
    }
    fx_prim2cons<MHD>(w, u);

    /* source terms: rhs = 0, then the static-gravity terms of
     * prj_src_monopole_gravity with the stage primitives (src/prj_src.c:32-139) */
    double rhs[6];
#pragma unroll
    for (int v = 0; v < 6; ++v) {
        rhs[v] = 0.0;
    }
    if (gravity) {
        const double *Ws = W + (size_t)(STAGE == 2 ? 1 : 0) * FX_NCELLS;
        const double *g = D.grav + (size_t)b * FX_GRAV_COUNT;
        const double g1 = g[c];
        const double g2 = g[FX_NCELLS + c];
        const double g3 = g[2 * FX_NCELLS + c];
        const double rho = Ws[(size_t)FX_RHO * kPlane + c];
        const double *vr = D.vr + (size_t)b * FX_VR_COUNT;
        rhs[FX_V1] += rho * g1;
        rhs[FX_V2] += rho * g2;
        rhs[FX_V3] += rho * g3;
        const double v_avg1 = (vr[fx_bidx(3, 0, i, j, k)] + vr[fx_bidx(3, 0, i + 1, j, k)]) * 0.5;
        const double v_avg2 = (vr[3 * FX_NCELLS + fx_bidx(3, 1, i, j, k)] +
            vr[3 * FX_NCELLS + fx_bidx(3, 1, i, j + 1, k)]) * 0.5;
        const double v_avg3 = (vr[6 * FX_NCELLS + fx_bidx(3, 2, i, j, k)] +
            vr[6 * FX_NCELLS + fx_bidx(3, 2, i, j, k + 1)]) * 0.5;
        rhs[FX_ETOT] += rho * (v_avg1 * g1 + v_avg2 * g2 + v_avg3 * g3);
    }
    if (store_rhs) {
        double *r = D.rhs + (size_t)b * FX_RHS_COUNT(nv);
#pragma unroll
        for (int v = 0; v < nv; ++v) {
            r[fx_bidx(nv, v, i, j, k)] = v < 6 ? rhs[v] : 0.0;
        }
    }

    /* dt_src from the start-of-step total energy,
     * prj_timeint_update_dt_src_values (src/prj_timeint.c:533-565) */
    const double dt_src = 0.02 * u[FX_ETOT] / (fabs(rhs[FX_ETOT]) + 1.0e-50);

    double un[9];
    if (STAGE != 2) {
#pragma unroll
        for (int v = 0; v < 6; ++v) {
            un[v] = u[v] + dt * (rhs[v] + fluxdiv[v]);
        }
    } else {
        double w1[9];
        double u1[9];
        const double *W1 = W + FX_NCELLS;
#pragma unroll
        for (int v = 0; v < nv; ++v) {
            w1[v] = W1[(size_t)v * kPlane + c];
        }
        fx_prim2cons<MHD>(w1, u1);
#pragma unroll
        for (int v = 0; v < 6; ++v) {
            const double u_trial = u1[v] + dt * (rhs[v] + fluxdiv[v]);
            un[v] = 0.5 * u[v] + 0.5 * u_trial;
        }
    }
    if (MHD) {
        /* cell B from the updated faces, src/prj_timeint.c:498-510 */
        const int bslot = STAGE == 1 ? 1 : 0;  /* slot the CT update wrote */
        const double *bf = D.Bf + (size_t)b * FX_BF_COUNT;
        const double *b1 = bf + (size_t)(0 * FX_NSTAGES + bslot) * FX_NFACES;
        const double *b2 = bf + (size_t)(1 * FX_NSTAGES + bslot) * FX_NFACES;
        const double *b3 = bf + (size_t)(2 * FX_NSTAGES + bslot) * FX_NFACES;
        un[FX_B1] = 0.5 * (b1[fx_face_idx(0, i, j, k)] + b1[fx_face_idx(0, i + 1, j, k)]);
        un[FX_B2] = 0.5 * (b2[fx_face_idx(1, i, j, k)] + b2[fx_face_idx(1, i, j + 1, k)]);
        un[FX_B3] = 0.5 * (b3[fx_face_idx(2, i, j, k)] + b3[fx_face_idx(2, i, j, k + 1)]);
        if (!isfinite(un[FX_B1]) || !isfinite(un[FX_B2]) || !isfinite(un[FX_B3])) {
            fx_fail(D.err, FX_ERR_B_NONFINITE, b, c);
        }
    }
    double wn[9];
    fx_cons2prim<MHD>(un, wn);
    double *Wd = D.W + (size_t)b * FX_W_COUNT(nv) + (size_t)(STAGE == 1 ? 1 : 0) * FX_NCELLS;
#pragma unroll
    for (int v = 0; v < nv; ++v) {
        Wd[(size_t)v * kPlane + c] = wn[v];
    }

    /* block-wide minimum of dt_src, then one atomic per CTA */
    __shared__ unsigned long long smin[4];
    unsigned long long key = fx_double_key(dt_src);
    if (dt_src != dt_src) {
        key = ~0ULL;
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
        const unsigned long long o = __shfl_down_sync(0xffffffffu, key, off);
        key = o < key ? o : key;
    }
    if ((threadIdx.x & 31) == 0) {
        smin[threadIdx.x >> 5] = key;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned long long m = smin[0];
        for (int q = 1; q < (int)(blockDim.x >> 5); ++q) {
            m = smin[q] < m ? smin[q] : m;
        }
        atomicMin(&D.red[1], m);
    }
}

/* ------------------------------------------------------------------------ */
/* EOS fill (eosvar = p, T, gamma from the stage primitives)                 */
/* ------------------------------------------------------------------------ */
__global__ void k_eos_fill(FxDev D, const int *__restrict__ blist, int wslot, int active_only)
{
    if (D.ctl->skip) {
        return;
    }
    const int b = blist[blockIdx.y];
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    int i, j, k;
    if (active_only) {
        if (t >= FX_BS * FX_BS * FX_BS) return;
        k = t % FX_BS;
        j = (t / FX_BS) % FX_BS;
        i = t / (FX_BS * FX_BS);
    } else {
        if (t >= FX_NCELLS) return;
        k = t % FX_PBS - FX_NG;
        j = (t / FX_PBS) % FX_PBS - FX_NG;
        i = t / (FX_PBS * FX_PBS) - FX_NG;
    }
    const int c = fx_lidx(i, j, k);
    const double *W = D.W + (size_t)b * FX_W_COUNT(D.nv) + (size_t)wslot * FX_NCELLS;
    const double rho = W[(size_t)FX_RHO * kPlane + c];
    const double eint = W[(size_t)FX_EINT * kPlane + c];
    if (rho == 0.0) {
        fx_fail(D.err, FX_ERR_EOS_ZERO_RHO, b, c);
    }
    const double g = D.gamma;
    double *e = D.eos + (size_t)b * FX_EOS_COUNT;
    e[fx_bidx(3, FX_EOS_P, i, j, k)] = fx_pressure(g, rho, eint);
    e[fx_bidx(3, FX_EOS_T, i, j, k)] = fx_temperature(g, eint);
    e[fx_bidx(3, FX_EOS_G, i, j, k)] = g;
}

/* ------------------------------------------------------------------------ */
/* dt = min over active cells of cfl / sum_d (|v_d| + c_s) / dx_d            */
/* ------------------------------------------------------------------------ */
__global__ void __launch_bounds__(256) k_calc_dt(FxDev D, const int *__restrict__ blist, int wslot, double cfl)
{
    const int b = blist[blockIdx.y];
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    unsigned long long key = ~0ULL;
    if (t < FX_BS * FX_BS * FX_BS) {
        const int k = t % FX_BS;
        const int j = (t / FX_BS) % FX_BS;
        const int i = t / (FX_BS * FX_BS);
        const int c = fx_lidx(i, j, k);
        const double *W = D.W + (size_t)b * FX_W_COUNT(D.nv) + (size_t)wslot * FX_NCELLS;
        const FxBlockDev &B = D.blk[b];
        const double g = D.gamma;
        const double rho = W[(size_t)FX_RHO * kPlane + c];
        const double p = fx_pressure(g, rho, W[(size_t)FX_EINT * kPlane + c]);
        const double cs = sqrt(g * p / rho);
        const double denom = (fabs(W[(size_t)FX_V1 * kPlane + c]) + cs) / B.dx[0] +
            (fabs(W[(size_t)FX_V2 * kPlane + c]) + cs) / B.dx[1] +
            (fabs(W[(size_t)FX_V3 * kPlane + c]) + cs) / B.dx[2];
        const double dt_cell = cfl / denom;
        if (dt_cell == dt_cell) {
            key = fx_double_key(dt_cell);
        }
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
        const unsigned long long o = __shfl_down_sync(0xffffffffu, key, off);
        key = o < key ? o : key;
    }
    __shared__ unsigned long long smin[8];
    if ((threadIdx.x & 31) == 0) {
        smin[threadIdx.x >> 5] = key;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned long long m = smin[0];
        for (int q = 1; q < (int)(blockDim.x >> 5); ++q) {
            m = smin[q] < m ? smin[q] : m;
        }
        atomicMin(&D.red[0], m);
    }
}

__global__ void k_reset_reductions(FxDev D, int which)
{
    /* initial values of the reference's reductions: dt_min = 1e99
     * (src/prj_timeint.c:2147), dt_src = 1e100 (src/main.c:491) */
    if (which & 1) D.red[0] = fx_double_key(1.0e99);
    if (which & 2) D.red[1] = fx_double_key(1.0e100);
}

__device__ __forceinline__ double fx_key_double(unsigned long long key)
{
    const unsigned long long bits = (key >> 63) ? (key & 0x7fffffffffffffffULL) : ~key;
    return __longlong_as_double((long long)bits);
}

/* dt selection of the driver loop, src/main.c:485-517 (no output events) */
__global__ void k_step_begin(FxDev D)
{
    FxCtl *c = D.ctl;
    if (!(c->time < c->t_end)) {
        c->skip = 1;
        return;
    }
    c->skip = 0;
    /* prj_timeint_calc_dt's minimum, times 6 for eSSPRK10_4 */
    const double dt_new = fx_key_double(D.red[0]) * c->dt_mult;
    if (c->dt_prev > 0.0) {
        const double dt_limit = c->dt_factor * c->dt_prev;
        c->dt_prev = dt_new <= dt_limit ? dt_new : dt_limit;
    } else {
        c->dt_prev = dt_new;
    }
    double dt_step = c->dt_prev;
    if (c->time + dt_step > c->t_end) {
        dt_step = c->t_end - c->time;
    }
    c->dt = dt_step;
    c->dt_stage = dt_step;
    D.red[1] = fx_double_key(1.0e100);
}

/* after the step: dt_src clamp and time advance, src/main.c:555-562 */
__global__ void k_step_end(FxDev D)
{
    FxCtl *c = D.ctl;
    if (c->skip) {
        return;
    }
    const double dt_src = fx_key_double(D.red[1]);
    c->dt_src = dt_src;
    if (c->cfl * dt_src < c->dt_prev) {
        c->dt_prev = c->cfl * dt_src;
    }
    c->time += c->dt;
    c->step += 1;
}

/* ------------------------------------------------------------------------ */
/* Ghost-fill programs                                                       */
/* ------------------------------------------------------------------------ */

/* prj_reconstruct_cell_for_prolongate_minmod (src/prj_reconstruct.h:111-143):
 * per axis base + slope * target, combined as vx + vy + vz - 2 base; target
 * offsets are +-1/4 of a coarse cell.  use_BJ = 1 takes fx_bj_cell /
 * fx_bj_face on the full 27-cell (3x3-face) stencil instead. */
__device__ __forceinline__ double fx_prolong_cell(const double *q, int c, double tx, double ty, double tz)
{
    const double base = q[c];
    const double vx = base + fx_minmod_slope(q[c - FX_PBS * FX_PBS], base, q[c + FX_PBS * FX_PBS]) * tx;
    const double vy = base + fx_minmod_slope(q[c - FX_PBS], base, q[c + FX_PBS]) * ty;
    const double vz = base + fx_minmod_slope(q[c - 1], base, q[c + 1]) * tz;
    return vx + vy + vz - 2.0 * base;
}

/* prj_reconstruct_face_for_prolongate_minmod (src/prj_reconstruct.h:222-246)
 * on the face stencil of direction d about face f: tangential axes t0 < t1
 * with face-index strides s0, s1 */
__device__ __forceinline__ double fx_prolong_face(const double *q, int f, int s0, int s1, double t0, double t1)
{
    const double base = q[f];
    const double vx = base + fx_minmod_slope(q[f - s0], base, q[f + s0]) * t0;
    const double vy = base + fx_minmod_slope(q[f - s1], base, q[f + s1]) * t1;
    return vx + vy - base;
}

/* BJ: the program may hold Barth-Jespersen prolongations (use_BJ); the
 * other instance keeps the copy-dominated wave kernel at its small register
 * count */
template <bool BJ>
__device__ __forceinline__ void fx_ghost_cell_op(const FxDev &D, const FxGop op, int wslot, int nvg)
{
    const int db = FX_CELL_BLOCK(op.dst);
    const int dc = FX_CELL_IDX(op.dst);
    const int sb = FX_CELL_BLOCK(op.src);
    const int sc = FX_CELL_IDX(op.src);
    double *Wd = D.W + (size_t)db * FX_W_COUNT(D.nv) + (size_t)wslot * FX_NCELLS;
    const double *Ws = D.W + (size_t)sb * FX_W_COUNT(D.nv) + (size_t)wslot * FX_NCELLS;
    if constexpr (BJ) {
        if (op.type == FX_GOP_PROLONG_BJ) {
            const double tx = (op.aux & 4) ? 0.25 : -0.25;
            const double ty = (op.aux & 2) ? 0.25 : -0.25;
            const double tz = (op.aux & 1) ? 0.25 : -0.25;
#pragma unroll 1
            for (int v = 0; v < nvg; ++v) {
                const double *q = Ws + (size_t)v * kPlane + sc;
                Wd[(size_t)v * kPlane + dc] = fx_bj_cell(
                    [q](int di, int dj, int dk) { return q[(di * FX_PBS + dj) * FX_PBS + dk]; }, tx, ty, tz);
            }
            return;
        }
    }
    /* every variable's value first, then the stores: the loads of all
     * variables are in flight together (the wave's operations are conflict
     * free, so no store of the wave feeds a load of it) */
    double val[FX_MAXVAR];
    switch (op.type) {
    case FX_GOP_COPY:
    case FX_GOP_COPY_NEG:
    case FX_GOP_COPY_USER:
#pragma unroll
        for (int v = 0; v < FX_MAXVAR; ++v) {
            if (v < nvg) val[v] = Ws[(size_t)v * kPlane + sc];
        }
        if (op.type == FX_GOP_COPY_NEG) {
#pragma unroll
            for (int v = 0; v < FX_MAXVAR; ++v) {
                if (v == op.aux) val[v] = -val[v];
            }
        } else if (op.type == FX_GOP_COPY_USER && op.aux) {
            val[FX_V1] = 5.0;
        }
        break;
    case FX_GOP_RESTRICT:
#pragma unroll
        for (int v = 0; v < FX_MAXVAR; ++v) {
            if (v >= nvg) continue;
            const double *q = Ws + (size_t)v * kPlane + sc;
            /* order of src/prj_boundary.c:238-261 */
            val[v] = 0.125 *
                (q[0] + q[1] + q[FX_PBS] + q[FX_PBS + 1] +
                 q[FX_PBS * FX_PBS] + q[FX_PBS * FX_PBS + 1] +
                 q[FX_PBS * FX_PBS + FX_PBS] + q[FX_PBS * FX_PBS + FX_PBS + 1]);
        }
        break;
    case FX_GOP_PROLONG: {
        /* target offsets of src/prj_boundary.c:318-320 */
        const double tx = (op.aux & 4) ? 0.25 : -0.25;
        const double ty = (op.aux & 2) ? 0.25 : -0.25;
        const double tz = (op.aux & 1) ? 0.25 : -0.25;
#pragma unroll
        for (int v = 0; v < FX_MAXVAR; ++v) {
            if (v < nvg) val[v] = fx_prolong_cell(Ws + (size_t)v * kPlane, sc, tx, ty, tz);
        }
        break;
    }
    default:
        return;
    }
#pragma unroll
    for (int v = 0; v < FX_MAXVAR; ++v) {
        if (v < nvg) Wd[(size_t)v * kPlane + dc] = val[v];
    }
}

__device__ __forceinline__ int fx_face_key_block(int key) { return key >> 15; }
__device__ __forceinline__ int fx_face_key_idx(int key) { return key & 32767; }

/* the value of one face operation (its loads) and where it goes; the store
 * is left to the caller, so that a thread can issue the loads of several
 * operations before their stores (the operations of a wave are conflict
 * free).  Null for an unknown type. */
__device__ __forceinline__ double *fx_ghost_face_value(const FxDev &D, const FxGop op, int bfslot, double &v)
{
    const int dir = op.aux & 3;
    const int db = fx_face_key_block(op.dst);
    const int df = fx_face_key_idx(op.dst);
    const int sb = fx_face_key_block(op.src);
    const int sf = fx_face_key_idx(op.src);
    double *Bd = D.Bf + (size_t)db * FX_BF_COUNT + ((size_t)dir * FX_NSTAGES + bfslot) * FX_NFACES;
    const double *Bs = D.Bf + (size_t)sb * FX_BF_COUNT + ((size_t)dir * FX_NSTAGES + bfslot) * FX_NFACES;
    if (op.type == FX_FOP_COPY) {
        v = Bs[sf];
        return Bd + df;
    }
    if (op.type == FX_FOP_RESTRICT) {
        /* 0.25*(s0 + s0+t1 + s0+t0 + s0+t0+t1), src/prj_boundary.c:738-764 */
        const int o1 = (op.aux >> 2) & 1023;   /* stride of tan1 */
        const int o0 = (op.aux >> 12) & 1023;  /* stride of tan0 */
        v = 0.25 * (Bs[sf] + Bs[sf + o1] + Bs[sf + o0] + Bs[sf + o0 + o1]);
        return Bd + df;
    }
    return nullptr;
}

/* face operations per thread of the wave kernel: a face copy moves one
 * double, so one operation per thread leaves too few loads in flight to
 * keep HBM busy */
constexpr int FX_GW_FACE_OPS = 4;

/* face-index offset of a unit step along axis a for faces of direction d */
__device__ __forceinline__ int fx_face_stride(int d, int a)
{
    return fx_face_idx(d, a == 0, a == 1, a == 2) - fx_face_idx(d, 0, 0, 0);
}

/* One Toth-Roe group: prj_mhd_prolong_bf_from_buffer (src/prj_mhd.c:374-512)
 * with prj_mhd_compute_buffer_inner_fluxes (src/prj_mhd.c:309-372), in the
 * reference's operation order.  Outer faces are area-weighted fluxes; kept
 * faces contribute their current fine value. */
__device__ __forceinline__ void fx_ghost_prolong_group(const FxDev &D, const FxPop &op, int slot)
{
    const int f0[3] = {(op.pos & 31) - FX_NG, ((op.pos >> 5) & 31) - FX_NG, ((op.pos >> 10) & 31) - FX_NG};
    const int c0[3] = {((op.pos >> 15) & 31) - FX_NG, ((op.pos >> 20) & 31) - FX_NG, ((op.pos >> 25) & 31) - FX_NG};
    const FxBlockDev &fb = D.blk[op.fine];
    const double area[3] = {fb.dx[1] * fb.dx[2], fb.dx[0] * fb.dx[2], fb.dx[0] * fb.dx[1]};
    /* outer fluxes o[d][side][a][b] */
    double o[3][2][2][2];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        const int t0 = d == 0 ? 1 : 0;
        const int t1 = d == 2 ? 1 : 2;
        double *Bfine = D.Bf + (size_t)op.fine * FX_BF_COUNT + ((size_t)d * FX_NSTAGES + slot) * FX_NFACES;
        const double *Bc = D.Bf + (size_t)op.coarse * FX_BF_COUNT + ((size_t)d * FX_NSTAGES + slot) * FX_NFACES;
        const int s0 = fx_face_stride(d, t0);
        const int s1 = fx_face_stride(d, t1);
#pragma unroll
        for (int side = 0; side < 2; ++side) {
            int y[3] = {c0[0], c0[1], c0[2]};
            y[d] += side;
            const int cf = fx_face_idx(d, y[0], y[1], y[2]);
#pragma unroll
            for (int a = 0; a < 2; ++a) {
#pragma unroll
                for (int b = 0; b < 2; ++b) {
                    const int q = 8 * d + 4 * side + 2 * a + b;
                    int x[3] = {f0[0], f0[1], f0[2]};
                    x[d] += 2 * side;
                    x[t0] += a;
                    x[t1] += b;
                    const int xf = fx_face_idx(d, x[0], x[1], x[2]);
                    double flux;
                    if ((op.keep >> q) & 1) {
                        flux = Bfine[xf] * area[d];
                    } else {
                        const double ta = a ? 0.25 : -0.25;
                        const double tb = b ? 0.25 : -0.25;
                        const double *qc = Bc + cf;
                        const double value = (op.flags & 1)
                            ? fx_bj_face([qc, s0, s1](int d0, int d1) { return qc[d0 * s0 + d1 * s1]; }, ta, tb)
                            : fx_prolong_face(Bc, cf, s0, s1, ta, tb);
                        flux = value * area[d];
                        if ((op.owrite >> q) & 1) {
                            Bfine[xf] = flux / area[d];
                        }
                    }
                    o[d][side][a][b] = flux;
                }
            }
        }
    }
    /* u[i][j][k] of the reference: u[0|2][j][k] = o[0][0|1][j][k],
     * v[i][0|2][k] = o[1][0|1][i][k], w[i][j][0|2] = o[2][0|1][i][j] */
    const double dx1s = fb.dx[0] * fb.dx[0];
    const double dx2s = fb.dx[1] * fb.dx[1];
    const double dx3s = fb.dx[2] * fb.dx[2];
    double Uxx = 0.0, Vyy = 0.0, Wzz = 0.0, Uxyz = 0.0, Vxyz = 0.0, Wxyz = 0.0;
#pragma unroll
    for (int i = 0; i < 2; ++i) {
        const double si = i ? 1.0 : -1.0;
#pragma unroll
        for (int j = 0; j < 2; ++j) {
            const double sj = j ? 1.0 : -1.0;
#pragma unroll
            for (int k = 0; k < 2; ++k) {
                const double sk = k ? 1.0 : -1.0;
                const double u = o[0][i][j][k];
                const double v = o[1][j][i][k];
                const double w = o[2][k][i][j];
                Uxx += si * sj * v + si * sk * w;
                Vyy += sj * sk * w + sj * si * u;
                Wzz += sk * si * u + sk * sj * v;
                Uxyz += si * sj * sk * u / (dx2s + dx3s);
                Vxyz += si * sj * sk * v / (dx1s + dx3s);
                Wxyz += si * sj * sk * w / (dx1s + dx2s);
            }
        }
    }
    Uxx *= 0.125;
    Vyy *= 0.125;
    Wzz *= 0.125;
    Uxyz *= 0.125;
    Vxyz *= 0.125;
    Wxyz *= 0.125;
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        const int t0 = d == 0 ? 1 : 0;
        const int t1 = d == 2 ? 1 : 2;
        double *Bfine = D.Bf + (size_t)op.fine * FX_BF_COUNT + ((size_t)d * FX_NSTAGES + slot) * FX_NFACES;
#pragma unroll
        for (int a = 0; a < 2; ++a) {
#pragma unroll
            for (int b = 0; b < 2; ++b) {
                const int q = 4 * d + 2 * a + b;
                if (!((op.iwrite >> q) & 1)) continue;
                const double sa = a ? 1.0 : -1.0;
                const double sb = b ? 1.0 : -1.0;
                double flux;
                if (d == 0) {        /* u[1][j][k], (a, b) = (j, k) */
                    flux = 0.5 * (o[0][1][a][b] + o[0][0][a][b]) + Uxx + sb * dx3s * Vxyz + sa * dx2s * Wxyz;
                } else if (d == 1) { /* v[i][1][k], (a, b) = (i, k) */
                    flux = 0.5 * (o[1][1][a][b] + o[1][0][a][b]) + Vyy + sa * dx1s * Wxyz + sb * dx3s * Uxyz;
                } else {             /* w[i][j][1], (a, b) = (i, j) */
                    flux = 0.5 * (o[2][1][a][b] + o[2][0][a][b]) + Wzz + sb * dx2s * Uxyz + sa * dx1s * Vxyz;
                }
                const double value = flux / area[d];
                int x[3] = {f0[0], f0[1], f0[2]};
                x[d] += 1;
                x[t0] += a;
                x[t1] += b;
                const int xf = fx_face_idx(d, x[0], x[1], x[2]);
                if (!isfinite(value)) {
                    fx_fail(D.err, FX_ERR_BF_NONFINITE, op.fine, xf);
                }
                Bfine[xf] = value;
            }
        }
    }
}

/* cell-centred field of one cell from its faces: prj_mhd_bf2bc_impl
 * (src/prj_mhd.c:555-603).  The metric factor sqrt(gamma) is 1 outside
 * dynamical GR; the reference's division by it is exact and omitted. */
__device__ __forceinline__ void fx_ghost_b_op(const FxDev &D, const FxBop op, int slot)
{
    double v[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        const int k0 = op.f[2 * d];
        const int k1 = op.f[2 * d + 1];
        const double *b0 = D.Bf + (size_t)fx_face_key_block(k0) * FX_BF_COUNT +
            ((size_t)d * FX_NSTAGES + slot) * FX_NFACES;
        const double *b1 = D.Bf + (size_t)fx_face_key_block(k1) * FX_BF_COUNT +
            ((size_t)d * FX_NSTAGES + slot) * FX_NFACES;
        v[d] = 0.5 * (b0[fx_face_key_idx(k0)] + b1[fx_face_key_idx(k1)]);
    }
    const int b = FX_CELL_BLOCK(op.dst);
    const int c = FX_CELL_IDX(op.dst);
    if (!isfinite(v[0]) || !isfinite(v[1]) || !isfinite(v[2])) {
        fx_fail(D.err, FX_ERR_B_NONFINITE, b, c);
    }
    double *W = D.W + (size_t)b * FX_W_COUNT(9) + (size_t)slot * FX_NCELLS;
    W[(size_t)FX_B1 * kPlane + c] = v[0];
    W[(size_t)FX_B2 * kPlane + c] = v[1];
    W[(size_t)FX_B3 * kPlane + c] = v[2];
}

/* face-prolongation groups of one wave (a separate kernel: the group
 * arithmetic would otherwise raise the register count, and so lower the
 * occupancy, of the copy-dominated wave kernel) */
__global__ void __launch_bounds__(128) k_ghost_groups(FxDev D, const FxPop *__restrict__ pops, int np, int slot)
{
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= np || D.ctl->skip) {
        return;
    }
    fx_ghost_prolong_group(D, pops[t], slot);
}

/* one conflict-free wave of the ghost fill: CTAs [0, nbc) run cell ops,
 * then face ops (FX_GW_FACE_OPS per thread) and cell-field ops.  At 6 CTAs
 * of 256 per SM the kernel keeps 40 registers without spills; on the 512-block
 * uniform fill this took 0.165 ms down to 0.148 ms. */
template <bool BJ>
__global__ void __launch_bounds__(256, 6) k_ghost_wave(FxDev D, const FxGop *__restrict__ cops, int nc,
    const FxGop *__restrict__ fops, int nf, const FxBop *__restrict__ bops, int nb, int slot, int nvg)
{
    if (D.ctl->skip) {
        return;
    }
    constexpr int UF = FX_GW_FACE_OPS;
    const int nbc = (nc + 255) / 256;
    const int nbf = (nf + 256 * UF - 1) / (256 * UF);
    int blk = blockIdx.x;
    if (blk < nbc) {
        const int t = blk * 256 + threadIdx.x;
        if (t < nc) fx_ghost_cell_op<BJ>(D, cops[t], slot, nvg);
        return;
    }
    blk -= nbc;
    if (blk < nbf) {
        /* operations t0 + 256 u, u < UF: every load first, then the stores */
        const int t0 = blk * 256 * UF + threadIdx.x;
        double v[UF];
        double *dst[UF];
#pragma unroll
        for (int u = 0; u < UF; ++u) {
            const int t = t0 + 256 * u;
            dst[u] = t < nf ? fx_ghost_face_value(D, fops[t], slot, v[u]) : nullptr;
        }
#pragma unroll
        for (int u = 0; u < UF; ++u) {
            if (dst[u]) *dst[u] = v[u];
        }
        return;
    }
    blk -= nbf;
    const int t = blk * 256 + threadIdx.x;
    if (t < nb) fx_ghost_b_op(D, bops[t], slot);
}

/* exchanges of a sharded mesh: one thread per listed element */
__device__ __forceinline__ double *fx_xelem(const FxDev &D, const FxXent &x, int slot, int q)
{
    switch (x.kind) {
    case 0:
        return D.W + (size_t)x.block * FX_W_COUNT(D.nv) + (size_t)slot * FX_NCELLS + (size_t)q * kPlane + x.idx;
    case 1: {
        const int dir = x.idx / FX_NFACES;
        return D.Bf + (size_t)x.block * FX_BF_COUNT + ((size_t)dir * FX_NSTAGES + slot) * FX_NFACES +
            (x.idx - dir * FX_NFACES);
    }
    case 2:
        return D.flux + (size_t)x.block * FX_FLUX_COUNT(D.nv) + x.idx + (size_t)q * FX_AOSOA_W;
    default:
        return D.emf + (size_t)x.block * FX_EMF_COUNT + x.idx;
    }
}

__device__ __forceinline__ int fx_xwidth(int kind) { return kind == 0 || kind == 2 ? 6 : 1; }

__global__ void k_xpack(FxDev D, const FxXent *__restrict__ ents, int n, double *__restrict__ buf, int slot)
{
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    const FxXent x = ents[t];
    for (int q = 0; q < fx_xwidth(x.kind); ++q) buf[x.off + q] = *fx_xelem(D, x, slot, q);
}

__global__ void k_xunpack(FxDev D, const FxXent *__restrict__ ents, int n, const double *__restrict__ buf, int slot)
{
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    const FxXent x = ents[t];
    for (int q = 0; q < fx_xwidth(x.kind); ++q) *fx_xelem(D, x, slot, q) = buf[x.off + q];
}

/* coarse/fine corrections */
__global__ void k_flux_correct(FxDev D, const FxCorr *__restrict__ recs, int n, int ncomp)
{
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n * ncomp || D.ctl->skip) {
        return;
    }
    const int r = t / ncomp;
    const int v = t - r * ncomp;
    const FxCorr rec = recs[r];
    /* entries index component 0 of a block's stacked flux array; component
     * v sits FX_AOSOA_W * v further in the AoSoA tile.  Sum order of
     * src/prj_riemann.c:1756-1761. */
    const double *s = D.flux + (size_t)rec.src_block * FX_FLUX_COUNT(D.nv) + (size_t)v * FX_AOSOA_W;
    double *d = D.flux + (size_t)rec.dst_block * FX_FLUX_COUNT(D.nv) + (size_t)v * FX_AOSOA_W;
    d[rec.dst] = 0.25 * (s[rec.src[0]] + s[rec.src[1]] + s[rec.src[2]] + s[rec.src[3]]);
}

__global__ void k_emf_correct(FxDev D, const FxCorr *__restrict__ recs, int n)
{
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n || D.ctl->skip) {
        return;
    }
    const FxCorr rec = recs[t];
    const double *s = D.emf + (size_t)rec.src_block * FX_EMF_COUNT;
    /* value = 0; value += e0; value += e1; value *= 0.5 (src/prj_mhd.c:904-910):
     * the leading 0.0 + makes a -0.0 pair sum to +0.0 */
    double value = 0.0;
    value += s[rec.src[0]];
    value += s[rec.src[1]];
    value *= 0.5;
    D.emf[(size_t)rec.dst_block * FX_EMF_COUNT + rec.dst] = value;
}

} /* namespace */


/* ------------------------------------------------------------------------ */
/* eSSPRK stored states (prj_timeint_eSSPRK_save_state / _blend_with_saved,  */
/* src/prj_timeint.c:2311-2444)                                              */
/* ------------------------------------------------------------------------ */

__device__ __forceinline__ double *fx_saved_w(const FxDev &D, int b, int which)
{
    return which == 1 ? D.W + (size_t)b * FX_W_COUNT(D.nv) + FX_NCELLS
                      : D.W2 + (size_t)b * D.nv * FX_NCELLS;
}

/* saved face array of direction d: stride of its faces is FX_NFACES */
__device__ __forceinline__ double *fx_saved_bf(const FxDev &D, int b, int d, int which)
{
    return which == 1 ? D.Bf + (size_t)b * FX_BF_COUNT + ((size_t)d * FX_NSTAGES + 1) * FX_NFACES
                      : D.Bf2 + ((size_t)b * 3 + d) * FX_NFACES;
}

/* W of the active cells (all variables) and every face of slot 0 */
__global__ void k_essprk_save(FxDev D, const int *__restrict__ blist, int which)
{
    if (D.ctl->skip) {
        return;
    }
    const int b = blist[blockIdx.y];
    const int nv = D.nv;
    const int ncell = FX_BS * FX_BS * FX_BS;
    const int nface = D.Bf ? 3 * FX_NFACES : 0;
    const double *W0 = D.W + (size_t)b * FX_W_COUNT(nv);
    double *Ws = fx_saved_w(D, b, which);
    const size_t wstride = which == 1 ? (size_t)FX_NSTAGES * FX_NCELLS : (size_t)FX_NCELLS;
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < nv * ncell + nface; t += gridDim.x * blockDim.x) {
        if (t < nv * ncell) {
            const int v = t / ncell;
            const int r = t - v * ncell;
            const int c = fx_lidx(r >> 8, (r >> 4) & 15, r & 15);
            Ws[(size_t)v * wstride + c] = W0[(size_t)v * kPlane + c];
        } else {
            const int q = t - nv * ncell;
            const int d = q / FX_NFACES;
            const int f = q - d * FX_NFACES;
            fx_saved_bf(D, b, d, which)[f] = D.Bf[(size_t)b * FX_BF_COUNT + (size_t)d * FX_NSTAGES * FX_NFACES + f];
        }
    }
}

/* prj_timeint_eSSPRK_blend_bf: active faces of slot 0 <- w saved + (1 - w) slot 0 */
__global__ void __launch_bounds__(128) k_essprk_blend_faces(FxDev D, const int *__restrict__ blist, int which,
    double w)
{
    if (D.ctl->skip) {
        return;
    }
    const int b = blist[blockIdx.y];
    constexpr int NF = (FX_BS + 1) * FX_BS * FX_BS;
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= 3 * NF) {
        return;
    }
    const int dir = t / NF;
    t -= dir * NF;
    const int x2 = dir == 2 ? FX_BS + 1 : FX_BS;
    const int x1 = dir == 1 ? FX_BS + 1 : FX_BS;
    const int k = t % x2;
    t /= x2;
    const int j = t % x1;
    const int i = t / x1;
    const int f = fx_face_idx(dir, i, j, k);
    const double cw = 1.0 - w;
    double *bf0 = D.Bf + (size_t)b * FX_BF_COUNT + (size_t)dir * FX_NSTAGES * FX_NFACES;
    bf0[f] = w * fx_saved_bf(D, b, dir, which)[f] + cw * bf0[f];
}

/* prj_timeint_eSSPRK_final_cell: conserved blend, field from the blended
 * faces, cons2prim into slot 0 */
template <bool MHD>
__global__ void __launch_bounds__(128) k_essprk_blend_cells(FxDev D, const int *__restrict__ blist, int which,
    double w)
{
    if (D.ctl->skip) {
        return;
    }
    const int b = blist[blockIdx.y];
    constexpr int nv = MHD ? 9 : 6;
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= FX_BS * FX_BS * FX_BS) {
        return;
    }
    const int i = t >> 8, j = (t >> 4) & 15, k = t & 15;
    const int c = fx_lidx(i, j, k);
    double *W0 = D.W + (size_t)b * FX_W_COUNT(nv);
    const double *Ws = fx_saved_w(D, b, which);
    const size_t wstride = which == 1 ? (size_t)FX_NSTAGES * FX_NCELLS : (size_t)FX_NCELLS;
    const double cw = 1.0 - w;
    double x[9], u[9], us[9];
#pragma unroll
    for (int v = 0; v < nv; ++v) x[v] = W0[(size_t)v * kPlane + c];
    fx_prim2cons<MHD>(x, u);
#pragma unroll
    for (int v = 0; v < nv; ++v) x[v] = Ws[(size_t)v * wstride + c];
    fx_prim2cons<MHD>(x, us);
#pragma unroll
    for (int v = 0; v < nv; ++v) u[v] = w * us[v] + cw * u[v];
    if (MHD) {
        /* prj_timeint_mhd_set_cons_b_from_bf (src/prj_timeint.c:498-510) on slot 0 */
        const double *bf = D.Bf + (size_t)b * FX_BF_COUNT;
        const double *b1 = bf;
        const double *b2 = bf + (size_t)1 * FX_NSTAGES * FX_NFACES;
        const double *b3 = bf + (size_t)2 * FX_NSTAGES * FX_NFACES;
        u[FX_B1] = 0.5 * (b1[fx_face_idx(0, i, j, k)] + b1[fx_face_idx(0, i + 1, j, k)]);
        u[FX_B2] = 0.5 * (b2[fx_face_idx(1, i, j, k)] + b2[fx_face_idx(1, i, j + 1, k)]);
        u[FX_B3] = 0.5 * (b3[fx_face_idx(2, i, j, k)] + b3[fx_face_idx(2, i, j, k + 1)]);
        if (!isfinite(u[FX_B1]) || !isfinite(u[FX_B2]) || !isfinite(u[FX_B3])) {
            fx_fail(D.err, FX_ERR_B_NONFINITE, b, c);
        }
    }
    fx_cons2prim<MHD>(u, x);
#pragma unroll
    for (int v = 0; v < nv; ++v) W0[(size_t)v * kPlane + c] = x[v];
}

/* ------------------------------------------------------------------------ */
/* launchers                                                                 */
/* ------------------------------------------------------------------------ */
static inline unsigned fx_blocks(int n, int tpb) { return (unsigned)((n + tpb - 1) / tpb); }

/* launch shapes of the face kernel: {threads per CTA, min CTAs per SM} */
static const int kFluxShapes[FX_FLUX_VARIANTS][2] = {{128, 4}, {128, 5}, {128, 6}, {256, 2}, {256, 3}, {64, 8}};

template <bool MHD, bool FULL, int TPB, int MINB, int RECON = FX_RECON_MC>
static void launch_flux_shape(const FxDev &D, const int *blist, int nlist, int ndir, int wslot,
    int bfslot, cudaStream_t s)
{
    const int nf = MHD ? (FX_BS + 1) * (FX_BS + 2) * (FX_BS + 2) : (FX_BS + 1) * FX_BS * FX_BS;
    const dim3 g(fx_blocks(nf, TPB), ndir, nlist);
    k_flux<MHD, FULL, TPB, MINB, RECON><<<g, TPB, 0, s>>>(D, blist, wslot, bfslot);
}

/* the autotuner's launch shapes (threads per CTA, minimum CTAs per SM) */
template <bool MHD, bool FULL, int RECON>
static void launch_flux_shapes(const FxDev &D, const int *blist, int nlist, int ndir, int wslot,
    int bfslot, int variant, cudaStream_t s)
{
    switch (variant) {
    case 1: launch_flux_shape<MHD, FULL, 128, 5, RECON>(D, blist, nlist, ndir, wslot, bfslot, s); break;
    case 2: launch_flux_shape<MHD, FULL, 128, 6, RECON>(D, blist, nlist, ndir, wslot, bfslot, s); break;
    case 3: launch_flux_shape<MHD, FULL, 256, 2, RECON>(D, blist, nlist, ndir, wslot, bfslot, s); break;
    case 4: launch_flux_shape<MHD, FULL, 256, 3, RECON>(D, blist, nlist, ndir, wslot, bfslot, s); break;
    case 5: launch_flux_shape<MHD, FULL, 64, 8, RECON>(D, blist, nlist, ndir, wslot, bfslot, s); break;
    default: launch_flux_shape<MHD, FULL, 128, 4, RECON>(D, blist, nlist, ndir, wslot, bfslot, s); break;
    }
}

/* Every reconstruction is compiled in every launch shape.  WENO-Z7 reads
 * three cells beyond each face's neighbours and exists in the
 * four-ghost-layer build only (the context rejects it elsewhere); its
 * register demand (about 180 per thread unbounded) makes the shape matter. */
template <bool MHD, bool FULL>
static void launch_flux_variant(const FxDev &D, const int *blist, int nlist, int ndir, int wslot,
    int bfslot, int variant, cudaStream_t s)
{
    if (D.recon == FX_RECON_WENO3) {
        launch_flux_shapes<MHD, FULL, FX_RECON_WENO3>(D, blist, nlist, ndir, wslot, bfslot, variant, s);
        return;
    }
#if FX_NG >= 4
    if (D.recon == FX_RECON_WENO7) {
        launch_flux_shapes<MHD, FULL, FX_RECON_WENO7>(D, blist, nlist, ndir, wslot, bfslot, variant, s);
        return;
    }
#endif
    launch_flux_shapes<MHD, FULL, FX_RECON_MC>(D, blist, nlist, ndir, wslot, bfslot, variant, s);
}

void fx_launch_flux(const FxDev &D, const int *blist, int nlist, int ndir, int wslot, int bfslot,
    int full, cudaStream_t s)
{
    if (nlist <= 0) return;
    if (D.br_mode != 0 && full && D.nv == 9 && D.recon == FX_RECON_MC) {
        /* the plain form recording or replaying its decisions */
        constexpr int nf = (FX_BS + 1) * (FX_BS + 2) * (FX_BS + 2);
        const dim3 g(fx_blocks(nf, 128), ndir, nlist);
        if (D.br_mode == 1) {
            k_flux<true, true, 128, 4, FX_RECON_MC, 1><<<g, 128, 0, s>>>(D, blist, wslot, bfslot);
        } else {
            k_flux<true, true, 128, 4, FX_RECON_MC, 2><<<g, 128, 0, s>>>(D, blist, wslot, bfslot);
        }
        return;
    }
    const int v = D.flux_variant;
    if (D.nv == 9) {
        if (full) launch_flux_variant<true, true>(D, blist, nlist, ndir, wslot, bfslot, v, s);
        else launch_flux_variant<true, false>(D, blist, nlist, ndir, wslot, bfslot, v, s);
    } else {
        if (full) launch_flux_variant<false, true>(D, blist, nlist, ndir, wslot, bfslot, v, s);
        else launch_flux_variant<false, false>(D, blist, nlist, ndir, wslot, bfslot, v, s);
    }
}

void fx_flux_shape(int variant, int *tpb, int *minb)
{
    const int v = variant >= 0 && variant < FX_FLUX_VARIANTS ? variant : 0;
    *tpb = kFluxShapes[v][0];
    *minb = kFluxShapes[v][1];
}

/* ------------------------------------------------------------------------ */
/* Dump payloads (prj_io_write_dump, src/prj_io.c:1994-2330)                */
/* ------------------------------------------------------------------------ */
/* The rows of the dump's Data, Eos and Bf datasets for the listed blocks,
 * packed per list position q at out + q * row: Data [v][cell] (stage slot 0
 * of W, cell = (i * 16 + j) * 16 + k over the active cells), Eos [v][cell]
 * (p, T, gamma from eosvar), then, when faces is set, Bf [d][face] (stage
 * slot 0, all faces). */
__global__ void __launch_bounds__(256) k_dump_pack(FxDev D, const int *__restrict__ blist, int faces,
    double *__restrict__ out)
{
    constexpr int NC = FX_BS * FX_BS * FX_BS;
    const int nv = D.nv;
    const size_t row = (size_t)(nv + 3) * NC + (faces ? (size_t)3 * FX_NFACES : 0);
    const int b = blist[blockIdx.y];
    double *o = out + (size_t)blockIdx.y * row;
    for (size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x; t < row; t += (size_t)gridDim.x * blockDim.x) {
        if (t < (size_t)(nv + 3) * NC) {
            const int v = (int)(t / NC);
            const int r = (int)(t - (size_t)v * NC);
            const int i = r / (FX_BS * FX_BS), j = (r / FX_BS) % FX_BS, k = r % FX_BS;
            if (v < nv) {
                o[t] = D.W[(size_t)b * FX_W_COUNT(nv) + (size_t)v * FX_NSTAGES * FX_NCELLS + fx_lidx(i, j, k)];
            } else {
                o[t] = D.eos[(size_t)b * FX_EOS_COUNT + fx_bidx(3, v - nv, i, j, k)];
            }
        } else {
            const size_t u = t - (size_t)(nv + 3) * NC;
            const int d = (int)(u / FX_NFACES);
            const int n = (int)(u - (size_t)d * FX_NFACES);
            o[t] = D.Bf[(size_t)b * FX_BF_COUNT + (size_t)d * FX_NSTAGES * FX_NFACES + n];
        }
    }
}

void fx_launch_dump_pack(const FxDev &D, const int *blist, int nlist, int faces, double *out, cudaStream_t s)
{
    if (nlist <= 0) return;
    k_dump_pack<<<dim3(64, nlist), 256, 0, s>>>(D, blist, faces, out);
}

/* ------------------------------------------------------------------------ */
/* Active-region state transfers: the cell-centred field after an upload    */
/* ------------------------------------------------------------------------ */
/* The cell-centred field of the listed blocks' active cells from their
 * faces, stage slot 0: prj_mhd_bf2bc_impl's arithmetic (src/prj_mhd.c:
 * 585-590; the metric factor is 1 outside dynamical GR) */
__global__ void __launch_bounds__(256) k_cell_field_active(FxDev D, const int *__restrict__ blist)
{
    constexpr int NC = FX_BS * FX_BS * FX_BS;
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= NC) {
        return;
    }
    const int b = blist[blockIdx.y];
    const int i = t / (FX_BS * FX_BS), j = (t / FX_BS) % FX_BS, k = t % FX_BS;
    const double *bf = D.Bf + (size_t)b * FX_BF_COUNT;
    const double *f1 = bf;
    const double *f2 = bf + (size_t)FX_NSTAGES * FX_NFACES;
    const double *f3 = bf + (size_t)2 * FX_NSTAGES * FX_NFACES;
    const double b1 = 0.5 * (f1[fx_face_idx(0, i, j, k)] + f1[fx_face_idx(0, i + 1, j, k)]);
    const double b2 = 0.5 * (f2[fx_face_idx(1, i, j, k)] + f2[fx_face_idx(1, i, j + 1, k)]);
    const double b3 = 0.5 * (f3[fx_face_idx(2, i, j, k)] + f3[fx_face_idx(2, i, j, k + 1)]);
    if (!isfinite(b1) || !isfinite(b2) || !isfinite(b3)) {
        fx_fail(D.err, FX_ERR_B_NONFINITE, b, fx_lidx(i, j, k));
    }
    double *w = D.W + (size_t)b * FX_W_COUNT(9) + fx_lidx(i, j, k);
    w[(size_t)FX_B1 * FX_NSTAGES * FX_NCELLS] = b1;
    w[(size_t)FX_B2 * FX_NSTAGES * FX_NCELLS] = b2;
    w[(size_t)FX_B3 * FX_NSTAGES * FX_NCELLS] = b3;
}

void fx_launch_cell_field_active(const FxDev &D, const int *blist, int nlist, cudaStream_t s)
{
    if (nlist <= 0) return;
    constexpr int NC = FX_BS * FX_BS * FX_BS;
    k_cell_field_active<<<dim3(fx_blocks(NC, 256), nlist), 256, 0, s>>>(D, blist);
}

void fx_launch_emf(const FxDev &D, const int *blist, int nlist, int wslot, int bfslot, cudaStream_t s)
{
    if (nlist <= 0) return;
    if (nlist < 16) {
        const int ne = 3 * FX_BS * (FX_BS + 1) * (FX_BS + 1);
        k_emf_edges<<<dim3(fx_blocks(ne, 128), nlist), 128, 0, s>>>(D, blist, wslot, bfslot);
        return;
    }
    k_emf<<<dim3(kEmfChunks, nlist), 256, 0, s>>>(D, blist, wslot, bfslot);
}

void fx_launch_bf_update(const FxDev &D, const int *blist, int nlist, int stage, cudaStream_t s)
{
    if (nlist <= 0) return;
    const int nf = (FX_BS + 1) * FX_BS * FX_BS;
    k_bf_update<<<dim3(fx_blocks(nf, 128), 3, nlist), 128, 0, s>>>(D, blist, stage);
}

void fx_launch_cell_update(const FxDev &D, const int *blist, int nlist, int stage,
    int gravity, int store_rhs, cudaStream_t s)
{
    if (nlist <= 0) return;
    const dim3 grid(fx_blocks(FX_BS * FX_BS * FX_BS, 128), nlist);
    if (D.nv == 9) {
        if (stage == 1) k_cell_update<true, 1><<<grid, 128, 0, s>>>(D, blist, gravity, store_rhs);
        else if (stage == 2) k_cell_update<true, 2><<<grid, 128, 0, s>>>(D, blist, gravity, store_rhs);
        else k_cell_update<true, 0><<<grid, 128, 0, s>>>(D, blist, gravity, store_rhs);
    } else {
        if (stage == 1) k_cell_update<false, 1><<<grid, 128, 0, s>>>(D, blist, gravity, store_rhs);
        else if (stage == 2) k_cell_update<false, 2><<<grid, 128, 0, s>>>(D, blist, gravity, store_rhs);
        else k_cell_update<false, 0><<<grid, 128, 0, s>>>(D, blist, gravity, store_rhs);
    }
}

void fx_launch_eos_fill(const FxDev &D, const int *blist, int nlist, int wslot, int active_only,
    cudaStream_t s)
{
    if (nlist <= 0) return;
    const int n = active_only ? FX_BS * FX_BS * FX_BS : FX_NCELLS;
    k_eos_fill<<<dim3(fx_blocks(n, 256), nlist), 256, 0, s>>>(D, blist, wslot, active_only);
}

void fx_launch_calc_dt(const FxDev &D, const int *blist, int nlist, int wslot, double cfl,
    cudaStream_t s)
{
    if (nlist <= 0) return;
    k_calc_dt<<<dim3(fx_blocks(FX_BS * FX_BS * FX_BS, 256), nlist), 256, 0, s>>>(D, blist, wslot, cfl);
}

void fx_launch_ghost_wave(const FxDev &D, const FxGop *cops, int nc, const FxGop *fops, int nf,
    const FxPop *pops, int np, const FxBop *bops, int nb, int slot, int nvg, cudaStream_t s)
{
    /* the operations of a wave are conflict free: the two launches may run
     * in either order */
    const unsigned grid = fx_blocks(nc, 256) + fx_blocks(nf, 256 * FX_GW_FACE_OPS) + fx_blocks(nb, 256);
    if (grid > 0) {
        if (D.use_bj) {
            k_ghost_wave<true><<<grid, 256, 0, s>>>(D, cops, nc, fops, nf, bops, nb, slot, nvg);
        } else {
            k_ghost_wave<false><<<grid, 256, 0, s>>>(D, cops, nc, fops, nf, bops, nb, slot, nvg);
        }
    }
    if (np > 0) {
        k_ghost_groups<<<fx_blocks(np, 128), 128, 0, s>>>(D, pops, np, slot);
    }
}

void fx_launch_xpack(const FxDev &D, const FxXent *ents, int n, double *buf, int slot, cudaStream_t s)
{
    if (n > 0) k_xpack<<<fx_blocks(n, 256), 256, 0, s>>>(D, ents, n, buf, slot);
}

void fx_launch_xunpack(const FxDev &D, const FxXent *ents, int n, const double *buf, int slot, cudaStream_t s)
{
    if (n > 0) k_xunpack<<<fx_blocks(n, 256), 256, 0, s>>>(D, ents, n, buf, slot);
}

void fx_launch_prolong_groups(const FxDev &D, const FxPop *pops, int np, int slot, cudaStream_t s)
{
    if (np > 0) {
        k_ghost_groups<<<fx_blocks(np, 128), 128, 0, s>>>(D, pops, np, slot);
    }
}

void fx_launch_flux_correct(const FxDev &D, const FxCorr *recs, int n, int ncomp, cudaStream_t s)
{
    if (n <= 0) return;
    k_flux_correct<<<fx_blocks(n * ncomp, 256), 256, 0, s>>>(D, recs, n, ncomp);
}

void fx_launch_emf_correct(const FxDev &D, const FxCorr *recs, int n, cudaStream_t s)
{
    if (n <= 0) return;
    k_emf_correct<<<fx_blocks(n, 256), 256, 0, s>>>(D, recs, n);
}

void fx_launch_reset_reductions(const FxDev &D, int which, cudaStream_t s)
{
    k_reset_reductions<<<1, 1, 0, s>>>(D, which);
}

void fx_launch_step_begin(const FxDev &D, cudaStream_t s)
{
    k_step_begin<<<1, 1, 0, s>>>(D);
}

void fx_launch_step_end(const FxDev &D, cudaStream_t s)
{
    k_step_end<<<1, 1, 0, s>>>(D);
}

namespace {
__global__ void k_set_dt(FxDev D, double dt)
{
    D.ctl->dt = dt;
    D.ctl->dt_stage = dt;
    D.ctl->skip = 0;
}

__global__ void k_stage_dt(FxDev D, double divisor)
{
    D.ctl->dt_stage = D.ctl->dt / divisor;
}

__global__ void k_set_ctl(FxDev D, FxCtl v)
{
    *D.ctl = v;
}
}

void fx_launch_set_dt(const FxDev &D, double dt, cudaStream_t s)
{
    k_set_dt<<<1, 1, 0, s>>>(D, dt);
}

void fx_launch_stage_dt(const FxDev &D, double divisor, cudaStream_t s)
{
    k_stage_dt<<<1, 1, 0, s>>>(D, divisor);
}

void fx_launch_essprk_save(const FxDev &D, const int *blist, int nlist, int which, cudaStream_t s)
{
    if (nlist <= 0) return;
    k_essprk_save<<<dim3(32, nlist), 256, 0, s>>>(D, blist, which);
}

void fx_launch_essprk_blend(const FxDev &D, const int *blist, int nlist, int which, double w, cudaStream_t s)
{
    if (nlist <= 0) return;
    if (D.nv == 9) {
        const int nf = 3 * (FX_BS + 1) * FX_BS * FX_BS;
        k_essprk_blend_faces<<<dim3(fx_blocks(nf, 128), nlist), 128, 0, s>>>(D, blist, which, w);
        k_essprk_blend_cells<true><<<dim3(fx_blocks(FX_BS * FX_BS * FX_BS, 128), nlist), 128, 0, s>>>(
            D, blist, which, w);
    } else {
        k_essprk_blend_cells<false><<<dim3(fx_blocks(FX_BS * FX_BS * FX_BS, 128), nlist), 128, 0, s>>>(
            D, blist, which, w);
    }
}

void fx_launch_set_ctl(const FxDev &D, FxCtl value, cudaStream_t s)
{
    k_set_ctl<<<1, 1, 0, s>>>(D, value);
}
