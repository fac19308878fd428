/*
 * Dynamic AMR, device half: the per-cell refinement vote of prj_amr_tag and
 * the data moves of prj_amr_adapt (prolongation onto new children,
 * restriction onto re-activated parents), each in the reference's double
 * operation order (compiled with --fmad=false):
 *
 *   k_amr_tag             prj_amr_tag pass 1, src/prj_amr.c:1611-1705, with the
 *                         estimators of src/prj_amr.c:930-1221
 *   k_amr_zero            prj_zero_block_arrays, src/prj_amr.c:220-233
 *   k_amr_copy_faces      the finer-neighbour face copies of
 *                         prj_amr_mhd_prolongate_bf_one, src/prj_amr.c:2000-2083
 *   (groups)              prj_mhd_prolong_bf_from_buffer through the ghost
 *                         fill's Toth-Roe group kernel
 *   k_amr_prolong_cells   prj_amr_prolongate, src/prj_amr.c:2239-2308, then
 *                         prj_amr_mhd_set_cons_b_from_bf (:1871-1913) and
 *                         prj_sync_primitive_from_conserved (:1399-1435)
 *   k_amr_restrict_faces  prj_amr_mhd_restrict_bf, src/prj_amr.c:2152-2237
 *   k_amr_restrict_cells  prj_amr_restrict, src/prj_amr.c:2310-2387, then the
 *                         same field and primitive sync
 *
 * The tag runs one CTA per block and reduces its votes in shared memory;
 * the prolongation stages the parent's conserved octant (10^3 cells with
 * the stencil halo) in shared memory, one CTA per child; the restriction
 * replays the reference's overlap loops per parent cell, one CTA per
 * (parent, i plane).
 */
#include <cuda_runtime.h>

#include "fx_kernels.h"
#include "fx_physics.cuh"

namespace {

constexpr int kPlane = FX_NSTAGES * FX_NCELLS;

__device__ __forceinline__ int clampi(int i)
{
    return i < -FX_NG ? -FX_NG : (i >= FX_BS + FX_NG ? FX_BS + FX_NG - 1 : i);
}

/* ------------------------------------------------------------------------ */
/* tag                                                                       */
/* ------------------------------------------------------------------------ */

/* one block's view for the estimators; eosvar values are those of the
 * ideal-gas fill (pressure, temperature, gamma) recomputed from W slot 0 */
template <bool MHD>
struct TagView {
    const double *W;
    const double *g;
    double gamma;
    double dx[3];

    /* prj_block_primitive_at (src/prj_amr.c:724-730): clamped */
    __device__ double prim(int v, int i, int j, int k) const
    {
        return W[(size_t)v * kPlane + fx_lidx(clampi(i), clampi(j), clampi(k))];
    }
    /* prj_amr_total_pressure_non_gr_at (src/prj_amr.c:805-819): unclamped */
    __device__ double ptot(int i, int j, int k) const
    {
        const int c = fx_lidx(i, j, k);
        double p = fx_pressure(gamma, W[c], W[(size_t)FX_EINT * kPlane + c]);
        if (MHD) {
            const double b1 = W[(size_t)FX_B1 * kPlane + c];
            const double b2 = W[(size_t)FX_B2 * kPlane + c];
            const double b3 = W[(size_t)FX_B3 * kPlane + c];
            p += 0.5 * (b1 * b1 + b2 * b2 + b3 * b3);
        }
        return p;
    }
    /* prj_loehner_cell_value (src/prj_amr.c:930-942) */
    __device__ double lohner_value(int var, int i, int j, int k) const
    {
        if (var == 0) return prim(FX_RHO, i, j, k);
        if (var == 2) return fx_temperature(gamma, W[(size_t)FX_EINT * kPlane + fx_lidx(i, j, k)]);
        return ptot(i, j, k);
    }
    /* prj_loehner_cell_indicator (src/prj_amr.c:944-1005) */
    __device__ double lohner(int var, double eps, int i, int j, int k) const
    {
        const double u0 = lohner_value(var, i, j, k);
        const double uxm = lohner_value(var, i - 1, j, k);
        const double uxp = lohner_value(var, i + 1, j, k);
        const double uym = lohner_value(var, i, j - 1, k);
        const double uyp = lohner_value(var, i, j + 1, k);
        const double uzm = lohner_value(var, i, j, k - 1);
        const double uzp = lohner_value(var, i, j, k + 1);
        const double num_x = uxp - 2.0 * u0 + uxm;
        const double num_y = uyp - 2.0 * u0 + uym;
        const double num_z = uzp - 2.0 * u0 + uzm;
        const double num_xy = 0.25 * (lohner_value(var, i + 1, j + 1, k) - lohner_value(var, i + 1, j - 1, k) -
            lohner_value(var, i - 1, j + 1, k) + lohner_value(var, i - 1, j - 1, k));
        const double num_xz = 0.25 * (lohner_value(var, i + 1, j, k + 1) - lohner_value(var, i + 1, j, k - 1) -
            lohner_value(var, i - 1, j, k + 1) + lohner_value(var, i - 1, j, k - 1));
        const double num_yz = 0.25 * (lohner_value(var, i, j + 1, k + 1) - lohner_value(var, i, j + 1, k - 1) -
            lohner_value(var, i, j - 1, k + 1) + lohner_value(var, i, j - 1, k - 1));
        const double den_x = fabs(uxp - u0) + fabs(u0 - uxm) + eps * (fabs(uxp) + 2.0 * fabs(u0) + fabs(uxm));
        const double den_y = fabs(uyp - u0) + fabs(u0 - uym) + eps * (fabs(uyp) + 2.0 * fabs(u0) + fabs(uym));
        const double den_z = fabs(uzp - u0) + fabs(u0 - uzm) + eps * (fabs(uzp) + 2.0 * fabs(u0) + fabs(uzm));
        const double numerator = num_x * num_x + num_y * num_y + num_z * num_z +
            2.0 * (num_xy * num_xy + num_xz * num_xz + num_yz * num_yz);
        const double denominator = den_x * den_x + den_y * den_y + den_z * den_z + 1.0e-14;
        return sqrt(numerator / denominator);
    }
    /* prj_block_sound_speed_at (src/prj_amr.c:840-862) */
    __device__ double sound_speed(int i, int j, int k) const
    {
        const double rho = prim(FX_RHO, i, j, k);
        const double eint = prim(FX_EINT, i, j, k);
        if (rho <= 0.0 || eint < 0.0) return 0.0;
        const double p = ptot(i, j, k);
        if (p <= 0.0 || gamma <= 0.0) return 0.0;
        return sqrt(gamma * p / rho);
    }
    /* prj_velocity_cell_indicator (src/prj_amr.c:1007-1038) */
    __device__ double velocity(int i, int j, int k) const
    {
        const double v1 = prim(FX_V1, i, j, k);
        const double v2 = prim(FX_V2, i, j, k);
        const double v3 = prim(FX_V3, i, j, k);
        const double cs = sound_speed(i, j, k);
        double m = 0.0;
        for (int axis = 0; axis < 3; ++axis) {
            for (int side = -1; side <= 1; side += 2) {
                const int di = axis == 0 ? side : 0;
                const int dj = axis == 1 ? side : 0;
                const int dk = axis == 2 ? side : 0;
                const double dv1 = v1 - prim(FX_V1, i + di, j + dj, k + dk);
                const double dv2 = v2 - prim(FX_V2, i + di, j + dj, k + dk);
                const double dv3 = v3 - prim(FX_V3, i + di, j + dj, k + dk);
                const double dv = sqrt(dv1 * dv1 + dv2 * dv2 + dv3 * dv3) / (cs + 1.0e-14);
                m = m > dv ? m : dv;
            }
        }
        return m;
    }
    /* prj_pressure_scale_height_cell_indicator, non-GR branch (src/prj_amr.c:1065-1144) */
    __device__ double scale_height(int i, int j, int k) const
    {
        if (g == nullptr) return 0.0;
        const int c = fx_lidx(i, j, k);
        const double rho = prim(FX_RHO, i, j, k);
        const double p = ptot(i, j, k);
        const double g1 = g[c];
        const double g2 = g[FX_NCELLS + c];
        const double g3 = g[2 * FX_NCELLS + c];
        const double accel = sqrt(g1 * g1 + g2 * g2 + g3 * g3);
        double cell = dx[0];
        if (dx[1] > cell) cell = dx[1];
        if (dx[2] > cell) cell = dx[2];
        if (rho <= 0.0 || p <= 0.0 || accel <= 0.0) return 0.0;
        const double hp = p / (rho * accel);
        if (hp <= 0.0) return 0.0;
        return cell / hp;
    }
    /* prj_fractional_jump_cell_indicator (src/prj_amr.c:1146-1202) */
    __device__ double jump_value(int var, int i, int j, int k) const
    {
        return var == 1 ? ptot(i, j, k) : W[fx_lidx(i, j, k)];
    }
    __device__ double jump(int var, int i, int j, int k) const
    {
        const double q0 = jump_value(var, i, j, k);
        double m = 0.0;
        if (q0 <= 0.0) return 0.0;
        for (int di = -1; di <= 1; ++di) {
            for (int dj = -1; dj <= 1; ++dj) {
                for (int dk = -1; dk <= 1; ++dk) {
                    if (di == 0 && dj == 0 && dk == 0) continue;
                    const double q = jump_value(var, i + di, j + dj, k + dk);
                    if (q <= 0.0) continue;
                    const double den = q0 < q ? q0 : q;
                    const double jv = fabs(q0 - q) / (den + 1.0e-14);
                    m = m > jv ? m : jv;
                }
            }
        }
        return m;
    }
    /* prj_amr_cell_indicator_for_estimator (src/prj_amr.c:1204-1221) */
    __device__ double indicator(const FxAmrTagCfg &cfg, int n, int i, int j, int k) const
    {
        switch (cfg.est[n]) {
        case 3: return jump(cfg.var[n], i, j, k);
        case 2: return scale_height(i, j, k);
        case 1: return velocity(i, j, k);
        default: return lohner(cfg.var[n], cfg.eps[n], i, j, k);
        }
    }
};

/* prj_amr_refine_boundary_mask_for_cell (src/prj_amr.c:120-144), buffer zone 2 */
__device__ __forceinline__ unsigned cell_mask(int i, int j, int k)
{
    unsigned m = 0u;
    if (i < 2) m |= 1u;
    if (i >= FX_BS - 2) m |= 2u;
    if (j < 2) m |= 4u;
    if (j >= FX_BS - 2) m |= 8u;
    if (k < 2) m |= 16u;
    if (k >= FX_BS - 2) m |= 32u;
    return m;
}

/* Pass 1 of prj_amr_tag for one block per CTA.  The reference's early exits
 * (cells skipped once the block votes to refine, the derefine scan stopped
 * at the first keeping cell) do not change the refine vote or the mask; the
 * derefine vote only matters for blocks that do not vote to refine. */
template <bool MHD>
__global__ void __launch_bounds__(256) k_amr_tag(FxDev D, const int *__restrict__ list,
    const int *__restrict__ has_parent, FxAmrTagCfg cfg, int32_t *__restrict__ votes)
{
    __shared__ unsigned s_mask;
    const int b = list[blockIdx.x];
    if (threadIdx.x == 0) s_mask = 0u;
    TagView<MHD> t;
    t.W = D.W + (size_t)b * FX_W_COUNT(D.nv);
    t.g = D.grav ? D.grav + (size_t)b * FX_GRAV_COUNT : nullptr;
    t.gamma = D.gamma;
    for (int a = 0; a < 3; ++a) t.dx[a] = D.blk[b].dx[a];
    __syncthreads();

    int refine = 0;
    int reach = 0;
    unsigned mask = 0u;
    for (int c = threadIdx.x; c < FX_BS * FX_BS * FX_BS; c += blockDim.x) {
        const int i = c >> 8, j = (c >> 4) & 15, k = c & 15;
        const unsigned cm = cell_mask(i, j, k);
        int hit = 0;
        if (cfg.reach > 0.0 && t.W[fx_lidx(i, j, k)] > cfg.reach) {
            hit = 1;
            reach = 1;
        }
        double sum = 0.0;
        for (int n = 0; n < cfg.ncrit; ++n) {
            if (cfg.rthr[n] <= 0.0) continue;
            sum += t.indicator(cfg, n, i, j, k) / cfg.rthr[n];
        }
        if (sum > 1.0) hit = 1;
        if (hit) {
            refine = 1;
            mask |= cm;
        }
    }
    if (mask) atomicOr(&s_mask, mask);
    refine = __syncthreads_or(refine);
    reach = __syncthreads_or(reach);

    int keep = 0;
    const bool scan = has_parent[blockIdx.x] && cfg.has_derefine && !reach;
    if (scan) {
        for (int c = threadIdx.x; c < 18 * 18 * 18 && !keep; c += blockDim.x) {
            const int i = c / 324 - 1, j = (c / 18) % 18 - 1, k = c % 18 - 1;
            double sum = 0.0;
            for (int n = 0; n < cfg.ncrit; ++n) {
                if (cfg.dthr[n] <= 0.0) continue;
                sum += t.indicator(cfg, n, i, j, k) / cfg.dthr[n];
            }
            if (sum >= 1.0) keep = 1;
        }
    }
    keep = __syncthreads_or(keep);
    if (threadIdx.x == 0) {
        votes[3 * blockIdx.x] = refine;
        votes[3 * blockIdx.x + 1] = (scan && !keep) ? -1 : 0;
        votes[3 * blockIdx.x + 2] = (int32_t)s_mask;
    }
}

/* ------------------------------------------------------------------------ */
/* remesh data moves                                                         */
/* ------------------------------------------------------------------------ */

__global__ void k_amr_zero(FxDev D, const int *__restrict__ blocks)
{
    const int b = blocks[blockIdx.y];
    const size_t nw = (size_t)FX_W_COUNT(D.nv);
    const size_t nbf = D.Bf ? (size_t)FX_BF_COUNT : 0;
    const size_t ne = (size_t)FX_EOS_COUNT;
    const size_t ng = D.grav ? (size_t)FX_GRAV_COUNT : 0;
    const size_t nw2 = D.W2 ? (size_t)D.nv * FX_NCELLS : 0;
    const size_t nb2 = D.Bf2 ? (size_t)3 * FX_NFACES : 0;
    const size_t total = nw + nbf + ne + ng + nw2 + nb2;
    for (size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x; e < total; e += (size_t)gridDim.x * blockDim.x) {
        size_t q = e;
        if (q < nw) {
            D.W[(size_t)b * nw + q] = 0.0;
            continue;
        }
        q -= nw;
        if (q < nbf) {
            D.Bf[(size_t)b * FX_BF_COUNT + q] = 0.0;
            continue;
        }
        q -= nbf;
        if (q < ne) {
            D.eos[(size_t)b * FX_EOS_COUNT + q] = 0.0;
            continue;
        }
        q -= ne;
        if (q < ng) {
            D.grav[(size_t)b * FX_GRAV_COUNT + q] = 0.0;
            continue;
        }
        q -= ng;
        if (q < nw2) {
            D.W2[(size_t)b * nw2 + q] = 0.0;
            continue;
        }
        q -= nw2;
        D.Bf2[(size_t)b * nb2 + q] = 0.0;
    }
}

/* 16 x 16 faces of one layer, both slots (prj_boundary_write_bf_face with
 * fidelity SAME onto cleared faces always writes) */
__global__ void __launch_bounds__(256) k_amr_copy_faces(FxDev D, const FxAmrCopyJob *__restrict__ jobs)
{
    const FxAmrCopyJob J = jobs[blockIdx.x];
    const int slot = blockIdx.y;
    const int t0 = (J.dir + 1) % 3;
    const int t1 = (J.dir + 2) % 3;
    const int i = threadIdx.x >> 4;
    const int j = threadIdx.x & 15;
    int src[3], dst[3];
    src[J.dir] = J.side ? 0 : FX_BS;
    dst[J.dir] = J.side ? FX_BS : 0;
    src[t0] = dst[t0] = i;
    src[t1] = dst[t1] = j;
    const double v = D.Bf[(size_t)J.src * FX_BF_COUNT + ((size_t)J.dir * FX_NSTAGES + slot) * FX_NFACES +
        fx_face_idx(J.dir, src[0], src[1], src[2])];
    const int df = fx_face_idx(J.dir, dst[0], dst[1], dst[2]);
    if (!isfinite(v)) fx_fail(D.err, FX_ERR_AMR_NONFINITE, J.child, df);
    D.Bf[(size_t)J.child * FX_BF_COUNT + ((size_t)J.dir * FX_NSTAGES + slot) * FX_NFACES + df] = v;
}

/* cell-centred field from the faces of slot 0 (prj_amr_mhd_set_cons_b_from_bf) */
__device__ __forceinline__ void face_average(const FxDev &D, int b, int i, int j, int k, double out[3])
{
    const double *bf = D.Bf + (size_t)b * FX_BF_COUNT;
    const double *b1 = bf + (size_t)(0 * FX_NSTAGES) * FX_NFACES;
    const double *b2 = bf + (size_t)(1 * FX_NSTAGES) * FX_NFACES;
    const double *b3 = bf + (size_t)(2 * FX_NSTAGES) * FX_NFACES;
    out[0] = 0.5 * (b1[fx_face_idx(0, i, j, k)] + b1[fx_face_idx(0, i + 1, j, k)]);
    out[1] = 0.5 * (b2[fx_face_idx(1, i, j, k)] + b2[fx_face_idx(1, i, j + 1, k)]);
    out[2] = 0.5 * (b3[fx_face_idx(2, i, j, k)] + b3[fx_face_idx(2, i, j, k + 1)]);
}

/* the tail shared by prolongation and restriction: field from faces, then
 * prj_sync_primitive_from_conserved with prj_apply_eint_floor
 * (src/prj_amr.c:872-928) */
template <bool MHD>
__device__ __forceinline__ void store_cell(const FxDev &D, int b, int i, int j, int k, double *u,
    double E_floor, double *inj)
{
    double *W = D.W + (size_t)b * FX_W_COUNT(D.nv);
    const int c = fx_lidx(i, j, k);
    if (MHD) {
        double bc[3];
        face_average(D, b, i, j, k, bc);
        if (!isfinite(bc[0]) || !isfinite(bc[1]) || !isfinite(bc[2])) {
            fx_fail(D.err, FX_ERR_AMR_NONFINITE, b, c);
        }
        u[FX_B1] = bc[0];
        u[FX_B2] = bc[1];
        u[FX_B3] = bc[2];
        W[(size_t)FX_B1 * kPlane + FX_NCELLS + c] = bc[0];
        W[(size_t)FX_B2 * kPlane + FX_NCELLS + c] = bc[1];
        W[(size_t)FX_B3 * kPlane + FX_NCELLS + c] = bc[2];
    }
    double w[FX_MAXVAR];
    fx_cons2prim<MHD>(u, w);
    double added = 0.0;
    if (E_floor > 0.0 && w[FX_RHO] > 0.0 && !(w[FX_EINT] >= E_floor)) {
        const double kinetic = 0.5 * (w[FX_V1] * w[FX_V1] + w[FX_V2] * w[FX_V2] + w[FX_V3] * w[FX_V3]);
        const double etot_old = u[FX_ETOT];
        double etot_new = w[FX_RHO] * (E_floor + kinetic);
        if (MHD) {
            const double magnetic = 0.5 * (w[FX_B1] * w[FX_B1] + w[FX_B2] * w[FX_B2] + w[FX_B3] * w[FX_B3]);
            etot_new = etot_new + magnetic;
        }
        w[FX_EINT] = E_floor;
        added = (etot_new - etot_old) * D.blk[b].vol;
    }
    if (inj != nullptr) inj[(i * FX_BS + j) * FX_BS + k] = added;
    for (int v = 0; v < (MHD ? 9 : 6); ++v) {
        W[(size_t)v * kPlane + c] = w[v];
    }
}

/* conserved prolongation: the parent's octant plus one halo cell (10^3) as
 * conserved variables in shared memory, then per child cell the minmod
 * prolongation of prj_reconstruct_cell_for_prolongate_minmod
 * (src/prj_reconstruct.h:111-143), or with use_BJ the Barth-Jespersen one
 * (:145-195) on the 27-cell stencil, the density guard, the face-average
 * field and the primitive sync */
template <bool MHD>
__global__ void __launch_bounds__(256) k_amr_prolong_cells(FxDev D, const FxAmrChildJob *__restrict__ jobs,
    double E_floor, double *inj)
{
    constexpr int NV = MHD ? 9 : 6;
    constexpr int R = 10;
    extern __shared__ double sU[]; /* [NV][R^3] */
    const FxAmrChildJob J = jobs[blockIdx.x];
    const int xo = J.oct & 1, yo = (J.oct >> 1) & 1, zo = (J.oct >> 2) & 1;
    const int o[3] = {xo * 8 - 1, yo * 8 - 1, zo * 8 - 1};
    const double *Wp = D.W + (size_t)J.parent * FX_W_COUNT(D.nv);
    for (int r = threadIdx.x; r < R * R * R; r += blockDim.x) {
        const int ri = r / (R * R), rj = (r / R) % R, rk = r % R;
        const int c = fx_lidx(clampi(o[0] + ri), clampi(o[1] + rj), clampi(o[2] + rk));
        double w[FX_MAXVAR], u[FX_MAXVAR];
        for (int v = 0; v < NV; ++v) w[v] = Wp[(size_t)v * kPlane + c];
        fx_prim2cons<MHD>(w, u);
        for (int v = 0; v < NV; ++v) sU[v * R * R * R + r] = u[v];
    }
    __syncthreads();
    double *injb = (inj != nullptr && E_floor > 0.0) ? inj + (size_t)blockIdx.x * FX_BS * FX_BS * FX_BS : nullptr;
    for (int t = threadIdx.x; t < FX_BS * FX_BS * FX_BS; t += blockDim.x) {
        const int i = t >> 8, j = (t >> 4) & 15, k = t & 15;
        const int gi = xo * FX_BS + i, gj = yo * FX_BS + j, gk = zo * FX_BS + k;
        const int r = ((gi / 2 - o[0]) * R + (gj / 2 - o[1])) * R + (gk / 2 - o[2]);
        const double tx = (gi % 2) == 0 ? -0.25 : 0.25;
        const double ty = (gj % 2) == 0 ? -0.25 : 0.25;
        const double tz = (gk % 2) == 0 ? -0.25 : 0.25;
        double u[FX_MAXVAR];
        for (int v = 0; v < NV; ++v) {
            const double *q = sU + v * R * R * R;
            if (D.use_bj) {
                const double *qr = q + r;
                u[v] = fx_bj_cell([qr](int di, int dj, int dk) { return qr[(di * R + dj) * R + dk]; }, tx, ty, tz);
                continue;
            }
            const double base = q[r];
            const double vx = base + fx_minmod_slope(q[r - R * R], base, q[r + R * R]) * tx;
            const double vy = base + fx_minmod_slope(q[r - R], base, q[r + R]) * ty;
            const double vz = base + fx_minmod_slope(q[r - 1], base, q[r + 1]) * tz;
            u[v] = vx + vy + vz - 2.0 * base;
        }
        if (u[FX_RHO] <= 0.0) u[FX_RHO] = 1.0e-10;
        store_cell<MHD>(D, J.child, i, j, k, u, E_floor, injb);
    }
}

/* prj_amr_mhd_face_bit / _face_local_index (src/prj_amr.c:2130-2150) */
__device__ __forceinline__ int face_bit(int g) { return g <= FX_BS ? 0 : 1; }
__device__ __forceinline__ int face_local(int g) { return g <= FX_BS ? g : g - FX_BS; }

/* one (parent, slot, dir) per CTA: clear the slot's faces, then write the
 * active faces as 0.25 times the sum of the four child faces in the
 * reference's order */
__global__ void __launch_bounds__(256) k_amr_restrict_faces(FxDev D, const FxAmrParentJob *__restrict__ jobs)
{
    const FxAmrParentJob J = jobs[blockIdx.z];
    const int slot = blockIdx.y;
    const int dir = blockIdx.x;
    double *dst = D.Bf + (size_t)J.parent * FX_BF_COUNT + ((size_t)dir * FX_NSTAGES + slot) * FX_NFACES;
    for (int f = threadIdx.x; f < FX_NFACES; f += blockDim.x) dst[f] = 0.0;
    __syncthreads();
    const int t0 = (dir + 1) % 3;
    const int t1 = (dir + 2) % 3;
    const int n0 = dir == 0 ? FX_BS + 1 : FX_BS;
    const int n1 = dir == 1 ? FX_BS + 1 : FX_BS;
    const int n2 = dir == 2 ? FX_BS + 1 : FX_BS;
    for (int f = threadIdx.x; f < n0 * n1 * n2; f += blockDim.x) {
        const int ci[3] = {f / (n1 * n2), (f / n2) % n1, f % n2};
        double sum = 0.0;
        for (int a = 0; a < 2; ++a) {
            for (int bb = 0; bb < 2; ++bb) {
                int g[3] = {2 * ci[0], 2 * ci[1], 2 * ci[2]};
                g[t0] += a;
                g[t1] += bb;
                int bit[3], loc[3];
                bit[dir] = face_bit(g[dir]);
                loc[dir] = face_local(g[dir]);
                bit[t0] = g[t0] / FX_BS;
                bit[t1] = g[t1] / FX_BS;
                loc[t0] = g[t0] - bit[t0] * FX_BS;
                loc[t1] = g[t1] - bit[t1] * FX_BS;
                const int child = J.children[bit[0] + 2 * bit[1] + 4 * bit[2]];
                const double v = D.Bf[(size_t)child * FX_BF_COUNT + ((size_t)dir * FX_NSTAGES + slot) * FX_NFACES +
                    fx_face_idx(dir, loc[0], loc[1], loc[2])];
                if (!isfinite(v)) fx_fail(D.err, FX_ERR_AMR_NONFINITE, child, fx_face_idx(dir, loc[0], loc[1], loc[2]));
                sum += v;
            }
        }
        dst[fx_face_idx(dir, ci[0], ci[1], ci[2])] = 0.25 * sum;
    }
}

/* prj_amr_restrict's overlap loops per parent cell, every conserved
 * variable at once (each keeps the reference's summation order); one CTA
 * per (parent, i plane), one thread per (j, k) */
template <bool MHD>
__global__ void __launch_bounds__(256) k_amr_restrict_cells(FxDev D, const FxAmrParentJob *__restrict__ jobs,
    double E_floor, double *inj)
{
    constexpr int NV = MHD ? 9 : 6;
    const FxAmrParentJob J = jobs[blockIdx.y];
    const FxBlockDev P = D.blk[J.parent];
    double *injb = (inj != nullptr && E_floor > 0.0) ? inj + (size_t)blockIdx.y * FX_BS * FX_BS * FX_BS : nullptr;
    const int i = blockIdx.x, j = threadIdx.x >> 4, k = threadIdx.x & 15;
    const double pvol = P.dx[0] * P.dx[1] * P.dx[2];
    const double pxmin = P.xmin[0] + (double)i * P.dx[0];
    const double pxmax = pxmin + P.dx[0];
    const double pymin = P.xmin[1] + (double)j * P.dx[1];
    const double pymax = pymin + P.dx[1];
    const double pzmin = P.xmin[2] + (double)k * P.dx[2];
    const double pzmax = pzmin + P.dx[2];
    double sum[FX_MAXVAR];
    for (int v = 0; v < NV; ++v) sum[v] = 0.0;
    for (int oct = 0; oct < 8; ++oct) {
        const int cb = J.children[oct];
        const FxBlockDev C = D.blk[cb];
        const double *Wc = D.W + (size_t)cb * FX_W_COUNT(D.nv);
        for (int fi = 0; fi < FX_BS; ++fi) {
            const double fxmin = C.xmin[0] + (double)fi * C.dx[0];
            const double fxmax = fxmin + C.dx[0];
            const double xover = (pxmax < fxmax ? pxmax : fxmax) - (pxmin > fxmin ? pxmin : fxmin);
            if (xover <= 0.0) continue;
            for (int fj = 0; fj < FX_BS; ++fj) {
                const double fymin = C.xmin[1] + (double)fj * C.dx[1];
                const double fymax = fymin + C.dx[1];
                const double yover = (pymax < fymax ? pymax : fymax) - (pymin > fymin ? pymin : fymin);
                if (yover <= 0.0) continue;
                for (int fk = 0; fk < FX_BS; ++fk) {
                    const double fzmin = C.xmin[2] + (double)fk * C.dx[2];
                    const double fzmax = fzmin + C.dx[2];
                    const double zover = (pzmax < fzmax ? pzmax : fzmax) - (pzmin > fzmin ? pzmin : fzmin);
                    if (zover > 0.0) {
                        const double ov = xover * yover * zover;
                        const int c = fx_lidx(fi, fj, fk);
                        double w[FX_MAXVAR], u[FX_MAXVAR];
                        for (int v = 0; v < NV; ++v) w[v] = Wc[(size_t)v * kPlane + c];
                        fx_prim2cons<MHD>(w, u);
                        for (int v = 0; v < NV; ++v) sum[v] += u[v] * ov;
                    }
                }
            }
        }
    }
    double u[FX_MAXVAR];
    for (int v = 0; v < NV; ++v) u[v] = sum[v] / pvol;
    store_cell<MHD>(D, J.parent, i, j, k, u, E_floor, injb);
}

} /* namespace */

void fx_launch_amr_tag(const FxDev &D, const int *list, const int *has_parent, int n,
    const FxAmrTagCfg &cfg, int32_t *votes, cudaStream_t s)
{
    if (n <= 0) return;
    if (D.nv == 9) {
        k_amr_tag<true><<<n, 256, 0, s>>>(D, list, has_parent, cfg, votes);
    } else {
        k_amr_tag<false><<<n, 256, 0, s>>>(D, list, has_parent, cfg, votes);
    }
}

void fx_launch_amr_zero(const FxDev &D, const int *blocks, int n, cudaStream_t s)
{
    if (n <= 0) return;
    k_amr_zero<<<dim3(64, n), 256, 0, s>>>(D, blocks);
}

void fx_launch_amr_copy_faces(const FxDev &D, const FxAmrCopyJob *jobs, int n, cudaStream_t s)
{
    if (n <= 0) return;
    k_amr_copy_faces<<<dim3(n, 2), 256, 0, s>>>(D, jobs);
}

void fx_launch_amr_prolong_cells(const FxDev &D, const FxAmrChildJob *jobs, int n, double E_floor,
    double *inj, cudaStream_t s)
{
    if (n <= 0) return;
    if (D.nv == 9) {
        const size_t smem = 9 * 1000 * sizeof(double);
        cudaFuncSetAttribute(k_amr_prolong_cells<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        k_amr_prolong_cells<true><<<n, 256, smem, s>>>(D, jobs, E_floor, inj);
    } else {
        const size_t smem = 6 * 1000 * sizeof(double);
        cudaFuncSetAttribute(k_amr_prolong_cells<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        k_amr_prolong_cells<false><<<n, 256, smem, s>>>(D, jobs, E_floor, inj);
    }
}

void fx_launch_amr_restrict_faces(const FxDev &D, const FxAmrParentJob *jobs, int n, cudaStream_t s)
{
    if (n <= 0 || D.Bf == nullptr) return;
    k_amr_restrict_faces<<<dim3(3, 2, n), 256, 0, s>>>(D, jobs);
}

void fx_launch_amr_restrict_cells(const FxDev &D, const FxAmrParentJob *jobs, int n, double E_floor,
    double *inj, cudaStream_t s)
{
    if (n <= 0) return;
    if (D.nv == 9) {
        k_amr_restrict_cells<true><<<dim3(FX_BS, n), 256, 0, s>>>(D, jobs, E_floor, inj);
    } else {
        k_amr_restrict_cells<false><<<dim3(FX_BS, n), 256, 0, s>>>(D, jobs, E_floor, inj);
    }
}
