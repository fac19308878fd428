/*
 * Discrete adjoint of the RK2 MHD step: host checks of the pointwise
 * vector-Jacobian products and (below) the reverse-pass kernels.
 */
#include <cuda_runtime.h>

#include "../../include/fornax_b200.h"
#include "fx_adjoint.cuh"

namespace {

void face_out_pack(const FxFaceOut &o, double *out)
{
    for (int v = 0; v < 9; ++v) {
        out[v] = o.F[v];
    }
    out[9] = o.v[0];
    out[10] = o.v[1];
    out[11] = o.v[2];
    out[12] = o.bv1;
    out[13] = o.bv2;
}

} // namespace

extern "C" int fx_face_eval_host(const double *w4, double bn, double gamma, double *out)
{
    if (!w4 || !out || !(gamma > 1.0)) {
        return FX_EINVAL;
    }
    FxFaceOut o;
    fxa_face_eval(w4, gamma, bn, o);
    face_out_pack(o, out);
    return FX_SUCCESS;
}

extern "C" int fx_face_vjp_host(const double *w4, double bn, double gamma, const double *out_bar,
    double *w4_bar, double *bn_bar)
{
    if (!w4 || !out_bar || !w4_bar || !bn_bar || !(gamma > 1.0)) {
        return FX_EINVAL;
    }
    for (int n = 0; n < 36; ++n) {
        w4_bar[n] = 0.0;
    }
    double bnb = 0.0;
    fxa_face_vjp(w4, gamma, bn, out_bar, w4_bar, bnb);
    *bn_bar = bnb;
    return FX_SUCCESS;
}

/* ------------------------------------------------------------------------ */
/* Reverse-pass kernels.  One reverse RK stage runs, in order: the ghost    */
/* fill adjoint on the stage's output slot, the cell update, the CT face    */
/* update, the edge EMFs and the face fluxes (recomputed from the stored    */
/* stage input, then reversed).  Adjoint arrays accumulate with atomics     */
/* where several forward outputs read one input.                             */
/* ------------------------------------------------------------------------ */
#include "fx_kernels.h"

namespace {

constexpr int kPlaneA = FX_NSTAGES * FX_NCELLS;

__device__ __forceinline__ int adj_axis_stride(int dir)
{
    return dir == 0 ? FX_PBS * FX_PBS : dir == 1 ? FX_PBS : 1;
}

/* local sweep variable -> global variable (as the forward face kernel) */
__device__ __forceinline__ int adj_gmap(int dir, int lv)
{
    if (lv >= 1 && lv <= 3) {
        return 1 + (dir + lv - 1) % 3;
    }
    if (lv >= 6) {
        return 6 + (dir + lv - 6) % 3;
    }
    return lv;
}

/* cell update of one stage (k_cell_update, no gravity) */
__global__ void __launch_bounds__(128) k_adj_cells(FxAdjDev A, const int *__restrict__ blist, int stage)
{
    const int b = blist[blockIdx.y];
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= FX_BS * FX_BS * FX_BS) {
        return;
    }
    const int k = t % FX_BS;
    const int j = (t / FX_BS) % FX_BS;
    const int i = t / (FX_BS * FX_BS);
    const int c = fx_lidx(i, j, k);
    const int dst = stage == 1 ? 1 : 0;
    const double *__restrict__ Wa = A.Waft + (size_t)b * FX_W_COUNT(9) + (size_t)dst * FX_NCELLS;
    const double *__restrict__ Wf = A.Wbef + (size_t)b * FX_W_COUNT(9);
    double *__restrict__ Wbb = A.Wb + (size_t)b * FX_W_COUNT(9);
    double wn[9], un[9], wb[9], ub[9];
    for (int v = 0; v < 9; ++v) {
        wn[v] = Wa[(size_t)v * kPlaneA + c];
        wb[v] = Wbb[(size_t)v * kPlaneA + (size_t)dst * FX_NCELLS + c];
        Wbb[(size_t)v * kPlaneA + (size_t)dst * FX_NCELLS + c] = 0.0;
    }
    fx_prim2cons<true>(wn, un);
    fxa_cons2prim_vjp(un, wb, ub);
    double u0b[9], w0[9];
    const double coef = stage == 1 ? A.dt : 0.5 * A.dt;
    const double ws = stage == 1 ? 1.0 : 0.5;
    for (int v = 0; v < 9; ++v) {
        u0b[v] = v < 6 ? ws * ub[v] : 0.0;
        w0[v] = Wf[(size_t)v * kPlaneA + c];
    }
    double wb0[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    fxa_prim2cons_vjp(w0, u0b, wb0);
    for (int v = 0; v < 9; ++v) {
        Wbb[(size_t)v * kPlaneA + c] += wb0[v];
    }
    if (stage == 2) {
        double w1[9];
        double wb1[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
        for (int v = 0; v < 9; ++v) {
            w1[v] = Wf[(size_t)v * kPlaneA + FX_NCELLS + c];
        }
        fxa_prim2cons_vjp(w1, u0b, wb1);
        for (int v = 0; v < 9; ++v) {
            Wbb[(size_t)v * kPlaneA + FX_NCELLS + c] += wb1[v];
        }
    }
    double *G = A.G + (size_t)b * FX_ADJ_G_COUNT;
    for (int v = 0; v < 6; ++v) {
        G[(size_t)v * FX_NCELLS + c] = coef * ub[v];
    }
    /* the updated cell field is the average of the updated faces: the face
     * kernel gathers half of each neighbour's field adjoint */
    for (int d = 0; d < 3; ++d) {
        G[(size_t)(6 + d) * FX_NCELLS + c] = ub[FX_B1 + d];
    }
}

/* CT face update of one stage (k_bf_update) */
__global__ void __launch_bounds__(128) k_adj_bf(FxAdjDev A, const int *__restrict__ blist, int stage)
{
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
    const int dst = stage == 1 ? 1 : 0;
    const int f = fx_face_idx(dir, i, j, k);
    double *bf = A.Bfb + (size_t)b * FX_BF_COUNT + (size_t)dir * FX_NSTAGES * FX_NFACES;
    /* stage-output face adjoint plus half the cell-field adjoints of the two
     * cells the face bounds (zero for ghost cells) */
    const double *GB = A.G + (size_t)b * FX_ADJ_G_COUNT + (size_t)(6 + dir) * FX_NCELLS;
    const int cu = fx_lidx(i, j, k);
    const int cl = fx_lidx(i - (dir == 0), j - (dir == 1), k - (dir == 2));
    const double bb = bf[(size_t)dst * FX_NFACES + f] + 0.5 * (GB[cu] + GB[cl]);
    double fac;
    if (stage == 1) {
        bf[f] += bb;
        bf[FX_NFACES + f] = 0.0;
        fac = A.dt;
    } else {
        bf[f] = 0.5 * bb;
        bf[FX_NFACES + f] += 0.5 * bb;
        fac = 0.5 * A.dt;
    }
    const FxBlockDev &B = A.blk[b];
    double *e = A.Eb + (size_t)b * FX_EMF_COUNT;
    double *e1 = e;
    double *e2 = e + FX_NEDGES;
    double *e3 = e + 2 * FX_NEDGES;
    const double g = fac * bb;
    if (dir == 0) {
        atomicAdd(&e3[fx_edge_idx(2, i, j + 1, k)], -g / B.dx[1]);
        atomicAdd(&e3[fx_edge_idx(2, i, j, k)], g / B.dx[1]);
        atomicAdd(&e2[fx_edge_idx(1, i, j, k + 1)], g / B.dx[2]);
        atomicAdd(&e2[fx_edge_idx(1, i, j, k)], -g / B.dx[2]);
    } else if (dir == 1) {
        atomicAdd(&e1[fx_edge_idx(0, i, j, k + 1)], -g / B.dx[2]);
        atomicAdd(&e1[fx_edge_idx(0, i, j, k)], g / B.dx[2]);
        atomicAdd(&e3[fx_edge_idx(2, i + 1, j, k)], g / B.dx[0]);
        atomicAdd(&e3[fx_edge_idx(2, i, j, k)], -g / B.dx[0]);
    } else {
        atomicAdd(&e2[fx_edge_idx(1, i + 1, j, k)], -g / B.dx[0]);
        atomicAdd(&e2[fx_edge_idx(1, i, j, k)], g / B.dx[0]);
        atomicAdd(&e1[fx_edge_idx(0, i, j + 1, k)], g / B.dx[1]);
        atomicAdd(&e1[fx_edge_idx(0, i, j, k)], -g / B.dx[1]);
    }
}

/* edge EMFs (k_emf with zero resistivity) */
__global__ void __launch_bounds__(128) k_adj_emf(FxAdjDev A, const int *__restrict__ blist, int stage)
{
    const int b = blist[blockIdx.y];
    constexpr int NE = FX_BS * (FX_BS + 1) * (FX_BS + 1);
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= 3 * NE) {
        return;
    }
    const int dir = t / NE;
    t -= dir * NE;
    const int x2 = dir == 2 ? FX_BS : FX_BS + 1;
    const int x1 = dir == 1 ? FX_BS : FX_BS + 1;
    int e[3];
    e[2] = t % x2;
    t /= x2;
    e[1] = t % x1;
    e[0] = t / x1;
    const double eb = A.Eb[(size_t)b * FX_EMF_COUNT + (size_t)dir * FX_NEDGES + fx_edge_idx(dir, e[0], e[1], e[2])];
    if (eb == 0.0) {
        return;
    }
    const int src = stage == 1 ? 0 : 1;
    const int up = (dir + 1) % 3;
    const int right = (dir + 2) % 3;
    const int su = adj_axis_stride(up);
    const int sr = adj_axis_stride(right);
    const int cells[4] = {fx_lidx(e[0], e[1], e[2]), 0, 0, 0};
    const int c0 = cells[0];
    const int cc[4] = {c0, c0 - su, c0 - su - sr, c0 - sr};
    const double *vrr = A.vr + (size_t)b * FX_VR_COUNT + (size_t)right * 3 * FX_NCELLS;
    const double *vru = A.vr + (size_t)b * FX_VR_COUNT + (size_t)up * 3 * FX_NCELLS;
    double vn[4];
    vn[0] = vrr[fx_bidx_cell(3, right, cc[0])];
    vn[1] = vru[fx_bidx_cell(3, up, cc[0])];
    vn[2] = vrr[fx_bidx_cell(3, right, cc[1])];
    vn[3] = vru[fx_bidx_cell(3, up, cc[3])];
    double fb[4] = {0, 0, 0, 0}, cb[4] = {0, 0, 0, 0};
    fxa_emf_upwind_vjp(vn, eb, fb, cb);
    double *b1r = A.bvb1 + (size_t)b * FX_BV_COUNT + (size_t)right * FX_NCELLS;
    double *b2u = A.bvb2 + (size_t)b * FX_BV_COUNT + (size_t)up * FX_NCELLS;
    atomicAdd(&b1r[cc[0]], fb[0]);
    atomicAdd(&b2u[cc[0]], fb[1]);
    atomicAdd(&b1r[cc[1]], fb[2]);
    atomicAdd(&b2u[cc[3]], fb[3]);
    /* cell EMF bA vB - bB vA, A = (dir + 1) % 3, B = (dir + 2) % 3 */
    const double *Wf = A.Wbef + (size_t)b * FX_W_COUNT(9) + (size_t)src * FX_NCELLS;
    double *Wbb = A.Wb + (size_t)b * FX_W_COUNT(9) + (size_t)src * FX_NCELLS;
    const int a = up;
    const int bb = right;
    for (int n = 0; n < 4; ++n) {
        const int c = cc[n];
        const double bA = Wf[(size_t)(FX_B1 + a) * kPlaneA + c];
        const double bB = Wf[(size_t)(FX_B1 + bb) * kPlaneA + c];
        const double vA = Wf[(size_t)(FX_V1 + a) * kPlaneA + c];
        const double vB = Wf[(size_t)(FX_V1 + bb) * kPlaneA + c];
        atomicAdd(&Wbb[(size_t)(FX_B1 + a) * kPlaneA + c], cb[n] * vB);
        atomicAdd(&Wbb[(size_t)(FX_V1 + bb) * kPlaneA + c], cb[n] * bA);
        atomicAdd(&Wbb[(size_t)(FX_B1 + bb) * kPlaneA + c], -cb[n] * vA);
        atomicAdd(&Wbb[(size_t)(FX_V1 + a) * kPlaneA + c], -cb[n] * bB);
    }
    (void)cells;
}

/* stencil access of one face for fxa_face_vjp_t: cell n at c0 + n s,
 * local variable lv at global variable adj_gmap(dir, lv) */
struct AdjCellLoad {
    const double *W;
    int dir, c0, s;
    __device__ __forceinline__ double operator()(int n, int lv) const
    {
        return W[(size_t)adj_gmap(dir, lv) * kPlaneA + c0 + n * s];
    }
};

struct AdjCellAcc {
    double *Wb;
    int dir, c0, s;
    __device__ __forceinline__ void operator()(int n, int lv, double x) const
    {
        if (x != 0.0) {
            atomicAdd(&Wb[(size_t)adj_gmap(dir, lv) * kPlaneA + c0 + n * s], x);
        }
    }
};

/* face fluxes (k_flux, MHD): recompute the face from the stored stage input
 * and reverse it.  Bounded to 128 registers (four resident CTAs per SM): the
 * reverse HLLD is latency-bound on dependent FP64 operations, and the
 * occupancy gained outweighs the spills (measured: 20 % faster than 255
 * registers). */
__global__ void __launch_bounds__(128, 4) k_adj_flux(FxAdjDev A, const int *__restrict__ blist, int stage)
{
    const int dir = blockIdx.y;
    const int b = blist[blockIdx.z];
    constexpr int T = FX_BS + 2;
    constexpr int NF = (FX_BS + 1) * T * T;
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= NF) {
        return;
    }
    const int e2 = dir == 2 ? FX_BS + 1 : T;
    const int e1 = dir == 1 ? FX_BS + 1 : T;
    const int k = (dir == 2 ? 0 : -1) + t % e2;
    t /= e2;
    const int j = (dir == 1 ? 0 : -1) + t % e1;
    const int i = (dir == 0 ? 0 : -1) + t / e1;
    const int s = adj_axis_stride(dir);
    const int cR = fx_lidx(i, j, k);
    const int cL = cR - s;
    const int src = stage == 1 ? 0 : 1;
    const FxBlockDev &B = A.blk[b];
    /* flux adjoint from the dt-scaled conserved-update adjoints of the two
     * cells: un(cR) gains +A/V F, un(cL) gains -A/V F */
    const double *G = A.G + (size_t)b * FX_ADJ_G_COUNT;
    const double av = B.area[dir] / B.vol;
    double ob[14];
    bool any = false;
    for (int lv = 0; lv < 6; ++lv) {
        const int gv = adj_gmap(dir, lv);
        ob[lv] = av * (G[(size_t)gv * FX_NCELLS + cR] - G[(size_t)gv * FX_NCELLS + cL]);
        any = any || ob[lv] != 0.0;
    }
    ob[6] = ob[7] = ob[8] = 0.0;
    ob[9] = ob[10] = ob[11] = 0.0;
    ob[12] = A.bvb1[(size_t)b * FX_BV_COUNT + (size_t)dir * FX_NCELLS + cR];
    ob[13] = A.bvb2[(size_t)b * FX_BV_COUNT + (size_t)dir * FX_NCELLS + cR];
    any = any || ob[12] != 0.0 || ob[13] != 0.0;
    if (!any) {
        return;
    }
    const double *Wf = A.Wbef + (size_t)b * FX_W_COUNT(9) + (size_t)src * FX_NCELLS;
    double *Wbb = A.Wb + (size_t)b * FX_W_COUNT(9) + (size_t)src * FX_NCELLS;
    const int f = fx_face_idx(dir, i, j, k);
    const double bn = A.Bfbef[(size_t)b * FX_BF_COUNT + ((size_t)dir * FX_NSTAGES + src) * FX_NFACES + f];
    double bnb = 0.0;
    fxa_face_vjp_t(AdjCellLoad{Wf, dir, cL - s, s}, AdjCellAcc{Wbb, dir, cL - s, s}, A.gamma, bn, ob, bnb);
    A.Bfb[(size_t)b * FX_BF_COUNT + ((size_t)dir * FX_NSTAGES + src) * FX_NFACES + f] += bnb;
}

/* transposed ghost wave: one thread per element the wave reads */
__global__ void __launch_bounds__(256) k_adj_gather(FxAdjDev A, const FxAdjSrc *__restrict__ csrc, int nc,
    const FxAdjSrc *__restrict__ fsrc, int nf, const FxAdjEnt *__restrict__ ents, int slot)
{
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t < nc) {
        const FxAdjSrc sr = csrc[t];
        double acc[6] = {0, 0, 0, 0, 0, 0};
        for (int q = sr.begin; q < sr.end; ++q) {
            const FxAdjEnt e = ents[q];
            const double *d = A.Wb + (size_t)FX_CELL_BLOCK(e.key) * FX_W_COUNT(9) + (size_t)slot * FX_NCELLS +
                FX_CELL_IDX(e.key);
            for (int v = 0; v < 6; ++v) {
                double x = d[(size_t)v * kPlaneA];
                if (e.kind == 1 + v) x = -x;
                if (e.kind == 16 && v == FX_V1) x = 0.0;
                acc[v] += x;
            }
        }
        double *w = A.Wb + (size_t)FX_CELL_BLOCK(sr.key) * FX_W_COUNT(9) + (size_t)slot * FX_NCELLS +
            FX_CELL_IDX(sr.key);
        for (int v = 0; v < 6; ++v) {
            w[(size_t)v * kPlaneA] += acc[v];
        }
        return;
    }
    const int u = t - nc;
    if (u < nf) {
        const FxAdjSrc sr = fsrc[u];
        double acc = 0.0;
        for (int q = sr.begin; q < sr.end; ++q) {
            const FxAdjEnt e = ents[q];
            if (e.kind == 0) {
                acc += A.Bfb[(size_t)(e.key >> 15) * FX_BF_COUNT + ((size_t)sr.dir * FX_NSTAGES + slot) * FX_NFACES +
                    (e.key & 32767)];
            } else {
                acc += 0.5 * A.Wb[(size_t)FX_CELL_BLOCK(e.key) * FX_W_COUNT(9) +
                    (size_t)(FX_B1 + e.kind - 1) * kPlaneA + (size_t)slot * FX_NCELLS + FX_CELL_IDX(e.key)];
            }
        }
        A.Bfb[(size_t)(sr.key >> 15) * FX_BF_COUNT + ((size_t)sr.dir * FX_NSTAGES + slot) * FX_NFACES +
            (sr.key & 32767)] += acc;
    }
}

__global__ void __launch_bounds__(256) k_adj_zero(FxAdjDev A, const FxGop *__restrict__ cops, int nc,
    const FxGop *__restrict__ fops, int nf, const FxBop *__restrict__ bops, int nb, int slot)
{
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t < nc) {
        const int key = cops[t].dst;
        double *d = A.Wb + (size_t)FX_CELL_BLOCK(key) * FX_W_COUNT(9) + (size_t)slot * FX_NCELLS + FX_CELL_IDX(key);
        for (int v = 0; v < 6; ++v) d[(size_t)v * kPlaneA] = 0.0;
        return;
    }
    t -= nc;
    if (t < nf) {
        const FxGop op = fops[t];
        A.Bfb[(size_t)(op.dst >> 15) * FX_BF_COUNT + ((size_t)(op.aux & 3) * FX_NSTAGES + slot) * FX_NFACES +
            (op.dst & 32767)] = 0.0;
        return;
    }
    t -= nf;
    if (t < nb) {
        const int key = bops[t].dst;
        double *d = A.Wb + (size_t)FX_CELL_BLOCK(key) * FX_W_COUNT(9) + (size_t)slot * FX_NCELLS + FX_CELL_IDX(key);
        for (int v = FX_B1; v <= FX_B3; ++v) d[(size_t)v * kPlaneA] = 0.0;
    }
}

inline unsigned adj_blocks(int n, int tpb) { return (unsigned)((n + tpb - 1) / tpb); }

} // namespace

void fx_launch_adj_cells(const FxAdjDev &A, const int *blist, int nlist, int stage, cudaStream_t s)
{
    k_adj_cells<<<dim3(adj_blocks(FX_BS * FX_BS * FX_BS, 128), nlist), 128, 0, s>>>(A, blist, stage);
}

void fx_launch_adj_bf(const FxAdjDev &A, const int *blist, int nlist, int stage, cudaStream_t s)
{
    k_adj_bf<<<dim3(adj_blocks(3 * (FX_BS + 1) * FX_BS * FX_BS, 128), nlist), 128, 0, s>>>(A, blist, stage);
}

void fx_launch_adj_emf(const FxAdjDev &A, const int *blist, int nlist, int stage, cudaStream_t s)
{
    k_adj_emf<<<dim3(adj_blocks(3 * FX_BS * (FX_BS + 1) * (FX_BS + 1), 128), nlist), 128, 0, s>>>(A, blist, stage);
}

void fx_launch_adj_flux(const FxAdjDev &A, const int *blist, int nlist, int stage, cudaStream_t s)
{
    k_adj_flux<<<dim3(adj_blocks((FX_BS + 1) * (FX_BS + 2) * (FX_BS + 2), 128), 3, nlist), 128, 0, s>>>(A, blist, stage);
}

void fx_launch_adj_gather(const FxAdjDev &A, const FxAdjSrc *csrc, int nc, const FxAdjSrc *fsrc, int nf,
    const FxAdjEnt *ents, int slot, cudaStream_t s)
{
    if (nc + nf <= 0) return;
    k_adj_gather<<<adj_blocks(nc + nf, 256), 256, 0, s>>>(A, csrc, nc, fsrc, nf, ents, slot);
}

void fx_launch_adj_zero(const FxAdjDev &A, const FxGop *cops, int nc, const FxGop *fops, int nf,
    const FxBop *bops, int nb, int slot, cudaStream_t s)
{
    const int n = nc + nf + nb;
    if (n <= 0) return;
    k_adj_zero<<<adj_blocks(n, 256), 256, 0, s>>>(A, cops, nc, fops, nf, bops, nb, slot);
}
