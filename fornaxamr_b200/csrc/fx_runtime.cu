/*
 * Context, device mirror, step sequencing and the C ABI of fornax_b200.
 *
 * Step sequence (prj_timeint_stage1/2, reference src/prj_timeint.c:2732-2973):
 *   face fluxes -> coarse/fine flux correction -> edge EMFs -> coarse/fine
 *   EMF correction -> CT face update -> cell update -> eos fill (active) ->
 *   ghost fill (cells, faces, bf2bc) -> eos fill (mesh).
 * FX_FORM_PLAIN launches the per-block phases once per block, in the
 * reference's loop order, and writes every block array the reference writes
 * (flux, v_riemann, Bv1/Bv2, emf, mhd_rhs, eosvar).  FX_FORM_BATCHED sweeps
 * each phase over all blocks in one launch, skips the eosvar writes (eosvar
 * is recomputed from W on download), and replays the whole step as one CUDA
 * graph.
 */
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <string>
#include <utility>
#include <vector>

#include "../../include/fornax_b200.h"
#include "fx_kernels.h"
#include "fx_physics.cuh"
#include "fx_amr.h"
#include "fx_plan.h"
#include "fx_transport.h"

/* one exchange of a sharded step on the device: the packed elements of all
 * peers (per-peer offsets in doubles) and the message buffers */
struct FxXdev {
    FxXent *d_send = nullptr, *d_recv = nullptr;
    int nsend = 0, nrecv = 0;
    double *sbuf = nullptr, *rbuf = nullptr;
    std::vector<size_t> soff, roff;
    bool any = false; /* some pair of ranks exchanges: every rank takes part */
};
enum { FX_XG = 0, FX_XF = 1, FX_XE = 2 }; /* ghost fill (cells + faces), flux, EMF */

struct fx_ctx {
    int device = 0;
    fx_config cfg{};
    int nv = 9;
    cudaStream_t stream = nullptr;
    /* the ghost-fill compiler's working buffers, kept from one adapt to the
     * next (created by the first fx_amr_adapt) */
    FxPlanWorkspace *plan_ws = nullptr;
    std::string err;
    int sticky = 0; /* a device-side physics failure was seen */

    int nblocks = 0;
    std::vector<fx_block_desc> blocks;
    FxPlan plan;
    FxDev D{};

    FxBlockDev *d_blk = nullptr;
    double *d_W = nullptr, *d_Bf = nullptr, *d_flux = nullptr, *d_vr = nullptr;
    double *d_bv1 = nullptr, *d_bv2 = nullptr, *d_emf = nullptr, *d_eos = nullptr;
    double *d_rhs = nullptr, *d_grav = nullptr;
    double *d_W2 = nullptr, *d_Bf2 = nullptr; /* eSSPRK10_4 stage slot 2 */
    int *d_ids = nullptr;
    int *d_active = nullptr;
    int nactive = 0;
    FxGop *d_cops = nullptr, *d_fops = nullptr;
    FxPop *d_pops = nullptr;
    FxBop *d_bops = nullptr;
    FxCorr *d_fcorr = nullptr, *d_ecorr = nullptr;
    /* element capacities of the seven program tables above (active list,
     * cell / face / group / cell-field ops, flux / EMF records): an adapt
     * reuses them when the new programs fit */
    size_t tab_cap[7] = {0, 0, 0, 0, 0, 0, 0};

    FxErr *d_err = nullptr;
    unsigned long long *d_red = nullptr;
    FxCtl *d_ctl = nullptr;
    FxErr *h_err = nullptr;
    unsigned long long *h_red = nullptr;
    FxCtl *h_ctl = nullptr;

    cudaGraphExec_t g_step = nullptr; /* batched RK2 step, dt from the control block */
    cudaGraphExec_t g_run = nullptr;  /* batched driver step (calc_dt + step + dt update) */
    int last_slot = 0;                /* W slot written by the last stage */

    /* discrete adjoint: states after every stage of the last
     * fx_adjoint_forward and the adjoint arrays */
    int adj_nsteps = 0;
    double adj_dt = 0.0;
    double *d_ckW = nullptr, *d_ckBf = nullptr, *d_ckVr = nullptr;
    double *d_Wb = nullptr, *d_Bfb = nullptr, *d_G = nullptr;
    double *d_bvb1 = nullptr, *d_bvb2 = nullptr, *d_Eb = nullptr;
    double adj_ms = 0.0;              /* device time of the last reverse sweep */
    /* transposed ghost waves for the adjoint (built on first use) */
    bool adj_ghost_ready = false;
    std::vector<int> adj_cbeg, adj_fbeg;
    FxAdjSrc *d_adj_csrc = nullptr, *d_adj_fsrc = nullptr;
    FxAdjEnt *d_adj_ents = nullptr;

    /* decision record / replay of the plain form (fx_branch_trace) */
    unsigned long long *d_br_words = nullptr, *d_br_edges = nullptr;
    int br_cap = 0;        /* stages the buffers hold */
    int br_nblocks = 0;    /* blocks they were sized for */
    int br_stage = 0;      /* next stage's slot */
    int br_recorded = 0;   /* stages of the last record */
    bool br_overflow = false;

    int cap = 0;                      /* blocks the per-block device arrays hold */
    /* dynamic AMR */
    bool amr_set = false;
    fx_amr_config amr{};
    double E_injected = 0.0;          /* eos->E_injected of the remesh floors */
    double amr_ms[6] = {0, 0, 0, 0, 0, 0}; /* host wall time of the phases of the last adapt */

    /* sharding: this context holds rank `rank`'s owned blocks (local ids
     * [0, nowned)) and its halo; g2l maps the mesh's block ids */
    int nranks = 1;
    int rank = 0;
    int nowned = 0;
    std::vector<int> g2l;
    FxXdev X[3];
    FxTransport *transport = nullptr;
    std::string xerr;                 /* first transport failure */
};

namespace {

int set_err(fx_ctx *c, int code, const char *fmt, ...)
{
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    if (c) c->err = buf;
    return code;
}

#define FX_CUDA(c, call)                                                                   \
    do {                                                                                    \
        cudaError_t e_ = (call);                                                            \
        if (e_ != cudaSuccess) {                                                            \
            return set_err((c), FX_ECUDA, "%s: %s", #call, cudaGetErrorString(e_));        \
        }                                                                                   \
    } while (0)

const char *err_message(int code)
{
    switch (code) {
    case FX_ERR_HLLD_RHO: return "prj_riemann_hlld: non-positive density";
    case FX_ERR_HLLD_P: return "prj_riemann_hlld: non-positive gas pressure";
    case FX_ERR_HLLD_GAMMA: return "prj_riemann_hlld: non-positive adiabatic index";
    case FX_ERR_HLLD_DISC: return "prj_riemann_hlld: negative fast-speed discriminant";
    case FX_ERR_HLLD_CF: return "prj_riemann_hlld: invalid fast speed";
    case FX_ERR_HLLD_ORDER: return "prj_riemann_hlld: invalid fast-wave ordering";
    case FX_ERR_HLLD_DENOM: return "prj_riemann_hlld: degenerate contact-speed denominator";
    case FX_ERR_HLLD_OUTER: return "prj_riemann_hlld: outer wave coincides with contact wave";
    case FX_ERR_HLLD_STARRHO: return "prj_riemann_hlld: invalid star density";
    case FX_ERR_HLLD_DSTAR: return "prj_riemann_hlld: invalid double-star density weights";
    case FX_ERR_EMF_NONFINITE: return "prj_mhd_emf_upwind: non-finite input or result";
    case FX_ERR_BF_NONFINITE: return "prj_timeint_mhd_ct_value: non-finite updated magnetic field";
    case FX_ERR_EOS_ZERO_RHO: return "prj_eos_fill_block: zero density";
    case FX_ERR_ETA: return "prj_timeint_mhd_fill_eta_mask: non-finite artificial eta";
    case FX_ERR_B_NONFINITE: return "non-finite cell-centered magnetic field";
    case FX_ERR_TIMEOUT: return "device wait timed out";
    case FX_ERR_AMR_NONFINITE: return "prj_amr_mhd: non-finite magnetic field in a remesh";
    default: return "unknown device failure";
    }
}

/* reads the device error word (the caller has synchronised) */
int check_device_error(fx_ctx *c)
{
    if (c->sticky) {
        return FX_EPHYSICS;
    }
    FX_CUDA(c, cudaMemcpyAsync(c->h_err, c->d_err, sizeof(FxErr), cudaMemcpyDeviceToHost, c->stream));
    FX_CUDA(c, cudaStreamSynchronize(c->stream));
    if (c->h_err->code != 0) {
        c->sticky = 1;
        return set_err(c, FX_EPHYSICS, "%s (block %d, index %d)", err_message(c->h_err->code),
            c->h_err->block, c->h_err->index);
    }
    return FX_SUCCESS;
}

int sync_and_check(fx_ctx *c)
{
    FX_CUDA(c, cudaGetLastError()); /* launch failures (configuration, resources) */
    FX_CUDA(c, cudaStreamSynchronize(c->stream));
    if (!c->xerr.empty()) return set_err(c, FX_ECOMM, "%s", c->xerr.c_str());
    return check_device_error(c);
}

template <typename T>
int dev_alloc(fx_ctx *c, T **p, size_t count)
{
    if (*p) {
        cudaFree(*p);
        *p = nullptr;
    }
    if (count == 0) {
        return FX_SUCCESS;
    }
    cudaError_t e = cudaMalloc((void **)p, count * sizeof(T));
    if (e != cudaSuccess) {
        *p = nullptr;
        return set_err(c, FX_ENOMEM, "cudaMalloc of %zu bytes failed: %s", count * sizeof(T),
            cudaGetErrorString(e));
    }
    return FX_SUCCESS;
}

void free_graphs(fx_ctx *c)
{
    if (c->g_step) {
        cudaGraphExecDestroy(c->g_step);
        c->g_step = nullptr;
    }
    if (c->g_run) {
        cudaGraphExecDestroy(c->g_run);
        c->g_run = nullptr;
    }
}

void free_mesh(fx_ctx *c)
{
    free_graphs(c);
    cudaFree(c->d_blk);
    cudaFree(c->d_W);
    cudaFree(c->d_Bf);
    cudaFree(c->d_flux);
    cudaFree(c->d_vr);
    cudaFree(c->d_bv1);
    cudaFree(c->d_bv2);
    cudaFree(c->d_emf);
    cudaFree(c->d_eos);
    cudaFree(c->d_rhs);
    cudaFree(c->d_grav);
    cudaFree(c->d_W2);
    cudaFree(c->d_Bf2);
    c->d_W2 = c->d_Bf2 = nullptr;
    cudaFree(c->d_ids);
    cudaFree(c->d_active);
    cudaFree(c->d_cops);
    cudaFree(c->d_fops);
    cudaFree(c->d_pops);
    cudaFree(c->d_bops);
    c->d_pops = nullptr;
    c->d_bops = nullptr;
    cudaFree(c->d_fcorr);
    cudaFree(c->d_ecorr);
    for (size_t &cap : c->tab_cap) cap = 0;
    c->d_blk = nullptr;
    c->d_W = c->d_Bf = c->d_flux = c->d_vr = c->d_bv1 = c->d_bv2 = nullptr;
    c->d_emf = c->d_eos = c->d_rhs = c->d_grav = nullptr;
    c->d_ids = c->d_active = nullptr;
    c->d_cops = c->d_fops = nullptr;
    c->d_fcorr = c->d_ecorr = nullptr;
    cudaFree(c->d_ckW);
    cudaFree(c->d_ckBf);
    cudaFree(c->d_ckVr);
    c->d_ckVr = nullptr;
    cudaFree(c->d_adj_csrc);
    cudaFree(c->d_adj_fsrc);
    cudaFree(c->d_adj_ents);
    c->d_adj_csrc = c->d_adj_fsrc = nullptr;
    c->d_adj_ents = nullptr;
    c->adj_ghost_ready = false;
    cudaFree(c->d_Wb);
    cudaFree(c->d_Bfb);
    cudaFree(c->d_G);
    cudaFree(c->d_bvb1);
    cudaFree(c->d_bvb2);
    cudaFree(c->d_Eb);
    c->d_ckW = c->d_ckBf = c->d_Wb = c->d_Bfb = c->d_G = nullptr;
    c->d_bvb1 = c->d_bvb2 = c->d_Eb = nullptr;
    c->adj_nsteps = 0;
    c->nblocks = 0;
    c->nactive = 0;
    c->cap = 0;
    for (FxXdev &x : c->X) {
        cudaFree(x.d_send);
        cudaFree(x.d_recv);
        cudaFree(x.sbuf);
        cudaFree(x.rbuf);
        x = FxXdev();
    }
    c->nranks = 1;
    c->rank = 0;
    c->nowned = 0;
    c->g2l.clear();
}

bool has_mesh(const fx_ctx *c) { return c && c->nblocks > 0 && c->d_W; }

/* device array of at least `count` elements, reusing the current one when it
 * is large enough (a grown one gets 1/8 headroom) */
template <typename T>
int dev_reserve(fx_ctx *c, T **p, size_t *cap, size_t count)
{
    if (*p && count <= *cap) {
        return FX_SUCCESS;
    }
    const size_t n = count + count / 8;
    int rc = dev_alloc(c, p, n);
    *cap = rc == FX_SUCCESS && *p ? n : 0;
    return rc;
}

/* a block index of the caller (the mesh's numbering) -> this context's;
 * a sharded context serves the blocks its rank owns */
int local_block(fx_ctx *c, int *b)
{
    if (c->nranks == 1) {
        if (*b < 0 || *b >= c->nblocks) return set_err(c, FX_EINVAL, "block %d out of range", *b);
        return FX_SUCCESS;
    }
    if (*b < 0 || *b >= (int)c->g2l.size() || c->g2l[*b] < 0 || c->g2l[*b] >= c->nowned) {
        return set_err(c, FX_EINVAL, "block %d is not owned by rank %d", *b, c->rank);
    }
    *b = c->g2l[*b];
    return FX_SUCCESS;
}

/* ---- phase sequencing ------------------------------------------------------ */

template <typename F>
void per_block(fx_ctx *c, int form, F &&fn)
{
    if (form == FX_FORM_PLAIN) {
        for (int b : c->plan.active) {
            fn(c->d_ids + b, 1);
        }
    } else {
        fn(c->d_active, c->nactive);
    }
}

/* the whole ghost fill of prj_boundary_fill_ghosts_and_bf: one launch per
 * conflict-free wave of the compiled program (a single launch on
 * single-level meshes) */
void ghost_fill(fx_ctx *c, int slot)
{
    const FxProgram &g = c->plan.ghost;
    for (int w = 0; w < g.nwaves(); ++w) {
        fx_launch_ghost_wave(c->D,
            c->d_cops + g.cell_begin[w], g.cell_begin[w + 1] - g.cell_begin[w],
            c->d_fops + g.face_begin[w], g.face_begin[w + 1] - g.face_begin[w],
            c->d_pops + g.p_begin[w], g.p_begin[w + 1] - g.p_begin[w],
            c->d_bops + g.b_begin[w], g.b_begin[w + 1] - g.b_begin[w], slot, 6, c->stream);
    }
}

/* coarse/fine flux corrections (prj_riemann_flux_send), wave by wave;
 * ncomp: flux components the face kernel stored */
void flux_correct(fx_ctx *c, int ncomp, cudaStream_t s)
{
    const std::vector<int> &wb = c->plan.flux_corr_begin;
    for (size_t w = 0; w + 1 < wb.size(); ++w) {
        fx_launch_flux_correct(c->D, c->d_fcorr + wb[w], wb[w + 1] - wb[w], ncomp, s);
    }
}

/* coarse/fine EMF corrections (prj_mhd_emf_send), wave by wave */
void emf_correct(fx_ctx *c, cudaStream_t s)
{
    const std::vector<int> &wb = c->plan.emf_corr_begin;
    for (size_t w = 0; w + 1 < wb.size(); ++w) {
        fx_launch_emf_correct(c->D, c->d_ecorr + wb[w], wb[w + 1] - wb[w], s);
    }
}

/* exchange k of a sharded step: pack, move, unpack (slot: the W / Bf stage
 * slot of a ghost-fill exchange) */
void shard_exchange(fx_ctx *c, int k, int slot)
{
    FxXdev &x = c->X[k];
    if (c->nranks == 1 || !x.any || !c->xerr.empty()) return;
    if (!c->transport) {
        c->xerr = "sharded mesh without a transport (fx_shard_attach_group / fx_shard_attach_nccl)";
        return;
    }
    fx_launch_xpack(c->D, x.d_send, x.nsend, x.sbuf, slot, c->stream);
    if (c->transport->exchange(k, x.sbuf, x.soff.data(), x.rbuf, x.roff.data(), c->stream)) {
        c->xerr = c->transport->err;
        return;
    }
    fx_launch_xunpack(c->D, x.d_recv, x.nrecv, x.rbuf, slot, c->stream);
}

/* minimum of the dt keys (first..first + count) over the ranks */
void shard_min(fx_ctx *c, int first, int count)
{
    if (c->nranks == 1 || !c->xerr.empty()) return;
    if (!c->transport) {
        c->xerr = "sharded mesh without a transport (fx_shard_attach_group / fx_shard_attach_nccl)";
        return;
    }
    if (c->transport->min_u64(c->d_red + first, count, c->stream)) c->xerr = c->transport->err;
}

/* one RK2 stage; dt is read from the control block */
void stage_seq(fx_ctx *c, int form, int stage)
{
    const int src = stage == 1 ? 0 : 1; /* W / Bf slot the fluxes read */
    const int dst = stage == 1 ? 1 : 0; /* W slot the update writes */
    cudaStream_t s = c->stream;
    const int full = form == FX_FORM_PLAIN ? 1 : 0;
    /* decisions are recorded / replayed by the plain form only, one slot
     * of the buffers per stage */
    const int br_mode = c->D.br_mode;
    if (br_mode && form != FX_FORM_PLAIN) {
        c->D.br_mode = 0;
    } else if (br_mode) {
        if (c->br_stage >= c->br_cap) {
            c->br_overflow = true;
            c->D.br_mode = 0;
        } else {
            c->D.br_off = (size_t)c->br_stage * c->nblocks * 3 * (FX_BS + 1) * (FX_BS + 2) * (FX_BS + 2);
            c->D.br_eoff = (size_t)c->br_stage * c->nblocks * 3 * FX_BS * (FX_BS + 1) * (FX_BS + 1);
            ++c->br_stage;
            if (br_mode == FX_BRANCH_RECORD) c->br_recorded = c->br_stage;
        }
    }
    per_block(c, form, [&](const int *l, int n) { fx_launch_flux(c->D, l, n, 3, src, src, full, s); });
    shard_exchange(c, FX_XF, src);
    flux_correct(c, full ? c->nv : 6, s);
    if (c->cfg.mhd) {
        per_block(c, form, [&](const int *l, int n) { fx_launch_emf(c->D, l, n, src, src, s); });
        shard_exchange(c, FX_XE, src);
        emf_correct(c, s);
        per_block(c, form, [&](const int *l, int n) { fx_launch_bf_update(c->D, l, n, stage, s); });
    }
    per_block(c, form, [&](const int *l, int n) {
        fx_launch_cell_update(c->D, l, n, stage, c->cfg.gravity, full, s);
    });
    if (form == FX_FORM_PLAIN) {
        per_block(c, form, [&](const int *l, int n) { fx_launch_eos_fill(c->D, l, n, dst, 1, s); });
    }
    shard_exchange(c, FX_XG, dst);
    ghost_fill(c, dst);
    if (form == FX_FORM_PLAIN) {
        per_block(c, form, [&](const int *l, int n) { fx_launch_eos_fill(c->D, l, n, dst, 0, s); });
    }
    c->last_slot = dst;
    if (!c->br_overflow) c->D.br_mode = br_mode;
}

/* the refill after a substep or a blend: eos (active) -> ghost fill -> eos
 * (mesh) on slot 0 */
void refill0(fx_ctx *c, int form)
{
    cudaStream_t s = c->stream;
    if (form == FX_FORM_PLAIN) {
        per_block(c, form, [&](const int *l, int n) { fx_launch_eos_fill(c->D, l, n, 0, 1, s); });
    }
    ghost_fill(c, 0);
    if (form == FX_FORM_PLAIN) {
        per_block(c, form, [&](const int *l, int n) { fx_launch_eos_fill(c->D, l, n, 0, 0, s); });
    }
}

/* one forward-Euler substep in place on slot 0, prj_timeint_eSSPRK_step
 * (src/prj_timeint.c:2452-2550); dt_stage holds dt / 6 */
void essprk_substep(fx_ctx *c, int form)
{
    cudaStream_t s = c->stream;
    const int full = form == FX_FORM_PLAIN ? 1 : 0;
    per_block(c, form, [&](const int *l, int n) { fx_launch_flux(c->D, l, n, 3, 0, 0, full, s); });
    flux_correct(c, full ? c->nv : 6, s);
    if (c->cfg.mhd) {
        per_block(c, form, [&](const int *l, int n) { fx_launch_emf(c->D, l, n, 0, 0, s); });
        emf_correct(c, s);
        per_block(c, form, [&](const int *l, int n) { fx_launch_bf_update(c->D, l, n, 0, s); });
    }
    per_block(c, form, [&](const int *l, int n) {
        fx_launch_cell_update(c->D, l, n, 0, c->cfg.gravity, full, s);
    });
    refill0(c, form);
}

void essprk_blend(fx_ctx *c, int form, int which, double w)
{
    per_block(c, form, [&](const int *l, int n) { fx_launch_essprk_blend(c->D, l, n, which, w, c->stream); });
    refill0(c, form);
}

void essprk_save(fx_ctx *c, int form, int which)
{
    per_block(c, form, [&](const int *l, int n) { fx_launch_essprk_save(c->D, l, n, which, c->stream); });
}

/* prj_timeint_eSSPRK10_4_advance (src/prj_timeint.c:2671-2729): Ketcheson's
 * eSSPRK(10,4) in its low-storage form with the reference's blend weights */
void essprk_seq(fx_ctx *c, int form)
{
    fx_launch_stage_dt(c->D, 6.0, c->stream);
    essprk_save(c, form, 1);
    for (int n = 0; n < 5; ++n) essprk_substep(c, form);
    essprk_save(c, form, 2);
    essprk_blend(c, form, 1, 3.0 / 5.0);
    for (int n = 0; n < 5; ++n) essprk_substep(c, form);
    essprk_blend(c, form, 2, 3.0 / 8.0);
    essprk_blend(c, form, 1, 1.0 / 25.0);
    c->last_slot = 0;
}

/* prj_timeint_step: the two RK2 stages or the eSSPRK10_4 advance */
void step_seq(fx_ctx *c, int form)
{
    if (c->cfg.integrator == FX_INT_ESSPRK10_4) {
        essprk_seq(c, form);
    } else {
        stage_seq(c, form, 1);
        stage_seq(c, form, 2);
    }
}

int build_step_graph(fx_ctx *c)
{
    if (c->g_step) {
        return FX_SUCCESS;
    }
    cudaGraph_t g;
    FX_CUDA(c, cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
    fx_launch_reset_reductions(c->D, 2, c->stream);
    step_seq(c, FX_FORM_BATCHED);
    FX_CUDA(c, cudaStreamEndCapture(c->stream, &g));
    cudaError_t e = cudaGraphInstantiate(&c->g_step, g, 0);
    cudaGraphDestroy(g);
    FX_CUDA(c, e);
    return FX_SUCCESS;
}

/* one batched driver step: calc_dt, dt selection, the step, dt_src clamp;
 * sharded, the dt and dt_src keys are minimised over the ranks */
void run_seq(fx_ctx *c, double cfl)
{
    fx_launch_reset_reductions(c->D, 1, c->stream);
    fx_launch_calc_dt(c->D, c->d_active, c->nactive, 0, cfl, c->stream);
    shard_min(c, 0, 1);
    fx_launch_step_begin(c->D, c->stream);
    step_seq(c, FX_FORM_BATCHED);
    shard_min(c, 1, 1);
    fx_launch_step_end(c->D, c->stream);
}

/* a sharded context whose transport cannot be captured runs eagerly */
bool eager(const fx_ctx *c) { return c->nranks > 1 && (!c->transport || !c->transport->capturable()); }

int build_run_graph(fx_ctx *c, double cfl)
{
    if (c->g_run) {
        return FX_SUCCESS;
    }
    cudaGraph_t g;
    FX_CUDA(c, cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
    run_seq(c, cfl);
    FX_CUDA(c, cudaStreamEndCapture(c->stream, &g));
    cudaError_t e = cudaGraphInstantiate(&c->g_run, g, 0);
    cudaGraphDestroy(g);
    FX_CUDA(c, e);
    return FX_SUCCESS;
}

int read_dt_src(fx_ctx *c, double *dt_src)
{
    FX_CUDA(c, cudaMemcpyAsync(c->h_red, c->d_red, 2 * sizeof(unsigned long long),
        cudaMemcpyDeviceToHost, c->stream));
    int rc = sync_and_check(c);
    if (rc) return rc;
    *dt_src = fx_key_to_double(c->h_red[1]);
    return FX_SUCCESS;
}

size_t w_count(const fx_ctx *c) { return (size_t)FX_W_COUNT(c->nv); }

/* stage slots of the host's block arrays: 2 (RK2), 3 (eSSPRK10_4).  The
 * device keeps slots 0-1 in the stacked W / Bf arrays and slot 2 in W2 /
 * Bf2. */
int host_ns(const fx_ctx *c) { return c->cfg.integrator == FX_INT_ESSPRK10_4 ? 3 : 2; }

/* factor of prj_timeint_calc_dt on the CFL minimum (src/prj_timeint.c:2246-2253) */
double dt_mult(const fx_ctx *c) { return c->cfg.integrator == FX_INT_ESSPRK10_4 ? 6.0 : 1.0; }

/* W of blocks [b0, b0 + nb) between host (host_ns slots per variable) and
 * device; state_only: slot 0 only */
int xfer_w(fx_ctx *c, int b0, int nb, double *host, cudaMemcpyKind kind, bool state_only)
{
    const int ns = host_ns(c);
    const size_t rows = (size_t)nb * c->nv;
    const size_t cell = sizeof(double) * FX_NCELLS;
    double *dev = c->d_W + (size_t)b0 * w_count(c);
    const int nslot = state_only ? 1 : 2;
    if (kind == cudaMemcpyHostToDevice) {
        FX_CUDA(c, cudaMemcpy2DAsync(dev, 2 * cell, host, ns * cell, nslot * cell, rows, kind, c->stream));
    } else {
        FX_CUDA(c, cudaMemcpy2DAsync(host, ns * cell, dev, 2 * cell, nslot * cell, rows, kind, c->stream));
    }
    if (ns == 3 && !state_only) {
        double *d2 = c->d_W2 + (size_t)b0 * c->nv * FX_NCELLS;
        if (kind == cudaMemcpyHostToDevice) {
            FX_CUDA(c, cudaMemcpy2DAsync(d2, cell, host + 2 * FX_NCELLS, 3 * cell, cell, rows, kind, c->stream));
        } else {
            FX_CUDA(c, cudaMemcpy2DAsync(host + 2 * FX_NCELLS, 3 * cell, d2, cell, cell, rows, kind, c->stream));
        }
    }
    return FX_SUCCESS;
}

/* Bf of blocks [b0, b0 + nb), rows (block, direction) */
int xfer_bf(fx_ctx *c, int b0, int nb, double *host, cudaMemcpyKind kind, bool state_only)
{
    const int ns = host_ns(c);
    const size_t rows = (size_t)nb * 3;
    const size_t face = sizeof(double) * FX_NFACES;
    double *dev = c->d_Bf + (size_t)b0 * FX_BF_COUNT;
    const int nslot = state_only ? 1 : 2;
    if (kind == cudaMemcpyHostToDevice) {
        FX_CUDA(c, cudaMemcpy2DAsync(dev, 2 * face, host, ns * face, nslot * face, rows, kind, c->stream));
    } else {
        FX_CUDA(c, cudaMemcpy2DAsync(host, ns * face, dev, 2 * face, nslot * face, rows, kind, c->stream));
    }
    if (ns == 3 && !state_only) {
        double *d2 = c->d_Bf2 + (size_t)b0 * 3 * FX_NFACES;
        if (kind == cudaMemcpyHostToDevice) {
            FX_CUDA(c, cudaMemcpy2DAsync(d2, face, host + 2 * FX_NFACES, 3 * face, face, rows, kind, c->stream));
        } else {
            FX_CUDA(c, cudaMemcpy2DAsync(host + 2 * FX_NFACES, 3 * face, d2, face, face, rows, kind, c->stream));
        }
    }
    return FX_SUCCESS;
}

/* one direction of one block's Bf (block->Bf[d]: host_ns slots) */
int xfer_bf_dir(fx_ctx *c, int b, int d, double *host, cudaMemcpyKind kind)
{
    const int ns = host_ns(c);
    double *dev = c->d_Bf + (size_t)b * FX_BF_COUNT + (size_t)d * FX_NSTAGES * FX_NFACES;
    const size_t n2 = (size_t)2 * FX_NFACES * sizeof(double);
    if (kind == cudaMemcpyHostToDevice) {
        FX_CUDA(c, cudaMemcpyAsync(dev, host, n2, kind, c->stream));
    } else {
        FX_CUDA(c, cudaMemcpyAsync(host, dev, n2, kind, c->stream));
    }
    if (ns == 3) {
        double *d2 = c->d_Bf2 + ((size_t)b * 3 + d) * FX_NFACES;
        const size_t n1 = (size_t)FX_NFACES * sizeof(double);
        if (kind == cudaMemcpyHostToDevice) {
            FX_CUDA(c, cudaMemcpyAsync(d2, host + 2 * FX_NFACES, n1, kind, c->stream));
        } else {
            FX_CUDA(c, cudaMemcpyAsync(host + 2 * FX_NFACES, d2, n1, kind, c->stream));
        }
    }
    return FX_SUCCESS;
}

/* (Re)allocates the per-block arrays for `cap` blocks.  The first `keep`
 * blocks of every array move over from the old allocation; the rest starts
 * at zero, so downloads of never-written entries are defined.  Every device
 * write goes on the context stream: the stream is non-blocking, so work on
 * the legacy default stream would not be ordered with it. */
template <typename T>
int regrow(fx_ctx *c, T **p, size_t per_block, int cap, int keep)
{
    T *old = *p;
    T *fresh = nullptr;
    const size_t n = per_block * (size_t)cap;
    if (n) {
        cudaError_t e = cudaMalloc((void **)&fresh, n * sizeof(T));
        if (e != cudaSuccess) {
            return set_err(c, FX_ENOMEM, "cudaMalloc of %zu bytes failed: %s", n * sizeof(T), cudaGetErrorString(e));
        }
        const size_t k = per_block * (size_t)keep;
        if (k && old) {
            FX_CUDA(c, cudaMemcpyAsync(fresh, old, k * sizeof(T), cudaMemcpyDeviceToDevice, c->stream));
        }
        FX_CUDA(c, cudaMemsetAsync(fresh + k, 0, (n - k) * sizeof(T), c->stream));
    }
    if (old) {
        FX_CUDA(c, cudaStreamSynchronize(c->stream));
        cudaFree(old);
    }
    *p = fresh;
    return FX_SUCCESS;
}

int alloc_block_arrays(fx_ctx *c, int cap, int keep)
{
    int rc;
    if ((rc = regrow(c, &c->d_blk, 1, cap, keep))) return rc;
    if ((rc = regrow(c, &c->d_W, w_count(c), cap, keep))) return rc;
    if ((rc = regrow(c, &c->d_flux, (size_t)FX_FLUX_COUNT(c->nv), cap, keep))) return rc;
    if ((rc = regrow(c, &c->d_vr, (size_t)FX_VR_COUNT, cap, keep))) return rc;
    if ((rc = regrow(c, &c->d_eos, (size_t)FX_EOS_COUNT, cap, keep))) return rc;
    if ((rc = regrow(c, &c->d_rhs, (size_t)FX_RHS_COUNT(c->nv), cap, keep))) return rc;
    if (c->cfg.mhd) {
        if ((rc = regrow(c, &c->d_Bf, (size_t)FX_BF_COUNT, cap, keep))) return rc;
        if ((rc = regrow(c, &c->d_bv1, (size_t)FX_BV_COUNT, cap, keep))) return rc;
        if ((rc = regrow(c, &c->d_bv2, (size_t)FX_BV_COUNT, cap, keep))) return rc;
        if ((rc = regrow(c, &c->d_emf, (size_t)FX_EMF_COUNT, cap, keep))) return rc;
    }
    if (c->cfg.gravity) {
        if ((rc = regrow(c, &c->d_grav, (size_t)FX_GRAV_COUNT, cap, keep))) return rc;
    }
    if (c->cfg.integrator == FX_INT_ESSPRK10_4) {
        if ((rc = regrow(c, &c->d_W2, (size_t)c->nv * FX_NCELLS, cap, keep))) return rc;
        if (c->cfg.mhd && (rc = regrow(c, &c->d_Bf2, (size_t)3 * FX_NFACES, cap, keep))) return rc;
    }
    if ((rc = regrow(c, &c->d_ids, 1, cap, 0))) return rc;
    c->cap = cap;
    return FX_SUCCESS;
}

/* Uploads the block geometry, the block and active lists and the compiled
 * programs of c->plan for the mesh in c->blocks, and points the device view
 * at the current arrays. */
int install_tables(fx_ctx *c)
{
    const int nblocks = c->nblocks;
    std::vector<FxBlockDev> hb(nblocks);
    for (int b = 0; b < nblocks; ++b) {
        for (int a = 0; a < 3; ++a) {
            hb[b].xmin[a] = c->blocks[b].xmin[a];
            hb[b].dx[a] = c->blocks[b].dx[a];
            hb[b].area[a] = c->blocks[b].area[a];
        }
        hb[b].vol = c->blocks[b].vol;
    }
    std::vector<int> ids(nblocks);
    for (int b = 0; b < nblocks; ++b) ids[b] = b;
    int rc;
    size_t *cap = c->tab_cap;
    if ((rc = dev_reserve(c, &c->d_active, &cap[0], (size_t)c->nactive))) return rc;
    if ((rc = dev_reserve(c, &c->d_cops, &cap[1], c->plan.ghost.cell_ops.size()))) return rc;
    if ((rc = dev_reserve(c, &c->d_fops, &cap[2], c->plan.ghost.face_ops.size()))) return rc;
    if ((rc = dev_reserve(c, &c->d_pops, &cap[3], c->plan.ghost.p_ops.size()))) return rc;
    if ((rc = dev_reserve(c, &c->d_bops, &cap[4], c->plan.ghost.b_ops.size()))) return rc;
    if ((rc = dev_reserve(c, &c->d_fcorr, &cap[5], c->plan.flux_corr.size()))) return rc;
    if ((rc = dev_reserve(c, &c->d_ecorr, &cap[6], c->plan.emf_corr.size()))) return rc;
    cudaStream_t s = c->stream;
    const cudaMemcpyKind h2d = cudaMemcpyHostToDevice;
    FX_CUDA(c, cudaMemcpyAsync(c->d_blk, hb.data(), (size_t)nblocks * sizeof(FxBlockDev), h2d, s));
    FX_CUDA(c, cudaMemcpyAsync(c->d_ids, ids.data(), (size_t)nblocks * sizeof(int), h2d, s));
    if (c->nactive) {
        FX_CUDA(c, cudaMemcpyAsync(c->d_active, c->plan.active.data(), (size_t)c->nactive * sizeof(int), h2d, s));
    }
    const FxProgram &g = c->plan.ghost;
    if (!g.cell_ops.empty()) {
        FX_CUDA(c, cudaMemcpyAsync(c->d_cops, g.cell_ops.data(), g.cell_ops.size() * sizeof(FxGop), h2d, s));
    }
    if (!g.face_ops.empty()) {
        FX_CUDA(c, cudaMemcpyAsync(c->d_fops, g.face_ops.data(), g.face_ops.size() * sizeof(FxGop), h2d, s));
    }
    if (!g.p_ops.empty()) {
        FX_CUDA(c, cudaMemcpyAsync(c->d_pops, g.p_ops.data(), g.p_ops.size() * sizeof(FxPop), h2d, s));
    }
    if (!g.b_ops.empty()) {
        FX_CUDA(c, cudaMemcpyAsync(c->d_bops, g.b_ops.data(), g.b_ops.size() * sizeof(FxBop), h2d, s));
    }
    if (!c->plan.flux_corr.empty()) {
        FX_CUDA(c, cudaMemcpyAsync(c->d_fcorr, c->plan.flux_corr.data(),
            c->plan.flux_corr.size() * sizeof(FxCorr), h2d, s));
    }
    if (!c->plan.emf_corr.empty()) {
        FX_CUDA(c, cudaMemcpyAsync(c->d_ecorr, c->plan.emf_corr.data(),
            c->plan.emf_corr.size() * sizeof(FxCorr), h2d, s));
    }
    /* the host vectors must outlive the copies */
    FX_CUDA(c, cudaStreamSynchronize(s));
    c->D.nblocks = nblocks;
    c->D.blk = c->d_blk;
    c->D.W = c->d_W;
    c->D.Bf = c->d_Bf;
    c->D.flux = c->d_flux;
    c->D.vr = c->d_vr;
    c->D.bv1 = c->d_bv1;
    c->D.bv2 = c->d_bv2;
    c->D.emf = c->d_emf;
    c->D.eos = c->d_eos;
    c->D.rhs = c->d_rhs;
    c->D.grav = c->d_grav;
    c->D.W2 = c->d_W2;
    c->D.Bf2 = c->d_Bf2;
    return FX_SUCCESS;
}

} /* namespace */

/* dynamic AMR helpers */
namespace {

bool amr_config_ok(const fx_amr_config &a, std::string *why)
{
    for (int d = 0; d < 3; ++d) {
        if (a.root_nx[d] <= 0) {
            *why = "root_nx must be positive";
            return false;
        }
    }
    for (int n = 0; n < FX_AMR_N; ++n) {
        const fx_amr_criterion &k = a.crit[n];
        if (!k.set) continue;
        if (k.estimator < FX_AMR_LOEHNER || k.estimator > FX_AMR_FRACTIONAL_JUMP) {
            *why = "unsupported estimator " + std::to_string(k.estimator);
            return false;
        }
        if (k.lohner_var < 0 || k.lohner_var > 2 || k.jump_var < 0 || k.jump_var > 1) {
            *why = "bad estimator variable";
            return false;
        }
    }
    return true;
}

FxAmrTagCfg tag_config(const fx_amr_config &a)
{
    FxAmrTagCfg t;
    std::memset(&t, 0, sizeof(t));
    for (int n = 0; n < FX_AMR_N; ++n) {
        const fx_amr_criterion &k = a.crit[n];
        if (!k.set) continue;
        const int m = t.ncrit++;
        t.est[m] = k.estimator;
        t.var[m] = k.estimator == FX_AMR_FRACTIONAL_JUMP ? k.jump_var : k.lohner_var;
        t.rthr[m] = k.refine_thresh;
        t.dthr[m] = k.derefine_thresh;
        t.eps[m] = k.lohner_eps;
        if (k.derefine_thresh > 0.0) t.has_derefine = 1;
    }
    t.reach = a.reach_density;
    return t;
}

/* device buffer holding a copy of a host vector for the duration of a call */
template <typename T>
struct DevVec {
    T *p = nullptr;
    ~DevVec() { cudaFree(p); }
    int load(fx_ctx *c, const std::vector<T> &v)
    {
        if (v.empty()) return FX_SUCCESS;
        FX_CUDA(c, cudaMalloc((void **)&p, v.size() * sizeof(T)));
        FX_CUDA(c, cudaMemcpyAsync(p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice, c->stream));
        return FX_SUCCESS;
    }
};

/* pass 1 of prj_amr_tag on the device: three int32 per block entry */
int amr_votes(fx_ctx *c, std::vector<int32_t> &votes)
{
    const int n = c->nactive;
    std::vector<int> hp(n);
    for (int i = 0; i < n; ++i) hp[i] = c->blocks[c->plan.active[i]].parent >= 0 ? 1 : 0;
    DevVec<int> d_hp;
    DevVec<int32_t> d_votes;
    int rc;
    if ((rc = d_hp.load(c, hp))) return rc;
    std::vector<int32_t> hv((size_t)3 * n, 0);
    if ((rc = d_votes.load(c, hv))) return rc;
    fx_launch_amr_tag(c->D, c->d_active, d_hp.p, n, tag_config(c->amr), d_votes.p, c->stream);
    if (n) {
        FX_CUDA(c, cudaMemcpyAsync(hv.data(), d_votes.p, hv.size() * sizeof(int32_t), cudaMemcpyDeviceToHost,
            c->stream));
    }
    if ((rc = sync_and_check(c))) return rc;
    votes.assign((size_t)3 * c->nblocks, 0);
    for (int i = 0; i < n; ++i) {
        const int b = c->plan.active[i];
        for (int q = 0; q < 3; ++q) votes[3 * b + q] = hv[3 * i + q];
    }
    return FX_SUCCESS;
}

/* Toth-Roe groups that prolong a new child's faces from its parent: 8^3
 * coarse cells of the child's octant, outer faces kept where the child
 * copied a finer neighbour's layer, every face stored once */
void child_groups(const FxAmrRefine &r, bool use_bj, std::vector<FxPop> &out)
{
    const int o[3] = {(r.oct & 1) * 8, ((r.oct >> 1) & 1) * 8, ((r.oct >> 2) & 1) * 8};
    for (int ci = o[0]; ci < o[0] + 8; ++ci) {
        for (int cj = o[1]; cj < o[1] + 8; ++cj) {
            for (int ck = o[2]; ck < o[2] + 8; ++ck) {
                const int f[3] = {2 * (ci - o[0]), 2 * (cj - o[1]), 2 * (ck - o[2])};
                FxPop p;
                std::memset(&p, 0, sizeof(p));
                p.fine = r.child;
                p.coarse = r.parent;
                p.pos = (f[0] + FX_NG) | ((f[1] + FX_NG) << 5) | ((f[2] + FX_NG) << 10) | ((ci + FX_NG) << 15) |
                    ((cj + FX_NG) << 20) | ((ck + FX_NG) << 25);
                for (int d = 0; d < 3; ++d) {
                    for (int side = 0; side < 2; ++side) {
                        const int x = f[d] + 2 * side;
                        const bool keep = (x == FX_BS && r.copy_src[2 * d + 1] >= 0) ||
                            (x == 0 && r.copy_src[2 * d] >= 0);
                        const bool store = side == 0 || x == FX_BS;
                        for (int q = 0; q < 4; ++q) {
                            const int bit = 8 * d + 4 * side + q;
                            if (keep) p.keep |= 1 << bit;
                            else if (store) p.owrite |= 1 << bit;
                        }
                    }
                }
                p.iwrite = 0xFFF;
                p.flags = use_bj ? 1 : 0;
                out.push_back(p);
            }
        }
    }
}

void drop_adjoint(fx_ctx *c)
{
    cudaFree(c->d_ckW);
    cudaFree(c->d_ckBf);
    cudaFree(c->d_ckVr);
    cudaFree(c->d_adj_csrc);
    cudaFree(c->d_adj_fsrc);
    cudaFree(c->d_adj_ents);
    cudaFree(c->d_Wb);
    cudaFree(c->d_Bfb);
    cudaFree(c->d_G);
    cudaFree(c->d_bvb1);
    cudaFree(c->d_bvb2);
    cudaFree(c->d_Eb);
    c->d_ckW = c->d_ckBf = c->d_ckVr = nullptr;
    c->d_adj_csrc = c->d_adj_fsrc = nullptr;
    c->d_adj_ents = nullptr;
    c->d_Wb = c->d_Bfb = c->d_G = c->d_bvb1 = c->d_bvb2 = c->d_Eb = nullptr;
    c->adj_ghost_ready = false;
    c->adj_nsteps = 0;
}

} /* namespace */

/* ========================================================================== */
/* C ABI                                                                      */
/* ========================================================================== */

extern "C" {

int fx_ghost_layers(void) { return FX_NG; }

int fx_create(int device, const fx_config *cfg, fx_ctx **out)
{
    if (!cfg || !out) {
        return FX_EINVAL;
    }
    *out = nullptr;
    if (cfg->mhd != 0 && cfg->mhd != 1) {
        return FX_EINVAL;
    }
    if (!(cfg->gamma > 0.0)) {
        return FX_EINVAL;
    }
    if ((cfg->recon != FX_RECON_MC && cfg->recon != FX_RECON_WENO3 && cfg->recon != FX_RECON_WENO7) ||
        (cfg->integrator != FX_INT_RK2 && cfg->integrator != FX_INT_ESSPRK10_4)) {
        return FX_EINVAL;
    }
    if (cfg->recon == FX_RECON_WENO7 && FX_NG < 4) {
        return FX_EINVAL; /* PRJ_RECON_WENO7 requires PRJ_NGHOST >= 4 (src/prj_defs.h:349-351) */
    }
    fx_ctx *c = new fx_ctx();
    c->device = device;
    c->cfg = *cfg;
    c->nv = cfg->mhd ? 9 : 6;
    if (cudaSetDevice(device) != cudaSuccess ||
        cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaMalloc((void **)&c->d_err, sizeof(FxErr)) != cudaSuccess ||
        cudaMalloc((void **)&c->d_red, 3 * sizeof(unsigned long long)) != cudaSuccess ||
        cudaMalloc((void **)&c->d_ctl, sizeof(FxCtl)) != cudaSuccess ||
        cudaMallocHost((void **)&c->h_err, sizeof(FxErr)) != cudaSuccess ||
        cudaMallocHost((void **)&c->h_red, 3 * sizeof(unsigned long long)) != cudaSuccess ||
        cudaMallocHost((void **)&c->h_ctl, sizeof(FxCtl)) != cudaSuccess) {
        fx_destroy(c);
        return FX_ECUDA;
    }
    cudaMemsetAsync(c->d_err, 0, sizeof(FxErr), c->stream);
    cudaMemsetAsync(c->d_ctl, 0, sizeof(FxCtl), c->stream);
    cudaMemsetAsync(c->d_red, 0, 3 * sizeof(unsigned long long), c->stream);
    if (cudaStreamSynchronize(c->stream) != cudaSuccess) {
        fx_destroy(c);
        return FX_ECUDA;
    }
    c->D.nv = c->nv;
    c->D.gamma = cfg->gamma;
    c->D.mhd_eta = cfg->mhd_eta;
    c->D.err = c->d_err;
    c->D.red = c->d_red;
    c->D.ctl = c->d_ctl;
    c->D.recon = cfg->recon;
    c->D.use_bj = cfg->use_bj != 0;
    {
        FxCtl v{};
        v.dt_mult = dt_mult(c);
        *c->h_ctl = v;
        fx_launch_set_ctl(c->D, v, c->stream);
        if (cudaStreamSynchronize(c->stream) != cudaSuccess) {
            fx_destroy(c);
            return FX_ECUDA;
        }
    }
    *out = c;
    return FX_SUCCESS;
}

void fx_destroy(fx_ctx *c)
{
    if (!c) {
        return;
    }
    fx_plan_workspace_free(c->plan_ws);
    c->plan_ws = nullptr;
    cudaSetDevice(c->device);
    if (c->stream) {
        cudaStreamSynchronize(c->stream);
    }
    free_mesh(c);
    delete c->transport;
    c->transport = nullptr;
    cudaFree(c->d_br_words);
    cudaFree(c->d_br_edges);
    cudaFree(c->d_err);
    cudaFree(c->d_red);
    cudaFree(c->d_ctl);
    cudaFreeHost(c->h_err);
    cudaFreeHost(c->h_red);
    cudaFreeHost(c->h_ctl);
    if (c->stream) {
        cudaStreamDestroy(c->stream);
    }
    delete c;
}

int fx_last_error(const fx_ctx *c, char *buf, size_t len)
{
    if (!c || !buf || len == 0) {
        return FX_EINVAL;
    }
    snprintf(buf, len, "%s", c->err.c_str());
    return FX_SUCCESS;
}

int fx_sync(fx_ctx *c)
{
    if (!c) return FX_EINVAL;
    return sync_and_check(c);
}

int fx_stream(fx_ctx *c, void **stream)
{
    if (!c || !stream) return FX_EINVAL;
    *stream = (void *)c->stream;
    return FX_SUCCESS;
}

int fx_set_mesh(fx_ctx *c, int nblocks, const fx_block_desc *blocks)
{
    if (!c || nblocks <= 0 || !blocks) {
        return c ? set_err(c, FX_EINVAL, "fx_set_mesh: empty mesh") : FX_EINVAL;
    }
    if (nblocks >= (1 << 16)) {
        return set_err(c, FX_EINVAL, "fx_set_mesh: at most 65535 blocks per device");
    }
    FX_CUDA(c, cudaSetDevice(c->device));
    FX_CUDA(c, cudaStreamSynchronize(c->stream));
    free_mesh(c);
    std::string perr;
    FxPlan plan;
    if (!fx_build_plan(c->cfg, nblocks, blocks, plan, &perr)) {
        return set_err(c, FX_EINVAL, "fx_set_mesh: %s", perr.c_str());
    }
    c->plan = std::move(plan);
    c->blocks.assign(blocks, blocks + nblocks);
    c->nblocks = nblocks;
    c->nactive = (int)c->plan.active.size();
    int rc;
    if ((rc = alloc_block_arrays(c, nblocks, 0))) return rc;
    if ((rc = install_tables(c))) return rc;
    c->last_slot = 0;
    return FX_SUCCESS;
}

int fx_shard_set_mesh(fx_ctx *c, int nblocks, const fx_block_desc *blocks, const int *owner, int nranks,
    int rank)
{
    if (!c || nblocks <= 0 || !blocks || !owner) {
        return c ? set_err(c, FX_EINVAL, "fx_shard_set_mesh: empty mesh") : FX_EINVAL;
    }
    if (c->cfg.integrator != FX_INT_RK2) {
        return set_err(c, FX_EINVAL, "fx_shard_set_mesh: sharded meshes run the RK2 integrator");
    }
    FX_CUDA(c, cudaSetDevice(c->device));
    FX_CUDA(c, cudaStreamSynchronize(c->stream));
    free_mesh(c);
    delete c->transport;
    c->transport = nullptr;
    c->xerr.clear();
    std::string perr;
    FxPlan plan;
    if (!fx_build_shard_plan(c->cfg, nblocks, blocks, owner, nranks, rank, plan, &perr)) {
        return set_err(c, FX_EINVAL, "fx_shard_set_mesh: %s", perr.c_str());
    }
    const FxShard &sh = plan.shard;
    const int nl = (int)sh.local_to_global.size();
    if (nl >= (1 << 16)) return set_err(c, FX_EINVAL, "fx_shard_set_mesh: at most 65535 blocks per device");
    c->blocks.resize(nl);
    for (int l = 0; l < nl; ++l) c->blocks[l] = blocks[sh.local_to_global[l]];
    c->nblocks = nl;
    c->nactive = (int)plan.active.size();
    int rc;
    if ((rc = alloc_block_arrays(c, nl, 0))) return rc;
    c->plan = std::move(plan);
    if ((rc = install_tables(c))) return rc;
    c->last_slot = 0;
    /* packed exchanges: ghost fill = cells (6 primitives) then faces, per
     * peer; flux entries (6 components); EMF entries */
    const FxShard &s2 = c->plan.shard;
    const int kinds[3][2] = {{FX_X_CELLS, FX_X_FACES}, {FX_X_FLUX, -1}, {FX_X_EMF, -1}};
    for (int x = 0; x < 3; ++x) {
        FxXdev &X = c->X[x];
        for (int dirn = 0; dirn < 2; ++dirn) {
            const FxXlist *lists = dirn == 0 ? s2.send : s2.recv;
            std::vector<FxXent> ents;
            std::vector<size_t> off(1, 0);
            size_t pos = 0;
            for (int p = 0; p < nranks; ++p) {
                for (int q = 0; q < 2; ++q) {
                    const int k = kinds[x][q];
                    if (k < 0) continue;
                    const int width = (k == FX_X_CELLS || k == FX_X_FLUX) ? 6 : 1;
                    const FxXlist &l = lists[k];
                    for (int e = l.begin[p]; e < l.begin[p + 1]; ++e) {
                        ents.push_back({l.el[e].block, l.el[e].idx, k, (int32_t)pos});
                        pos += width;
                    }
                }
                off.push_back(pos);
            }
            if (pos >= (size_t)1 << 31) return set_err(c, FX_ETOOBIG, "fx_shard_set_mesh: exchange too large");
            FxXent **d = dirn == 0 ? &X.d_send : &X.d_recv;
            double **buf = dirn == 0 ? &X.sbuf : &X.rbuf;
            if ((rc = dev_alloc(c, d, ents.size()))) return rc;
            if ((rc = dev_alloc(c, buf, pos))) return rc;
            if (!ents.empty()) {
                FX_CUDA(c, cudaMemcpy(*d, ents.data(), ents.size() * sizeof(FxXent), cudaMemcpyHostToDevice));
            }
            (dirn == 0 ? X.nsend : X.nrecv) = (int)ents.size();
            (dirn == 0 ? X.soff : X.roff) = off;
        }
        X.any = s2.any[kinds[x][0]] || (kinds[x][1] >= 0 && s2.any[kinds[x][1]]);
    }
    c->nranks = nranks;
    c->rank = rank;
    c->nowned = s2.nowned;
    c->g2l.assign(nblocks, -1);
    for (int l = 0; l < nl; ++l) c->g2l[s2.local_to_global[l]] = l;
    return FX_SUCCESS;
}

int fx_shard_attach_group(fx_ctx *c, fx_shard_group *g)
{
    if (!c || !g) return c ? set_err(c, FX_EINVAL, "fx_shard_attach_group: null group") : FX_EINVAL;
    if (c->nranks == 1 || fx_group_size(g) != c->nranks) {
        return set_err(c, FX_EINVAL, "fx_shard_attach_group: the group size must equal the mesh's rank count");
    }
    delete c->transport;
    c->transport = fx_transport_group(g, c->rank);
    free_graphs(c);
    return FX_SUCCESS;
}

int fx_shard_attach_nccl(fx_ctx *c, const unsigned char id[128])
{
    if (!c || !id) return c ? set_err(c, FX_EINVAL, "fx_shard_attach_nccl: null id") : FX_EINVAL;
    if (c->nranks == 1 && !c->nblocks) return set_err(c, FX_ENOMESH, "fx_shard_attach_nccl: no sharded mesh");
    std::string err;
    FxTransport *t = fx_transport_nccl(c->nranks, c->rank, id, c->device, &err);
    if (!t) return set_err(c, FX_ECOMM, "fx_shard_attach_nccl: %s", err.c_str());
    delete c->transport;
    c->transport = t;
    free_graphs(c);
    return FX_SUCCESS;
}

int fx_nccl_unique_id(unsigned char id[128])
{
    if (!id) return FX_EINVAL;
    std::string err;
    return fx_transport_nccl_id(id, &err) ? FX_ECOMM : FX_SUCCESS;
}

fx_shard_group *fx_shard_group_create(int nranks) { return fx_group_new(nranks); }

void fx_shard_group_destroy(fx_shard_group *g) { fx_group_delete(g); }

int fx_shard_info(fx_ctx *c, int *nowned, int *nlocal, long long *doubles_per_step)
{
    if (!has_mesh(c)) return c ? set_err(c, FX_ENOMESH, "no mesh") : FX_EINVAL;
    if (nowned) *nowned = c->nranks > 1 ? c->nowned : c->nactive;
    if (nlocal) *nlocal = c->nblocks;
    if (doubles_per_step) {
        /* sent per RK2 step: two stages, each with every exchange */
        long long n = 0;
        for (const FxXdev &x : c->X) {
            if (x.any && !x.soff.empty()) n += (long long)x.soff.back();
        }
        *doubles_per_step = 2 * n;
    }
    return FX_SUCCESS;
}

namespace {

/* fx_plan_export / fx_shard_export of a built plan */
int export_plan(const FxPlan &plan, int which, int32_t *ops, int *nops, int32_t *wave_begin, int *nwaves)
{
    const FxProgram &g = plan.ghost;
    if (which >= 7) {
        const FxShard &sh = plan.shard;
        if (which == 7) {
            const std::vector<int> &m = sh.local_to_global;
            if (ops && (int)m.size() <= *nops && !m.empty()) std::memcpy(ops, m.data(), m.size() * sizeof(int));
            *nops = (int)m.size();
            *nwaves = sh.nowned;
            return FX_SUCCESS;
        }
        const FxXlist &l = which < 12 ? sh.send[which - 8] : sh.recv[which - 12];
        if (ops && (int)l.el.size() <= *nops && !l.el.empty()) {
            std::memcpy(ops, l.el.data(), l.el.size() * sizeof(FxXel));
        }
        if (wave_begin && sh.nranks <= *nwaves) {
            std::memcpy(wave_begin, l.begin.data(), l.begin.size() * sizeof(int));
        }
        *nops = (int)l.el.size();
        *nwaves = sh.nranks;
        return FX_SUCCESS;
    }
    if (which <= 1 || which == 4 || which == 6) {
        const void *data = which == 0 ? (const void *)g.cell_ops.data() :
            which == 1 ? (const void *)g.face_ops.data() :
            which == 4 ? (const void *)g.b_ops.data() : (const void *)g.p_ops.data();
        const size_t count = which == 0 ? g.cell_ops.size() : which == 1 ? g.face_ops.size() :
            which == 4 ? g.b_ops.size() : g.p_ops.size();
        const size_t size = which == 4 ? sizeof(FxBop) : which == 6 ? sizeof(FxPop) : sizeof(FxGop);
        const std::vector<int> &wb = which == 0 ? g.cell_begin : which == 1 ? g.face_begin :
            which == 4 ? g.b_begin : g.p_begin;
        if (ops && (int)count <= *nops && count) {
            std::memcpy(ops, data, count * size);
        }
        if (wave_begin && g.nwaves() <= *nwaves) {
            std::memcpy(wave_begin, wb.data(), wb.size() * sizeof(int));
        }
        *nops = (int)count;
        *nwaves = g.nwaves();
    } else if (which == 5) {
        /* statistics: emitted cell ops, emitted face ops, rewired, dead */
        if (ops && *nops >= 4) {
            ops[0] = (int32_t)plan.stats.emitted_cell_ops;
            ops[1] = (int32_t)plan.stats.emitted_face_ops;
            ops[2] = (int32_t)plan.stats.rewired;
            ops[3] = (int32_t)plan.stats.dead;
        }
        *nops = 4;
        *nwaves = g.nwaves();
    } else {
        const std::vector<FxCorr> &r = which == 2 ? plan.flux_corr : plan.emf_corr;
        const std::vector<int> &wb = which == 2 ? plan.flux_corr_begin : plan.emf_corr_begin;
        const int nw = (int)wb.size() - 1;
        if (ops && (int)r.size() <= *nops) {
            std::memcpy(ops, r.data(), r.size() * sizeof(FxCorr));
        }
        if (wave_begin && nw <= *nwaves) {
            std::memcpy(wave_begin, wb.data(), wb.size() * sizeof(int));
        }
        *nops = (int)r.size();
        *nwaves = nw;
    }
    return FX_SUCCESS;
}

} /* namespace */

int fx_plan_export(const fx_config *cfg, int nblocks, const fx_block_desc *blocks, int which,
    int32_t *ops, int *nops, int32_t *wave_begin, int *nwaves)
{
    if (!cfg || nblocks <= 0 || !blocks || !nops || !nwaves || which < 0 || which > 6) {
        return FX_EINVAL;
    }
    FxPlan plan;
    std::string perr;
    const bool corr_only = which == 2 || which == 3;
    if (!(corr_only ? fx_build_corrections(*cfg, nblocks, blocks, plan, &perr) :
                      fx_build_plan(*cfg, nblocks, blocks, plan, &perr))) {
        return FX_EINVAL;
    }
    return export_plan(plan, which, ops, nops, wave_begin, nwaves);
}

int fx_shard_export(const fx_config *cfg, int nblocks, const fx_block_desc *blocks, const int *owner,
    int nranks, int rank, int which, int32_t *ops, int *nops, int32_t *wave_begin, int *nwaves)
{
    if (!cfg || nblocks <= 0 || !blocks || !owner || !nops || !nwaves || which < 0 || which > 15 ||
        which == 5) {
        return FX_EINVAL;
    }
    FxPlan plan;
    std::string perr;
    if (!fx_build_shard_plan(*cfg, nblocks, blocks, owner, nranks, rank, plan, &perr)) {
        return FX_EINVAL;
    }
    return export_plan(plan, which, ops, nops, wave_begin, nwaves);
}

int fx_upload_block(fx_ctx *c, int b, const double *W, const double *const Bf[3],
    const double *const grav[3])
{
    if (!has_mesh(c)) return c ? set_err(c, FX_ENOMESH, "no mesh") : FX_EINVAL;
    int rc;
    if ((rc = local_block(c, &b))) return rc;
    if (W && (rc = xfer_w(c, b, 1, const_cast<double *>(W), cudaMemcpyHostToDevice, false))) return rc;
    if (Bf && c->cfg.mhd) {
        for (int d = 0; d < 3; ++d) {
            if (Bf[d] && (rc = xfer_bf_dir(c, b, d, const_cast<double *>(Bf[d]), cudaMemcpyHostToDevice))) return rc;
        }
    }
    if (grav && c->d_grav) {
        for (int d = 0; d < 3; ++d) {
            if (grav[d]) {
                FX_CUDA(c, cudaMemcpyAsync(c->d_grav + (size_t)b * FX_GRAV_COUNT + (size_t)d * FX_NCELLS,
                    grav[d], (size_t)FX_NCELLS * sizeof(double), cudaMemcpyHostToDevice, c->stream));
            }
        }
    }
    FX_CUDA(c, cudaStreamSynchronize(c->stream));
    return FX_SUCCESS;
}

int fx_download_block(fx_ctx *c, int b, double *W, double *eosvar, double *const Bf[3])
{
    if (!has_mesh(c)) return c ? set_err(c, FX_ENOMESH, "no mesh") : FX_EINVAL;
    int rc;
    if ((rc = local_block(c, &b))) return rc;
    if (W && (rc = xfer_w(c, b, 1, W, cudaMemcpyDeviceToHost, false))) return rc;
    if (eosvar) {
        fx_launch_eos_fill(c->D, c->d_ids + b, 1, c->last_slot, 0, c->stream);
        FX_CUDA(c, cudaMemcpyAsync(eosvar, c->d_eos + (size_t)b * FX_EOS_COUNT, FX_EOS_COUNT * sizeof(double),
            cudaMemcpyDeviceToHost, c->stream));
    }
    if (Bf && c->cfg.mhd) {
        for (int d = 0; d < 3; ++d) {
            if (Bf[d] && (rc = xfer_bf_dir(c, b, d, Bf[d], cudaMemcpyDeviceToHost))) return rc;
        }
    }
    return sync_and_check(c);
}

int fx_upload_all(fx_ctx *c, const double *W_all, const double *Bf_all)
{
    if (c && c->nranks > 1) return set_err(c, FX_EINVAL, "%s: not available on a sharded mesh", __func__);
    if (!has_mesh(c)) return c ? set_err(c, FX_ENOMESH, "no mesh") : FX_EINVAL;
    int rc;
    if (W_all && (rc = xfer_w(c, 0, c->nblocks, const_cast<double *>(W_all), cudaMemcpyHostToDevice, false))) return rc;
    if (Bf_all && c->cfg.mhd &&
        (rc = xfer_bf(c, 0, c->nblocks, const_cast<double *>(Bf_all), cudaMemcpyHostToDevice, false))) return rc;
    return FX_SUCCESS;
}

int fx_download_all(fx_ctx *c, double *W_all, double *Bf_all)
{
    if (c && c->nranks > 1) return set_err(c, FX_EINVAL, "%s: not available on a sharded mesh", __func__);
    if (!has_mesh(c)) return c ? set_err(c, FX_ENOMESH, "no mesh") : FX_EINVAL;
    int rc;
    if (W_all && (rc = xfer_w(c, 0, c->nblocks, W_all, cudaMemcpyDeviceToHost, false))) return rc;
    if (Bf_all && c->cfg.mhd && (rc = xfer_bf(c, 0, c->nblocks, Bf_all, cudaMemcpyDeviceToHost, false))) return rc;
    return sync_and_check(c);
}

int fx_upload_state(fx_ctx *c, const double *W_all, const double *Bf_all)
{
    if (c && c->nranks > 1) return set_err(c, FX_EINVAL, "%s: not available on a sharded mesh", __func__);
    if (!has_mesh(c)) return c ? set_err(c, FX_ENOMESH, "no mesh") : FX_EINVAL;
    int rc;
    if (W_all && (rc = xfer_w(c, 0, c->nblocks, const_cast<double *>(W_all), cudaMemcpyHostToDevice, true))) return rc;
    if (Bf_all && c->cfg.mhd &&
        (rc = xfer_bf(c, 0, c->nblocks, const_cast<double *>(Bf_all), cudaMemcpyHostToDevice, true))) return rc;
    return FX_SUCCESS;
}

int fx_download_state(fx_ctx *c, double *W_all, double *Bf_all)
{
    if (c && c->nranks > 1) return set_err(c, FX_EINVAL, "%s: not available on a sharded mesh", __func__);
    if (!has_mesh(c)) return c ? set_err(c, FX_ENOMESH, "no mesh") : FX_EINVAL;
    int rc;
    if (W_all && (rc = xfer_w(c, 0, c->nblocks, W_all, cudaMemcpyDeviceToHost, true))) return rc;
    if (Bf_all && c->cfg.mhd && (rc = xfer_bf(c, 0, c->nblocks, Bf_all, cudaMemcpyDeviceToHost, true))) return rc;
    return FX_SUCCESS;
}

/* Copies of slot 0's active region by the copy engines: for W one 3-D copy
 * per variable over blocks, for Bf one per direction over blocks; every
 * copied row is the whole span of one i-plane's active rows (ghost columns
 * along k included), 2.5-2.7 KB, so the engines run at full rate.  Every
 * block entry (active or not) is covered.  Host -> device leaves out the
 * cell-centred field (MHD; recomputed from the faces), device -> host
 * copies every variable. */
int dma_active(fx_ctx *c, double *W_all, double *Bf_all, cudaMemcpyKind kind)
{
    constexpr size_t P = FX_PBS;
    constexpr size_t G = FX_NG;
    constexpr size_t B = FX_BS;
    const size_t hs = (size_t)host_ns(c);
    const size_t nb = (size_t)c->nblocks;
    const bool up = kind == cudaMemcpyHostToDevice;
    auto copy3d = [&](double *host, size_t host_ysize, double *dev, size_t dev_ysize, size_t pitch_el,
                      size_t width_el, size_t height, size_t depth) -> cudaError_t {
        cudaMemcpy3DParms p{};
        cudaPitchedPtr h = make_cudaPitchedPtr(host, pitch_el * sizeof(double), width_el * sizeof(double), host_ysize);
        cudaPitchedPtr d = make_cudaPitchedPtr(dev, pitch_el * sizeof(double), width_el * sizeof(double), dev_ysize);
        p.srcPtr = up ? h : d;
        p.dstPtr = up ? d : h;
        p.extent = make_cudaExtent(width_el * sizeof(double), height, depth);
        p.kind = kind;
        return cudaMemcpy3DAsync(&p, c->stream);
    };
    if (W_all) {
        /* cell (i, j, k) = (i + G) P^2 + (j + G) P + (k + G); rows: i-planes of
         * the active j range, z: blocks, one copy per variable */
        const size_t off = G * P * P + G * P;
        const size_t nvar = (up && c->cfg.mhd) ? (size_t)FX_B1 : (size_t)c->nv;
        for (size_t v = 0; v < nvar; ++v) {
            const size_t hoff = v * hs * FX_NCELLS + off;
            const size_t doff = v * FX_NSTAGES * FX_NCELLS + off;
            FX_CUDA(c, copy3d(W_all + hoff, (size_t)c->nv * hs * P, c->d_W + doff, (size_t)c->nv * FX_NSTAGES * P,
                P * P, B * P, B, nb));
        }
    }
    if (Bf_all && c->cfg.mhd) {
        for (int d = 0; d < 3; ++d) {
            /* face strides: i-planes P^2 (d = 0) or P (P + 1); rows P (d = 0, 1) or P + 1 */
            const size_t plane = d == 0 ? P * P : P * (P + 1);
            const size_t row = d == 2 ? P + 1 : P;
            const size_t nplanes = d == 0 ? B + 1 : B;
            const size_t nrows = d == 1 ? B + 1 : B;
            const size_t off = G * plane + G * row;
            const size_t hoff = (size_t)d * hs * FX_NFACES + off;
            const size_t doff = (size_t)d * FX_NSTAGES * FX_NFACES + off;
            FX_CUDA(c, copy3d(Bf_all + hoff, 3 * hs * FX_NFACES / plane, c->d_Bf + doff,
                3 * (size_t)FX_NSTAGES * FX_NFACES / plane, plane, nrows * row, nplanes, nb));
        }
    }
    return FX_SUCCESS;
}

int fx_upload_state_active(fx_ctx *c, const double *W_all, const double *Bf_all)
{
    if (c && c->nranks > 1) return set_err(c, FX_EINVAL, "%s: not available on a sharded mesh", __func__);
    if (!has_mesh(c)) return c ? set_err(c, FX_ENOMESH, "no mesh") : FX_EINVAL;
    if (!W_all) return set_err(c, FX_EINVAL, "%s: W_all is required", __func__);
    int rc = dma_active(c, const_cast<double *>(W_all), const_cast<double *>(Bf_all), cudaMemcpyHostToDevice);
    if (rc) return rc;
    if (c->cfg.mhd) {
        if (!Bf_all) return set_err(c, FX_EINVAL, "%s: Bf_all is required in MHD runs", __func__);
        fx_launch_cell_field_active(c->D, c->d_active, c->nactive, c->stream);
    }
    /* the ghost cells and faces of slot 0 from the active ones: the fill
     * that produced the host's ghost zones (src/main.c:446) */
    return fx_boundary_fill_ghosts_and_bf(c, 1, 0);
}

int fx_download_state_active(fx_ctx *c, double *W_all, double *Bf_all)
{
    if (c && c->nranks > 1) return set_err(c, FX_EINVAL, "%s: not available on a sharded mesh", __func__);
    if (!has_mesh(c)) return c ? set_err(c, FX_ENOMESH, "no mesh") : FX_EINVAL;
    if (!W_all) return set_err(c, FX_EINVAL, "%s: W_all is required", __func__);
    const int rc = dma_active(c, W_all, Bf_all, cudaMemcpyDeviceToHost);
    return rc ? rc : sync_and_check(c);
}

int fx_dump_gather(fx_ctx *c, double *data, double *eos, double *bf)
{
    if (c && c->nranks > 1) return set_err(c, FX_EINVAL, "%s: not available on a sharded mesh", __func__);
    if (!has_mesh(c)) return c ? set_err(c, FX_ENOMESH, "no mesh") : FX_EINVAL;
    if (!data && !eos && !bf) return set_err(c, FX_EINVAL, "%s: no output", __func__);
    const int faces = (bf && c->cfg.mhd) ? 1 : 0;
    const size_t nc = (size_t)FX_BS * FX_BS * FX_BS;
    const size_t nw = (size_t)c->nv * nc;
    const size_t row = nw + 3 * nc + (faces ? (size_t)3 * FX_NFACES : 0);
    const size_t n = (size_t)c->nactive;
    if (n == 0) return FX_SUCCESS;
    /* eosvar of the stored state (the batched form does not keep it) */
    fx_launch_eos_fill(c->D, c->d_active, c->nactive, 0, 1, c->stream);
    double *d = nullptr;
    cudaError_t e = cudaMalloc((void **)&d, n * row * sizeof(double));
    if (e != cudaSuccess) {
        cudaGetLastError();
        return set_err(c, FX_ENOMEM, "%s: no room for the %zu-byte staging buffer", __func__, n * row * sizeof(double));
    }
    std::vector<double> h(n * row);
    fx_launch_dump_pack(c->D, c->d_active, c->nactive, faces, d, c->stream);
    e = cudaMemcpyAsync(h.data(), d, n * row * sizeof(double), cudaMemcpyDeviceToHost, c->stream);
    const cudaError_t e2 = cudaStreamSynchronize(c->stream);
    cudaFree(d);
    if (e != cudaSuccess || e2 != cudaSuccess) {
        cudaGetLastError();
        return set_err(c, FX_ECUDA, "%s: %s", __func__, cudaGetErrorString(e != cudaSuccess ? e : e2));
    }
    std::vector<int> act(n);
    FX_CUDA(c, cudaMemcpy(act.data(), c->d_active, n * sizeof(int), cudaMemcpyDeviceToHost));
    for (size_t q = 0; q < n; ++q) {
        const size_t b = (size_t)act[q];
        const double *r = h.data() + q * row;
        if (data) std::memcpy(data + b * nw, r, nw * sizeof(double));
        if (eos) std::memcpy(eos + b * 3 * nc, r + nw, 3 * nc * sizeof(double));
        if (faces) std::memcpy(bf + b * 3 * FX_NFACES, r + nw + 3 * nc, 3 * (size_t)FX_NFACES * sizeof(double));
    }
    return sync_and_check(c);
}

int fx_dump_metadata(int nblocks, const fx_block_desc *blocks, double *meta)
{
    if (nblocks < 0 || (nblocks > 0 && (!blocks || !meta))) return FX_EINVAL;
    for (int b = 0; b < nblocks; ++b) {
        const fx_block_desc &k = blocks[b];
        double *m = meta + (size_t)b * FX_DUMP_METADATA_SIZE;
        std::fill(m, m + FX_DUMP_METADATA_SIZE, 0.0);
        m[0] = (double)k.id;
        m[2] = (double)k.level;
        m[3] = (double)k.active;
        for (int a = 0; a < 3; ++a) {
            m[4 + a] = k.xmin[a];
            m[7 + a] = k.xmax[a];
            m[10 + a] = k.dx[a];
        }
        m[13] = (double)k.parent;
        for (int o = 0; o < 8; ++o) m[15 + o] = (double)k.children[o];
        int idx = 23;
        for (int n = 0; n < 56; ++n) {
            const int id = k.slot[n].id;
            m[idx++] = (double)id;
            ++idx; /* the slot's rank: 0 */
            const bool nb = id >= 0 && id < nblocks;
            for (int a = 0; a < 3; ++a) m[idx++] = nb ? blocks[id].xmin[a] : 0.0;
            for (int a = 0; a < 3; ++a) m[idx++] = nb ? blocks[id].xmax[a] : 0.0;
            for (int a = 0; a < 3; ++a) m[idx++] = nb ? blocks[id].dx[a] : 0.0;
        }
    }
    return FX_SUCCESS;
}

int fx_download_array(fx_ctx *c, int b, int which, int dir, double *out)
{
    if (c && c->nranks > 1) return set_err(c, FX_EINVAL, "%s: not available on a sharded mesh", __func__);
    if (!has_mesh(c)) return c ? set_err(c, FX_ENOMESH, "no mesh") : FX_EINVAL;
    if (b < 0 || b >= c->nblocks || dir < 0 || dir > 2 || !out) {
        return set_err(c, FX_EINVAL, "fx_download_array: bad arguments");
    }
    const double *src = nullptr;
    size_t count = 0;
    const size_t nv = (size_t)c->nv;
    switch (which) {
    case FX_ARR_W: {
        int rc = xfer_w(c, b, 1, out, cudaMemcpyDeviceToHost, false);
        return rc ? rc : sync_and_check(c);
    }
    case FX_ARR_EOSVAR: src = c->d_eos + (size_t)b * FX_EOS_COUNT; count = FX_EOS_COUNT; break;
    case FX_ARR_RHS: src = c->d_rhs + (size_t)b * FX_RHS_COUNT(nv); count = FX_RHS_COUNT(nv); break;
    case FX_ARR_FLUX: src = c->d_flux + (size_t)b * FX_FLUX_COUNT(nv) + (size_t)dir * nv * FX_NCELLS;
        count = nv * FX_NCELLS; break;
    case FX_ARR_VRIEMANN: src = c->d_vr + (size_t)b * FX_VR_COUNT + (size_t)dir * 3 * FX_NCELLS;
        count = 3 * FX_NCELLS; break;
    case FX_ARR_GRAV:
        if (!c->d_grav) return set_err(c, FX_EINVAL, "no gravity arrays");
        src = c->d_grav + (size_t)b * FX_GRAV_COUNT + (size_t)dir * FX_NCELLS; count = FX_NCELLS; break;
    case FX_ARR_BF:
    case FX_ARR_BV1:
    case FX_ARR_BV2:
    case FX_ARR_EMF:
        if (!c->cfg.mhd) return set_err(c, FX_EINVAL, "field arrays exist only in MHD runs");
        if (which == FX_ARR_BF) {
            int rc = xfer_bf_dir(c, b, dir, out, cudaMemcpyDeviceToHost);
            return rc ? rc : sync_and_check(c);
        } else if (which == FX_ARR_EMF) {
            src = c->d_emf + (size_t)b * FX_EMF_COUNT + (size_t)dir * FX_NEDGES;
            count = FX_NEDGES;
        } else {
            src = (which == FX_ARR_BV1 ? c->d_bv1 : c->d_bv2) + (size_t)b * FX_BV_COUNT + (size_t)dir * FX_NCELLS;
            count = FX_NCELLS;
        }
        break;
    default:
        return set_err(c, FX_EINVAL, "fx_download_array: unknown array %d", which);
    }
    FX_CUDA(c, cudaMemcpyAsync(out, src, count * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    return sync_and_check(c);
}

/* ---- per-block reference entry points ---------------------------------------- */

static int check_block(fx_ctx *c, int b)
{
    if (!has_mesh(c)) return c ? set_err(c, FX_ENOMESH, "no mesh") : FX_EINVAL;
    if (b < 0 || b >= c->nblocks) return set_err(c, FX_EINVAL, "block %d out of range", b);
    return FX_SUCCESS;
}

int fx_flux_update(fx_ctx *c, int b, int w_slot, int use_bf1)
{
    if (c && c->nranks > 1) return set_err(c, FX_EINVAL, "%s: not available on a sharded mesh", __func__);
    int rc = check_block(c, b);
    if (rc) return rc;
    if (w_slot < 0 || w_slot > 1 || use_bf1 < 0 || use_bf1 > 1) return set_err(c, FX_EINVAL, "bad slot");
    fx_launch_set_dt(c->D, 0.0, c->stream);
    fx_launch_flux(c->D, c->d_ids + b, 1, 3, w_slot, use_bf1, 1, c->stream);
    return FX_SUCCESS;
}

int fx_mhd_update_emf(fx_ctx *c, int b, int stage)
{
    if (c && c->nranks > 1) return set_err(c, FX_EINVAL, "%s: not available on a sharded mesh", __func__);
    int rc = check_block(c, b);
    if (rc) return rc;
    if (!c->cfg.mhd || stage < 0 || stage > 1) return set_err(c, FX_EINVAL, "bad emf call");
    fx_launch_set_dt(c->D, 0.0, c->stream);
    fx_launch_emf(c->D, c->d_ids + b, 1, stage, stage, c->stream);
    return FX_SUCCESS;
}

int fx_mhd_update_bf(fx_ctx *c, int b, int stage, double dt)
{
    if (c && c->nranks > 1) return set_err(c, FX_EINVAL, "%s: not available on a sharded mesh", __func__);
    int rc = check_block(c, b);
    if (rc) return rc;
    if (!c->cfg.mhd || (stage != 1 && stage != 2)) return set_err(c, FX_EINVAL, "bad bf update call");
    fx_launch_set_dt(c->D, dt, c->stream);
    fx_launch_bf_update(c->D, c->d_ids + b, 1, stage, c->stream);
    return FX_SUCCESS;
}

int fx_update_cells(fx_ctx *c, int b, int stage, double dt, double *dt_src)
{
    if (c && c->nranks > 1) return set_err(c, FX_EINVAL, "%s: not available on a sharded mesh", __func__);
    int rc = check_block(c, b);
    if (rc) return rc;
    if (stage != 1 && stage != 2) return set_err(c, FX_EINVAL, "bad stage");
    fx_launch_set_dt(c->D, dt, c->stream);
    if (dt_src) fx_launch_reset_reductions(c->D, 2, c->stream);
    fx_launch_cell_update(c->D, c->d_ids + b, 1, stage, c->cfg.gravity, 1, c->stream);
    c->last_slot = stage == 1 ? 1 : 0;
    if (dt_src) {
        double v;
        rc = read_dt_src(c, &v);
        if (rc) return rc;
        if (v < *dt_src) *dt_src = v;
    }
    return FX_SUCCESS;
}

int fx_riemann_flux_send(fx_ctx *c)
{
    if (c && c->nranks > 1) return set_err(c, FX_EINVAL, "%s: not available on a sharded mesh", __func__);
    if (!has_mesh(c)) return c ? set_err(c, FX_ENOMESH, "no mesh") : FX_EINVAL;
    fx_launch_set_dt(c->D, 0.0, c->stream);
    flux_correct(c, c->nv, c->stream);
    return FX_SUCCESS;
}

int fx_mhd_emf_send(fx_ctx *c)
{
    if (c && c->nranks > 1) return set_err(c, FX_EINVAL, "%s: not available on a sharded mesh", __func__);
    if (!has_mesh(c)) return c ? set_err(c, FX_ENOMESH, "no mesh") : FX_EINVAL;
    fx_launch_set_dt(c->D, 0.0, c->stream);
    emf_correct(c, c->stream);
    return FX_SUCCESS;
}

int fx_eos_fill_active_cells(fx_ctx *c, int stage)
{
    if (c && c->nranks > 1) return set_err(c, FX_EINVAL, "%s: not available on a sharded mesh", __func__);
    if (!has_mesh(c)) return c ? set_err(c, FX_ENOMESH, "no mesh") : FX_EINVAL;
    const int slot = stage > 0 ? stage - 1 : 0;
    if (slot > 1) return set_err(c, FX_EINVAL, "bad stage");
    fx_launch_set_dt(c->D, 0.0, c->stream);
    fx_launch_eos_fill(c->D, c->d_active, c->nactive, slot, 1, c->stream);
    return FX_SUCCESS;
}

int fx_eos_fill_mesh(fx_ctx *c, int stage)
{
    if (c && c->nranks > 1) return set_err(c, FX_EINVAL, "%s: not available on a sharded mesh", __func__);
    if (!has_mesh(c)) return c ? set_err(c, FX_ENOMESH, "no mesh") : FX_EINVAL;
    const int slot = stage > 0 ? stage - 1 : 0;
    if (slot > 1) return set_err(c, FX_EINVAL, "bad stage");
    fx_launch_set_dt(c->D, 0.0, c->stream);
    fx_launch_eos_fill(c->D, c->d_active, c->nactive, slot, 0, c->stream);
    return FX_SUCCESS;
}

int fx_boundary_fill_ghosts_and_bf(fx_ctx *c, int stage, int use_bf1)
{
    if (!has_mesh(c)) return c ? set_err(c, FX_ENOMESH, "no mesh") : FX_EINVAL;
    const int slot = stage > 0 ? stage - 1 : 0;
    if (slot > 1 || use_bf1 < 0 || use_bf1 > 1) return set_err(c, FX_EINVAL, "bad stage");
    if (c->cfg.mhd && slot != use_bf1) {
        return set_err(c, FX_EINVAL, "fx_boundary_fill_ghosts_and_bf: W slot and Bf slot must agree");
    }
    fx_launch_set_dt(c->D, 0.0, c->stream);
    if (c->nranks > 1) {
        /* sharded: every rank takes part (the exchange before the fill) */
        shard_exchange(c, FX_XG, slot);
        ghost_fill(c, slot);
        return sync_and_check(c);
    }
    ghost_fill(c, slot);
    return FX_SUCCESS;
}

/* ---- time integration ----------------------------------------------------------- */

int fx_calc_dt(fx_ctx *c, double cfl, double *dt)
{
    if (!has_mesh(c)) return c ? set_err(c, FX_ENOMESH, "no mesh") : FX_EINVAL;
    if (!dt) return set_err(c, FX_EINVAL, "null dt");
    fx_launch_reset_reductions(c->D, 1, c->stream);
    fx_launch_calc_dt(c->D, c->d_active, c->nactive, 0, cfl, c->stream);
    shard_min(c, 0, 1);
    FX_CUDA(c, cudaMemcpyAsync(c->h_red, c->d_red, 2 * sizeof(unsigned long long), cudaMemcpyDeviceToHost,
        c->stream));
    int rc = sync_and_check(c);
    if (rc) return rc;
    *dt = fx_key_to_double(c->h_red[0]) * dt_mult(c);
    return FX_SUCCESS;
}

int fx_stage(fx_ctx *c, int form, int stage, double dt, double *dt_src)
{
    if (c && c->nranks > 1 && form != FX_FORM_BATCHED) {
        return set_err(c, FX_EINVAL, "%s: a sharded mesh runs the batched form", __func__);
    }
    if (!has_mesh(c)) return c ? set_err(c, FX_ENOMESH, "no mesh") : FX_EINVAL;
    if (c->cfg.integrator != FX_INT_RK2) return set_err(c, FX_EINVAL, "fx_stage: RK2 stages only");
    if ((form != FX_FORM_PLAIN && form != FX_FORM_BATCHED) || (stage != 1 && stage != 2)) {
        return set_err(c, FX_EINVAL, "fx_stage: bad form or stage");
    }
    fx_launch_set_dt(c->D, dt, c->stream);
    fx_launch_reset_reductions(c->D, 2, c->stream);
    stage_seq(c, form, stage);
    shard_min(c, 1, 1);
    if (dt_src) return read_dt_src(c, dt_src);
    return c->xerr.empty() ? FX_SUCCESS : set_err(c, FX_ECOMM, "%s", c->xerr.c_str());
}

int fx_step(fx_ctx *c, int form, double dt, double *dt_src)
{
    if (c && c->nranks > 1 && form != FX_FORM_BATCHED) {
        return set_err(c, FX_EINVAL, "%s: a sharded mesh runs the batched form", __func__);
    }
    if (!has_mesh(c)) return c ? set_err(c, FX_ENOMESH, "no mesh") : FX_EINVAL;
    if (form != FX_FORM_PLAIN && form != FX_FORM_BATCHED) {
        return set_err(c, FX_EINVAL, "fx_step: bad form");
    }
    if (c->sticky) return FX_EPHYSICS;
    fx_launch_set_dt(c->D, dt, c->stream);
    if (form == FX_FORM_PLAIN || eager(c)) {
        fx_launch_reset_reductions(c->D, 2, c->stream);
        step_seq(c, form);
    } else {
        int rc = build_step_graph(c);
        if (rc) return rc;
        FX_CUDA(c, cudaGraphLaunch(c->g_step, c->stream));
        c->last_slot = 0;
    }
    shard_min(c, 1, 1);
    if (dt_src) return read_dt_src(c, dt_src);
    return c->xerr.empty() ? FX_SUCCESS : set_err(c, FX_ECOMM, "%s", c->xerr.c_str());
}

int fx_run(fx_ctx *c, int form, int nsteps, double cfl, double dt_factor, double t_end, double *state)
{
    if (c && c->nranks > 1 && form != FX_FORM_BATCHED) {
        return set_err(c, FX_EINVAL, "%s: a sharded mesh runs the batched form", __func__);
    }
    if (!has_mesh(c)) return c ? set_err(c, FX_ENOMESH, "no mesh") : FX_EINVAL;
    if (!state || nsteps < 0) return set_err(c, FX_EINVAL, "fx_run: bad arguments");
    if (form == FX_FORM_PLAIN) {
        double time = state[0], dt = state[1];
        long long step = (long long)state[2];
        for (int n = 0; n < nsteps && time < t_end; ++n) {
            double dt_new;
            int rc = fx_calc_dt(c, cfl, &dt_new);
            if (rc) return rc;
            if (dt > 0.0) {
                const double dt_limit = dt_factor * dt;
                dt = dt_new <= dt_limit ? dt_new : dt_limit;
            } else {
                dt = dt_new;
            }
            double dt_step = dt;
            if (time + dt_step > t_end) dt_step = t_end - time;
            double dt_src = 1.0e100;
            rc = fx_step(c, FX_FORM_PLAIN, dt_step, &dt_src);
            if (rc) return rc;
            if (cfl * dt_src < dt) dt = cfl * dt_src;
            time += dt_step;
            step += 1;
        }
        state[0] = time;
        state[1] = dt;
        state[2] = (double)step;
        return FX_SUCCESS;
    }
    if (form != FX_FORM_BATCHED) return set_err(c, FX_EINVAL, "fx_run: bad form");
    if (c->g_run && c->h_ctl->cfl != cfl) {
        free_graphs(c);
    }
    FxCtl v{};
    v.time = state[0];
    v.dt_prev = state[1];
    v.step = (long long)state[2];
    v.cfl = cfl;
    v.dt_factor = dt_factor;
    v.t_end = t_end;
    v.dt_src = 1.0e100;
    v.dt_mult = dt_mult(c);
    *c->h_ctl = v;
    fx_launch_set_ctl(c->D, v, c->stream);
    int rc;
    if (eager(c)) {
        for (int n = 0; n < nsteps; ++n) run_seq(c, cfl);
    } else {
        if ((rc = build_run_graph(c, cfl))) return rc;
        for (int n = 0; n < nsteps; ++n) {
            FX_CUDA(c, cudaGraphLaunch(c->g_run, c->stream));
        }
    }
    c->last_slot = 0;
    FX_CUDA(c, cudaMemcpyAsync(c->h_ctl, c->d_ctl, sizeof(FxCtl), cudaMemcpyDeviceToHost, c->stream));
    rc = sync_and_check(c);
    if (rc) return rc;
    state[0] = c->h_ctl->time;
    state[1] = c->h_ctl->dt_prev;
    state[2] = (double)c->h_ctl->step;
    c->h_ctl->cfl = cfl;
    return FX_SUCCESS;
}

int fx_time_phase(fx_ctx *c, int phase, int reps, double dt, double *ms)
{
    if (!has_mesh(c)) return c ? set_err(c, FX_ENOMESH, "no mesh") : FX_EINVAL;
    if (!ms || reps <= 0 || phase < 0 || phase > FX_PHASE_STEP) return set_err(c, FX_EINVAL, "bad phase");
    if ((phase == FX_PHASE_EMF || phase == FX_PHASE_CT) && !c->cfg.mhd) {
        return set_err(c, FX_EINVAL, "phase needs an MHD run");
    }
    if (phase == FX_PHASE_STEP) {
        int rc = build_step_graph(c);
        if (rc) return rc;
    }
    cudaStream_t s = c->stream;
    auto launch = [&]() {
        switch (phase) {
        case FX_PHASE_FLUX: fx_launch_flux(c->D, c->d_active, c->nactive, 3, 0, 0, 0, s); break;
        case FX_PHASE_EMF: fx_launch_emf(c->D, c->d_active, c->nactive, 0, 0, s); break;
        case FX_PHASE_CT: fx_launch_bf_update(c->D, c->d_active, c->nactive, 1, s); break;
        case FX_PHASE_CELLS: fx_launch_cell_update(c->D, c->d_active, c->nactive, 1, c->cfg.gravity, 0, s); break;
        case FX_PHASE_GHOST: ghost_fill(c, 1); break;
        default: cudaGraphLaunch(c->g_step, s); break;
        }
    };
    fx_launch_set_dt(c->D, dt, s);
    launch();
    cudaEvent_t e0, e1;
    FX_CUDA(c, cudaEventCreate(&e0));
    FX_CUDA(c, cudaEventCreate(&e1));
    FX_CUDA(c, cudaEventRecord(e0, s));
    for (int r = 0; r < reps; ++r) {
        launch();
    }
    FX_CUDA(c, cudaEventRecord(e1, s));
    FX_CUDA(c, cudaEventSynchronize(e1));
    float t = 0.0f;
    FX_CUDA(c, cudaEventElapsedTime(&t, e0, e1));
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    *ms = (double)t / reps;
    if (phase == FX_PHASE_STEP) c->last_slot = 0;
    return check_device_error(c);
}

int fx_autotune(fx_ctx *c, double *times_ms, int n, int *choice)
{
    if (!has_mesh(c) || !choice) return c ? set_err(c, FX_EINVAL, "fx_autotune: no mesh") : FX_EINVAL;
    cudaStream_t s = c->stream;
    cudaEvent_t e0, e1;
    FX_CUDA(c, cudaEventCreate(&e0));
    FX_CUDA(c, cudaEventCreate(&e1));
    fx_launch_set_dt(c->D, 0.0, s);
    int best = 0;
    double best_ms = 1.0e30;
    for (int v = 0; v < FX_FLUX_VARIANTS; ++v) {
        c->D.flux_variant = v;
        fx_launch_flux(c->D, c->d_active, c->nactive, 3, 0, 0, 0, s);
        FX_CUDA(c, cudaEventRecord(e0, s));
        for (int r = 0; r < 3; ++r) {
            fx_launch_flux(c->D, c->d_active, c->nactive, 3, 0, 0, 0, s);
        }
        FX_CUDA(c, cudaEventRecord(e1, s));
        FX_CUDA(c, cudaEventSynchronize(e1));
        float t = 0.0f;
        FX_CUDA(c, cudaEventElapsedTime(&t, e0, e1));
        const double ms = (double)t / 3.0;
        if (times_ms && v < n) times_ms[v] = ms;
        if (ms < best_ms) {
            best_ms = ms;
            best = v;
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    c->D.flux_variant = best;
    free_graphs(c); /* captured graphs hold the previous launch shape */
    *choice = best;
    return check_device_error(c);
}

int fx_branch_trace(fx_ctx *c, int mode, int max_stages, unsigned long long *flips)
{
    if (!c) return FX_EINVAL;
    if (!has_mesh(c)) return set_err(c, FX_ENOMESH, "no mesh");
    if (!c->cfg.mhd || c->cfg.recon != FX_RECON_MC || c->cfg.integrator != FX_INT_RK2 || c->nranks > 1) {
        return set_err(c, FX_EINVAL, "fx_branch_trace: MHD, MC, RK2, one rank only");
    }
    if (mode == FX_BRANCH_OFF) {
        const int was = c->D.br_mode;
        c->D.br_mode = 0;
        free_graphs(c);
        if (c->br_overflow) {
            c->br_overflow = false;
            return set_err(c, FX_ETOOBIG, "fx_branch_trace: more stages than the %d recorded", c->br_cap);
        }
        if (flips) {
            *flips = 0;
            if (was == FX_BRANCH_REPLAY) {
                FX_CUDA(c, cudaMemcpyAsync(c->h_red + 2, c->d_red + 2, sizeof(unsigned long long),
                    cudaMemcpyDeviceToHost, c->stream));
                const int rc = sync_and_check(c);
                if (rc) return rc;
                *flips = c->h_red[2];
            }
        }
        return FX_SUCCESS;
    }
    const size_t faces = (size_t)c->nblocks * 3 * (FX_BS + 1) * (FX_BS + 2) * (FX_BS + 2);
    const size_t edges = (size_t)c->nblocks * 3 * FX_BS * (FX_BS + 1) * (FX_BS + 1);
    if (mode == FX_BRANCH_RECORD) {
        if (max_stages <= 0) return set_err(c, FX_EINVAL, "fx_branch_trace: max_stages must be positive");
        if (c->br_cap != max_stages || c->br_nblocks != c->nblocks) {
            cudaFree(c->d_br_words);
            cudaFree(c->d_br_edges);
            c->d_br_words = c->d_br_edges = nullptr;
            c->br_cap = 0;
            if (cudaMalloc((void **)&c->d_br_words, faces * max_stages * sizeof(unsigned long long)) != cudaSuccess ||
                cudaMalloc((void **)&c->d_br_edges, edges * max_stages * sizeof(unsigned long long)) != cudaSuccess) {
                cudaGetLastError();
                cudaFree(c->d_br_words);
                cudaFree(c->d_br_edges);
                c->d_br_words = c->d_br_edges = nullptr;
                return set_err(c, FX_ENOMEM, "fx_branch_trace: no room for %d stages of decisions", max_stages);
            }
            c->br_cap = max_stages;
            c->br_nblocks = c->nblocks;
        }
        c->br_recorded = 0;
    } else if (mode == FX_BRANCH_REPLAY) {
        if (!c->d_br_words || c->br_nblocks != c->nblocks || c->br_recorded == 0) {
            return set_err(c, FX_EINVAL, "fx_branch_trace: nothing recorded to replay");
        }
        FX_CUDA(c, cudaMemsetAsync(c->d_red + 2, 0, sizeof(unsigned long long), c->stream));
    } else {
        return set_err(c, FX_EINVAL, "fx_branch_trace: unknown mode %d", mode);
    }
    c->br_stage = 0;
    c->br_overflow = false;
    c->D.br_mode = mode;
    c->D.br_words = c->d_br_words;
    c->D.br_edges = c->d_br_edges;
    c->D.br_flips = c->d_red + 2;
    free_graphs(c); /* captured graphs hold the previous device view */
    return FX_SUCCESS;
}

int fx_set_flux_shape(fx_ctx *c, int variant)
{
    if (!c) return FX_EINVAL;
    if (variant < 0 || variant >= FX_FLUX_VARIANTS) {
        return set_err(c, FX_EINVAL, "fx_set_flux_shape: variant %d outside [0, %d)", variant, FX_FLUX_VARIANTS);
    }
    c->D.flux_variant = variant;
    free_graphs(c);
    return FX_SUCCESS;
}

/* ---- dynamic AMR ---------------------------------------------------------------- */

int fx_amr_configure(fx_ctx *c, const fx_amr_config *amr)
{
    if (c && c->nranks > 1) return set_err(c, FX_EINVAL, "%s: not available on a sharded mesh", __func__);
    if (!c || !amr) return c ? set_err(c, FX_EINVAL, "fx_amr_configure: null config") : FX_EINVAL;
    std::string why;
    if (!amr_config_ok(*amr, &why)) return set_err(c, FX_EINVAL, "fx_amr_configure: %s", why.c_str());
    c->amr = *amr;
    c->amr_set = true;
    return FX_SUCCESS;
}

int fx_amr_tag(fx_ctx *c, int32_t *refine_flag)
{
    if (c && c->nranks > 1) return set_err(c, FX_EINVAL, "%s: not available on a sharded mesh", __func__);
    if (!has_mesh(c)) return c ? set_err(c, FX_ENOMESH, "no mesh") : FX_EINVAL;
    if (!c->amr_set) return set_err(c, FX_EINVAL, "fx_amr_tag: fx_amr_configure first");
    if (!refine_flag) return set_err(c, FX_EINVAL, "fx_amr_tag: null output");
    std::vector<int32_t> votes;
    int rc;
    fx_launch_set_dt(c->D, 0.0, c->stream);
    if ((rc = amr_votes(c, votes))) return rc;
    fx_amr_flags(c->amr, c->nblocks, c->blocks.data(), votes.data(), refine_flag);
    return FX_SUCCESS;
}

int fx_amr_adapt(fx_ctx *c, int *changed)
{
    if (c && c->nranks > 1) return set_err(c, FX_EINVAL, "%s: not available on a sharded mesh", __func__);
    if (!has_mesh(c)) return c ? set_err(c, FX_ENOMESH, "no mesh") : FX_EINVAL;
    if (!c->amr_set) return set_err(c, FX_EINVAL, "fx_amr_adapt: fx_amr_configure first");
    if (changed) *changed = 0;
    int rc;
    using clk = std::chrono::steady_clock;
    auto ms_since = [](clk::time_point t) { return std::chrono::duration<double, std::milli>(clk::now() - t).count(); };
    const clk::time_point t_start = clk::now();
    for (double &x : c->amr_ms) x = 0.0;
    fx_launch_set_dt(c->D, 0.0, c->stream);
    std::vector<int32_t> votes;
    if ((rc = amr_votes(c, votes))) return rc;
    c->amr_ms[0] = ms_since(t_start);
    clk::time_point t = clk::now();
    FxAmrResult res;
    std::string err;
    const int capacity = std::min(c->amr.max_blocks > 0 ? c->amr.max_blocks : 65535, 65535);
    if ((rc = fx_amr_remesh(c->cfg, c->amr, c->nblocks, c->blocks.data(), votes.data(), capacity, res, &err))) {
        return set_err(c, rc, "fx_amr_adapt: %s", err.c_str());
    }
    c->amr_ms[1] = ms_since(t);
    if (!res.changed) {
        c->amr_ms[5] = ms_since(t_start);
        return FX_SUCCESS;
    }
    t = clk::now();
    const int nb = (int)res.blocks.size();
    if (nb > c->cap) {
        const int grown = std::min(std::max(nb, c->cap + c->cap / 4), capacity);
        if ((rc = alloc_block_arrays(c, grown, c->nblocks))) return rc;
        c->D.blk = c->d_blk;
        c->D.W = c->d_W;
        c->D.Bf = c->d_Bf;
        c->D.flux = c->d_flux;
        c->D.vr = c->d_vr;
        c->D.bv1 = c->d_bv1;
        c->D.bv2 = c->d_bv2;
        c->D.emf = c->d_emf;
        c->D.eos = c->d_eos;
        c->D.rhs = c->d_rhs;
        c->D.grav = c->d_grav;
        c->D.W2 = c->d_W2;
        c->D.Bf2 = c->d_Bf2;
    }
    /* geometry of the new block list, read by the data kernels */
    std::vector<FxBlockDev> hb(nb);
    for (int b = 0; b < nb; ++b) {
        for (int a = 0; a < 3; ++a) {
            hb[b].xmin[a] = res.blocks[b].xmin[a];
            hb[b].dx[a] = res.blocks[b].dx[a];
            hb[b].area[a] = res.blocks[b].area[a];
        }
        hb[b].vol = res.blocks[b].vol;
    }
    FX_CUDA(c, cudaMemcpyAsync(c->d_blk, hb.data(), (size_t)nb * sizeof(FxBlockDev), cudaMemcpyHostToDevice,
        c->stream));
    c->D.nblocks = nb;

    /* device jobs */
    std::vector<int> children;
    std::vector<FxAmrChildJob> cjobs;
    std::vector<FxAmrCopyJob> copies;
    std::vector<FxPop> pops;
    for (const FxAmrRefine &r : res.refine) {
        children.push_back(r.child);
        FxAmrChildJob j;
        j.child = r.child;
        j.parent = r.parent;
        j.oct = r.oct;
        j.pad = 0;
        cjobs.push_back(j);
        if (c->cfg.mhd) {
            for (int q = 0; q < 6; ++q) {
                if (r.copy_src[q] < 0) continue;
                FxAmrCopyJob cp;
                cp.child = r.child;
                cp.src = r.copy_src[q];
                cp.dir = q / 2;
                cp.side = q % 2;
                copies.push_back(cp);
            }
            child_groups(r, c->cfg.use_bj != 0, pops);
        }
    }
    std::vector<FxAmrParentJob> pjobs;
    for (const FxAmrCoarsen &k : res.coarsen) {
        FxAmrParentJob j;
        std::memset(&j, 0, sizeof(j));
        j.parent = k.parent;
        for (int o = 0; o < 8; ++o) j.children[o] = k.children[o];
        pjobs.push_back(j);
    }
    DevVec<int> d_children;
    DevVec<FxAmrChildJob> d_cjobs;
    DevVec<FxAmrCopyJob> d_copies;
    DevVec<FxPop> d_pops;
    DevVec<FxAmrParentJob> d_pjobs;
    if ((rc = d_children.load(c, children))) return rc;
    if ((rc = d_cjobs.load(c, cjobs))) return rc;
    if ((rc = d_copies.load(c, copies))) return rc;
    if ((rc = d_pops.load(c, pops))) return rc;
    if ((rc = d_pjobs.load(c, pjobs))) return rc;
    const double floor = c->amr.E_floor;
    const size_t ninj = floor > 0.0 ? (cjobs.size() + pjobs.size()) * (size_t)(FX_BS * FX_BS * FX_BS) : 0;
    double *d_inj = nullptr;
    if (ninj) FX_CUDA(c, cudaMalloc((void **)&d_inj, ninj * sizeof(double)));
    cudaStream_t s = c->stream;
    fx_launch_amr_zero(c->D, d_children.p, (int)children.size(), s);
    if (c->cfg.mhd) {
        fx_launch_amr_copy_faces(c->D, d_copies.p, (int)copies.size(), s);
        fx_launch_prolong_groups(c->D, d_pops.p, (int)pops.size(), 0, s);
        fx_launch_prolong_groups(c->D, d_pops.p, (int)pops.size(), 1, s);
    }
    fx_launch_amr_prolong_cells(c->D, d_cjobs.p, (int)cjobs.size(), floor, d_inj, s);
    fx_launch_amr_restrict_faces(c->D, d_pjobs.p, (int)pjobs.size(), s);
    fx_launch_amr_restrict_cells(c->D, d_pjobs.p, (int)pjobs.size(), floor,
        d_inj ? d_inj + cjobs.size() * (size_t)(FX_BS * FX_BS * FX_BS) : nullptr, s);
    FX_CUDA(c, cudaGetLastError());
    c->amr_ms[2] = ms_since(t);

    /* the ghost fill of the new mesh compiles while the device moves data */
    t = clk::now();
    FxPlan plan;
    if (!c->plan_ws) c->plan_ws = fx_plan_workspace_new();
    if (!fx_build_plan(c->cfg, nb, res.blocks.data(), plan, &err, c->plan_ws)) {
        cudaFree(d_inj);
        return set_err(c, FX_EINVAL, "fx_amr_adapt: %s", err.c_str());
    }
    free_graphs(c);
    drop_adjoint(c);
    {
        /* the retired plan's program arrays take the next adapt's program */
        FxPlan old = std::move(c->plan);
        c->plan = std::move(plan);
        fx_plan_workspace_recycle(c->plan_ws, std::move(old));
    }
    c->blocks = std::move(res.blocks);
    c->nblocks = nb;
    c->nactive = (int)c->plan.active.size();
    c->amr_ms[3] = ms_since(t);
    t = clk::now();
    if ((rc = install_tables(c))) {
        cudaFree(d_inj);
        return rc;
    }
    /* the driver's refill of a changed mesh (src/main.c:599-606) */
    fx_launch_set_dt(c->D, 0.0, s);
    fx_launch_eos_fill(c->D, c->d_active, c->nactive, 0, 1, s);
    ghost_fill(c, 0);
    fx_launch_eos_fill(c->D, c->d_active, c->nactive, 0, 0, s);
    c->last_slot = 0;
    if (ninj) {
        /* prj_sync_primitive_from_conserved sums the floor's energy over the
         * regenerated blocks in block order, cells in (i, j, k) order */
        std::vector<double> inj(ninj);
        FX_CUDA(c, cudaMemcpyAsync(inj.data(), d_inj, ninj * sizeof(double), cudaMemcpyDeviceToHost, s));
        rc = sync_and_check(c);
        cudaFree(d_inj);
        if (rc) return rc;
        std::vector<std::pair<int, size_t>> order;
        for (size_t j = 0; j < cjobs.size(); ++j) order.emplace_back(cjobs[j].child, j);
        for (size_t j = 0; j < pjobs.size(); ++j) order.emplace_back(pjobs[j].parent, cjobs.size() + j);
        std::sort(order.begin(), order.end());
        double local = 0.0;
        for (const auto &e : order) {
            const double *v = inj.data() + e.second * (size_t)(FX_BS * FX_BS * FX_BS);
            for (int q = 0; q < FX_BS * FX_BS * FX_BS; ++q) local += v[q];
        }
        if (local != 0.0) c->E_injected += local;
    } else if ((rc = sync_and_check(c))) {
        return rc;
    }
    c->amr_ms[4] = ms_since(t);
    c->amr_ms[5] = ms_since(t_start);
    if (changed) *changed = 1;
    return FX_SUCCESS;
}

int fx_amr_timings(fx_ctx *c, double *ms)
{
    if (!c || !ms) return c ? set_err(c, FX_EINVAL, "null argument") : FX_EINVAL;
    for (int q = 0; q < 6; ++q) ms[q] = c->amr_ms[q];
    return FX_SUCCESS;
}

int fx_get_mesh(fx_ctx *c, int capacity, fx_block_desc *out, int *nblocks)
{
    if (!c || !nblocks) return c ? set_err(c, FX_EINVAL, "fx_get_mesh: null argument") : FX_EINVAL;
    *nblocks = c->nblocks;
    if (out && capacity >= c->nblocks && c->nblocks) {
        std::memcpy(out, c->blocks.data(), (size_t)c->nblocks * sizeof(fx_block_desc));
    }
    return FX_SUCCESS;
}

int fx_amr_energy_injected(fx_ctx *c, double *e)
{
    if (!c || !e) return c ? set_err(c, FX_EINVAL, "null argument") : FX_EINVAL;
    *e = c->E_injected;
    return FX_SUCCESS;
}

int fx_mesh_slot_geometry(int nblocks, fx_block_desc *blocks)
{
    if (nblocks < 0 || (nblocks > 0 && !blocks)) return FX_EINVAL;
    for (int i = 0; i < nblocks; ++i) {
        for (int s = 0; s < 56; ++s) {
            fx_slot &sl = blocks[i].slot[s];
            if (sl.id < 0) {
                const int32_t id = sl.id;
                std::memset(&sl, 0, sizeof(sl));
                sl.id = id;
                continue;
            }
            if (sl.id >= nblocks || !fx_neighbor_geometry(blocks[i], blocks[sl.id], sl)) return FX_EINVAL;
        }
    }
    return FX_SUCCESS;
}

int fx_amr_remesh_host(const fx_config *cfg, const fx_amr_config *amr, int nblocks, const fx_block_desc *in,
    const int32_t *votes, int32_t *flags, int capacity, fx_block_desc *out, int *nout)
{
    if (!cfg || !amr || nblocks <= 0 || !in || !votes || !out || !nout || capacity <= 0) return FX_EINVAL;
    std::string why;
    if (!amr_config_ok(*amr, &why)) return FX_EINVAL;
    FxAmrResult res;
    const int rc = fx_amr_remesh(*cfg, *amr, nblocks, in, votes, capacity, res, &why);
    if (rc) return rc;
    if (flags) std::memcpy(flags, res.flags.data(), (size_t)nblocks * sizeof(int32_t));
    if (!res.changed) {
        std::memcpy(out, in, (size_t)nblocks * sizeof(fx_block_desc));
        *nout = nblocks;
        return FX_SUCCESS;
    }
    if ((int)res.blocks.size() > capacity) return FX_ETOOBIG;
    std::memcpy(out, res.blocks.data(), res.blocks.size() * sizeof(fx_block_desc));
    *nout = (int)res.blocks.size();
    return FX_SUCCESS;
}

int fx_info(fx_ctx *c, int what, long long *value)
{
    if (!has_mesh(c) || !value) return c ? set_err(c, FX_EINVAL, "fx_info: no mesh") : FX_EINVAL;
    const FxProgram &g = c->plan.ghost;
    /* ghost launches: per wave one for cell/face/cell-field ops and one for
     * face-prolongation groups, when present */
    long long gw = 0;
    for (int w = 0; w < g.nwaves(); ++w) {
        const bool ops = g.cell_begin[w + 1] > g.cell_begin[w] || g.face_begin[w + 1] > g.face_begin[w] ||
            g.b_begin[w + 1] > g.b_begin[w];
        gw += (ops ? 1 : 0) + (g.p_begin[w + 1] > g.p_begin[w] ? 1 : 0);
    }
    /* correction launches: one per non-empty wave */
    const long long corr = (long long)std::max<size_t>(c->plan.flux_corr_begin.size(), 1) - 1 +
        (c->cfg.mhd ? (long long)std::max<size_t>(c->plan.emf_corr_begin.size(), 1) - 1 : 0);
    const long long mhd = c->cfg.mhd ? 1 : 0;
    const bool ess = c->cfg.integrator == FX_INT_ESSPRK10_4;
    switch (what) {
    case 0:
        if (ess) {
            /* reset + stage dt + 2 saves + 10 x (flux + emf + ct + cells +
             * ghost waves) + 3 x (blend + ghost waves) */
            *value = 2 + 2 + 10 * (1 + 2 * mhd + 1 + corr + gw) + 3 * (1 + mhd + gw);
        } else { /* reset + 2 x (flux + emf + ct + cells + ghost waves) */
            *value = 1 + 2 * (1 + 2 * mhd + 1 + corr + gw);
        }
        break;
    case 1: /* set_dt + reset + 2 x (per-block phases + eos fills) + ghost waves */
        *value = 2 + 2 * ((long long)c->nactive * (1 + 2 * mhd + 1 + 2) + corr + gw);
        break;
    case 2: *value = (long long)g.cell_ops.size(); break;
    case 3: *value = (long long)g.face_ops.size(); break;
    case 4: *value = g.nwaves(); break;
    case 5: *value = (long long)g.b_ops.size(); break;
    default: return set_err(c, FX_EINVAL, "fx_info: unknown query");
    }
    return FX_SUCCESS;
}

} /* extern "C" */

/* ---- discrete adjoint ------------------------------------------------------ */

namespace {

/* the reverse pass covers what the forward step does on single-level MHD
 * meshes without gravity or resistivity: copy-type ghost operations, no
 * coarse/fine transfers */
int adj_supported(fx_ctx *c)
{
    if (!c->cfg.mhd || c->cfg.gravity || c->cfg.mhd_eta != 0.0) {
        return set_err(c, FX_EINVAL, "the adjoint covers MHD runs without gravity or resistivity");
    }
    if (c->cfg.integrator != FX_INT_RK2 || c->cfg.recon != FX_RECON_MC) {
        return set_err(c, FX_EINVAL, "the adjoint covers the RK2 / MC build");
    }
    const FxProgram &g = c->plan.ghost;
    bool ok = g.p_ops.empty() && c->plan.flux_corr.empty() && c->plan.emf_corr.empty();
    for (const FxGop &op : g.cell_ops) {
        ok = ok && (op.type == FX_GOP_COPY || op.type == FX_GOP_COPY_NEG || op.type == FX_GOP_COPY_USER);
    }
    for (const FxGop &op : g.face_ops) {
        ok = ok && op.type == FX_FOP_COPY;
    }
    if (!ok) {
        return set_err(c, FX_EINVAL, "the adjoint covers single-level meshes (no coarse/fine neighbours)");
    }
    return FX_SUCCESS;
}

/* the ghost program's waves transposed into gathers (FxAdjSrc / FxAdjEnt) */
int build_adj_ghost(fx_ctx *c)
{
    if (c->adj_ghost_ready) {
        return FX_SUCCESS;
    }
    const FxProgram &g = c->plan.ghost;
    std::vector<FxAdjSrc> cs, fs;
    std::vector<FxAdjEnt> ents;
    c->adj_cbeg.assign(1, 0);
    c->adj_fbeg.assign(1, 0);
    std::vector<std::pair<int64_t, FxAdjEnt>> list;
    for (int w = 0; w < g.nwaves(); ++w) {
        list.clear();
        for (int q = g.cell_begin[w]; q < g.cell_begin[w + 1]; ++q) {
            const FxGop &op = g.cell_ops[q];
            int kind = 0;
            if (op.type == FX_GOP_COPY_NEG) kind = 1 + op.aux;
            if (op.type == FX_GOP_COPY_USER && op.aux) kind = 16;
            list.push_back({(int64_t)op.src, FxAdjEnt{op.dst, kind}});
        }
        std::stable_sort(list.begin(), list.end(),
            [](const std::pair<int64_t, FxAdjEnt> &a, const std::pair<int64_t, FxAdjEnt> &b) { return a.first < b.first; });
        for (size_t q = 0; q < list.size();) {
            FxAdjSrc sr{(int32_t)list[q].first, 0, (int32_t)ents.size(), 0};
            while (q < list.size() && list[q].first == sr.key) {
                ents.push_back(list[q].second);
                ++q;
            }
            sr.end = (int32_t)ents.size();
            cs.push_back(sr);
        }
        c->adj_cbeg.push_back((int)cs.size());
        list.clear();
        for (int q = g.face_begin[w]; q < g.face_begin[w + 1]; ++q) {
            const FxGop &op = g.face_ops[q];
            list.push_back({((int64_t)op.src << 2) | (op.aux & 3), FxAdjEnt{op.dst, 0}});
        }
        for (int q = g.b_begin[w]; q < g.b_begin[w + 1]; ++q) {
            const FxBop &op = g.b_ops[q];
            for (int d = 0; d < 3; ++d) {
                for (int h = 0; h < 2; ++h) {
                    list.push_back({((int64_t)op.f[2 * d + h] << 2) | d, FxAdjEnt{op.dst, 1 + d}});
                }
            }
        }
        std::stable_sort(list.begin(), list.end(),
            [](const std::pair<int64_t, FxAdjEnt> &a, const std::pair<int64_t, FxAdjEnt> &b) { return a.first < b.first; });
        for (size_t q = 0; q < list.size();) {
            const int64_t key = list[q].first;
            FxAdjSrc sr{(int32_t)(key >> 2), (int32_t)(key & 3), (int32_t)ents.size(), 0};
            while (q < list.size() && list[q].first == key) {
                ents.push_back(list[q].second);
                ++q;
            }
            sr.end = (int32_t)ents.size();
            fs.push_back(sr);
        }
        c->adj_fbeg.push_back((int)fs.size());
    }
    int rc;
    if ((rc = dev_alloc(c, &c->d_adj_csrc, cs.size()))) return rc;
    if ((rc = dev_alloc(c, &c->d_adj_fsrc, fs.size()))) return rc;
    if ((rc = dev_alloc(c, &c->d_adj_ents, ents.size()))) return rc;
    const cudaMemcpyKind h2d = cudaMemcpyHostToDevice;
    if (!cs.empty()) FX_CUDA(c, cudaMemcpyAsync(c->d_adj_csrc, cs.data(), cs.size() * sizeof(FxAdjSrc), h2d, c->stream));
    if (!fs.empty()) FX_CUDA(c, cudaMemcpyAsync(c->d_adj_fsrc, fs.data(), fs.size() * sizeof(FxAdjSrc), h2d, c->stream));
    if (!ents.empty()) FX_CUDA(c, cudaMemcpyAsync(c->d_adj_ents, ents.data(), ents.size() * sizeof(FxAdjEnt), h2d, c->stream));
    FX_CUDA(c, cudaStreamSynchronize(c->stream));
    c->adj_ghost_ready = true;
    return FX_SUCCESS;
}

/* adjoint of the whole ghost fill of `slot`: waves in reverse order, each a
 * gather into the elements it read followed by clearing its destinations */
void adj_ghost(fx_ctx *c, const FxAdjDev &A, int slot)
{
    const FxProgram &g = c->plan.ghost;
    for (int w = g.nwaves() - 1; w >= 0; --w) {
        fx_launch_adj_gather(A, c->d_adj_csrc + c->adj_cbeg[w], c->adj_cbeg[w + 1] - c->adj_cbeg[w],
            c->d_adj_fsrc + c->adj_fbeg[w], c->adj_fbeg[w + 1] - c->adj_fbeg[w], c->d_adj_ents, slot, c->stream);
        fx_launch_adj_zero(A, c->d_cops + g.cell_begin[w], g.cell_begin[w + 1] - g.cell_begin[w],
            c->d_fops + g.face_begin[w], g.face_begin[w + 1] - g.face_begin[w],
            c->d_bops + g.b_begin[w], g.b_begin[w + 1] - g.b_begin[w], slot, c->stream);
    }
}

/* the reverse sweep over all stored stages; the adjoint of the final
 * state is in d_Wb / d_Bfb on entry, that of the stored initial state on
 * return.  Device time of the sweep goes to c->adj_ms. */
int adjoint_reverse(fx_ctx *c)
{
    const size_t nb = (size_t)c->nblocks;
    const size_t wn = nb * w_count(c);
    const size_t bn = nb * FX_BF_COUNT;
    cudaStream_t s = c->stream;
    FxAdjDev A{};
    A.blk = c->d_blk;
    A.gamma = c->cfg.gamma;
    A.dt = c->adj_dt;
    A.Wb = c->d_Wb;
    A.Bfb = c->d_Bfb;
    A.G = c->d_G;
    A.bvb1 = c->d_bvb1;
    A.bvb2 = c->d_bvb2;
    A.Eb = c->d_Eb;
    cudaEvent_t e0, e1;
    FX_CUDA(c, cudaEventCreate(&e0));
    FX_CUDA(c, cudaEventCreate(&e1));
    FX_CUDA(c, cudaEventRecord(e0, s));
    for (int n = c->adj_nsteps - 1; n >= 0; --n) {
        for (int stage = 2; stage >= 1; --stage) {
            const size_t k = 2 * (size_t)n + stage;
            const int dst = stage == 1 ? 1 : 0;
            A.Wbef = c->d_ckW + (k - 1) * wn;
            A.Bfbef = c->d_ckBf + (k - 1) * bn;
            A.Waft = c->d_ckW + k * wn;
            A.vr = c->d_ckVr + (k - 1) * nb * FX_VR_COUNT;
            adj_ghost(c, A, dst);
            fx_launch_adj_cells(A, c->d_active, c->nactive, stage, s);
            FX_CUDA(c, cudaMemsetAsync(c->d_Eb, 0, nb * FX_EMF_COUNT * sizeof(double), s));
            fx_launch_adj_bf(A, c->d_active, c->nactive, stage, s);
            FX_CUDA(c, cudaMemsetAsync(c->d_bvb1, 0, nb * FX_BV_COUNT * sizeof(double), s));
            FX_CUDA(c, cudaMemsetAsync(c->d_bvb2, 0, nb * FX_BV_COUNT * sizeof(double), s));
            fx_launch_adj_emf(A, c->d_active, c->nactive, stage, s);
            fx_launch_adj_flux(A, c->d_active, c->nactive, stage, s);
        }
    }
    FX_CUDA(c, cudaEventRecord(e1, s));
    FX_CUDA(c, cudaEventSynchronize(e1));
    float ms = 0.0f;
    cudaEventElapsedTime(&ms, e0, e1);
    c->adj_ms = ms;
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    return check_device_error(c);
}

} // namespace

int fx_adjoint_forward(fx_ctx *c, int nsteps, double dt)
{
    if (c && c->nranks > 1) return set_err(c, FX_EINVAL, "%s: not available on a sharded mesh", __func__);
    if (!has_mesh(c)) return c ? set_err(c, FX_ENOMESH, "no mesh") : FX_EINVAL;
    if (nsteps < 1 || !(dt > 0.0)) return set_err(c, FX_EINVAL, "fx_adjoint_forward: nsteps >= 1 and dt > 0");
    int rc = adj_supported(c);
    if (rc) return rc;
    if ((rc = build_adj_ghost(c))) return rc;
    const size_t nb = (size_t)c->nblocks;
    const size_t wn = nb * w_count(c);
    const size_t bn = nb * FX_BF_COUNT;
    const size_t nck = 2 * (size_t)nsteps + 1;
    if (c->adj_nsteps != nsteps || !c->d_ckW) {
        if ((rc = dev_alloc(c, &c->d_ckW, nck * wn))) return rc;
        if ((rc = dev_alloc(c, &c->d_ckBf, nck * bn))) return rc;
        if ((rc = dev_alloc(c, &c->d_ckVr, (nck - 1) * nb * FX_VR_COUNT))) return rc;
    }
    cudaStream_t s = c->stream;
    const cudaMemcpyKind d2d = cudaMemcpyDeviceToDevice;
    FX_CUDA(c, cudaMemcpyAsync(c->d_ckW, c->d_W, wn * sizeof(double), d2d, s));
    FX_CUDA(c, cudaMemcpyAsync(c->d_ckBf, c->d_Bf, bn * sizeof(double), d2d, s));
    for (int n = 0; n < nsteps; ++n) {
        for (int stage = 1; stage <= 2; ++stage) {
            fx_launch_set_dt(c->D, dt, s);
            stage_seq(c, FX_FORM_BATCHED, stage);
            const size_t k = 2 * (size_t)n + stage;
            FX_CUDA(c, cudaMemcpyAsync(c->d_ckW + k * wn, c->d_W, wn * sizeof(double), d2d, s));
            FX_CUDA(c, cudaMemcpyAsync(c->d_ckBf + k * bn, c->d_Bf, bn * sizeof(double), d2d, s));
            /* the stage's face velocities: their signs pick the upwind EMF
             * terms the reverse pass differentiates */
            FX_CUDA(c, cudaMemcpyAsync(c->d_ckVr + (k - 1) * nb * FX_VR_COUNT, c->d_vr,
                nb * FX_VR_COUNT * sizeof(double), d2d, s));
        }
    }
    c->adj_nsteps = nsteps;
    c->adj_dt = dt;
    return sync_and_check(c);
}

int fx_adjoint_backward(fx_ctx *c, const double *W_bar, const double *Bf_bar, double *W_bar_out,
    double *Bf_bar_out, int initial_fill)
{
    if (c && c->nranks > 1) return set_err(c, FX_EINVAL, "%s: not available on a sharded mesh", __func__);
    if (!has_mesh(c)) return c ? set_err(c, FX_ENOMESH, "no mesh") : FX_EINVAL;
    if (c->adj_nsteps < 1 || !c->d_ckW) return set_err(c, FX_EINVAL, "fx_adjoint_backward: no stored forward pass");
    if (!W_bar || !W_bar_out || !Bf_bar_out) return set_err(c, FX_EINVAL, "fx_adjoint_backward: null array");
    const size_t nb = (size_t)c->nblocks;
    const size_t wn = nb * w_count(c);
    const size_t bn = nb * FX_BF_COUNT;
    int rc;
    if (!c->d_Wb) {
        if ((rc = dev_alloc(c, &c->d_Wb, wn))) return rc;
        if ((rc = dev_alloc(c, &c->d_Bfb, bn))) return rc;
        if ((rc = dev_alloc(c, &c->d_G, nb * FX_ADJ_G_COUNT))) return rc;
        if ((rc = dev_alloc(c, &c->d_bvb1, nb * FX_BV_COUNT))) return rc;
        if ((rc = dev_alloc(c, &c->d_bvb2, nb * FX_BV_COUNT))) return rc;
        if ((rc = dev_alloc(c, &c->d_Eb, nb * FX_EMF_COUNT))) return rc;
    }
    cudaStream_t s = c->stream;
    FX_CUDA(c, cudaMemcpyAsync(c->d_Wb, W_bar, wn * sizeof(double), cudaMemcpyHostToDevice, s));
    if (Bf_bar) {
        FX_CUDA(c, cudaMemcpyAsync(c->d_Bfb, Bf_bar, bn * sizeof(double), cudaMemcpyHostToDevice, s));
    } else {
        FX_CUDA(c, cudaMemsetAsync(c->d_Bfb, 0, bn * sizeof(double), s));
    }
    FX_CUDA(c, cudaMemsetAsync(c->d_G, 0, nb * FX_ADJ_G_COUNT * sizeof(double), s));
    rc = adjoint_reverse(c);
    if (rc) return rc;
    FxAdjDev A{};
    A.blk = c->d_blk;
    A.Wb = c->d_Wb;
    A.Bfb = c->d_Bfb;
    if (initial_fill) {
        adj_ghost(c, A, 0);
    }
    FX_CUDA(c, cudaMemcpyAsync(W_bar_out, c->d_Wb, wn * sizeof(double), cudaMemcpyDeviceToHost, s));
    FX_CUDA(c, cudaMemcpyAsync(Bf_bar_out, c->d_Bfb, bn * sizeof(double), cudaMemcpyDeviceToHost, s));
    return sync_and_check(c);
}

int fx_adjoint_time(fx_ctx *c, double *ms)
{
    if (!c || !ms) return FX_EINVAL;
    *ms = c->adj_ms;
    return FX_SUCCESS;
}
