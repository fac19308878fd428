/*
 * Host-visible declarations shared by the runtime and the kernels.
 */
#ifndef FX_KERNELS_H
#define FX_KERNELS_H

#include <cuda_runtime.h>
#include <stdint.h>

#include "fx_layout.h"

struct FxErr;

/* Step control block in device memory.  Stepping kernels read dt from here
 * (so a captured graph is dt-independent) and return at once when `skip` is
 * set (the device-resident driver loop reached t_end). */
struct FxCtl {
    double dt;        /* dt of the current step */
    double time;      /* simulation time (driver loop) */
    double dt_prev;   /* sim.dt of the reference driver */
    double cfl;
    double dt_factor;
    double t_end;
    double dt_src;    /* last step's dt_src */
    long long step;
    int skip;
    int pad;
    double dt_stage;  /* dt of the stage kernels: dt (RK2) or dt / 6 (eSSPRK10_4 substeps) */
    double dt_mult;   /* factor on the CFL minimum: 1 (RK2) or 6 (eSSPRK10_4) */
};

/* per-block geometry on the device */
struct FxBlockDev {
    double xmin[3];
    double dx[3];
    double vol;
    double area[3];
};

/* device view of one mesh: stacked per-block arrays in the reference layout */
struct FxDev {
    int nv;       /* primitive/conserved variables per cell: 9 (MHD) or 6 */
    int nblocks;
    double gamma;
    double mhd_eta;
    const FxBlockDev *blk;
    double *W;    /* [b][v][stage][cell]           (WIDX) */
    double *Bf;   /* [b][dir][stage][face]         (FACE_IDX) */
    double *flux; /* [b][dir][AoSoA nc=nv]         (VIDX) */
    double *vr;   /* [b][dir][AoSoA nc=3]          (VRIDX) */
    double *bv1;  /* [b][dir][cell]                (IDX) */
    double *bv2;
    double *emf;  /* [b][dir][edge]                (EDGE_IDX) */
    double *eos;  /* [b][AoSoA nc=3]               (EIDX) */
    double *rhs;  /* [b][AoSoA nc=nv]              (MHDVIDX) */
    double *grav; /* [b][dir][cell] or null        (IDX) */
    FxErr *err;
    unsigned long long *red;  /* [0] dt min key, [1] dt_src min key */
    FxCtl *ctl;
    int flux_variant;         /* launch shape of the face kernel (autotuned) */
    int recon;                /* FX_RECON_MC or FX_RECON_WENO3 */
    int use_bj;               /* Barth-Jespersen prolongation limiter (refinement) */
    /* decisions of the plain form's face and edge kernels (MHD, MC):
     * br_mode 0 none, 1 record into / 2 replay from br_words (one word per
     * face, at br_off + (b * 3 + dir) * faces per direction + face) and
     * br_edges (likewise per edge, br_eoff); replays count the decisions
     * whose comparison differs from the recorded one in br_flips */
    int br_mode;
    size_t br_off, br_eoff;
    unsigned long long *br_words, *br_edges, *br_flips;
    double *W2;   /* eSSPRK10_4 stage slot 2 of W: [b][v][cell] (null for RK2) */
    double *Bf2;  /* eSSPRK10_4 stage slot 2 of Bf: [b][dir][face] (null for RK2 or hydro) */
};

#define FX_FLUX_VARIANTS 6
/* threads per CTA and min resident CTAs per SM of a face-kernel variant */
void fx_flux_shape(int variant, int *tpb, int *minb);

/* One element operation of a ghost-fill program.  dst/src pack
 * FX_CELL_KEY(block, cell) for cell ops, or (block << 15) | face for face ops
 * (with the face direction in `aux` bits 0-1). */
enum FxGopType {
    FX_GOP_COPY = 0,        /* dst <- src (all ghost vars) */
    FX_GOP_COPY_NEG = 1,    /* dst <- src, normal velocity aux negated (reflect) */
    FX_GOP_COPY_USER = 2,   /* dst <- src, then v1 = 5 (reference PRJ_BC_USER) */
    FX_GOP_RESTRICT = 3,    /* dst <- 1/8 sum of the 2x2x2 cells at src */
    FX_GOP_PROLONG = 4,     /* dst <- minmod-limited linear from src and its 6 axis neighbours,
                               target offsets +-1/4 from aux bits 2, 1, 0 (set: +) */
    FX_GOP_PROLONG_BJ = 5,  /* dst <- Barth-Jespersen-limited linear from src and its 26
                               neighbours, target offsets as FX_GOP_PROLONG */
    FX_FOP_COPY = 8,        /* face: dst <- src */
    FX_FOP_RESTRICT = 9,    /* face: dst <- 1/4 sum of 4 fine faces */
    FX_FOP_PROLONG = 10     /* face: divergence-free prolongation value */
};

struct FxGop {
    int32_t dst;
    int32_t src;
    int32_t aux;
    int32_t type;
};

/* cell-centred field of one cell from its six faces (bf2bc of one cell):
 * dst = FX_CELL_KEY(block, cell); f[2d], f[2d+1] = (block << 15) | face of the
 * lower and upper face along d (after copy propagation they may point at
 * the faces those were copied from) */
struct FxBop {
    int32_t dst;
    int32_t f[6];
    int32_t pad;
};

/* Divergence-preserving prolongation of the face field onto one 2x2x2 group
 * of fine cells (prj_mhd_prolong_bf_from_buffer, src/prj_mhd.c:374-512).
 * pos packs the fine corner (fi, fj, fk) and the coarse cell (ci, cj, ck),
 * each biased by FX_NG, in 5 bits apiece: fi | fj << 5 | fk << 10 | ci << 15 |
 * cj << 20 | ck << 25.  Outer face q = 8 d + 4 s + 2 a + b is the face of
 * direction d on side s (s = 1: index +2 along d) at tangential offsets
 * (a, b) in increasing axis order; inner face q = 4 d + 2 a + b.  keep bit
 * q: outer face q keeps the fine block's value (its fidelity is above
 * COARSER); owrite bit q: outer face q is stored; iwrite bit q: inner face q
 * is stored.  The masks come from the data-independent fidelity replay.
 * flags bit 0: the outer faces take the Barth-Jespersen limiter on the 3x3
 * tangential stencil (use_BJ), else minmod on the 5-point cross. */
struct FxPop {
    int32_t fine;
    int32_t coarse;
    int32_t pos;
    int32_t keep;
    int32_t owrite;
    int32_t iwrite;
    int32_t flags;
    int32_t pad;
};

/* coarse/fine correction records: entry dst of block dst_block <- 0.25 *
 * sum of 4 (flux) or 0.5 * sum of 2 (emf) entries of block src_block.
 * Indices are into one block's stacked array: dir * nv * 8000 + VIDX(0, ..)
 * for fluxes (component v sits 4 v further), dir * 8820 + EDGE_IDX for
 * EMFs. */
struct FxCorr {
    int32_t dst_block;
    int32_t dst;
    int32_t src_block;
    int32_t src[4];
    int32_t pad;
};

/* one element of a packed exchange between ranks of a sharded mesh: kind 0
 * a cell (the 6 ghost-filled primitives of W slot `slot`, idx the cell), 1 a
 * face (Bf slot `slot`, idx = dir * 8400 + face), 2 a flux entry (the 6
 * components the batched face kernel stores, idx their component-0 entry),
 * 3 an EMF entry; off: its first double in the message buffer */
struct FxXent {
    int32_t block;
    int32_t idx;
    int32_t kind;
    int32_t off;
};

/* cell keys: (block << FX_CELL_BITS) | cell, with the cell index below
 * 2^FX_CELL_BITS (8000 cells of a 20^3 block, 13824 of a 24^3 one) */
#define FX_CELL_BITS (FX_NCELLS <= 8192 ? 13 : 14)
#define FX_CELL_KEY(b, c) (((b) << FX_CELL_BITS) | (c))
#define FX_CELL_BLOCK(key) ((key) >> FX_CELL_BITS)
#define FX_CELL_IDX(key) ((key) & ((1 << FX_CELL_BITS) - 1))

/* launchers (fx_kernels.cu); all asynchronous on `s` */
void fx_launch_flux(const FxDev &D, const int *blist, int nlist, int ndir, int wslot, int bfslot,
    int full, cudaStream_t s);
void fx_launch_emf(const FxDev &D, const int *blist, int nlist, int wslot, int bfslot, cudaStream_t s);
/* stage 1, 2: the RK2 stages; stage 0: an eSSPRK forward-Euler substep in
 * place on slot 0 (prj_timeint_mhd_update_bf stage 0 and the stage-1 cell
 * update writing slot 0) */
void fx_launch_bf_update(const FxDev &D, const int *blist, int nlist, int stage, cudaStream_t s);
void fx_launch_cell_update(const FxDev &D, const int *blist, int nlist, int stage,
    int gravity, int store_rhs, cudaStream_t s);
/* dt_stage = dt / divisor in the control block */
void fx_launch_stage_dt(const FxDev &D, double divisor, cudaStream_t s);
/* prj_timeint_eSSPRK_save_state (src/prj_timeint.c:2311-2352): W of the
 * active cells and every Bf face of slot 0 into saved state `which` (1: slot
 * 1, 2: W2 / Bf2) */
void fx_launch_essprk_save(const FxDev &D, const int *blist, int nlist, int which, cudaStream_t s);
/* prj_timeint_eSSPRK_blend_with_saved, cell and face part
 * (src/prj_timeint.c:2354-2444): slot 0 <- w saved + (1 - w) slot 0 */
void fx_launch_essprk_blend(const FxDev &D, const int *blist, int nlist, int which, double w,
    cudaStream_t s);
void fx_launch_eos_fill(const FxDev &D, const int *blist, int nlist, int wslot, int active_only,
    cudaStream_t s);
void fx_launch_calc_dt(const FxDev &D, const int *blist, int nlist, int wslot, double cfl,
    cudaStream_t s);
/* one wave of the ghost fill (cell ops, face ops, face-prolongation groups
 * and cell-field ops) */
void fx_launch_ghost_wave(const FxDev &D, const FxGop *cops, int nc, const FxGop *fops, int nf,
    const FxPop *pops, int np, const FxBop *bops, int nb, int slot, int nvg, cudaStream_t s);
/* gather the listed elements into buf / scatter buf into them */
void fx_launch_xpack(const FxDev &D, const FxXent *ents, int n, double *buf, int slot, cudaStream_t s);
void fx_launch_xunpack(const FxDev &D, const FxXent *ents, int n, const double *buf, int slot, cudaStream_t s);
/* one wave of correction records; ncomp flux components per record */
/* the dump rows (Data, Eos, optionally Bf) of the listed blocks, packed
 * contiguously per list position */
void fx_launch_dump_pack(const FxDev &D, const int *blist, int nlist, int faces, double *out, cudaStream_t s);
/* cell-centred field of the listed blocks' active cells from the faces (slot 0) */
void fx_launch_cell_field_active(const FxDev &D, const int *blist, int nlist, cudaStream_t s);
void fx_launch_flux_correct(const FxDev &D, const FxCorr *recs, int n, int ncomp, cudaStream_t s);
void fx_launch_emf_correct(const FxDev &D, const FxCorr *recs, int n, cudaStream_t s);
void fx_launch_reset_reductions(const FxDev &D, int which, cudaStream_t s);
/* device-resident driver: dt selection before a step, dt_src clamp and time
 * advance after it (src/main.c:513-562) */
void fx_launch_step_begin(const FxDev &D, cudaStream_t s);
void fx_launch_step_end(const FxDev &D, cudaStream_t s);
/* stream-ordered write of a host-chosen dt into the control block */
void fx_launch_set_dt(const FxDev &D, double dt, cudaStream_t s);
/* controlled driver state set-up */
void fx_launch_set_ctl(const FxDev &D, FxCtl value, cudaStream_t s);

/* ordered-integer keys for atomicMin over doubles */
static inline double fx_key_to_double(unsigned long long key)
{
    unsigned long long bits = (key >> 63) ? (key & 0x7fffffffffffffffULL) : ~key;
    double d;
    __builtin_memcpy(&d, &bits, sizeof(d));
    return d;
}


/* ---- discrete adjoint (fx_adjoint.cu) ------------------------------------ */

/* device view of one reverse stage: the stored states before and after the
 * stage (stacked per-block W and Bf arrays, both slots) and the adjoint
 * arrays (same layouts; G holds, per cell, the dt-scaled adjoints of the
 * six updated conserved variables and the adjoints of the three updated
 * cell-field components, [b][v][cell]) */
struct FxAdjDev {
    const FxBlockDev *blk;
    double gamma;
    double dt;
    const double *Wbef;
    const double *Bfbef;
    const double *Waft;
    double *Wb;
    double *Bfb;
    double *G;
    double *bvb1;
    double *bvb2;
    double *Eb;
    const double *vr; /* face velocities recomputed from Wbef (normal component) */
};

#define FX_ADJ_G_COUNT (9 * FX_NCELLS)

/* A ghost-fill wave transposed into gathers (its adjoint): for every element the wave reads,
 * the list of operations reading it.  Cell sources: entries (dst cell key,
 * kind) with kind 0 copy, 1 + v copy with variable v negated, 16 copy with
 * v1 replaced (no sensitivity to v1).  Face sources: entries (key, kind)
 * with kind 0 = face copy to face key dst (direction in the source's
 * aux), 1 + d = half of cell key's field component d. */
struct FxAdjEnt {
    int32_t key;
    int32_t kind;
};

struct FxAdjSrc {
    int32_t key;   /* cell key, or face key */
    int32_t dir;   /* faces: direction */
    int32_t begin; /* entries [begin, end) */
    int32_t end;
};

void fx_launch_adj_gather(const FxAdjDev &A, const FxAdjSrc *csrc, int nc, const FxAdjSrc *fsrc, int nf,
    const FxAdjEnt *ents, int slot, cudaStream_t s);
/* zero the wave's destinations: cell ops (variables 0-5), face ops, and the
 * field components of cell-field ops */
void fx_launch_adj_zero(const FxAdjDev &A, const FxGop *cops, int nc, const FxGop *fops, int nf,
    const FxBop *bops, int nb, int slot, cudaStream_t s);
void fx_launch_adj_cells(const FxAdjDev &A, const int *blist, int nlist, int stage, cudaStream_t s);
void fx_launch_adj_bf(const FxAdjDev &A, const int *blist, int nlist, int stage, cudaStream_t s);
void fx_launch_adj_emf(const FxAdjDev &A, const int *blist, int nlist, int stage, cudaStream_t s);
void fx_launch_adj_flux(const FxAdjDev &A, const int *blist, int nlist, int stage, cudaStream_t s);

/* ---- dynamic AMR ----------------------------------------------------------- */

/* refinement criteria of prj_amr_tag, the set entries of the reference's
 * amr_* arrays in index order */
struct FxAmrTagCfg {
    int ncrit;
    int est[4];        /* estimator */
    int var[4];        /* Loehner variable (estimator 0) or jump variable (3) */
    double rthr[4];    /* refine threshold, <= 0: not summed for refinement */
    double dthr[4];    /* derefine threshold, <= 0: not summed for derefinement */
    double eps[4];     /* Loehner epsilon */
    double reach;      /* amr_reach_highest_level_at_density, <= 0: off */
    int has_derefine;  /* some criterion has a derefine threshold > 0 */
    int pad;
};

/* a child block to fill from its parent (oct: octant, x fastest) */
struct FxAmrChildJob {
    int32_t child;
    int32_t parent;
    int32_t oct;
    int32_t pad;
};

/* one face layer (16 x 16 faces of direction dir) a new child copies from
 * a finer neighbour of its parent: side 1 writes child index 16 from the
 * neighbour's index 0, side 0 index 0 from index 16 */
struct FxAmrCopyJob {
    int32_t child;
    int32_t src;
    int32_t dir;
    int32_t side;
};

/* a parent to fill from its eight children */
struct FxAmrParentJob {
    int32_t parent;
    int32_t children[8];
    int32_t pad[3];
};

/* votes[3 i .. 3 i + 2] = refine vote, derefine vote, boundary side mask of
 * block list[i] (pass 1 of prj_amr_tag); has_parent[i]: the block may
 * derefine */
void fx_launch_amr_tag(const FxDev &D, const int *list, const int *has_parent, int n,
    const FxAmrTagCfg &cfg, int32_t *votes, cudaStream_t s);
/* zeroes W, Bf, eosvar and grav of the listed blocks (prj_zero_block_arrays) */
void fx_launch_amr_zero(const FxDev &D, const int *blocks, int n, cudaStream_t s);
/* both stage slots of every job */
void fx_launch_amr_copy_faces(const FxDev &D, const FxAmrCopyJob *jobs, int n, cudaStream_t s);
/* Toth-Roe groups of the ghost fill kernel, for one stage slot */
void fx_launch_prolong_groups(const FxDev &D, const FxPop *pops, int np, int slot, cudaStream_t s);
/* conserved prolongation, face-average field, cons2prim and energy floor of
 * new children; inj (4096 per job) receives the floor's energy per cell
 * when E_floor > 0 */
void fx_launch_amr_prolong_cells(const FxDev &D, const FxAmrChildJob *jobs, int n, double E_floor,
    double *inj, cudaStream_t s);
/* face restriction of both stage slots onto re-activated parents */
void fx_launch_amr_restrict_faces(const FxDev &D, const FxAmrParentJob *jobs, int n, cudaStream_t s);
/* volume-weighted conserved restriction, face-average field, cons2prim and
 * energy floor of re-activated parents */
void fx_launch_amr_restrict_cells(const FxDev &D, const FxAmrParentJob *jobs, int n, double E_floor,
    double *inj, cudaStream_t s);

#endif
