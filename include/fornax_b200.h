/*
 * fornax_b200 -- B200 (sm_100a) implementation of FornaxAMR's per-block
 * Godunov MHD update behind a plain C ABI.
 *
 * The library keeps a device mirror of a FornaxAMR mesh: for every block the
 * primitive array W_mhd (2 RK stages), the face field Bf (2 stages) and the
 * static gravity array, in exactly the reference's per-block layout
 * (reference src/prj_defs.h:383-453), plus device-side scratch in the same
 * layout for flux, v_riemann, Bv1/Bv2, emf, eosvar and mhd_rhs.  A host that
 * owns prj_block data uploads it once, steps on the device, and downloads
 * when it needs the state (I/O, diagnostics).
 *
 * Build variants of the reference map onto run-time settings:
 *   PRJ_MHD=1 -> fx_config.mhd = 1 (NHYDRO = 9, HLLD, constrained transport)
 *   PRJ_MHD=0 -> fx_config.mhd = 0 (NHYDRO = 6, HLLC)
 *   PRJ_RECON_HYDRO -> fx_config.recon (MC, WENO-Z3, or WENO-Z7 in the
 *                      four-ghost-layer library)
 *   TIME_INTEGRATION -> fx_config.integrator (RK2 or eSSPRK10_4)
 *   prj_mesh.use_BJ -> fx_config.use_bj (Barth-Jespersen instead of minmod
 *                      in the coarse-to-fine prolongation of cells and faces)
 *   PRJ_NGHOST -> the library: libfornax_b200.so (2 layers, 20^3 block
 *                 arrays) or libfornax_b200_ng4.so (4 layers, 24^3);
 *                 fx_ghost_layers() reports which one is loaded
 * Fixed: PRJ_BLOCK_SIZE = 16, ideal-gas EOS with a run-time
 * adiabatic index, no radiation, no GR.  The number of stage slots of the
 * block W and Bf arrays (NS below) is 2 for RK2 and 3 for eSSPRK10_4.
 *
 * Every entry point returns 0 on success and a positive FX_E* code on
 * failure; fx_last_error() returns the message.  Device-side physics
 * failures (the reference's exit(1) paths) are reported by the next call
 * that synchronises (fx_sync, fx_step, fx_calc_dt, downloads) with
 * FX_EPHYSICS and the reference's message text.
 *
 * Threading: one context per host thread and device; calls on a context are
 * not thread-safe (the reference's hot path is single-threaded per rank and
 * keeps non-reentrant static scratch, src/prj_flux.c:385, 2155-2171).
 */
#ifndef FORNAX_B200_H
#define FORNAX_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define FX_API_VERSION 1

/* return codes */
#define FX_SUCCESS 0
#define FX_EINVAL 1     /* bad argument */
#define FX_ECUDA 2      /* CUDA runtime error */
#define FX_ENOMESH 3    /* no mesh set */
#define FX_EPHYSICS 4   /* device-side physics failure (reference exit path) */
#define FX_ENOMEM 5     /* device allocation failed */
#define FX_ETOOBIG 6    /* request exceeds a fixed capacity (FX_NOALLOC_MAX_BLOCKS) */
#define FX_ECOMM 7      /* exchange between ranks of a sharded mesh failed */

/* execution forms of a step */
#define FX_FORM_PLAIN 0    /* per-block kernel launches in the reference's loop order */
#define FX_FORM_BATCHED 1  /* every phase swept over all blocks, replayed as one CUDA graph */

/* boundary condition types, values of enum prj_bc_type (src/prj_defs.h:518-523) */
#define FX_BC_OUTFLOW 0
#define FX_BC_REFLECT 1
#define FX_BC_USER 2
#define FX_BC_PERIODIC 3

/* block-level array selectors for fx_download_array */
#define FX_ARR_W 0        /* NHYDRO * 2 * 8000, WIDX */
#define FX_ARR_EOSVAR 1   /* 3 * 8000, EIDX (AoSoA) */
#define FX_ARR_FLUX 4     /* per dir: NHYDRO * 8000, VIDX (AoSoA) */
#define FX_ARR_VRIEMANN 5 /* per dir: 3 * 8000, VRIDX (AoSoA) */
#define FX_ARR_GRAV 6     /* per dir: 8000, IDX */
#define FX_ARR_BF 7       /* per dir: 2 * 8400, FACE_IDX */
#define FX_ARR_BV1 8      /* per dir: 8000, IDX */
#define FX_ARR_BV2 9      /* per dir: 8000, IDX */
#define FX_ARR_EMF 10     /* per dir: 8820, EDGE_IDX */
#define FX_ARR_RHS 3      /* NHYDRO * 8000, MHDVIDX (AoSoA) */

typedef struct fx_ctx fx_ctx;

/* One neighbour slot: the fields of prj_neighbor (src/prj_types.h:73-100)
 * that the ghost fill and the coarse/fine corrections read. */
typedef struct fx_slot {
    int32_t id;         /* neighbour block index into the block array, -1 if none */
    int32_t rel_level;  /* neighbour level minus this block's level: -1, 0, +1 */
    int32_t type;       /* 0 none, 1 face, 2 edge, 3 corner */
    int8_t send_loc_start[3];
    int8_t send_loc_end[3];
    int8_t recv_loc_start[3];
    int8_t recv_loc_end[3];
} fx_slot;

/* One block of the mesh (prj_block, src/prj_types.h:151-213: geometry,
 * the 56 neighbour slots and the refinement tree). */
typedef struct fx_block_desc {
    int32_t id;         /* < 0: unused entry */
    int32_t level;
    int32_t active;     /* 1 for leaf blocks that are stepped */
    int32_t rank;       /* must be 0 (one device, one rank) */
    double xmin[3];
    double xmax[3];
    double dx[3];
    double vol;
    double area[3];
    fx_slot slot[56];
    int32_t parent;     /* parent block index, -1 for root blocks */
    int32_t children[8];/* child block indices in octant order (x fastest), -1 if none */
    int32_t can_refine; /* prj_block.can_refine: 0 keeps the block from refining */
} fx_block_desc;

/* reconstruction (PRJ_RECON_HYDRO, src/prj_defs.h:299-301) */
#define FX_RECON_MC 0      /* PRJ_RECON_MC: monotonised-central slopes */
#define FX_RECON_WENO3 1   /* PRJ_RECON_WENO3: WENO-Z3 face values (src/prj_reconstruct.h:383-423) */
#define FX_RECON_WENO7 2   /* PRJ_RECON_WENO7: WENO-Z7 face values (src/prj_reconstruct.h:425-521);
                              needs four ghost layers: the library built with FX_NG=4
                              (libfornax_b200_ng4.so, 24^3 block arrays) */
/* time integration (TIME_INTEGRATION, src/prj_defs.h:135-150) */
#define FX_INT_RK2 0           /* RK2: two stages, block arrays with 2 stage slots */
#define FX_INT_ESSPRK10_4 1    /* eSSPRK10_4 (the reference's default): ten forward-Euler
                                * substeps of dt / 6 with three stored states; block W and
                                * Bf arrays carry 3 stage slots (PRJ_BLOCK_NSTAGES = 3) */

/* Run-time configuration (compile-time switches of the reference). */
typedef struct fx_config {
    int32_t mhd;        /* 1: PRJ_MHD=1 build, 0: hydro build */
    int32_t gravity;    /* 1: apply the static gravity source from uploaded grav arrays */
    double gamma;       /* ideal-gas adiabatic index of the user EOS */
    double coord[6];    /* domain: x1min, x1max, x2min, x2max, x3min, x3max (prj_coord) */
    int32_t bc[6];      /* x1 inner, x1 outer, x2 inner, x2 outer, x3 inner, x3 outer */
    double mhd_eta;     /* prj_mesh.mhd_eta */
    int32_t recon;      /* FX_RECON_MC, FX_RECON_WENO3 or FX_RECON_WENO7 */
    int32_t integrator; /* FX_INT_RK2 or FX_INT_ESSPRK10_4 */
    int32_t use_bj;     /* prj_mesh.use_BJ: 1 selects the Barth-Jespersen limiter of
                         * prj_reconstruct_{cell,face}_for_prolongate_bj
                         * (src/prj_reconstruct.h:145-313) in the ghost fill's and the
                         * refinement's prolongation, 0 the minmod limiter */
    int32_t pad;
} fx_config;

/* ---- context -------------------------------------------------------------- */

/* Ghost layers of this build (the reference's compile-time PRJ_NGHOST):
 * 2 for libfornax_b200.so (20^3 block arrays), 4 for libfornax_b200_ng4.so
 * (24^3, needed by FX_RECON_WENO7).  Every per-block size in this header
 * (8000 cells, 8400 faces, 8820 edges) is that of the 2-layer build; the
 * 4-layer build uses 13824, 14400 and 15000. */
int fx_ghost_layers(void);

/* Creates a context on `device`.  Replaces nothing: the reference has no
 * device; this owns the stream, the device mirror and the step graphs.
 * FX_EINVAL for FX_RECON_WENO7 in the 2-layer build. */
int fx_create(int device, const fx_config *cfg, fx_ctx **out);
void fx_destroy(fx_ctx *ctx);
int fx_last_error(const fx_ctx *ctx, char *buf, size_t len);
/* Waits for all queued work and reports device-side physics failures. */
int fx_sync(fx_ctx *ctx);
/* The CUDA stream (cudaStream_t) all work is queued on, for host-side timing. */
int fx_stream(fx_ctx *ctx, void **stream);

/* ---- mesh ------------------------------------------------------------------ */

/* Mirrors the block list and neighbour slots of a prj_mesh
 * (src/prj_types.h:465-503; slots built by prj_neighbor_compute_geometry,
 * src/prj_mesh.c:46-243).  Allocates device storage and compiles the ghost
 * fill of prj_boundary_fill_ghosts_and_bf (src/prj_boundary.c:1150-1241) and
 * the coarse/fine flux and EMF corrections (src/prj_riemann.c:1700-1768,
 * src/prj_mhd.c:1003-1029) into device programs. */
int fx_set_mesh(fx_ctx *ctx, int nblocks, const fx_block_desc *blocks);

/* Host-only inspection of the compiled ghost fill (no device needed).
 * which = 0: cell program, 1: face program, 2: flux corrections,
 * 3: EMF corrections, 4: cell-field (bf2bc) operations, 5: compiler
 * statistics, 6: face-prolongation groups.  Call with NULL buffers to get
 * *nops and *nwaves; then ops receives 4 int32 per operation for 0/1
 * (dst, src, aux, type) and 8 for 2/3/4/6, and wave_begin nwaves + 1
 * offsets. */
int fx_plan_export(const fx_config *cfg, int nblocks, const fx_block_desc *blocks, int which,
    int32_t *ops, int *nops, int32_t *wave_begin, int *nwaves);

/* ---- sharding over ranks (one GPU per rank) ---------------------------------
 * The reference decomposes the block list over MPI ranks (block->rank,
 * prj_mpi_decompose, src/prj_mpi.c:375-470) and exchanges ghost zones
 * (prj_mpi_post/wait_ghosts_and_bf, src/prj_boundary.c:1184-1222), the
 * coarse/fine flux and EMF records (prj_mpi_exchange_fluxes_and_emf,
 * src/prj_mpi.c:4601) and the dt minimum (src/prj_mpi.c:4765-4778).  Here
 * owner[b] assigns every active block to a rank; each rank runs its part of
 * the single-device ghost-fill and correction programs (the operations into
 * its blocks and, transitively, the operations on other ranks' blocks whose
 * values they read) after receiving the values its part reads from other
 * ranks' blocks.  Every rank then holds, for its blocks, exactly the values
 * of the single-device step.
 *
 * Host-only inspection of rank `rank`'s part (no device needed): which 0-4,
 * 6 as fx_plan_export (programs in the rank's local block numbering: owned
 * blocks first, then the halo); 7: local -> global block map (*nops
 * entries, *nwaves = owned blocks); 8 + k / 12 + k: the send / receive list
 * of exchange k (0 cells, 1 faces, 2 flux entries, 3 EMF entries) as
 * (local block, index) pairs with per-peer offsets in wave_begin (nranks + 1
 * entries, *nwaves = nranks).  No counterpart in the reference. */
int fx_shard_export(const fx_config *cfg, int nblocks, const fx_block_desc *blocks, const int *owner,
    int nranks, int rank, int which, int32_t *ops, int *nops, int32_t *wave_begin, int *nwaves);

/* Sets rank `rank`'s part of a mesh sharded over nranks ranks (owner[b]:
 * the rank of active block b; contiguous runs of the reference's Morton
 * order are the natural choice): device storage for the owned blocks and
 * the halo, the rank's programs and exchange buffers.  Afterwards
 * fx_upload_block / fx_download_block take the mesh's block indices of
 * owned blocks, and fx_calc_dt, fx_step and fx_run (batched form, RK2) run
 * the rank's part of every step, exchanging with the other ranks through
 * the attached transport: every rank must make the same calls in the same
 * order; fx_boundary_fill_ghosts_and_bf fills the ghost zones of the owned
 * blocks (with its exchange).  The other per-block drop-in calls, whole-mesh
 * copies, dynamic AMR and the adjoint are not available on a sharded mesh.  No counterpart in the
 * reference (its ranks are MPI processes over one prj_mesh). */
int fx_shard_set_mesh(fx_ctx *ctx, int nblocks, const fx_block_desc *blocks, const int *owner, int nranks,
    int rank);

/* Transports.  A group emulates nranks ranks inside one process (one host
 * thread per rank, each driving its own context, possibly on one GPU):
 * exchanges are device-to-device copies between the contexts' buffers with
 * host barriers (a rank that does not arrive within 120 s fails the
 * exchange with FX_ECOMM); steps run without graphs.  NCCL runs one process
 * per GPU: rank 0 makes the unique id (fx_nccl_unique_id), the host shares
 * it (e.g. torch.distributed), every rank attaches; exchanges are
 * send/recv groups and dt minima all-reduces on the context's stream, and
 * whole steps are captured as CUDA graphs.  libnccl.so.2 is loaded when
 * first needed. */
typedef struct fx_shard_group fx_shard_group;
fx_shard_group *fx_shard_group_create(int nranks);
void fx_shard_group_destroy(fx_shard_group *group);
int fx_shard_attach_group(fx_ctx *ctx, fx_shard_group *group);
int fx_nccl_unique_id(unsigned char id[128]);
int fx_shard_attach_nccl(fx_ctx *ctx, const unsigned char id[128]);

/* owned blocks, local blocks (owned + halo) and the doubles this rank sends
 * per RK2 step over all exchanges */
int fx_shard_info(fx_ctx *ctx, int *nowned, int *nlocal, long long *doubles_per_step);

/* Host <-> device copies of one block, in the reference's per-block layout:
 * W = block->W_mhd (NHYDRO * NS * 8000 doubles), Bf[d] = block->Bf[d]
 * (NS * 8400 doubles each, may be NULL for hydro), grav[d] = block->grav[d]
 * (8000 doubles each, may be NULL); NS = 2 (RK2) or 3 (eSSPRK10_4). */
int fx_upload_block(fx_ctx *ctx, int block, const double *W, const double *const Bf[3],
    const double *const grav[3]);
/* eosvar (3 * 8000, may be NULL) is recomputed from W of the last stage,
 * exactly what prj_eos_fill_active_cells + prj_eos_fill_mesh leave there. */
int fx_download_block(fx_ctx *ctx, int block, double *W, double *eosvar, double *const Bf[3]);
/* Whole-mesh copies: W_all is nblocks consecutive W arrays, Bf_all nblocks
 * consecutive 3 * NS * 8400 arrays (d-major); either may be NULL. */
int fx_upload_all(fx_ctx *ctx, const double *W_all, const double *Bf_all);
int fx_download_all(fx_ctx *ctx, double *W_all, double *Bf_all);
/* Same host layout as fx_upload_all / fx_download_all, but only stage slot 0
 * of W and Bf moves: the state a host driver sees between calls to
 * prj_timeint_step (slot 1 is the step's scratch). */
int fx_upload_state(fx_ctx *ctx, const double *W_all, const double *Bf_all);
int fx_download_state(fx_ctx *ctx, double *W_all, double *Bf_all);
/* ---- dump payloads ------------------------------------------------------------ */

/* Values per block of the dump's MetaData dataset (src/prj_io.c:19). */
#define FX_DUMP_METADATA_SIZE 639

/* The contents of prj_io_write_dump's datasets (src/prj_io.c:1994-2330,
 * dump_format_version 4), gathered from the device state for a host that
 * writes them into its own container (the HDF5 library is not linked here):
 *   data  [nblocks][NHYDRO][16^3]: Data, stage slot 0 of W at the active
 *         cells, cell = (i 16 + j) 16 + k;
 *   eos   [nblocks][3][16^3]: Eos, pressure, temperature and adiabatic index
 *         (eosvar) at the active cells, from that state;
 *   bf    [nblocks][3][NFACES]: Bf (the reference writes it in its
 *         PRJ_MHD_DEBUG builds), stage slot 0 of every face.
 * Rows of entries that are not active blocks are left untouched (the
 * reference never writes them: zero-fill the arrays first for its file
 * contents).  Any argument may be NULL; bf is ignored without MHD. */
int fx_dump_gather(fx_ctx *ctx, double *data, double *eos, double *bf);

/* The MetaData rows of prj_io_fill_metadata (src/prj_io.c:1133-1165) for a
 * mesh description (e.g. from fx_get_mesh): id, rank 0, level, active,
 * xmin[3], xmax[3], dx[3], parent, 0, children[8], then per slot the
 * neighbour id, rank 0 and the neighbour's xmin[3], xmax[3], dx[3] (zeros
 * for a free slot).  Host only. */
int fx_dump_metadata(int nblocks, const fx_block_desc *blocks, double *meta);

/* The state through its active region: stage slot 0 of the 16^3 active
 * cells and of the active faces (17 x 16 x 16 per direction), in the host
 * layout of fx_upload_state, moved by the copy engines as whole rows of the
 * active (i, j) range (the ghost columns along k of those rows included) --
 * about half of fx_upload_state's bytes each way for 16^3 blocks with two
 * ghost layers.  fx_upload_state_active leaves out the cell-centred field
 * in MHD runs and sets it from the faces as prj_mhd_bf2bc does (Bf_all is
 * then required), then runs the ghost fill of slot 0
 * (prj_boundary_fill_ghosts_and_bf with stage 1 and the stage-0 field).
 * fx_download_state_active copies every variable and synchronises; the
 * rest of the host arrays (the other ghost entries, other slots) is left
 * untouched.  The ghost fill does not write every ghost entry: a few of the
 * outermost ghost faces and corner cells keep the values the set-up gave
 * them, in the reference as here.  Make one full transfer (fx_upload_state
 * or fx_upload_all) first; from then on the device state after
 * fx_upload_state_active equals the one fx_upload_state gives whenever the
 * host's ghost zones come from that fill, as they do after every reference
 * step.  Page-locked host arrays make the copies asynchronous and fast;
 * pageable ones work at the copy engines' staged rate. */
int fx_upload_state_active(fx_ctx *ctx, const double *W_all, const double *Bf_all);
int fx_download_state_active(fx_ctx *ctx, double *W_all, double *Bf_all);
/* Any block array, including the step's scratch, for inspection. */
int fx_download_array(fx_ctx *ctx, int block, int which, int dir, double *out);

/* ---- reference entry points (plain, per block) ----------------------------- */

/* prj_flux_update (src/prj_flux.h:4-5): face fluxes, v_riemann, Bv1/Bv2 of
 * one block from W slot w_slot and Bf slot use_bf1. */
int fx_flux_update(fx_ctx *ctx, int block, int w_slot, int use_bf1);
/* prj_timeint_mhd_update_emf (src/prj_timeint.c:292-413): edge EMFs of one
 * block at stage slot `stage`. */
int fx_mhd_update_emf(fx_ctx *ctx, int block, int stage);
/* prj_timeint_mhd_update_bf (src/prj_timeint.c:448-495), stage 1 or 2. */
int fx_mhd_update_bf(fx_ctx *ctx, int block, int stage, double dt);
/* prj_src_update + the per-cell stage update loops (src/prj_timeint.c:1255-1349,
 * 1562-1654) of one block; folds the block's dt_src into *dt_src if non-NULL
 * (synchronises). */
int fx_update_cells(fx_ctx *ctx, int block, int stage, double dt, double *dt_src);
/* prj_riemann_flux_send (src/prj_riemann.c:1700-1768). */
int fx_riemann_flux_send(fx_ctx *ctx);
/* prj_mhd_emf_send (src/prj_mhd.c:1003-1029). */
int fx_mhd_emf_send(fx_ctx *ctx);
/* prj_eos_fill_active_cells / prj_eos_fill_mesh (src/prj_eos.c:1112-1162);
 * `stage` is the reference's stage argument (slot = stage - 1). */
int fx_eos_fill_active_cells(fx_ctx *ctx, int stage);
int fx_eos_fill_mesh(fx_ctx *ctx, int stage);
/* prj_boundary_fill_ghosts_and_bf (src/prj_boundary.h:17-18). */
int fx_boundary_fill_ghosts_and_bf(fx_ctx *ctx, int stage, int use_bf1);

/* ---- time integration ------------------------------------------------------- */

/* prj_timeint_calc_dt (src/prj_timeint.h:15-16): min over active cells
 * (times 6 for eSSPRK10_4, src/prj_timeint.c:2250-2251). */
int fx_calc_dt(fx_ctx *ctx, double cfl, double *dt);
/* prj_timeint_stage1 / prj_timeint_stage2 (src/prj_timeint.h:17-20); RK2 only. */
int fx_stage(fx_ctx *ctx, int form, int stage, double dt, double *dt_src);
/* prj_timeint_step (src/prj_timeint.h:31-33): one RK2 step, or one
 * eSSPRK10_4 step (prj_timeint_eSSPRK10_4_advance, src/prj_timeint.c:2671-2729).
 * *dt_src (may be NULL) receives the minimum source time step.
 * FX_FORM_BATCHED replays a captured CUDA graph; it does not synchronise
 * unless dt_src != NULL. */
int fx_step(fx_ctx *ctx, int form, double dt, double *dt_src);
/* The driver loop of src/main.c:485-562 without I/O: calc_dt, dt growth
 * limit dt_factor, clip to t_end, step, dt_src clamp; device resident.
 * state[0..2] = time, dt, step on entry and on return. */
int fx_run(fx_ctx *ctx, int form, int nsteps, double cfl, double dt_factor, double t_end,
    double *state);

/* ---- allocation-free timestep ----------------------------------------------- */

/* Capacity of fx_calc_dt_noalloc: at most this many listed blocks per call. */
#define FX_NOALLOC_MAX_BLOCKS 65536

/* The timestep of fx_calc_dt / prj_timeint_calc_dt (src/prj_timeint.h:15-16)
 * for a host that keeps the block state in its own device memory and may not
 * allocate device memory while it steps (for instance one whose device
 * memory comes from a fixed pool sized at start-up).  No counterpart in the
 * reference, which has no device; nothing is allocated, here or by the
 * library calls it makes.
 *
 *   W           device; block b's W_mhd in the reference layout (src/prj_defs.h
 *               WIDX): NHYDRO variables (9 if mhd else 6) x NS stage slots x
 *               NCELLS cells, block b at W + b * NHYDRO * NS * NCELLS, where
 *               NS = 2 for FX_INT_RK2 and 3 for FX_INT_ESSPRK10_4 (the
 *               reference's PRJ_BLOCK_NSTAGES) and NCELLS = (16 + 2 NG)^3 with
 *               NG = fx_ghost_layers() of the loaded library (8000 cells in
 *               libfornax_b200.so, 13824 in libfornax_b200_ng4.so); stage
 *               slot 0 is read
 *   integrator  FX_INT_RK2 or FX_INT_ESSPRK10_4: the stage slots of W and the
 *               factor the minimum is multiplied by (1, or 6 as the
 *               reference does for eSSPRK10_4, src/prj_timeint.c:2250-2251)
 *   dx          device; dx[3b + d] = cell width of block b along d
 *   nblocks     the number of blocks present in W and dx
 *   blocks      device; nlist block indices to reduce over (the active
 *               blocks), or NULL for blocks 0 .. nlist-1; an index outside
 *               [0, nblocks) is not read and makes the result NaN
 *   stream      cudaStream_t the two kernels are queued on (NULL: default stream)
 *   dt          device; receives the minimum (1e99 if no cell gives a finite
 *               value) times the integrator's factor, stream-ordered: the
 *               call does not synchronise
 *
 * Returns FX_ETOOBIG, before any device work, when nlist exceeds
 * FX_NOALLOC_MAX_BLOCKS, and FX_EINVAL for null pointers, nblocks <= 0,
 * nlist <= 0, mhd not 0/1, an unknown integrator, gamma <= 1 or cfl <= 0.
 * A CUDA error already pending in the calling thread is left in place and
 * reported as FX_ECUDA without queueing anything; a failed launch returns
 * FX_ECUDA.  The scratch is one fixed 512 KiB device array per device,
 * written in full by each call before it is read, so it needs no clearing.
 * The first call on a device resolves its address with cudaGetSymbolAddress
 * (with that device current) and keeps it for the life of the process; make
 * that first call before any stream capture, and do not call the function
 * after a cudaDeviceReset of that device (the array's address may change).
 * Calls on one device share the scratch: two calls whose kernels overlap
 * (different streams or host threads) race and give wrong results, so order
 * them on one stream or serialise them. */
int fx_calc_dt_noalloc(const double *W, int mhd, int integrator, const double *dx, int nblocks,
    const int *blocks, int nlist, double gamma, double cfl, void *stream, double *dt);

/* ---- dynamic AMR ---------------------------------------------------------------- */

/* Refinement criteria: the amr_* arrays of prj_mesh (src/prj_types.h:482-490),
 * PRJ_AMR_N = 4 entries, summed as sum_n indicator_n / thresh_n per cell. */
#define FX_AMR_N 4
#define FX_AMR_LOEHNER 0                /* PRJ_AMR_ESTIMATOR_LOEHNER */
#define FX_AMR_VELOCITY 1               /* PRJ_AMR_ESTIMATOR_VELOCITY */
#define FX_AMR_PRESSURE_SCALE_HEIGHT 2  /* PRJ_AMR_ESTIMATOR_PRESSURE_SCALE_HEIGHT */
#define FX_AMR_FRACTIONAL_JUMP 3        /* PRJ_AMR_ESTIMATOR_FRACTIONAL_JUMP */
#define FX_AMR_VAR_DENSITY 0            /* Loehner / jump variable: density */
#define FX_AMR_VAR_PRESSURE 1           /* gas + magnetic pressure */
#define FX_AMR_VAR_TEMPERATURE 2        /* Loehner only */

typedef struct fx_amr_criterion {
    int32_t set;             /* amr_criterion_set */
    int32_t estimator;       /* FX_AMR_LOEHNER .. FX_AMR_FRACTIONAL_JUMP */
    int32_t lohner_var;      /* amr_lohner_var */
    int32_t jump_var;        /* amr_fractional_jump_var */
    double refine_thresh;    /* <= 0: not a refinement criterion */
    double derefine_thresh;  /* <= 0: not a derefinement criterion */
    double lohner_eps;
} fx_amr_criterion;

typedef struct fx_amr_config {
    int32_t root_nx[3];      /* prj_mesh.root_nx: root blocks per axis */
    int32_t max_level;       /* < 0: unlimited */
    int32_t max_blocks;      /* prj_mesh.nblocks_max: capacity of the block array */
    int32_t pad;
    double min_dx;           /* <= 0: no cell-size floor */
    double reach_density;    /* amr_reach_highest_level_at_density, <= 0: off */
    double E_floor;          /* internal-energy floor after a remesh, <= 0: off */
    fx_amr_criterion crit[FX_AMR_N];
} fx_amr_config;

/* Sets the refinement parameters and the refinement tree of the mirrored
 * mesh (the parent/children/can_refine of the last fx_set_mesh).  The
 * prolongation limiter is fx_config.use_bj; the angular-resolution cap and
 * the Z4c estimator are not supported. */
int fx_amr_configure(fx_ctx *ctx, const fx_amr_config *amr);
/* prj_amr_tag (src/prj_amr.c:1581-1782) on the device state (W slot 0 after a
 * step or a fill): refine_flag[b] for every block entry (+1 refine, -1
 * derefine, 0 keep) after the per-block caps, before 2:1 balance. */
int fx_amr_tag(fx_ctx *ctx, int32_t *refine_flag);
/* prj_amr_adapt (src/prj_amr.c:2576-2706) followed by the driver's refill of
 * a changed mesh (src/main.c:599-606): tags on the device, balances and
 * rebuilds the block tree and neighbour slots on the host, prolongs and
 * restricts the cell and face data on the device, recompiles the ghost fill
 * and fills the ghosts of slot 0.  *changed = 1 if the mesh changed.  From
 * the first call on, the context keeps the ghost-fill compiler's working
 * buffers in host memory (about 1.7 MB per MHD block entry of the largest
 * adapted mesh: 4.1 GB for 2352 entries, plus the program arrays of the
 * previous mesh's ghost fill) so that later adapts reuse them instead of
 * faulting in fresh pages; fx_destroy releases them. */
int fx_amr_adapt(fx_ctx *ctx, int *changed);
/* The mirrored mesh: *nblocks entries (unused ones have id < 0) are written
 * to out if capacity allows; *nblocks is always set. */
int fx_get_mesh(fx_ctx *ctx, int capacity, fx_block_desc *out, int *nblocks);
/* Energy added by the E_floor of all remeshes so far (eos->E_injected). */
int fx_amr_energy_injected(fx_ctx *ctx, double *e);
/* Host wall time (ms) of the phases of the last fx_amr_adapt: ms[0] device
 * tag (with its read-back), ms[1] host remesh, ms[2] data moves queued
 * (and any array growth), ms[3] ghost-fill compile of the new mesh (the data
 * moves run on the device meanwhile), ms[4] tables, refill and
 * synchronisation, ms[5] total. */
int fx_amr_timings(fx_ctx *ctx, double *ms);

/* Host-only remesh (no device): the block-tree half of prj_amr_adapt for
 * given per-block tag votes.  votes[3 b .. 3 b + 2] = refine vote (0/1),
 * derefine vote (0/-1) and the boundary side mask of block b, as pass 1 of
 * prj_amr_tag leaves them.  flags (nblocks, may be NULL) receives the tag
 * result (after the caps); out (capacity entries) the adapted mesh, *nout
 * its block count.  Returns FX_ETOOBIG when the mesh outgrows
 * amr->max_blocks or capacity. */
int fx_amr_remesh_host(const fx_config *cfg, const fx_amr_config *amr, int nblocks,
    const fx_block_desc *in, const int32_t *votes, int32_t *flags, int capacity, fx_block_desc *out,
    int *nout);

/* Neighbour-slot geometry of a mesh whose slot ids are set: for every slot
 * with id >= 0, its type, relative level and send/recv boxes
 * (prj_neighbor_compute_geometry, src/prj_mesh.c:46-243); slots with id < 0
 * are reset to the empty slot (type 0, level 0, zero boxes).  Returns
 * FX_EINVAL for an id outside [0, nblocks) or neighbours more than one
 * level apart.  The product's mesh builders use this one restatement. */
int fx_mesh_slot_geometry(int nblocks, fx_block_desc *blocks);

/* Decision record and replay of the plain form (no reference counterpart;
 * for checking the discrete adjoint against finite differences).  The
 * update is smooth in the state except where a decision switches: the MC
 * limiter's candidate for each reconstructed quantity, the HLLD
 * wave-speed arguments, clamped discriminants, fan region, bn_small,
 * contact side, single or double star, degenerate outer-star denominators
 * and the sign of bn (src/prj_reconstruct.h:355-375,
 * src/prj_riemann.c:117-440), and each edge's upwind directions
 * (src/prj_mhd.c:627-680).
 *   FX_BRANCH_RECORD: the following plain-form RK2 stages (at most
 *     max_stages) record every face's and edge's decisions;
 *   FX_BRANCH_REPLAY: the following plain-form stages take those decisions
 *     instead of evaluating them -- the map with its branches frozen at the
 *     recorded state, whose derivative the adjoint computes -- and count the
 *     decisions that would have come out otherwise;
 *   FX_BRANCH_OFF: back to the solver as it stands; after a replay *flips
 *     (may be NULL) receives that count.  FX_ETOOBIG if more stages ran
 *     than were recorded.
 * MHD, MC, RK2, one rank; the batched form is not affected. */
#define FX_BRANCH_OFF 0
#define FX_BRANCH_RECORD 1
#define FX_BRANCH_REPLAY 2
int fx_branch_trace(fx_ctx *ctx, int mode, int max_stages, unsigned long long *flips);

/* ---- measurement --------------------------------------------------------------- */

/* phases for fx_time_phase: the batched sweep of one phase over all blocks */
#define FX_PHASE_FLUX 0      /* one face-flux launch (all three directions) */
#define FX_PHASE_EMF 1       /* edge EMFs */
#define FX_PHASE_CT 2        /* CT face update, stage 1 */
#define FX_PHASE_CELLS 3     /* cell update, stage 1 */
#define FX_PHASE_GHOST 4     /* ghost fill of stage slot 1 (all waves) */
#define FX_PHASE_STEP 5      /* one batched RK2 step (graph) */

/* Times `reps` back-to-back launches of one phase with CUDA events on the
 * context's stream (after one untimed launch); *ms = average per launch.
 * Phases 0-4 rewrite the stage-1 scratch only, so repeating them leaves the
 * mesh state unchanged; phase 5 advances the state by reps steps with dt. */
int fx_time_phase(fx_ctx *ctx, int phase, int reps, double dt, double *ms);

/* Autotuner: times every compiled launch shape of the face-flux kernel (the
 * dominant phase) on the current mesh and keeps the fastest for all later
 * steps.  times_ms (may be NULL) receives up to `n` per-shape times, *choice
 * the chosen shape.  The shapes compute identical results. */
int fx_autotune(fx_ctx *ctx, double *times_ms, int n, int *choice);
/* Forces face-kernel launch shape `variant` (0 .. 5, the autotuner's
 * choices: one thread per face at various CTA sizes and register budgets).
 * All shapes compute identical results. */
int fx_set_flux_shape(fx_ctx *ctx, int variant);

/* what = 0: kernel launches per batched step, 1: per plain step,
 * 2/3: ghost cell/face operations, 4: ghost-fill waves, 5: cell-field
 * (bf2bc) operations */
int fx_info(fx_ctx *ctx, int what, long long *value);

/* ---- discrete adjoint ---------------------------------------------------------- */

/* No counterpart in the reference (it has no adjoint): reverse-mode
 * derivatives of the batched RK2 step for single-level MHD meshes without
 * gravity or resistivity.
 *
 * fx_adjoint_forward runs nsteps batched RK2 steps with the fixed time step
 * dt from the current state and stores the state after every stage (W and
 * Bf, both slots) and the stage's face velocities: (2 nsteps + 1) * nblocks
 * * (9 * 2 * 8000 + 3 * 2 * 8400) + 2 nsteps * nblocks * 72000 doubles of
 * device memory. */
int fx_adjoint_forward(fx_ctx *ctx, int nsteps, double dt);
/* Reverse pass over the stored steps.  W_bar / Bf_bar (host, the layout of
 * fx_upload_all; Bf_bar may be NULL for zero) hold d J / d (final state);
 * W_bar_out / Bf_bar_out receive d J / d (state at fx_adjoint_forward's
 * entry).  With initial_fill = 1 the adjoint of one more ghost fill of slot
 * 0 is applied last, so the result is with respect to the state before the
 * driver's initial fill (the ghost entries then carry no sensitivity).
 * Limiter and Riemann-fan branches are those of the stored forward pass. */
int fx_adjoint_backward(fx_ctx *ctx, const double *W_bar, const double *Bf_bar, double *W_bar_out,
    double *Bf_bar_out, int initial_fill);
/* Device time (ms, CUDA events) of the last reverse sweep, without the
 * host transfers. */
int fx_adjoint_time(fx_ctx *ctx, double *ms);

/* ---- adjoint building blocks (host) ----------------------------------------- */

/* Host evaluation of one face of the face-flux kernel, for checks of the
 * discrete adjoint (no counterpart in the reference): w4[n * 9 + v] are the
 * local-frame primitives of the four stencil cells n = 0..3 along the sweep
 * (v = 0 rho, 1 normal velocity, 2-3 transverse velocities, 4 eint, 5 ye,
 * 7-8 transverse field; 6 unused), bn the face-normal field.  MC
 * reconstruction of every variable and of the cell pressures, then HLLD
 * (prj_riemann_hlld, src/prj_riemann.c:321-440).  out[14] = local flux[9],
 * face velocity[3], Bv1, Bv2. */
int fx_face_eval_host(const double *w4, double bn, double gamma, double *out);
/* Its vector-Jacobian product: w4_bar[36] and *bn_bar = out_bar^T d out /
 * d (w4, bn), on the smooth piece the evaluation lies on. */
int fx_face_vjp_host(const double *w4, double bn, double gamma, const double *out_bar,
    double *w4_bar, double *bn_bar);

#ifdef __cplusplus
}
#endif

#endif
