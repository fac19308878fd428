/*
 * Ghost-fill compiler: turns a mesh description into device programs.
 */
#ifndef FX_PLAN_H
#define FX_PLAN_H

#include <string>
#include <vector>

#include "../../include/fornax_b200.h"
#include "fx_kernels.h"

/* The ghost fill as waves of element operations.  Operations inside one
 * wave touch disjoint elements (no read/write or write/write overlap), so a
 * wave runs as one parallel kernel; waves run in order.  Each wave holds
 * cell operations (primitives 0..5), face operations, face-prolongation
 * groups and cell-field operations (bf2bc of one cell). */
struct FxProgram {
    std::vector<FxGop> cell_ops;
    std::vector<FxGop> face_ops;
    std::vector<FxPop> p_ops;
    std::vector<FxBop> b_ops;
    std::vector<int> cell_begin; /* per wave: [begin, next begin) into cell_ops */
    std::vector<int> face_begin;
    std::vector<int> p_begin;
    std::vector<int> b_begin;
    int nwaves() const { return cell_begin.empty() ? 0 : (int)cell_begin.size() - 1; }
};

struct FxPlanStats {
    long long emitted_cell_ops = 0; /* writes that land in the reference sequence */
    long long emitted_face_ops = 0;
    long long rewired = 0;          /* copies redirected to an earlier source */
    long long dead = 0;             /* overwritten before any read: dropped */
};

/* One element of a sharded exchange, in the receiving or sending rank's
 * local block numbering.  idx: the cell (cells; the ghost-filled primitives
 * move), dir * 8400 + face (faces), the component-0 entry of the block's
 * stacked flux array (flux; every stored component moves) or the entry of
 * its EMF array (emf). */
struct FxXel {
    int32_t block;
    int32_t idx;
};

/* elements exchanged with each peer rank p: el[begin[p], begin[p + 1]) */
struct FxXlist {
    std::vector<FxXel> el;
    std::vector<int> begin;
};

enum { FX_X_CELLS = 0, FX_X_FACES = 1, FX_X_FLUX = 2, FX_X_EMF = 3, FX_X_KINDS = 4 };

/* A rank's part of a sharded mesh.  Local blocks are the owned active blocks
 * (first, in mesh order) and then the halo: other ranks' blocks that the
 * rank's programs read or write.  send[k] lists what this rank packs for
 * each peer before exchange k, recv[k] what it unpacks into its halo; both
 * sides of a pair order the elements by global block and index, so the
 * lists match without being exchanged. */
struct FxShard {
    int nranks = 1;
    int rank = 0;
    int nowned = 0;
    std::vector<int> local_to_global;
    FxXlist send[FX_X_KINDS];
    FxXlist recv[FX_X_KINDS];
    bool any[FX_X_KINDS] = {false, false, false, false}; /* some pair of ranks exchanges kind k */
};

struct FxPlan {
    FxProgram ghost;
    FxPlanStats stats;
    std::vector<FxCorr> flux_corr;  /* prj_riemann_flux_send records, by wave */
    std::vector<FxCorr> emf_corr;   /* prj_mhd_emf_send records, by wave */
    std::vector<int> flux_corr_begin; /* per wave offsets (+1 closing entry) */
    std::vector<int> emf_corr_begin;
    std::vector<int> active;        /* active block indices in mesh order */
    FxShard shard;                  /* sharded plans only */
};

#define FX_MAX_RANKS 16

/* The ghost-fill compiler's large working buffers (element versions and
 * fidelities, the recorded sequence and its per-thread parts, the wave
 * arrays, the cell-field operations per thread, the sort scratch), kept between
 * compiles: a later compile reuses their memory instead of faulting in
 * fresh pages, which is about a fifth of a compile of a few thousand
 * blocks.  Holds about 1.7 MB of host memory per MHD block entry of the
 * largest mesh compiled with it (4.1 GB for 2352 entries). */
struct FxPlanWorkspace;
FxPlanWorkspace *fx_plan_workspace_new();
void fx_plan_workspace_free(FxPlanWorkspace *ws);
/* hands a plan that is no longer used to the workspace: the next compile
 * writes its ghost-fill program into that plan's arrays */
void fx_plan_workspace_recycle(FxPlanWorkspace *ws, FxPlan &&old);

/* Builds the plan.  Returns false and sets *err for meshes the device path
 * does not handle (e.g. non-outflow field boundaries in an MHD run, which the
 * reference rejects too).  ws (may be null) lends the working buffers; the
 * plan is the same with or without it. */
bool fx_build_plan(const fx_config &cfg, int nblocks, const fx_block_desc *blocks,
    FxPlan &plan, std::string *err, FxPlanWorkspace *ws = nullptr);

/* The part of the single-device plan that rank `rank` of `nranks` runs when
 * owner[b] gives the rank of every block: the ghost-fill operations that
 * write its blocks and, transitively, the operations on other ranks' blocks
 * that produce what they read; the correction records likewise; renumbered
 * to the rank's local blocks, with the exchange lists (plan.shard).  Running
 * the parts on all ranks with the exchanges reproduces the single-device
 * plan's values on every owned block. */
bool fx_build_shard_plan(const fx_config &cfg, int nblocks, const fx_block_desc *blocks,
    const int *owner, int nranks, int rank, FxPlan &plan, std::string *err);

/* Only the coarse/fine flux and EMF correction records of the plan (fast:
 * no ghost-fill replay); the other members stay empty. */
bool fx_build_corrections(const fx_config &cfg, int nblocks, const fx_block_desc *blocks,
    FxPlan &plan, std::string *err);

#endif
