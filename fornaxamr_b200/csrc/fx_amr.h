/*
 * Dynamic AMR: host half (block tree, 2:1 balance, neighbour slots) and the
 * device jobs it hands to the prolongation / restriction kernels.
 */
#ifndef FX_AMR_H
#define FX_AMR_H

#include <string>
#include <vector>

#include "../../include/fornax_b200.h"

/* One child created by prj_amr_refine_block (src/prj_amr.c:2389-2504).
 * copy_src[2 d + s]: the finer face neighbour of the parent whose face
 * layer the child copies onto its side s (0: index 0, 1: index 16) of
 * direction d before the divergence-free prolongation
 * (prj_amr_mhd_prolongate_bf_one, src/prj_amr.c:1981-2108), or -1. */
struct FxAmrRefine {
    int child;
    int parent;
    int oct;
    int copy_src[6];
};

/* One parent re-activated by prj_amr_coarsen_block (src/prj_amr.c:2506-2574). */
struct FxAmrCoarsen {
    int parent;
    int children[8];
};

struct FxAmrResult {
    bool changed = false;
    std::vector<fx_block_desc> blocks;   /* the adapted mesh */
    std::vector<FxAmrRefine> refine;     /* in creation order */
    std::vector<FxAmrCoarsen> coarsen;   /* in coarsening order */
    std::vector<int32_t> flags;          /* prj_amr_tag's refine_flag per input entry */
};

/* The block-tree half of prj_amr_adapt (src/prj_amr.c:2576-2706) for
 * per-block tag votes (pass 1 of prj_amr_tag: refine vote, derefine vote,
 * boundary side mask, three int32 per block).  Returns FX_SUCCESS or an
 * FX_E* code with *err set. */
int fx_amr_remesh(const fx_config &cfg, const fx_amr_config &amr, int nblocks,
    const fx_block_desc *blocks, const int32_t *votes, int capacity, FxAmrResult &res,
    std::string *err);

/* prj_neighbor_compute_geometry (src/prj_mesh.c:46-243): type, relative
 * level and send/recv boxes of neighbour b in slot s of block a; false when
 * the levels differ by more than one. */
bool fx_neighbor_geometry(const fx_block_desc &a, const fx_block_desc &b, fx_slot &s);

/* prj_amr_tag passes 2-4 (src/prj_amr.c:1707-1774) alone: refine_flag per
 * block from the pass-1 votes. */
void fx_amr_flags(const fx_amr_config &amr, int nblocks, const fx_block_desc *blocks,
    const int32_t *votes, int32_t *flags);

#endif
