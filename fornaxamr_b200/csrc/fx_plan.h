/*
 * Ghost-fill compiler: turns a mesh description into device programs.
 */
#ifndef FX_PLAN_H
#define FX_PLAN_H

#include <string>
#include <vector>

#include "../../include/fornax_b200.h"
#include "fx_kernels.h"

/* A program is a list of element operations grouped into waves.  Operations
 * inside one wave touch disjoint elements (no read/write or write/write
 * overlap), so a wave runs as one parallel kernel; waves run in order. */
struct FxProgram {
    std::vector<FxGop> ops;
    std::vector<int> wave_begin; /* ops of wave w are [wave_begin[w], wave_begin[w+1]) */
    int nwaves() const { return wave_begin.empty() ? 0 : (int)wave_begin.size() - 1; }
};

struct FxPlan {
    FxProgram cells;                /* W ghost cells (primitive vars except cell B) */
    FxProgram faces;                /* Bf ghost faces (MHD) */
    std::vector<FxCorr> flux_corr;  /* prj_riemann_flux_send records */
    std::vector<FxCorr> emf_corr;   /* prj_mhd_emf_send records */
    std::vector<int> active;        /* active block indices in mesh order */
};

/* Builds the plan.  Returns false and sets *err for meshes the device path
 * does not handle (e.g. non-outflow field boundaries in an MHD run, which the
 * reference rejects too). */
bool fx_build_plan(const fx_config &cfg, int nblocks, const fx_block_desc *blocks,
    FxPlan &plan, std::string *err);

#endif
