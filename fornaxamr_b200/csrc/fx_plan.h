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

struct FxPlan {
    FxProgram ghost;
    FxPlanStats stats;
    std::vector<FxCorr> flux_corr;  /* prj_riemann_flux_send records, by wave */
    std::vector<FxCorr> emf_corr;   /* prj_mhd_emf_send records, by wave */
    std::vector<int> flux_corr_begin; /* per wave offsets (+1 closing entry) */
    std::vector<int> emf_corr_begin;
    std::vector<int> active;        /* active block indices in mesh order */
};

/* Builds the plan.  Returns false and sets *err for meshes the device path
 * does not handle (e.g. non-outflow field boundaries in an MHD run, which the
 * reference rejects too). */
bool fx_build_plan(const fx_config &cfg, int nblocks, const fx_block_desc *blocks,
    FxPlan &plan, std::string *err);

/* Only the coarse/fine flux and EMF correction records of the plan (fast:
 * no ghost-fill replay); the other members stay empty. */
bool fx_build_corrections(const fx_config &cfg, int nblocks, const fx_block_desc *blocks,
    FxPlan &plan, std::string *err);

#endif
