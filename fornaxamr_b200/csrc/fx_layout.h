/*
 * Per-block memory layout of the device mirror.
 *
 * The device keeps every block array in exactly the reference's per-block
 * layout so that offsets agree between a host prj_block and its device copy:
 *   - block geometry: BLOCK_SIZE=16 active cells, NGHOST=2, so 20 cells per
 *     axis with ghosts (reference src/prj_defs.h:383-388);
 *   - LIDX: untiled cell index, k fastest (src/prj_defs.h:392-393);
 *   - FACE_IDX / EDGE_IDX: staggered face and edge indices, one extra point
 *     along the staggered axis (src/prj_defs.h:394-405);
 *   - BIDX: AoSoA cell buffers [i][j][k/4][var][k%4] with lane width 4
 *     (src/prj_defs.h:419-434), used by flux, v_riemann, eosvar, rhs;
 *   - WIDX: primitives stage-major per variable, v*NSTAGES*NCELLS + cell
 *     (src/prj_defs.h:451-453).
 * These index formulas are the interface the drop-in must honour, so they
 * are restated here with the same meaning.  Blocks are stacked: block b's
 * array starts at base + b * per_block_count.
 */
#ifndef FX_LAYOUT_H
#define FX_LAYOUT_H

#ifdef __CUDACC__
#define FX_HD __host__ __device__ __forceinline__
#else
#define FX_HD static inline
#endif

#define FX_BS 16
#ifndef FX_NG
#define FX_NG 2                              /* 4 for the WENO-Z7 build (PRJ_NGHOST) */
#endif
#define FX_PBS (FX_BS + 2 * FX_NG)          /* 20 */
#define FX_NCELLS (FX_PBS * FX_PBS * FX_PBS) /* 8000 */
#define FX_NFACES ((FX_PBS + 1) * FX_PBS * FX_PBS) /* 8400 */
#define FX_NEDGES ((FX_PBS + 1) * (FX_PBS + 1) * FX_PBS) /* 8820 */
#define FX_NSTAGES 2
#define FX_AOSOA_W 4
#define FX_AOSOA_KT (FX_PBS / FX_AOSOA_W) /* 5 */
#define FX_NSLOTS 56
#define FX_MAXVAR 9

/* primitive / conserved variable slots (src/prj_defs.h:466-494) */
#define FX_RHO 0
#define FX_V1 1
#define FX_V2 2
#define FX_V3 3
#define FX_EINT 4
#define FX_ETOT 4
#define FX_YE 5
#define FX_B1 6
#define FX_B2 7
#define FX_B3 8

/* eosvar components */
#define FX_EOS_P 0
#define FX_EOS_T 1
#define FX_EOS_G 2

/* ideal-gas temperature scale of the reference's ideal EOS provider */
#define FX_IDEAL_ENERGY_SCALE 0.95655684e18

FX_HD int fx_lidx(int i, int j, int k)
{
    return ((i + FX_NG) * FX_PBS + (j + FX_NG)) * FX_PBS + (k + FX_NG);
}

FX_HD int fx_face_idx(int dir, int i, int j, int k)
{
    return dir == 0 ? ((i + FX_NG) * FX_PBS * FX_PBS + (j + FX_NG) * FX_PBS + (k + FX_NG))
         : dir == 1 ? ((i + FX_NG) * (FX_PBS + 1) * FX_PBS + (j + FX_NG) * FX_PBS + (k + FX_NG))
                    : ((i + FX_NG) * FX_PBS * (FX_PBS + 1) + (j + FX_NG) * (FX_PBS + 1) + (k + FX_NG));
}

FX_HD int fx_edge_idx(int dir, int i, int j, int k)
{
    return dir == 0 ? ((i + FX_NG) * (FX_PBS + 1) * (FX_PBS + 1) + (j + FX_NG) * (FX_PBS + 1) + (k + FX_NG))
         : dir == 1 ? ((i + FX_NG) * FX_PBS * (FX_PBS + 1) + (j + FX_NG) * (FX_PBS + 1) + (k + FX_NG))
                    : ((i + FX_NG) * (FX_PBS + 1) * FX_PBS + (j + FX_NG) * FX_PBS + (k + FX_NG));
}

/* AoSoA index of component v of an nc-component cell buffer */
FX_HD int fx_bidx(int nc, int v, int i, int j, int k)
{
    const int kk = k + FX_NG;
    return ((((i + FX_NG) * FX_PBS + (j + FX_NG)) * FX_AOSOA_KT + kk / FX_AOSOA_W) * nc + v) *
        FX_AOSOA_W + kk % FX_AOSOA_W;
}

/* same AoSoA index from an untiled cell index */
FX_HD int fx_bidx_cell(int nc, int v, int cell)
{
    const int row = cell / FX_PBS;
    const int kk = cell - row * FX_PBS;
    return ((row * FX_AOSOA_KT + kk / FX_AOSOA_W) * nc + v) * FX_AOSOA_W + kk % FX_AOSOA_W;
}

/* per-block element counts of the stacked device arrays */
#define FX_W_COUNT(nv) ((nv) * FX_NSTAGES * FX_NCELLS)
#define FX_BF_COUNT (3 * FX_NSTAGES * FX_NFACES)
#define FX_FLUX_COUNT(nv) (3 * (nv) * FX_NCELLS)
#define FX_VR_COUNT (3 * 3 * FX_NCELLS)
#define FX_BV_COUNT (3 * FX_NCELLS)
#define FX_EMF_COUNT (3 * FX_NEDGES)
#define FX_EOS_COUNT (3 * FX_NCELLS)
#define FX_RHS_COUNT(nv) ((nv) * FX_NCELLS)
#define FX_GRAV_COUNT (3 * FX_NCELLS)

#endif
