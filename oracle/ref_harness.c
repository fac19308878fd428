/*
 * Oracle harness around the reference FornaxAMR C core.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is compiled (by oracle/Makefile)
 * together with the reference's own unmodified sources into
 * oracle/_ref/libprjref_{mhd,hydro}.so.  Only tests/, the smoke check and the
 * CPU-baseline leg of bench.py load that library, and only as the checker or
 * the timed CPU reference; the product never links it.
 *
 * What it adds on top of the reference core:
 *   - the ideal-gas user EOS provider (the USER provider ABI of
 *     src/prj_eos.h:78-85) with a run-time adiabatic index; the arithmetic is
 *     the one of problems/prj_problem_ideal_eos.h:6-32;
 *   - problem set-ups for the workloads the GPU build is measured on (Sod tube,
 *     seeded Fourier-mode MHD, static-AMR magnetised blast, collapse profile),
 *     following the reference's own patterns: uniform root mesh from
 *     prj_mesh_init (src/prj_mesh.c:1438), ball-overlap static refinement as in
 *     problems/prj_problem_sedov.c:139-181, and B = curl A on faces as in
 *     src/prj_mhd.c:77-156, 1184-1231;
 *   - the driver's initialisation and step loop of src/main.c:354-562 without
 *     I/O;
 *   - accessors that expose block arrays and neighbour slots to ctypes, and
 *     thin wrappers around single reference kernels (HLLD, HLLC, MC slope,
 *     upwind EMF, prim<->cons) for golden-vector generation.
 */
#define _POSIX_C_SOURCE 199309L
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

#include "prj.h"

/* ------------------------------------------------------------------------ */
/* Ideal-gas user EOS provider with a run-time gamma.                        */
/* ------------------------------------------------------------------------ */

#define RH_IDEAL_ENERGY_SCALE 0.95655684e18

static double rh_gamma = 5.0 / 3.0;

void eos_rty(double rho, double temperature, double ye,
    double *eint, double *pressure, double *gamma, double *eta,
    double deint[3], double dpressure[3])
{
    const double g = rh_gamma;
    (void)ye;
    *eint = RH_IDEAL_ENERGY_SCALE * temperature / (g - 1.0);
    *pressure = rho * RH_IDEAL_ENERGY_SCALE * temperature;
    *gamma = g;
    *eta = 0.0;
    deint[0] = 0.0;
    deint[1] = RH_IDEAL_ENERGY_SCALE / (g - 1.0);
    deint[2] = 0.0;
    dpressure[0] = RH_IDEAL_ENERGY_SCALE * temperature;
    dpressure[1] = rho * RH_IDEAL_ENERGY_SCALE;
    dpressure[2] = 0.0;
}

void eos_rey(double rho, double eint, double ye,
    double *temperature, double *pressure, double *gamma)
{
    const double g = rh_gamma;
    (void)ye;
    *temperature = (g - 1.0) * eint / RH_IDEAL_ENERGY_SCALE;
    *pressure = (g - 1.0) * rho * eint;
    *gamma = g;
}

/* ------------------------------------------------------------------------ */
/* Parameters of a workload.                                                 */
/* ------------------------------------------------------------------------ */

enum {
    RH_CFG_SOD = 1,
    RH_CFG_FOURIER_MHD = 2,
    RH_CFG_AMR_BLAST = 3,
    RH_CFG_COLLAPSE = 4
};

typedef struct rh_params {
    int config;
    int root[3];
    int max_level;
    int max_blocks;
    double xmin[3];
    double xmax[3];
    double gamma;
    double cfl;
    double dt_factor;
    double t_end;
    /* Fourier-mode workload */
    int nmodes;
    int kmax;
    double amp_rho;
    double amp_v;
    double amp_A;
    unsigned long long seed_rho;
    unsigned long long seed_v;
    unsigned long long seed_A;
    /* static refinement: level L blocks overlapping the ball of radius
     * refine_radius[L] about center are refined (until max_level) */
    double center[3];
    double refine_radius[4];
    /* blast */
    double p_in;
    double p_out;
    double r_in;
    double B0[3];
    /* collapse */
    double rho_c;
    double r0;
    double K;
    double beta;
    double gm_point;
    int bc[6];          /* prj_bc_type per side: x1 inner, x1 outer, ..., x3 outer (0 outflow) */
} rh_params;

static prj_sim g_sim;
static prj_mpi g_mpi;
static rh_params g_par;
static int g_ready = 0;

/* ------------------------------------------------------------------------ */
/* Seeded mode sums (splitmix64, the generator of src/prj_perturbation.c:5-20)*/
/* ------------------------------------------------------------------------ */

static unsigned long long rh_splitmix64(unsigned long long *state)
{
    unsigned long long z;

    *state += 0x9E3779B97F4A7C15ULL;
    z = *state;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    return z ^ (z >> 31);
}

static double rh_uniform01(unsigned long long *state)
{
    return (double)(rh_splitmix64(state) >> 11) * (1.0 / 9007199254740992.0);
}

#define RH_MAX_MODES 64

typedef struct rh_modes {
    int n;
    double k[RH_MAX_MODES][3];
    double phase[RH_MAX_MODES];
    double dir[RH_MAX_MODES][3];
    double amp;
} rh_modes;

/* Draw n modes: integer wave vector with 1 <= |k|_inf <= kmax, phase in
 * [0, 2pi), unit direction; every mode carries amplitude amp_total / n. */
static void rh_draw_modes(rh_modes *m, int n, int kmax, double amp_total,
    unsigned long long seed)
{
    unsigned long long st = seed;
    int q;

    if (n > RH_MAX_MODES) {
        n = RH_MAX_MODES;
    }
    m->n = n;
    m->amp = n > 0 ? amp_total / (double)n : 0.0;
    for (q = 0; q < n; ++q) {
        int kx, ky, kz;
        double d0, d1, d2, dn;

        do {
            kx = (int)(rh_splitmix64(&st) % (unsigned long long)(2 * kmax + 1)) - kmax;
            ky = (int)(rh_splitmix64(&st) % (unsigned long long)(2 * kmax + 1)) - kmax;
            kz = (int)(rh_splitmix64(&st) % (unsigned long long)(2 * kmax + 1)) - kmax;
        } while (kx == 0 && ky == 0 && kz == 0);
        m->k[q][0] = (double)kx;
        m->k[q][1] = (double)ky;
        m->k[q][2] = (double)kz;
        m->phase[q] = 2.0 * M_PI * rh_uniform01(&st);
        do {
            d0 = rh_uniform01(&st) - 0.5;
            d1 = rh_uniform01(&st) - 0.5;
            d2 = rh_uniform01(&st) - 0.5;
            dn = sqrt(d0 * d0 + d1 * d1 + d2 * d2);
        } while (dn < 1.0e-3);
        m->dir[q][0] = d0 / dn;
        m->dir[q][1] = d1 / dn;
        m->dir[q][2] = d2 / dn;
    }
}

/* Scalar sum: sum_q amp * cos(2 pi k.x + phase). */
static double rh_mode_scalar(const rh_modes *m, double x, double y, double z)
{
    double s = 0.0;
    int q;

    for (q = 0; q < m->n; ++q) {
        double arg = 2.0 * M_PI * (m->k[q][0] * x + m->k[q][1] * y + m->k[q][2] * z) +
            m->phase[q];
        s += m->amp * cos(arg);
    }
    return s;
}

/* Vector sum: sum_q amp * cos(2 pi k.x + phase) * dir_q. */
static void rh_mode_vector(const rh_modes *m, double x, double y, double z, double out[3])
{
    int q;

    out[0] = 0.0;
    out[1] = 0.0;
    out[2] = 0.0;
    for (q = 0; q < m->n; ++q) {
        double arg = 2.0 * M_PI * (m->k[q][0] * x + m->k[q][1] * y + m->k[q][2] * z) +
            m->phase[q];
        double c = m->amp * cos(arg);
        out[0] += c * m->dir[q][0];
        out[1] += c * m->dir[q][1];
        out[2] += c * m->dir[q][2];
    }
}

/* ------------------------------------------------------------------------ */
/* Problem set-up                                                            */
/* ------------------------------------------------------------------------ */

static int rh_block_live(const prj_block *b)
{
    return b != 0 && b->id >= 0 && b->active == 1 && b->W_mhd != 0;
}

static void rh_store_prim(prj_block *b, int i, int j, int k, const double *w)
{
    double u[PRJ_NVAR_CONS];

    prj_block_store_prim_cell(b, 0, i, j, k, w);
    prj_block_store_prim_cell(b, 1, i, j, k, w);
    prj_eos_prim2cons(&g_sim.eos, (double *)w, u);
    prj_block_store_cons_cell(b, i, j, k, u);
}

static double rh_cell_x(const prj_block *b, int axis, int idx)
{
    return b->xmin[axis] + ((double)idx + 0.5) * b->dx[axis];
}

/* Same rule as problems/prj_problem_sedov.c:20-44. */
static int rh_block_overlaps_ball(const prj_block *block, const double c[3], double radius)
{
    double d[3] = {0.0, 0.0, 0.0};
    int a;

    if (block == 0 || block->id < 0 || block->active != 1) {
        return 0;
    }
    for (a = 0; a < 3; ++a) {
        if (block->xmin[a] > c[a]) {
            d[a] = block->xmin[a] - c[a];
        } else if (block->xmax[a] < c[a]) {
            d[a] = c[a] - block->xmax[a];
        }
    }
    return d[0] * d[0] + d[1] * d[1] + d[2] * d[2] < radius * radius;
}

static void rh_ensure_allocated(prj_mesh *mesh)
{
    int b;

    for (b = 0; b < mesh->nblocks; ++b) {
        prj_block *block = &mesh->blocks[b];

        if (block->id >= 0 && block->active == 1 && block->W_mhd == 0) {
            prj_block_alloc_data(block);
            prj_block_setup_geometry(block, &mesh->coord);
            prj_mesh_update_block_r_com(block, mesh);
        }
    }
}

/* Zero the state arrays of every allocated block.  Refinement prolongs the
 * parents' (not yet initialised) arrays into the children and checks them
 * for finite values; fresh heap memory is zero, recycled memory need not be,
 * so a second setup in one process would otherwise fail. */
static void rh_zero_state(prj_mesh *mesh)
{
    int b;

    for (b = 0; b < mesh->nblocks; ++b) {
        prj_block *block = &mesh->blocks[b];

        if (block->W_mhd == 0) {
            continue;
        }
        memset(block->W_mhd, 0, sizeof(double) * (size_t)PRJ_NVAR_MHD_PRIM * PRJ_BLOCK_NSTAGES *
            PRJ_BLOCK_NCELLS);
        if (block->eosvar != 0) {
            memset(block->eosvar, 0, sizeof(double) * (size_t)PRJ_NVAR_EOSVAR * PRJ_BLOCK_NCELLS);
        }
#if PRJ_MHD
        {
            int d;
            for (d = 0; d < 3; ++d) {
                if (block->Bf[d] != 0) {
                    memset(block->Bf[d], 0, sizeof(double) * (size_t)PRJ_BLOCK_NSTAGES * PRJ_BLOCK_NFACES);
                }
            }
        }
#endif
    }
}

/* Static refinement in the pattern of problems/prj_problem_sedov.c:139-181. */
static void rh_static_refine(void)
{
    int level;

    for (level = 0; level < g_sim.mesh.max_level; ++level) {
        int b;
        int any = 0;

        rh_zero_state(&g_sim.mesh);

        for (b = 0; b < g_sim.mesh.nblocks; ++b) {
            prj_block *block = &g_sim.mesh.blocks[b];

            if (block->id < 0 || block->active != 1 || block->level != level) {
                continue;
            }
            block->refine_flag = 0;
            if (rh_block_overlaps_ball(block, g_par.center, g_par.refine_radius[level])) {
                block->refine_flag = 1;
                any = 1;
            }
        }
        if (!any) {
            break;
        }
        prj_amr_enforce_two_to_one(&g_sim.mesh, &g_mpi);
        if (prj_amr_refine_marked_blocks(&g_sim.mesh, &g_mpi) == 0) {
            break;
        }
        prj_amr_init_neighbors(&g_sim.mesh);
        rh_ensure_allocated(&g_sim.mesh);
    }
    prj_mesh_update_max_active_level(&g_sim.mesh);
}

#if PRJ_MHD
typedef void (*rh_apot_fn)(double x, double y, double z, double A[3]);

static rh_modes g_modes_A;

static void rh_apot_modes(double x, double y, double z, double A[3])
{
    rh_mode_vector(&g_modes_A, x, y, z, A);
}

/* A = (0, 0, Bx*y - By*x) gives the uniform field B = (Bx, By, 0). */
static void rh_apot_uniform(double x, double y, double z, double A[3])
{
    (void)z;
    A[0] = 0.0;
    A[1] = 0.0;
    A[2] = g_par.B0[0] * y - g_par.B0[1] * x;
}

/* Weak dipole-like loop: A_phi = B0 * r0^3 * R / (r^2 + r0^2)^1.5 with
 * R = sqrt(x^2 + y^2) (so A_phi proportional to r sin(theta)/(r^2+r0^2)^1.5),
 * written in Cartesian components A = A_phi * (-y/R, x/R, 0). */
static void rh_apot_dipole(double x, double y, double z, double A[3])
{
    double r2 = x * x + y * y + z * z;
    double s = r2 + g_par.r0 * g_par.r0;
    double f = g_par.B0[0] * g_par.r0 * g_par.r0 * g_par.r0 / (s * sqrt(s));

    A[0] = -y * f;
    A[1] = x * f;
    A[2] = 0.0;
}

/* Edge coordinate rule of src/prj_mhd.c:43-48. */
static double rh_edge_coord(const prj_block *block, int axis, int component, int index)
{
    double offset = axis == component ? 0.5 : 0.0;

    return block->xmin[axis] + ((double)index + offset) * block->dx[axis];
}

/* B = curl A on faces.  A is stored on edges, restricted on coarse/fine edges
 * by the reference's own prj_mhd_emf_send, and differenced with the discrete
 * curl of src/prj_mhd.c:106-142; then Bf is copied to the second stage slot
 * and the cell-centred B is rebuilt (src/prj_mhd.c:1184-1231). */
static void rh_init_bfield(rh_apot_fn apot)
{
    int b;

    for (b = 0; b < g_sim.mesh.nblocks; ++b) {
        prj_block *block = &g_sim.mesh.blocks[b];
        int d, i, j, k;

        if (!rh_block_live(block)) {
            continue;
        }
        for (d = 0; d < 3; ++d) {
            prj_fill(block->emf[d], (size_t)PRJ_BLOCK_NEDGES, 0.0);
        }
        for (i = -PRJ_NGHOST; i < PRJ_BLOCK_SIZE + PRJ_NGHOST; ++i) {
            for (j = -PRJ_NGHOST; j < PRJ_BLOCK_SIZE + PRJ_NGHOST; ++j) {
                for (k = -PRJ_NGHOST; k < PRJ_BLOCK_SIZE + PRJ_NGHOST; ++k) {
                    for (d = 0; d < 3; ++d) {
                        double A[3];

                        apot(rh_edge_coord(block, X1DIR, d, i),
                            rh_edge_coord(block, X2DIR, d, j),
                            rh_edge_coord(block, X3DIR, d, k), A);
                        block->emf[d][EDGE_IDX(d, i, j, k)] = A[d];
                    }
                }
            }
        }
    }
    prj_mhd_emf_send(&g_sim.mesh, &g_mpi);
    for (b = 0; b < g_sim.mesh.nblocks; ++b) {
        prj_block *block = &g_sim.mesh.blocks[b];
        const int lo = -PRJ_NGHOST;
        const int hi = PRJ_BLOCK_SIZE + PRJ_NGHOST - 1;
        int d, i, j, k, n;

        if (!rh_block_live(block)) {
            continue;
        }
        for (d = 0; d < 3; ++d) {
            prj_fill(block->Bf[d], (size_t)PRJ_BLOCK_NFACES, 0.0);
        }
        for (i = lo; i < hi; ++i) {
            for (j = lo; j < hi; ++j) {
                for (k = lo; k < hi; ++k) {
                    double *e1 = block->emf[X1DIR];
                    double *e2 = block->emf[X2DIR];
                    double *e3 = block->emf[X3DIR];
                    double B1 = (e3[EDGE_IDX(X3DIR, i, j + 1, k)] - e3[EDGE_IDX(X3DIR, i, j, k)]) / block->dx[1] -
                        (e2[EDGE_IDX(X2DIR, i, j, k + 1)] - e2[EDGE_IDX(X2DIR, i, j, k)]) / block->dx[2];
                    double B2 = (e1[EDGE_IDX(X1DIR, i, j, k + 1)] - e1[EDGE_IDX(X1DIR, i, j, k)]) / block->dx[2] -
                        (e3[EDGE_IDX(X3DIR, i + 1, j, k)] - e3[EDGE_IDX(X3DIR, i, j, k)]) / block->dx[0];
                    double B3 = (e2[EDGE_IDX(X2DIR, i + 1, j, k)] - e2[EDGE_IDX(X2DIR, i, j, k)]) / block->dx[0] -
                        (e1[EDGE_IDX(X1DIR, i, j + 1, k)] - e1[EDGE_IDX(X1DIR, i, j, k)]) / block->dx[1];

                    block->Bf[X1DIR][FACE_IDX(X1DIR, i, j, k)] = B1;
                    block->Bf[X2DIR][FACE_IDX(X2DIR, i, j, k)] = B2;
                    block->Bf[X3DIR][FACE_IDX(X3DIR, i, j, k)] = B3;
                }
            }
        }
        for (d = 0; d < 3; ++d) {
            double *bf1 = prj_block_bf_stage(block, d, 1);

            for (n = 0; n < PRJ_BLOCK_NFACES; ++n) {
                bf1[n] = block->Bf[d][n];
            }
            prj_fill(block->emf[d], (size_t)PRJ_BLOCK_NEDGES, 0.0);
        }
        prj_mhd_bf2bc_all_mesh(&g_sim.eos, &g_sim.mesh, block, 0);
        prj_mhd_bf2bc_all_mesh(&g_sim.eos, &g_sim.mesh, block, 1);
    }
}
#endif

static void rh_fill_prims(void (*cell)(const prj_block *, int, int, int, double *))
{
    int b;

    for (b = 0; b < g_sim.mesh.nblocks; ++b) {
        prj_block *block = &g_sim.mesh.blocks[b];
        int i, j, k;

        if (!rh_block_live(block)) {
            continue;
        }
        for (i = -PRJ_NGHOST; i < PRJ_BLOCK_SIZE + PRJ_NGHOST; ++i) {
            for (j = -PRJ_NGHOST; j < PRJ_BLOCK_SIZE + PRJ_NGHOST; ++j) {
                for (k = -PRJ_NGHOST; k < PRJ_BLOCK_SIZE + PRJ_NGHOST; ++k) {
                    double w[PRJ_NVAR_PRIM];
                    int v;

                    for (v = 0; v < PRJ_NVAR_PRIM; ++v) {
                        w[v] = 0.0;
                    }
                    cell(block, i, j, k, w);
                    rh_store_prim(block, i, j, k, w);
                }
            }
        }
    }
}

static void rh_cell_sod(const prj_block *b, int i, int j, int k, double *w)
{
    double x = rh_cell_x(b, 0, i);
    double rho = x < 0.5 ? 1.0 : 0.125;
    double p = x < 0.5 ? 1.0 : 0.1;

    (void)j;
    (void)k;
    w[PRJ_PRIM_RHO] = rho;
    w[PRJ_PRIM_EINT] = p / ((g_par.gamma - 1.0) * rho);
    w[PRJ_PRIM_YE] = 0.1;
}

static rh_modes g_modes_rho;
static rh_modes g_modes_v;

static void rh_cell_fourier(const prj_block *b, int i, int j, int k, double *w)
{
    double x = rh_cell_x(b, 0, i);
    double y = rh_cell_x(b, 1, j);
    double z = rh_cell_x(b, 2, k);
    double v[3];
    double rho = 1.0 + rh_mode_scalar(&g_modes_rho, x, y, z);

    rh_mode_vector(&g_modes_v, x, y, z, v);
    w[PRJ_PRIM_RHO] = rho;
    w[PRJ_PRIM_V1] = v[0];
    w[PRJ_PRIM_V2] = v[1];
    w[PRJ_PRIM_V3] = v[2];
    w[PRJ_PRIM_EINT] = 1.0 / ((g_par.gamma - 1.0) * rho);
    w[PRJ_PRIM_YE] = 0.1;
}

static void rh_cell_blast(const prj_block *b, int i, int j, int k, double *w)
{
    double x = rh_cell_x(b, 0, i) - g_par.center[0];
    double y = rh_cell_x(b, 1, j) - g_par.center[1];
    double z = rh_cell_x(b, 2, k) - g_par.center[2];
    double r = sqrt(x * x + y * y + z * z);
    double p = r < g_par.r_in ? g_par.p_in : g_par.p_out;

    w[PRJ_PRIM_RHO] = 1.0;
    w[PRJ_PRIM_EINT] = p / ((g_par.gamma - 1.0) * 1.0);
    w[PRJ_PRIM_YE] = 0.1;
}

static void rh_cell_collapse(const prj_block *b, int i, int j, int k, double *w)
{
    double x = rh_cell_x(b, 0, i);
    double y = rh_cell_x(b, 1, j);
    double z = rh_cell_x(b, 2, k);
    double r = sqrt(x * x + y * y + z * z);
    double q = r / g_par.r0;
    double s = 1.0 + q * q;
    double rho = g_par.rho_c / (s * sqrt(s));
    double p = g_par.K * pow(rho, g_par.gamma);
    double cs = sqrt(g_par.gamma * p / rho);
    double vr = -0.1 * cs * r / (r + g_par.r0);
    double inv_r = r > 0.0 ? 1.0 / r : 0.0;

    w[PRJ_PRIM_RHO] = rho;
    w[PRJ_PRIM_V1] = vr * x * inv_r;
    w[PRJ_PRIM_V2] = vr * y * inv_r;
    w[PRJ_PRIM_V3] = vr * z * inv_r;
    w[PRJ_PRIM_EINT] = p / ((g_par.gamma - 1.0) * rho);
    w[PRJ_PRIM_YE] = 0.1;
}

/* Static gravitational acceleration g = -G M(<r) x / r^3 with a point mass
 * plus the enclosed mass of the profile rho_c/(1+(r/r0)^2)^1.5, written once
 * into block->grav (the reference's src term reads it each stage,
 * src/prj_src.c:32-139). */
static void rh_fill_gravity(void)
{
    int b;

    for (b = 0; b < g_sim.mesh.nblocks; ++b) {
        prj_block *block = &g_sim.mesh.blocks[b];
        int i, j, k;

        if (!rh_block_live(block)) {
            continue;
        }
        for (i = -PRJ_NGHOST; i < PRJ_BLOCK_SIZE + PRJ_NGHOST; ++i) {
            for (j = -PRJ_NGHOST; j < PRJ_BLOCK_SIZE + PRJ_NGHOST; ++j) {
                for (k = -PRJ_NGHOST; k < PRJ_BLOCK_SIZE + PRJ_NGHOST; ++k) {
                    double x = rh_cell_x(block, 0, i);
                    double y = rh_cell_x(block, 1, j);
                    double z = rh_cell_x(block, 2, k);
                    double r = sqrt(x * x + y * y + z * z);
                    double a = r / g_par.r0;
                    /* enclosed mass of rho_c (1 + a^2)^-1.5: 4 pi rho_c r0^3 (asinh(a) - a / sqrt(1 + a^2)) */
                    double menc = 4.0 * M_PI * g_par.rho_c * g_par.r0 * g_par.r0 * g_par.r0 *
                        (asinh(a) - a / sqrt(1.0 + a * a));
                    double gmag = r > 0.0 ? -(g_par.gm_point + menc) / (r * r * r) : 0.0;
                    int idx = IDX(i, j, k);

                    block->grav[0][idx] = gmag * x;
                    block->grav[1][idx] = gmag * y;
                    block->grav[2][idx] = gmag * z;
                }
            }
        }
    }
}

static void rh_set_defaults(void)
{
    int a;

    memset(&g_sim, 0, sizeof(g_sim));
    g_sim.coord.x1min = g_par.xmin[0];
    g_sim.coord.x1max = g_par.xmax[0];
    g_sim.coord.x2min = g_par.xmin[1];
    g_sim.coord.x2max = g_par.xmax[1];
    g_sim.coord.x3min = g_par.xmin[2];
    g_sim.coord.x3max = g_par.xmax[2];
    g_sim.bc.bc_x1_inner = g_par.bc[0];
    g_sim.bc.bc_x1_outer = g_par.bc[1];
    g_sim.bc.bc_x2_inner = g_par.bc[2];
    g_sim.bc.bc_x2_outer = g_par.bc[3];
    g_sim.bc.bc_x3_inner = g_par.bc[4];
    g_sim.bc.bc_x3_outer = g_par.bc[5];
    g_sim.cfl = g_par.cfl;
    g_sim.dt_factor = g_par.dt_factor;
    g_sim.t_end = g_par.t_end;
    g_sim.output_dt = -1.0;
    g_sim.restart_dt = -1.0;
    g_sim.dt_gw = -1.0;
    g_sim.max_steps = 1000000000;
    g_sim.amr_interval = -1;
    g_sim.grav.use_multipole_gravity = 0;
    for (a = 0; a < 3; ++a) {
        g_sim.mesh.root_nx[a] = g_par.root[a];
        g_sim.mesh.periodic[a] = 0;
    }
    g_sim.mesh.max_level = g_par.max_level;
    g_sim.mesh.max_blocks = g_par.max_blocks > 0 ? g_par.max_blocks :
        g_par.root[0] * g_par.root[1] * g_par.root[2];
    g_sim.mesh.use_BJ = 0;
    g_sim.mesh.E_floor = -1.0;
    g_sim.mesh.mhd_eta = 0.0;
    g_sim.mesh.amr_init_scale_factor = 0.5;
    g_sim.mesh.amr_reach_highest_level_at_density = -1.0;
    g_sim.eos.kind = PRJ_EOS_KIND_IDEAL;
#if PRJ_MHD
    g_sim.mhd_init_type = PRJ_MHD_INIT_UNIFORM;
    g_sim.mhd_B_norm = 0.0;
    g_sim.mhd_B_scale = 1.0;
#endif
}

void rh_teardown(void)
{
    if (g_ready) {
        prj_mesh_destroy(&g_sim.mesh);
        g_ready = 0;
    }
}

/* Build the workload and run the driver's initialisation
 * (src/main.c:359-448 minus I/O and gravity solver). Returns 0 on success. */
int rh_setup(const rh_params *p)
{
    if (p == 0) {
        return 1;
    }
    rh_teardown();
    g_par = *p;
    rh_gamma = p->gamma;
    rh_set_defaults();
    prj_mpi_init(0, 0, &g_mpi);
    prj_timeint_init(&PRJ_TIMEINT_TABLEAU_NAME);
    prj_eos_init(&g_sim.eos, &g_mpi);
    if (prj_mesh_init(&g_sim.mesh, p->root[0], p->root[1], p->root[2],
            p->max_level, &g_sim.coord, 0) != 0) {
        return 2;
    }
    if (p->max_level > 0) {
        rh_static_refine();
    }
    switch (p->config) {
    case RH_CFG_SOD:
        rh_fill_prims(rh_cell_sod);
        break;
    case RH_CFG_FOURIER_MHD:
        rh_draw_modes(&g_modes_rho, p->nmodes, p->kmax, p->amp_rho, p->seed_rho);
        rh_draw_modes(&g_modes_v, p->nmodes, p->kmax, p->amp_v, p->seed_v);
        rh_fill_prims(rh_cell_fourier);
#if PRJ_MHD
        rh_draw_modes(&g_modes_A, p->nmodes, p->kmax, p->amp_A, p->seed_A);
        rh_init_bfield(rh_apot_modes);
#endif
        break;
    case RH_CFG_AMR_BLAST:
        rh_fill_prims(rh_cell_blast);
#if PRJ_MHD
        rh_init_bfield(rh_apot_uniform);
#endif
        break;
    case RH_CFG_COLLAPSE:
        rh_fill_prims(rh_cell_collapse);
        rh_fill_gravity();
#if PRJ_MHD
        rh_init_bfield(rh_apot_dipole);
#endif
        break;
    default:
        return 3;
    }
    prj_mpi_decompose(&g_sim.mesh, &g_mpi);
    prj_mpi_prepare(&g_sim.mesh, &g_mpi);
    prj_eos_fill_active_cells(&g_sim.mesh, &g_sim.eos, &g_mpi, 1, PRJ_EOS_CTX_MAIN);
    g_sim.mesh.time_seconds = g_sim.time;
    prj_boundary_fill_ghosts_and_bf(&g_sim.mesh, &g_mpi, &g_sim.bc, 1, 0, &g_sim.eos, 0,
        &g_sim.rad, PRJ_BOUNDARY_TIMER_SCOPE_NONE);
    prj_eos_fill_mesh(&g_sim.mesh, &g_sim.eos, &g_mpi, 1, PRJ_EOS_CTX_MAIN);
    g_sim.time = 0.0;
    g_sim.dt = 0.0;
    g_sim.step = 0;
    g_ready = 1;
    return 0;
}

/* ------------------------------------------------------------------------ */
/* Stepping                                                                  */
/* ------------------------------------------------------------------------ */

double rh_calc_dt(void)
{
    return prj_timeint_calc_dt(&g_sim.mesh, &g_sim.eos, &g_sim.rad, &g_mpi, g_sim.cfl,
        &PRJ_TIMEINT_TABLEAU_NAME);
}

/* One RK2 step with a given dt (prj_timeint_step, src/prj_timeint.c:3221). */
void rh_step(double dt, double *dt_src)
{
    double local = 1.0e100;

    g_sim.mesh.time_seconds = g_sim.time;
    prj_timeint_step(&g_sim.mesh, &g_sim.coord, &g_sim.bc, &g_sim.eos, &g_sim.rad,
        &g_sim.grav, &g_mpi, &PRJ_TIMEINT_TABLEAU_NAME, dt, &local, 0);
    if (dt_src != 0) {
        *dt_src = prj_mpi_min_dt(&g_mpi, local);
    }
}

/* Single stages, for stage-level comparisons. */
void rh_stage(int which, double dt, double *dt_src)
{
    double local = 1.0e100;

    if (which == 1) {
        prj_timeint_stage1(&g_sim.mesh, &g_sim.coord, &g_sim.bc, &g_sim.eos, &g_sim.rad,
            &g_sim.grav, &g_mpi, dt, &local, 0);
    } else {
        prj_timeint_stage2(&g_sim.mesh, &g_sim.coord, &g_sim.bc, &g_sim.eos, &g_sim.rad,
            &g_sim.grav, &g_mpi, dt, &local, 0);
    }
    if (dt_src != 0) {
        *dt_src = local;
    }
}

/* The driver loop of src/main.c:485-562 (no output, no AMR adapt).
 * state[0..2] = time, dt, step on return.  Runs at most nsteps steps. */
int rh_run(int nsteps, double *state)
{
    int n = 0;

    while (g_sim.time < g_sim.t_end && n < nsteps) {
        double dt_new = rh_calc_dt();
        double dt_step;
        double dt_src = 1.0e100;

        if (g_sim.dt > 0.0) {
            double dt_limit = g_sim.dt_factor * g_sim.dt;

            g_sim.dt = dt_new <= dt_limit ? dt_new : dt_limit;
        } else {
            g_sim.dt = dt_new;
        }
        dt_step = g_sim.dt;
        if (g_sim.time + dt_step > g_sim.t_end) {
            dt_step = g_sim.t_end - g_sim.time;
        }
        rh_step(dt_step, &dt_src);
        if (g_sim.cfl * dt_src < g_sim.dt) {
            g_sim.dt = g_sim.cfl * dt_src;
        }
        g_sim.time += dt_step;
        g_sim.step += 1;
        n += 1;
    }
    if (state != 0) {
        state[0] = g_sim.time;
        state[1] = g_sim.dt;
        state[2] = (double)g_sim.step;
    }
    return n;
}

/* Wall time of n plain steps at a fixed dt (CPU baseline timing). */
double rh_time_steps(int nsteps, double dt)
{
    struct timespec t0, t1;
    int n;

    clock_gettime(CLOCK_MONOTONIC, &t0);
    for (n = 0; n < nsteps; ++n) {
        rh_step(dt, 0);
    }
    clock_gettime(CLOCK_MONOTONIC, &t1);
    return (double)(t1.tv_sec - t0.tv_sec) + 1.0e-9 * (double)(t1.tv_nsec - t0.tv_nsec);
}

/* ------------------------------------------------------------------------ */
/* Accessors                                                                 */
/* ------------------------------------------------------------------------ */

int rh_nblocks(void) { return g_ready ? g_sim.mesh.nblocks : 0; }
int rh_nhydro(void) { return PRJ_NHYDRO; }
int rh_block_size(void) { return PRJ_BLOCK_SIZE; }
int rh_nghost(void) { return PRJ_NGHOST; }
int rh_aosoa_w(void) { return PRJ_AOSOA_W; }
int rh_nstages(void) { return PRJ_BLOCK_NSTAGES; }
double rh_sim_time(void) { return g_sim.time; }
double rh_sim_dt(void) { return g_sim.dt; }

/* ints[0..3] = id, level, active, rank; dbl[0..12] = xmin[3], xmax[3], dx[3], vol, area[3] */
int rh_block_geom(int b, int *ints, double *dbl)
{
    const prj_block *block;
    int a;

    if (!g_ready || b < 0 || b >= g_sim.mesh.nblocks) {
        return 1;
    }
    block = &g_sim.mesh.blocks[b];
    ints[0] = block->id;
    ints[1] = block->level;
    ints[2] = block->active;
    ints[3] = block->rank;
    for (a = 0; a < 3; ++a) {
        dbl[a] = block->xmin[a];
        dbl[3 + a] = block->xmax[a];
        dbl[6 + a] = block->dx[a];
        dbl[10 + a] = block->area[a];
    }
    dbl[9] = block->vol;
    return 0;
}

/* 56 slots x 15 ints: id, rel_level, type, send_start[3], send_end[3], recv_start[3], recv_end[3] */
int rh_block_slots(int b, int *out)
{
    const prj_block *block;
    int n, a;

    if (!g_ready || b < 0 || b >= g_sim.mesh.nblocks) {
        return 1;
    }
    block = &g_sim.mesh.blocks[b];
    for (n = 0; n < 56; ++n) {
        const prj_neighbor *s = &block->slot[n];
        int *o = &out[n * 15];

        o[0] = s->id;
        o[1] = s->rel_level;
        o[2] = s->type;
        for (a = 0; a < 3; ++a) {
            o[3 + a] = s->send_loc_start[a];
            o[6 + a] = s->send_loc_end[a];
            o[9 + a] = s->recv_loc_start[a];
            o[12 + a] = s->recv_loc_end[a];
        }
    }
    return 0;
}

enum {
    RH_ARR_W = 0,
    RH_ARR_EOSVAR = 1,
    RH_ARR_U = 2,
    RH_ARR_RHS = 3,
    RH_ARR_FLUX = 4,
    RH_ARR_VRIEMANN = 5,
    RH_ARR_GRAV = 6,
    RH_ARR_BF = 7,
    RH_ARR_BV1 = 8,
    RH_ARR_BV2 = 9,
    RH_ARR_EMF = 10
};

/* Raw pointer to a block array (the reference's per-block layout); NULL when
 * the array does not exist in this build. */
double *rh_block_array(int b, int which, int dir)
{
    prj_block *block;

    if (!g_ready || b < 0 || b >= g_sim.mesh.nblocks || dir < 0 || dir > 2) {
        return 0;
    }
    block = &g_sim.mesh.blocks[b];
    switch (which) {
    case RH_ARR_W: return block->W_mhd;
    case RH_ARR_EOSVAR: return block->eosvar;
    case RH_ARR_U: return block->U_mhd;
    case RH_ARR_RHS: return block->mhd_rhs;
    case RH_ARR_FLUX: return block->flux[dir];
    case RH_ARR_VRIEMANN: return block->v_riemann[dir];
    case RH_ARR_GRAV: return block->grav[dir];
#if PRJ_MHD
    case RH_ARR_BF: return block->Bf[dir];
    case RH_ARR_BV1: return block->Bv1[dir];
    case RH_ARR_BV2: return block->Bv2[dir];
    case RH_ARR_EMF: return block->emf[dir];
#endif
    default: return 0;
    }
}

/* The reference's ghost fill followed by its eos fill of the mesh
 * (src/prj_timeint.c:2829-2834 with stage arguments). */
void rh_fill_ghosts(int stage, int use_bf1)
{
    prj_boundary_fill_ghosts_and_bf(&g_sim.mesh, &g_mpi, &g_sim.bc, stage, use_bf1, &g_sim.eos, 0,
        &g_sim.rad, PRJ_BOUNDARY_TIMER_SCOPE_NONE);
    prj_eos_fill_mesh(&g_sim.mesh, &g_sim.eos, &g_mpi, stage, PRJ_EOS_CTX_MAIN);
}

/* Run-time resistivity of the mesh (prj_mesh.mhd_eta, src/prj_types.h:497),
 * which the EMF update adds to the artificial eta of each edge
 * (src/prj_timeint.c:404-408, 525). */
void rh_set_mhd_eta(double eta)
{
    g_sim.mesh.mhd_eta = eta;
}

/* prj_mesh.use_BJ (the prolongation limiter of the ghost fill and of
 * prj_amr_adapt); kept by rh_amr_configure, reset by rh_setup */
void rh_set_use_bj(int on)
{
    g_sim.mesh.use_BJ = on != 0;
}

/* The driver's set-up refill (src/main.c:437-448) after the caller has
 * rewritten stage-0 cells or faces: eos of the active cells, ghost fill
 * with the cell field from the faces, eos of the whole mesh. */
void rh_refill(void)
{
    prj_eos_fill_active_cells(&g_sim.mesh, &g_sim.eos, &g_mpi, 1, PRJ_EOS_CTX_MAIN);
    prj_boundary_fill_ghosts_and_bf(&g_sim.mesh, &g_mpi, &g_sim.bc, 1, 0, &g_sim.eos, 0,
        &g_sim.rad, PRJ_BOUNDARY_TIMER_SCOPE_NONE);
    prj_eos_fill_mesh(&g_sim.mesh, &g_sim.eos, &g_mpi, 1, PRJ_EOS_CTX_MAIN);
}

#ifdef PRJ_FX_WRAP
/* The drop-in build: refresh the host arrays from the device (resident mode). */
#include "prj_fx.h"
void rh_dropin_to_host(void)
{
    prj_fx_to_host(&g_sim.mesh);
}
#endif

/* The coarse/fine corrections of a stage (src/prj_timeint.c:2750, 528). */
void rh_flux_send(void)
{
    prj_riemann_flux_send(&g_sim.mesh, &g_mpi);
}

void rh_emf_send(void)
{
#if PRJ_MHD
    prj_mhd_emf_send(&g_sim.mesh, &g_mpi);
#endif
}

/* Per-block reference phases, for phase-level parity tests. */
void rh_flux_update(int b, int w_slot, int use_bf1)
{
    prj_block *block = &g_sim.mesh.blocks[b];

    prj_flux_update(&g_sim.eos, &g_sim.rad, &g_sim.mesh, block,
        prj_block_prim_stage(block, w_slot), block->eosvar, block->flux, use_bf1);
}

/* ------------------------------------------------------------------------ */
/* Single-kernel wrappers for golden vectors                                 */
/* ------------------------------------------------------------------------ */

double rh_mc_slope(double qm, double q0, double qp)
{
    return prj_reconstruct_mc_face_slope(qm, q0, qp);
}

#if PRJ_MHD
/* out[0..8] flux, out[9..11] v_face, out[12] Bv1, out[13] Bv2 */
void rh_hlld(const double *WL, const double *WR, double pL, double pR,
    double gL, double gR, double bn, double *out)
{
    double wl[PRJ_NVAR_PRIM];
    double wr[PRJ_NVAR_PRIM];
    int v;

    for (v = 0; v < PRJ_NVAR_PRIM; ++v) {
        wl[v] = WL[v];
        wr[v] = WR[v];
    }
    wl[PRJ_PRIM_B1] = bn;
    wr[PRJ_PRIM_B1] = bn;
    prj_riemann_hlld(wl, wr, pL, pR, gL, gR, &g_sim.eos, bn, out, &out[9],
        &out[12], &out[13], 0.0, 0.0, 0.0);
}

static double rh_emf_store[3][PRJ_BLOCK_NEDGES];

double rh_emf_upwind(const double *face, const double *cell, const double *vn)
{
    prj_block blk;

    memset(&blk, 0, sizeof(blk));
    blk.emf[0] = rh_emf_store[0];
    blk.emf[1] = rh_emf_store[1];
    blk.emf[2] = rh_emf_store[2];
    blk.dx[0] = blk.dx[1] = blk.dx[2] = 1.0;
    return prj_mhd_emf_upwind(&blk, 0, 0, 0, 0, face, cell, vn, 0, 0.0);
}
#endif

/* out[0..NHYDRO-1] flux, out[NHYDRO..NHYDRO+2] v_face */
void rh_hllc(const double *WL, const double *WR, double pL, double pR,
    double gL, double gR, double du, double dv, double dw, double *out)
{
    prj_riemann_hllc(WL, WR, pL, pR, gL, gR, &g_sim.eos, out, &out[PRJ_NHYDRO], du, dv, dw);
}

void rh_prim2cons(const double *w, double *u)
{
    prj_eos_prim2cons(&g_sim.eos, (double *)w, u);
}

void rh_cons2prim(const double *u, double *w)
{
    prj_eos_cons2prim(&g_sim.eos, (double *)u, w);
}

void rh_set_gamma(double g)
{
    rh_gamma = g;
}

/* eos_quantities of prj_eos_rey (src/prj_eos.c:772): [T, p, gamma] */
void rh_eos_rey(double rho, double eint, double ye, double *out)
{
    double q[PRJ_EOS_NQUANT];

    prj_eos_rey(&g_sim.eos, rho, eint, ye, q, PRJ_EOS_CTX_MAIN);
    out[0] = q[PRJ_EOS_TEMPERATURE];
    out[1] = q[PRJ_EOS_PRESSURE];
    out[2] = q[PRJ_EOS_GAMMA];
}

/* ------------------------------------------------------------------------ */
/* Dynamic AMR (src/prj_amr.c) driven the way src/main.c:565-607 drives it.   */
/* ------------------------------------------------------------------------ */

typedef struct rh_amr {
    int max_level;
    double min_dx;
    double reach_density;   /* amr_reach_highest_level_at_density */
    double E_floor;
    int set[PRJ_AMR_N];
    int estimator[PRJ_AMR_N];
    int lohner_var[PRJ_AMR_N];
    int jump_var[PRJ_AMR_N];
    double refine_thresh[PRJ_AMR_N];
    double derefine_thresh[PRJ_AMR_N];
    double lohner_eps[PRJ_AMR_N];
} rh_amr;

int rh_amr_n(void) { return PRJ_AMR_N; }

void rh_amr_configure(const rh_amr *a)
{
    int n;

    g_sim.mesh.max_level = a->max_level;
    g_sim.mesh.min_dx = a->min_dx;
    g_sim.mesh.amr_reach_highest_level_at_density = a->reach_density;
    g_sim.mesh.E_floor = a->E_floor;
    g_sim.mesh.use_amr_angular_resolution_limit = 0;
    g_sim.mesh.amr_init_refine_fn = 0;
    for (n = 0; n < PRJ_AMR_N; ++n) {
        g_sim.mesh.amr_criterion_set[n] = a->set[n];
        g_sim.mesh.amr_estimator[n] = a->estimator[n];
        g_sim.mesh.amr_lohner_var[n] = a->lohner_var[n];
        g_sim.mesh.amr_fractional_jump_var[n] = a->jump_var[n];
        g_sim.mesh.amr_refine_thresh[n] = a->refine_thresh[n];
        g_sim.mesh.amr_derefine_thresh[n] = a->derefine_thresh[n];
        g_sim.mesh.amr_lohner_eps[n] = a->lohner_eps[n];
    }
}

/* prj_amr_tag alone: flags[b] = refine_flag of every block afterwards (the
 * votes after the caps, before 2:1 balance).  The flags are cleared again. */
void rh_amr_tag(int *flags)
{
    int b;

    prj_amr_tag(&g_sim.mesh, &g_sim.eos, &g_mpi);
    for (b = 0; b < g_sim.mesh.nblocks; ++b) {
        flags[b] = g_sim.mesh.blocks[b].refine_flag;
        if (g_sim.mesh.blocks[b].id >= 0) {
            g_sim.mesh.blocks[b].refine_flag = 0;
        }
    }
}

/* prj_amr_adapt followed by the driver's refill after a changed mesh
 * (src/main.c:571-606 without output, radiation and gravity).  Returns the
 * block_changed flag. */
int rh_amr_adapt(void)
{
    int changed = prj_amr_adapt(&g_sim.mesh, &g_sim.eos, &g_mpi);

    if (changed) {
        prj_mpi_rebalance(&g_sim.mesh, &g_mpi);
        prj_eos_fill_active_cells(&g_sim.mesh, &g_sim.eos, &g_mpi, 1, PRJ_EOS_CTX_AMR);
        prj_boundary_fill_ghosts_and_bf(&g_sim.mesh, &g_mpi, &g_sim.bc, 1, 0,
            &g_sim.eos, 0, &g_sim.rad, PRJ_BOUNDARY_TIMER_SCOPE_NONE);
        prj_eos_fill_mesh(&g_sim.mesh, &g_sim.eos, &g_mpi, 1, PRJ_EOS_CTX_AMR);
    }
    return changed;
}

/* The driver loop of src/main.c:485-607 with an adapt every amr_interval
 * steps (counted by the global step number).  state as rh_run; state[3]
 * counts the adapts that changed the mesh. */
int rh_run_amr(int nsteps, int amr_interval, double *state)
{
    int n = 0;
    int changes = 0;

    while (g_sim.time < g_sim.t_end && n < nsteps) {
        double dt_new = rh_calc_dt();
        double dt_step;
        double dt_src = 1.0e100;

        if (g_sim.dt > 0.0) {
            double dt_limit = g_sim.dt_factor * g_sim.dt;

            g_sim.dt = dt_new <= dt_limit ? dt_new : dt_limit;
        } else {
            g_sim.dt = dt_new;
        }
        dt_step = g_sim.dt;
        if (g_sim.time + dt_step > g_sim.t_end) {
            dt_step = g_sim.t_end - g_sim.time;
        }
        rh_step(dt_step, &dt_src);
        if (g_sim.cfl * dt_src < g_sim.dt) {
            g_sim.dt = g_sim.cfl * dt_src;
        }
        g_sim.time += dt_step;
        g_sim.step += 1;
        n += 1;
        if (amr_interval > 0 && g_sim.step % amr_interval == 0) {
            changes += rh_amr_adapt();
        }
    }
    if (state != 0) {
        state[0] = g_sim.time;
        state[1] = g_sim.dt;
        state[2] = (double)g_sim.step;
        state[3] = (double)changes;
    }
    return n;
}

/* out[0] parent, out[1..8] children, out[9] refine_flag, out[10] can_refine */
int rh_block_tree(int b, int *out)
{
    const prj_block *block;
    int n;

    if (!g_ready || b < 0 || b >= g_sim.mesh.nblocks) {
        return 1;
    }
    block = &g_sim.mesh.blocks[b];
    out[0] = block->parent;
    for (n = 0; n < 8; ++n) {
        out[1 + n] = block->children[n];
    }
    out[9] = block->refine_flag;
    out[10] = block->can_refine;
    return 0;
}

double rh_E_injected(void) { return g_sim.eos.E_injected; }
int rh_max_blocks(void) { return g_sim.mesh.nblocks_max; }

/* WENO-Z3 face value of the reference (src/prj_reconstruct.h:383-423) */
double rh_weno3_face(double qm, double q0, double qp, double target)
{
    return prj_reconstruct_weno3_face(qm, q0, qp, target);
}
