/*
 * prj_fx: FornaxAMR's timestep reduction and RK step on the device through
 * the fornax_b200 C ABI (see prj_fx.h for the contract).
 *
 * Per driver step in the default mirror mode: prj_timeint_calc_dt uploads
 * the host's block state and reduces on the device; prj_timeint_step runs
 * the step (one CUDA graph in the batched form) and downloads W, eosvar and
 * Bf of the active blocks.  A change of the mesh (blocks refined,
 * coarsened, renumbered or re-linked by the host) is detected from a
 * signature of the block tree and its neighbour slots, so any adapt --
 * including one that keeps the block count -- sends the new mesh before the
 * next device call.
 */
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "prj_fx.h"
#include "fornax_b200.h"

static fx_ctx *g_fx;
static int g_form = FX_FORM_BATCHED;
static int g_mode = PRJ_FX_MIRROR;
static int g_gravity;
static int g_have_mesh;
static uint64_t g_sig;        /* signature of the mesh the context holds */
static int g_host_newer = 1;  /* the host arrays may differ from the device's */

static void prj_fx_check(int rc, const char *where)
{
    if (rc != FX_SUCCESS) {
        char msg[512];

        msg[0] = '\0';
        if (g_fx != 0) {
            fx_last_error(g_fx, msg, sizeof msg);
        }
        fprintf(stderr, "prj_fx: %s failed (code %d): %s\n", where, rc, msg);
        exit(EXIT_FAILURE);
    }
}

/* 64-bit FNV-1a over 32-bit words */
static uint64_t prj_fx_mix(uint64_t h, const void *p, size_t nbytes)
{
    const unsigned char *c = (const unsigned char *)p;
    size_t i;

    for (i = 0; i + 4 <= nbytes; i += 4) {
        uint32_t w;

        memcpy(&w, c + i, 4);
        h ^= w;
        h *= 1099511628211ULL;
    }
    for (; i < nbytes; ++i) {
        h ^= c[i];
        h *= 1099511628211ULL;
    }
    return h;
}

/* Everything fx_set_mesh reads that an adapt can change: the entries'
 * ids, levels, activity, tree links, extents and every slot's neighbour. */
static uint64_t prj_fx_mesh_signature(const prj_mesh *mesh)
{
    uint64_t h = 1469598103934665603ULL;
    int b;
    int n;

    h = prj_fx_mix(h, &mesh->nblocks, sizeof mesh->nblocks);
    for (b = 0; b < mesh->nblocks; ++b) {
        const prj_block *k = &mesh->blocks[b];

        h = prj_fx_mix(h, &k->id, sizeof k->id);
        h = prj_fx_mix(h, &k->level, sizeof k->level);
        h = prj_fx_mix(h, &k->active, sizeof k->active);
        h = prj_fx_mix(h, &k->parent, sizeof k->parent);
        h = prj_fx_mix(h, k->children, sizeof k->children);
        h = prj_fx_mix(h, k->xmin, sizeof k->xmin);
        h = prj_fx_mix(h, k->dx, sizeof k->dx);
        for (n = 0; n < 56; ++n) {
            h = prj_fx_mix(h, &k->slot[n].id, sizeof k->slot[n].id);
        }
    }
    return h;
}

/* prj_block / prj_neighbor -> fx_block_desc / fx_slot */
static void prj_fx_desc(const prj_mesh *mesh, fx_block_desc *d)
{
    int b;
    int a;
    int n;

    for (b = 0; b < mesh->nblocks; ++b) {
        const prj_block *k = &mesh->blocks[b];

        d[b].id = k->id;
        d[b].level = k->level;
        d[b].active = k->active;
        d[b].rank = 0;
        for (a = 0; a < 3; ++a) {
            d[b].xmin[a] = k->xmin[a];
            d[b].xmax[a] = k->xmax[a];
            d[b].dx[a] = k->dx[a];
            d[b].area[a] = k->area[a];
        }
        d[b].vol = k->vol;
        d[b].parent = k->parent;
        for (n = 0; n < 8; ++n) {
            d[b].children[n] = k->children[n];
        }
        d[b].can_refine = k->can_refine;
        for (n = 0; n < 56; ++n) {
            const prj_neighbor *s = &k->slot[n];
            fx_slot *t = &d[b].slot[n];

            t->id = s->id;
            t->rel_level = s->rel_level;
            t->type = s->type;
            for (a = 0; a < 3; ++a) {
                t->send_loc_start[a] = s->send_loc_start[a];
                t->send_loc_end[a] = s->send_loc_end[a];
                t->recv_loc_start[a] = s->recv_loc_start[a];
                t->recv_loc_end[a] = s->recv_loc_end[a];
            }
        }
    }
}

static int prj_fx_has_gravity(const prj_mesh *mesh)
{
    int b;
    int d;
    int c;

    for (b = 0; b < mesh->nblocks; ++b) {
        const prj_block *k = &mesh->blocks[b];

        if (k->id < 0 || k->active != 1) {
            continue;
        }
        for (d = 0; d < 3; ++d) {
            if (k->grav[d] == 0) {
                continue;
            }
            for (c = 0; c < PRJ_BLOCK_NCELLS; ++c) {
                if (k->grav[d][c] != 0.0) {
                    return 1;
                }
            }
        }
    }
    return 0;
}

static void prj_fx_create(const prj_mesh *mesh, const prj_bc *bc, prj_eos *eos)
{
    fx_config cfg;
    double q[PRJ_EOS_NQUANT];

    if (g_fx != 0) {
        return;
    }
    if (fx_ghost_layers() != PRJ_NGHOST || PRJ_BLOCK_SIZE != 16) {
        fprintf(stderr, "prj_fx: the loaded library has %d ghost layers, this build PRJ_NGHOST = %d "
            "(block size %d, 16 required)\n", fx_ghost_layers(), PRJ_NGHOST, PRJ_BLOCK_SIZE);
        exit(EXIT_FAILURE);
    }
    memset(&cfg, 0, sizeof cfg);
    cfg.mhd = PRJ_MHD;
    /* the ideal gas's adiabatic index, from the EOS itself */
    prj_eos_rey(eos, 1.0, 1.0, 0.1, q, PRJ_EOS_CTX_MAIN);
    cfg.gamma = q[PRJ_EOS_GAMMA];
    g_gravity = prj_fx_has_gravity(mesh);
    cfg.gravity = g_gravity;
    cfg.coord[0] = mesh->coord.x1min;
    cfg.coord[1] = mesh->coord.x1max;
    cfg.coord[2] = mesh->coord.x2min;
    cfg.coord[3] = mesh->coord.x2max;
    cfg.coord[4] = mesh->coord.x3min;
    cfg.coord[5] = mesh->coord.x3max;
    cfg.bc[0] = bc->bc_x1_inner;
    cfg.bc[1] = bc->bc_x1_outer;
    cfg.bc[2] = bc->bc_x2_inner;
    cfg.bc[3] = bc->bc_x2_outer;
    cfg.bc[4] = bc->bc_x3_inner;
    cfg.bc[5] = bc->bc_x3_outer;
    cfg.mhd_eta = mesh->mhd_eta;
    cfg.use_bj = mesh->use_BJ != 0;
#if PRJ_RECON_HYDRO == PRJ_RECON_WENO7
    cfg.recon = FX_RECON_WENO7;
#elif PRJ_RECON_HYDRO == PRJ_RECON_WENO3
    cfg.recon = FX_RECON_WENO3;
#else
    cfg.recon = FX_RECON_MC;
#endif
#if TIME_INTEGRATION == PRJ_TIMEINT_ESSPRK10_4
    cfg.integrator = FX_INT_ESSPRK10_4;
#elif TIME_INTEGRATION == PRJ_TIMEINT_RK2
    cfg.integrator = FX_INT_RK2;
#else
#error "prj_fx: RK2 or eSSPRK10_4 builds only"
#endif
    prj_fx_check(fx_create(0, &cfg, &g_fx), "fx_create");
    g_have_mesh = 0;
    g_host_newer = 1;
}

static void prj_fx_upload(const prj_mesh *mesh)
{
    int b;

    for (b = 0; b < mesh->nblocks; ++b) {
        prj_block *k = &mesh->blocks[b];
        const double *gr[3];

        if (k->id < 0 || k->W_mhd == 0) {
            continue;
        }
        gr[0] = k->grav[0];
        gr[1] = k->grav[1];
        gr[2] = k->grav[2];
#if PRJ_MHD
        {
            const double *bf[3] = {k->Bf[0], k->Bf[1], k->Bf[2]};

            prj_fx_check(fx_upload_block(g_fx, b, k->W_mhd, bf, g_gravity ? gr : 0), "fx_upload_block");
        }
#else
        prj_fx_check(fx_upload_block(g_fx, b, k->W_mhd, 0, g_gravity ? gr : 0), "fx_upload_block");
#endif
    }
    g_host_newer = 0;
}

static void prj_fx_download(const prj_mesh *mesh)
{
    int b;

    for (b = 0; b < mesh->nblocks; ++b) {
        prj_block *k = &mesh->blocks[b];

        if (k->id < 0 || k->active != 1) {
            continue;
        }
#if PRJ_MHD
        {
            double *bf[3] = {k->Bf[0], k->Bf[1], k->Bf[2]};

            prj_fx_check(fx_download_block(g_fx, b, k->W_mhd, k->eosvar, bf), "fx_download_block");
        }
#else
        prj_fx_check(fx_download_block(g_fx, b, k->W_mhd, k->eosvar, 0), "fx_download_block");
#endif
    }
}

/* Sends a changed mesh and, where the device is not current, the state. */
static void prj_fx_sync_in(const prj_mesh *mesh)
{
    const uint64_t sig = prj_fx_mesh_signature(mesh);

    if (!g_have_mesh || sig != g_sig) {
        fx_block_desc *d = (fx_block_desc *)calloc((size_t)mesh->nblocks, sizeof *d);

        if (d == 0) {
            fprintf(stderr, "prj_fx: out of host memory for the mesh description\n");
            exit(EXIT_FAILURE);
        }
        prj_fx_desc(mesh, d);
        prj_fx_check(fx_set_mesh(g_fx, mesh->nblocks, d), "fx_set_mesh");
        free(d);
        g_sig = sig;
        g_have_mesh = 1;
        g_host_newer = 1;
    }
    if (g_host_newer) {
        prj_fx_upload(mesh);
    }
}

void prj_fx_configure(int form, int mode)
{
    if (form != FX_FORM_BATCHED && form != FX_FORM_PLAIN) {
        fprintf(stderr, "prj_fx_configure: unknown form %d\n", form);
        exit(EXIT_FAILURE);
    }
    if (mode != PRJ_FX_MIRROR && mode != PRJ_FX_RESIDENT) {
        fprintf(stderr, "prj_fx_configure: unknown mode %d\n", mode);
        exit(EXIT_FAILURE);
    }
    g_form = form;
    g_mode = mode;
}

void prj_fx_to_host(const prj_mesh *mesh)
{
    if (g_fx != 0 && g_have_mesh) {
        prj_fx_download(mesh);
    }
}

void prj_fx_to_device(const prj_mesh *mesh)
{
    if (g_fx != 0) {
        g_host_newer = 1;
        prj_fx_sync_in(mesh);
    }
}

void prj_fx_release(void)
{
    if (g_fx != 0) {
        fx_destroy(g_fx);
        g_fx = 0;
    }
    g_have_mesh = 0;
    g_host_newer = 1;
}

int prj_fx_active(void)
{
    return g_fx != 0;
}

double prj_fx_timeint_calc_dt(const prj_mesh *mesh, prj_eos *eos, const prj_rad *rad,
    const prj_mpi *mpi, double cfl, const prj_timeint_imex_tableau *tableau)
{
    double dt = 0.0;

    (void)eos;
    (void)rad;
    (void)mpi;
    (void)tableau;
    if (g_fx == 0) {
        fprintf(stderr, "prj_fx_timeint_calc_dt: no device context (the first step creates it)\n");
        exit(EXIT_FAILURE);
    }
    if (g_mode == PRJ_FX_MIRROR) {
        prj_fx_sync_in(mesh);
    } else if (!g_have_mesh || prj_fx_mesh_signature(mesh) != g_sig) {
        prj_fx_sync_in(mesh);
    }
    prj_fx_check(fx_calc_dt(g_fx, cfl, &dt), "fx_calc_dt");
    return dt;
}

void prj_fx_timeint_step(prj_mesh *mesh, const prj_coord *coord, const prj_bc *bc, prj_eos *eos,
    prj_rad *rad, prj_grav *grav, prj_mpi *mpi, const prj_timeint_imex_tableau *tableau,
    double dt, double *dt_src, prj_timer *timer)
{
    double src = 1.0e100;

    (void)coord;
    (void)rad;
    (void)grav;
    (void)mpi;
    (void)tableau;
    (void)timer;
    prj_fx_create(mesh, bc, eos);
    prj_fx_sync_in(mesh);
    prj_fx_check(fx_step(g_fx, g_form, dt, dt_src != 0 ? &src : 0), "fx_step");
    if (dt_src != 0 && src < *dt_src) {
        *dt_src = src;
    }
    if (g_mode == PRJ_FX_MIRROR) {
        prj_fx_download(mesh);
        g_host_newer = 1;
    }
}

#ifdef PRJ_FX_WRAP
/* Link-time replacement (-Wl,--wrap=prj_timeint_step,--wrap=prj_timeint_calc_dt):
 * the reference's callers reach these instead of the originals.  Before the
 * first step has created the device context (it needs the boundary
 * conditions the step receives), the timestep comes from the reference's own
 * reduction on the host arrays, which hold the state at that point. */
double __real_prj_timeint_calc_dt(const prj_mesh *mesh, prj_eos *eos, const prj_rad *rad,
    const prj_mpi *mpi, double cfl, const prj_timeint_imex_tableau *tableau);

double __wrap_prj_timeint_calc_dt(const prj_mesh *mesh, prj_eos *eos, const prj_rad *rad,
    const prj_mpi *mpi, double cfl, const prj_timeint_imex_tableau *tableau)
{
    if (!prj_fx_active()) {
        return __real_prj_timeint_calc_dt(mesh, eos, rad, mpi, cfl, tableau);
    }
    return prj_fx_timeint_calc_dt(mesh, eos, rad, mpi, cfl, tableau);
}

void __wrap_prj_timeint_step(prj_mesh *mesh, const prj_coord *coord, const prj_bc *bc, prj_eos *eos,
    prj_rad *rad, prj_grav *grav, prj_mpi *mpi, const prj_timeint_imex_tableau *tableau,
    double dt, double *dt_src, prj_timer *timer)
{
    prj_fx_timeint_step(mesh, coord, bc, eos, rad, grav, mpi, tableau, dt, dt_src, timer);
}
#endif
