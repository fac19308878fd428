/*
 * prj_fx: the binding of fornax_b200 into the FornaxAMR C code.
 *
 * Compiled with the reference's own headers (prj.h) into its build and
 * linked with libfornax_b200 (libfornax_b200_ng4 for a PRJ_NGHOST = 4
 * build).  The two entry points below have the signatures of the functions
 * they replace (src/prj_timeint.h:15-16 and 31-33), so the reference's
 * driver loop (src/main.c:485-562) calls the device through them unchanged,
 * either by a build switch in prj_timeint_step / prj_timeint_calc_dt or by
 * linking with
 *     -Wl,--wrap=prj_timeint_step,--wrap=prj_timeint_calc_dt
 * and compiling prj_fx.c with -DPRJ_FX_WRAP (no reference source edited).
 *
 * Supported builds: PRJ_MHD 0/1, RK2 or eSSPRK10_4, MC / WENO-Z3 / WENO-Z7
 * reconstruction, the ideal-gas EOS (its adiabatic index is read from the
 * EOS at start-up), one rank.  Errors follow the reference's fail-fast
 * convention: the library's message on stderr, then exit(EXIT_FAILURE).
 */
#ifndef PRJ_FX_H
#define PRJ_FX_H

#include "prj.h"

/* Where the block state lives between driver steps.
 *   PRJ_FX_MIRROR (default): the host's prj_block arrays stay current: the
 *     state is uploaded before the step's timestep reduction (or the step,
 *     if no reduction came first) and W, eosvar and Bf are downloaded after
 *     every step, so host code between steps (an adapt on the host, a dump)
 *     sees and may change the state as with the reference.
 *   PRJ_FX_RESIDENT: the device keeps the state across steps; the host's
 *     arrays are refreshed only by prj_fx_to_host(), and host changes reach
 *     the device only through prj_fx_to_device() (a changed mesh -- blocks
 *     refined, coarsened or re-linked -- is detected and uploaded by itself).
 * In both modes the device writes W, Bf and eosvar of the active blocks;
 * the scratch arrays (flux, v_riemann, emf, Bv, mhd_rhs) are not copied
 * back. */
#define PRJ_FX_MIRROR 0
#define PRJ_FX_RESIDENT 1

/* form: FX_FORM_BATCHED (default: one CUDA graph per step) or
 * FX_FORM_PLAIN (per-block launches).  Call before the first step or
 * between steps; changing the mode syncs the host first. */
void prj_fx_configure(int form, int mode);

/* RESIDENT mode: copy W, eosvar and Bf of the active blocks to the host /
 * to the device. */
void prj_fx_to_host(const prj_mesh *mesh);
void prj_fx_to_device(const prj_mesh *mesh);

/* Frees the device context (the next step creates a new one). */
void prj_fx_release(void);

/* 1 once a step has created the device context (it needs the boundary
 * conditions the step receives), else 0. */
int prj_fx_active(void);

/* prj_timeint_calc_dt (src/prj_timeint.h:15-16) on the device. */
double prj_fx_timeint_calc_dt(const prj_mesh *mesh, prj_eos *eos, const prj_rad *rad,
    const prj_mpi *mpi, double cfl, const prj_timeint_imex_tableau *tableau);

/* prj_timeint_step (src/prj_timeint.h:31-33) on the device; *dt_src is
 * lowered to the step's source time-step minimum like the reference's. */
void prj_fx_timeint_step(prj_mesh *mesh, const prj_coord *coord, const prj_bc *bc, prj_eos *eos,
    prj_rad *rad, prj_grav *grav, prj_mpi *mpi, const prj_timeint_imex_tableau *tableau,
    double dt, double *dt_src, prj_timer *timer);

#endif
