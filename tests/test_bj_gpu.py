"""The Barth-Jespersen prolongation limiter (prj_mesh.use_BJ = 1,
src/prj_reconstruct.h:145-313) on the device against the reference built
from its sources (the oracle), through the C ABI.

use_BJ changes every coarse-to-fine prolongation: the ghost fill's cell
prolongation (27-cell stencil, src/prj_boundary.c:79-96), the outer faces
of its Toth-Roe groups (3x3 tangential face stencil, src/prj_mhd.c:238-305)
and, in prj_amr_adapt, the conserved prolongation onto new children
(src/prj_amr.c:2239-2308) and their face groups (:2084-2103).  Each case
sets it on both sides and compares the full state of every active block bit
for bit; a reference run with the minmod limiter from the same state shows
that the limiter changed the result.

The limiter acts on each conserved variable separately, so a refinement of
the blast front leaves negative internal energies in some new cells, and the
reference then exits at the next Riemann solve ("non-positive gas
pressure").  The refinement cases therefore set the internal-energy floor
of prj_sync_primitive_from_conserved (E_FLOOR), which the device must apply
to the same cells with the same injected energy.
"""
import numpy as np
import pytest

import fornaxamr_b200 as fx
from oracle import ref as R
from tests import helpers as H
from tests.test_amr_gpu import CRITERIA, assert_active_state_equal, assert_mesh_equal, configure

pytestmark = pytest.mark.gpu

AMR3 = dict(root=3, radii=(0.25, 0.1))
E_FLOOR = 1.0e-3


def make_ctx(ref, p, mhd):
    desc = H.ref_desc(ref)
    coord = [p.xmin[0], p.xmax[0], p.xmin[1], p.xmax[1], p.xmin[2], p.xmax[2]]
    ctx = fx.Context(mhd, p.gamma, coord, bc=tuple(p.bc), use_bj=True)
    ctx.set_mesh(desc)
    W, Bf = H.ref_state(ref)
    ctx.upload_all(np.ascontiguousarray(W), None if Bf is None else np.ascontiguousarray(Bf))
    return ctx


def minmod_state(ref, p, nsteps):
    """the reference's state after nsteps from the same set-up, minmod limiter"""
    ref.setup(p)
    ref.run(nsteps)
    return H.ref_state(ref)


@pytest.mark.parametrize("form", [fx.FORM_PLAIN, fx.FORM_BATCHED])
@pytest.mark.parametrize("mhd", [True, False])
def test_static_amr_steps_with_barth_jespersen_match_reference(ref_mhd, ref_hydro, mhd, form):
    ref = ref_mhd if mhd else ref_hydro
    p = R.params_amr_blast(**AMR3) if mhd else R.params_amr_blast(root=2, radii=(0.3, 0.1))
    nsteps = 3
    W_mm, _ = minmod_state(ref, p, nsteps)
    ref.setup(p)
    ref.set_use_bj(True)
    ctx = make_ctx(ref, p, mhd)
    try:
        n, t_ref, dt_ref, st_ref = ref.run(nsteps)
        st = ctx.run(form, nsteps, p.cfl, p.dt_factor, p.t_end, (0.0, 0.0, 0.0))
        assert st == (t_ref, dt_ref, st_ref)
        assert_active_state_equal(ctx, ref, mhd)
        W_bj, _ = H.ref_state(ref)
        assert not np.array_equal(W_bj, W_mm)
    finally:
        ref.set_use_bj(False)
        ctx.close()


def minmod_refined_state(ref, p):
    """the reference's state after 2 steps and one refinement, minmod limiter"""
    ref.setup(p)
    ref.run(2)
    c = CRITERIA[0][0]
    ref.amr_configure(R.amr_params(2, [dict(estimator=c["estimator"], refine=c["refine"],
                                            derefine=c["derefine"], lohner_var=c["var"],
                                            jump_var=min(c["var"], 1), eps=0.1)], E_floor=E_FLOOR))
    assert ref.amr_adapt()
    return H.ref_state(ref)


def test_refine_then_coarsen_with_barth_jespersen_matches_reference(ref_mhd):
    p = R.params_amr_blast(root=2, max_level=1, radii=(0.4,))
    W_mm, Bf_mm = minmod_refined_state(ref_mhd, p)
    ref_mhd.setup(p)
    _, t0, dt0, st0 = ref_mhd.run(2)
    ref_mhd.set_use_bj(True)
    ctx = make_ctx(ref_mhd, p, True)
    try:
        configure(ctx, ref_mhd, p, CRITERIA[0], 2, E_floor=E_FLOOR)
        assert ctx.amr_adapt() == bool(ref_mhd.amr_adapt()) is True
        assert ctx.amr_energy_injected() == ref_mhd.E_injected() != 0.0
        assert_mesh_equal(ctx, ref_mhd)
        assert_active_state_equal(ctx, ref_mhd, True)
        W_bj, Bf_bj = H.ref_state(ref_mhd)
        assert W_bj.shape == W_mm.shape and not np.array_equal(W_bj, W_mm) and not np.array_equal(Bf_bj, Bf_mm)
        n, t_ref, dt_ref, st_ref = ref_mhd.run(1)
        assert ctx.run(fx.FORM_BATCHED, 1, p.cfl, p.dt_factor, p.t_end, (t0, dt0, st0)) == (t_ref, dt_ref, st_ref)
        assert_active_state_equal(ctx, ref_mhd, True)
        configure(ctx, ref_mhd, p, CRITERIA[5], 2, E_floor=E_FLOOR)
        assert ctx.amr_adapt() == bool(ref_mhd.amr_adapt()) is True
        assert_mesh_equal(ctx, ref_mhd)
        assert_active_state_equal(ctx, ref_mhd, True)
    finally:
        ref_mhd.set_use_bj(False)
        ctx.close()


def test_driver_loop_with_adapts_and_barth_jespersen_matches_reference(ref_mhd):
    """src/main.c's loop with amr_interval = 2 under use_BJ: the refinement
    prolongation and every later ghost fill take the limiter."""
    p = R.params_amr_blast(root=2, max_level=1, radii=(0.4,))
    ref_mhd.setup(p)
    ref_mhd.set_use_bj(True)
    ctx = make_ctx(ref_mhd, p, True)
    try:
        configure(ctx, ref_mhd, p, [dict(estimator=R.EST_LOEHNER, refine=0.25, derefine=0.1, var=1)], 2,
                  E_floor=E_FLOOR)
        n, t_ref, dt_ref, st_ref, changes = ref_mhd.run_amr(6, 2)
        state, mine = ctx.run_amr(fx.FORM_BATCHED, 6, 2, p.cfl, p.dt_factor, p.t_end, (0.0, 0.0, 0.0))
        assert mine == changes and changes >= 1
        assert state == (t_ref, dt_ref, st_ref)
        assert ctx.amr_energy_injected() == ref_mhd.E_injected()
        assert_mesh_equal(ctx, ref_mhd)
        assert_active_state_equal(ctx, ref_mhd, True)
    finally:
        ref_mhd.set_use_bj(False)
        ctx.close()


def test_hydro_refine_with_barth_jespersen_matches_reference(ref_hydro):
    p = R.params_amr_blast(root=2, max_level=1, radii=(0.4,))
    ref_hydro.setup(p)
    _, t, dt, st = ref_hydro.run(2)
    ref_hydro.set_use_bj(True)
    ctx = make_ctx(ref_hydro, p, False)
    try:
        configure(ctx, ref_hydro, p, CRITERIA[0], 2, E_floor=E_FLOOR)
        assert ctx.amr_adapt() == bool(ref_hydro.amr_adapt()) is True
        assert_mesh_equal(ctx, ref_hydro)
        assert_active_state_equal(ctx, ref_hydro, False)
        n, t_ref, dt_ref, st_ref = ref_hydro.run(1)
        assert ctx.run(fx.FORM_BATCHED, 1, p.cfl, p.dt_factor, p.t_end, (t, dt, st)) == (t_ref, dt_ref, st_ref)
        assert_active_state_equal(ctx, ref_hydro, False)
    finally:
        ref_hydro.set_use_bj(False)
        ctx.close()
