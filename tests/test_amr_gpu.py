"""Dynamic AMR on the device against the reference's prj_amr_tag and
prj_amr_adapt (the oracle, compiled from the reference's sources), through
the C ABI.

Each test builds a workload with the reference, uploads its mesh (with the
refinement tree) and state, and then tags / adapts / steps both sides the
same way.  Tag flags, the adapted mesh (entries, geometry, neighbour slots,
tree) and the full W and Bf arrays of every active block must agree bit for
bit: the prolongation, restriction and field reconstruction run the
reference's double operations in its order (--fmad=false).
"""
import numpy as np
import pytest

import fornaxamr_b200 as fx
from fornaxamr_b200 import mesh
from oracle import ref as R
from tests import helpers as H

pytestmark = pytest.mark.gpu

L = R.EST_LOEHNER


def make_ctx(ref, p, mhd, gravity=False):
    desc = H.ref_desc(ref)
    coord = [p.xmin[0], p.xmax[0], p.xmin[1], p.xmax[1], p.xmin[2], p.xmax[2]]
    ctx = fx.Context(mhd, p.gamma, coord, bc=tuple(p.bc), gravity=gravity)
    ctx.set_mesh(desc)
    W, Bf = H.ref_state(ref)
    for b in range(W.shape[0]):
        grav = [ref.grav(b, d) for d in range(3)] if gravity else None
        ctx.upload_block(b, W[b].ravel(), None if Bf is None else [Bf[b, d].ravel() for d in range(3)], grav)
    return ctx


def configure(ctx, ref, p, crits, max_level, reach=-1.0, E_floor=-1.0):
    ctx.amr_configure(fx.amr_config(tuple(p.root), max_level, crits, reach_density=reach, E_floor=E_floor))
    ref.amr_configure(R.amr_params(max_level, [
        dict(estimator=c["estimator"], refine=c["refine"], derefine=c["derefine"], lohner_var=c.get("var", 1),
             jump_var=min(c.get("var", 1), 1), eps=c.get("eps", 0.1)) for c in crits],
        reach_density=reach, E_floor=E_floor))


def assert_mesh_equal(ctx, ref):
    i2, g2, s2 = ref.mesh_arrays()
    t2 = ref.tree_arrays()
    got = ctx.get_mesh()
    mi, mg, ms = mesh.desc_to_arrays(got)
    assert i2.shape == mi.shape
    assert np.array_equal(i2, mi)
    assert np.array_equal(g2, mg)
    assert np.array_equal(s2, ms)
    assert np.array_equal(t2[:, [0, 1, 2, 3, 4, 5, 6, 7, 8, 10]], mesh.desc_tree(got))


def assert_active_state_equal(ctx, ref, mhd):
    W_ref, Bf_ref = H.ref_state(ref)
    nb, nv = W_ref.shape[0], W_ref.shape[1]
    W = np.empty((nb, nv, 2, H.NCELLS))
    Bf = np.empty((nb, 3, 2, H.NFACES)) if mhd else None
    ctx.download_all(W, Bf)
    ints, _, _ = ref.mesh_arrays()
    act = ints[:, 2] == 1
    assert np.array_equal(W[act], W_ref[act])
    if mhd:
        assert np.array_equal(Bf[act], Bf_ref[act])


def blast(ref, root=2):
    p = R.params_amr_blast(root=root, max_level=1, radii=(0.4,))
    ref.setup(p)
    return p


CRITERIA = [
    [dict(estimator=L, refine=0.3, derefine=0.1, var=1)],
    [dict(estimator=L, refine=0.2, derefine=0.05, var=0, eps=0.05)],
    [dict(estimator=L, refine=0.05, derefine=0.01, var=2, eps=0.01)],
    [dict(estimator=R.EST_VELOCITY, refine=0.05, derefine=0.01)],
    [dict(estimator=R.EST_FRACTIONAL_JUMP, refine=0.5, derefine=0.1, var=0),
     dict(estimator=R.EST_FRACTIONAL_JUMP, refine=0.2, derefine=0.05, var=1)],
    [dict(estimator=L, refine=100.0, derefine=100.0, var=1)],
]


@pytest.mark.parametrize("case", range(len(CRITERIA)))
def test_tag_flags_match_reference(ref_mhd, case):
    p = blast(ref_mhd)
    ref_mhd.run(2)
    ctx = make_ctx(ref_mhd, p, True)
    configure(ctx, ref_mhd, p, CRITERIA[case], 2)
    assert np.array_equal(ctx.amr_tag(), ref_mhd.amr_tag())
    ctx.close()


def test_tag_density_trigger_and_scale_height_match_reference(ref_mhd):
    p = R.params_collapse(root=2, max_level=1, radii=(0.4,))
    ref_mhd.setup(p)
    ref_mhd.run(1)
    ctx = make_ctx(ref_mhd, p, True, gravity=True)
    for crits, reach in (([dict(estimator=R.EST_PRESSURE_SCALE_HEIGHT, refine=0.05, derefine=0.01)], -1.0),
                         ([dict(estimator=L, refine=100.0, derefine=0.2, var=0)], 1.0e9)):
        configure(ctx, ref_mhd, p, crits, 3, reach=reach)
        assert np.array_equal(ctx.amr_tag(), ref_mhd.amr_tag())
    ctx.close()


def test_refine_then_coarsen_matches_reference(ref_mhd):
    p = blast(ref_mhd)
    _, t0, dt0, st0 = ref_mhd.run(2)
    ctx = make_ctx(ref_mhd, p, True)
    configure(ctx, ref_mhd, p, CRITERIA[0], 2)
    assert ctx.amr_adapt() == bool(ref_mhd.amr_adapt()) is True
    assert_mesh_equal(ctx, ref_mhd)
    assert_active_state_equal(ctx, ref_mhd, True)
    # step the refined mesh, then coarsen everything that may coarsen
    n, t_ref, dt_ref, st_ref = ref_mhd.run(1)
    t, dt, st = ctx.run(fx.FORM_BATCHED, 1, p.cfl, p.dt_factor, p.t_end, (t0, dt0, st0))
    assert (t, dt, st) == (t_ref, dt_ref, st_ref)
    configure(ctx, ref_mhd, p, CRITERIA[5], 2)
    assert ctx.amr_adapt() == bool(ref_mhd.amr_adapt()) is True
    assert_mesh_equal(ctx, ref_mhd)
    assert_active_state_equal(ctx, ref_mhd, True)
    ctx.close()


def test_driver_loop_with_adapts_matches_reference(ref_mhd):
    """src/main.c's loop with amr_interval = 2: calc_dt, step, dt_src clamp,
    and prj_amr_adapt plus the refill after every second step."""
    p = blast(ref_mhd)
    ctx = make_ctx(ref_mhd, p, True)
    configure(ctx, ref_mhd, p, [dict(estimator=L, refine=0.25, derefine=0.1, var=1),
                                dict(estimator=R.EST_VELOCITY, refine=0.5, derefine=0.05)], 2)
    n, t_ref, dt_ref, st_ref, changes = ref_mhd.run_amr(6, 2)
    state, mine = ctx.run_amr(fx.FORM_BATCHED, 6, 2, p.cfl, p.dt_factor, p.t_end, (0.0, 0.0, 0.0))
    assert mine == changes and changes >= 1
    assert state == (t_ref, dt_ref, st_ref)
    assert_mesh_equal(ctx, ref_mhd)
    assert_active_state_equal(ctx, ref_mhd, True)
    assert ctx.amr_timings()["total"] > 0.0
    ctx.close()


def test_energy_floor_after_remesh_matches_reference(ref_mhd):
    p = blast(ref_mhd)
    ref_mhd.run(1)
    ctx = make_ctx(ref_mhd, p, True)
    W, _ = H.ref_state(ref_mhd)
    ints, _, _ = ref_mhd.mesh_arrays()
    act = W[ints[:, 2] == 1, 4, 0].reshape(-1, 20, 20, 20)[:, 2:18, 2:18, 2:18]
    floor = float(np.median(act))  # a good part of the regenerated cells get floored
    configure(ctx, ref_mhd, p, CRITERIA[0], 2, E_floor=floor)
    assert ctx.amr_adapt() == bool(ref_mhd.amr_adapt()) is True
    assert ctx.amr_energy_injected() == ref_mhd.E_injected() != 0.0
    assert_active_state_equal(ctx, ref_mhd, True)
    ctx.close()


def test_hydro_refine_and_coarsen_match_reference(ref_hydro):
    p = R.params_amr_blast(root=2, max_level=1, radii=(0.4,))
    ref_hydro.setup(p)
    _, t, dt, st = ref_hydro.run(2)
    ctx = make_ctx(ref_hydro, p, False)
    for crits in (CRITERIA[0], CRITERIA[5]):
        configure(ctx, ref_hydro, p, crits, 2)
        assert np.array_equal(ctx.amr_tag(), ref_hydro.amr_tag())
        assert ctx.amr_adapt() == bool(ref_hydro.amr_adapt())
        assert_mesh_equal(ctx, ref_hydro)
        assert_active_state_equal(ctx, ref_hydro, False)
        n, t_ref, dt_ref, st_ref = ref_hydro.run(1)
        t, dt, st = ctx.run(fx.FORM_BATCHED, 1, p.cfl, p.dt_factor, p.t_end, (t, dt, st))
        assert (t, dt, st) == (t_ref, dt_ref, st_ref)
    assert_active_state_equal(ctx, ref_hydro, False)
    ctx.close()
