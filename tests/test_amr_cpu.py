"""Dynamic AMR on the CPU: the host half of fx_amr_adapt against the
reference's prj_amr_tag / prj_amr_adapt (compiled from its own sources).

The reference runs a magnetised blast on a 2^3-root mesh with one static
level; between adapts it steps the state forward.  The per-block votes of
pass 1 of prj_amr_tag come from the oracle's restatement (fx_oracle.c, on
the reference's own state); the library turns them into refine flags (tag
passes 2-4) and a new mesh (2:1 balance, refinement, coarsening, neighbour
rebuild).  Flags must equal the reference's prj_amr_tag result and the new
mesh (block entries, geometry, slots with their send/recv boxes, parent and
children) must equal the reference's after prj_amr_adapt, entry by entry.
The sequence covers refinement with boundary-mask propagation to coarser
neighbours, coarsening of whole levels, every estimator without gravity and
the density trigger.
"""
import numpy as np
import pytest

import fornaxamr_b200 as fx
from fornaxamr_b200 import mesh
from oracle import ref as R
from oracle import restate as RS
from tests import helpers as H

COORD = (-0.7, 0.7, -0.7, 0.7, -0.7, 0.7)


def _ref_amr(crits, max_level, reach):
    return R.amr_params(max_level, [dict(estimator=c["estimator"], refine=c["refine"], derefine=c["derefine"],
                                         lohner_var=c.get("var", 1), jump_var=min(c.get("var", 1), 1),
                                         eps=c.get("eps", 0.1)) for c in crits],
                        reach_density=reach)


def _adapt_and_compare(ref, crits, max_level, reach=-1.0):
    O = RS.Restatement()
    W, _ = H.ref_state(ref)
    ints, geom, slots = ref.mesh_arrays()
    tree = ref.tree_arrays()
    votes = O.amr_votes(9, 5.0 / 3.0, W, None, geom[:, 6:9], ints[:, 2] == 1, tree[:, 0], crits, reach)
    desc = mesh.desc_from_arrays(ints, geom, slots, tree)
    cfg = fx.make_config(True, 5.0 / 3.0, COORD)
    amr = fx.amr_config((2, 2, 2), max_level, crits, reach_density=reach)
    flags, new = fx.amr_remesh_host(cfg, amr, desc, votes)

    ref.amr_configure(_ref_amr(crits, max_level, reach))
    assert np.array_equal(flags, ref.amr_tag())
    changed = ref.amr_adapt()
    i2, g2, s2 = ref.mesh_arrays()
    t2 = ref.tree_arrays()
    mi, mg, ms = mesh.desc_to_arrays(new)
    mt = mesh.desc_tree(new)
    assert i2.shape == mi.shape
    assert np.array_equal(i2, mi)
    assert np.array_equal(g2, mg)
    assert np.array_equal(s2, ms)
    assert np.array_equal(t2[:, [0, 1, 2, 3, 4, 5, 6, 7, 8, 10]], mt)
    return changed, flags


def test_remesh_sequence_matches_reference(ref_mhd):
    ref_mhd.setup(R.params_amr_blast(root=2, max_level=1, radii=(0.4,)))
    ref_mhd.run(2)
    L = R.EST_LOEHNER
    changed, flags = _adapt_and_compare(ref_mhd, [dict(estimator=L, refine=0.3, derefine=0.1, var=1)], 2)
    assert changed and (flags > 0).sum() > 4  # refinement spread to neighbours by the boundary mask
    ref_mhd.run(1)
    changed, flags = _adapt_and_compare(ref_mhd, [dict(estimator=L, refine=100.0, derefine=100.0, var=1)], 2)
    assert changed and (flags < 0).sum() > 0
    ref_mhd.run(1)
    _adapt_and_compare(ref_mhd, [dict(estimator=R.EST_VELOCITY, refine=0.05, derefine=0.01),
                                 dict(estimator=R.EST_FRACTIONAL_JUMP, refine=0.5, derefine=0.1, var=0)], 2)
    ref_mhd.run(1)
    _adapt_and_compare(ref_mhd, [dict(estimator=L, refine=0.2, derefine=0.05, var=2, eps=0.01)], 3)
    ref_mhd.run(1)
    _adapt_and_compare(ref_mhd, [dict(estimator=L, refine=100.0, derefine=0.5, var=0)], 3, reach=1.05)
    ref_mhd.run(1)
    _adapt_and_compare(ref_mhd, [dict(estimator=R.EST_FRACTIONAL_JUMP, refine=100.0, derefine=100.0, var=1)], 3)


def test_remesh_without_changes_returns_the_input(ref_mhd):
    ref_mhd.setup(R.params_amr_blast(root=2, max_level=1, radii=(0.4,)))
    ints, geom, slots = ref_mhd.mesh_arrays()
    desc = mesh.desc_from_arrays(ints, geom, slots, ref_mhd.tree_arrays())
    cfg = fx.make_config(True, 5.0 / 3.0, COORD)
    amr = fx.amr_config((2, 2, 2), 1, [dict(estimator=fx.AMR_LOEHNER, refine=0.5, derefine=0.2)])
    votes = np.zeros((len(desc), 3), dtype=np.int32)
    flags, new = fx.amr_remesh_host(cfg, amr, desc, votes)
    assert not flags.any()
    assert np.array_equal(mesh.desc_to_arrays(new)[2], slots)


def test_remesh_reports_block_capacity():
    blocks = mesh.uniform_mesh((2, 2, 2), (0, 1, 0, 1, 0, 1))
    desc = mesh.to_desc(blocks)
    cfg = fx.make_config(True, 5.0 / 3.0, (0, 1, 0, 1, 0, 1))
    amr = fx.amr_config((2, 2, 2), 1, [dict(estimator=fx.AMR_LOEHNER)], max_blocks=12)
    votes = np.zeros((8, 3), dtype=np.int32)
    votes[:, 0] = 1
    with pytest.raises(fx.FxError) as e:
        fx.amr_remesh_host(cfg, amr, desc, votes)
    assert e.value.code == 6  # FX_ETOOBIG: prj_find_free_block_slot's capacity exit


def test_static_mesh_builder_fills_the_tree():
    blocks = mesh.static_amr_mesh((2, 2, 2), COORD, 1, mesh.ball_refiner((0.1, 0.05, 0.0), (0.4,)))
    t = mesh.desc_tree(mesh.to_desc(blocks))
    for n, b in enumerate(blocks):
        assert t[n, 0] == b.parent
        assert list(t[n, 1:9]) == b.children
