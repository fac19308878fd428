"""The product's workload generators build the same initial state as the
oracle harness (same recipes, separate code)."""
import numpy as np

from oracle import ref as R
from tests import helpers as H


def test_fourier_mhd_initial_state_matches_oracle(ref_mhd):
    from fornaxamr_b200 import mesh, problems
    p = R.params_fourier(root=2, nmodes=8, kmax=3)
    ref_mhd.setup(p)
    W_ref, Bf_ref = H.ref_state(ref_mhd)
    blocks = mesh.uniform_mesh((2, 2, 2), (0, 1, 0, 1, 0, 1))
    W, Bf = problems.fourier_mhd(blocks, nmodes=8, kmax=3)
    act = H.active_cells()
    # active cells are untouched by the oracle's initial ghost fill
    assert H.max_rel_err(W[:, :, 0][..., act], W_ref[:, :, 0][..., act]) < 1e-13
    for d in range(3):
        fa = H.active_faces(d)
        assert H.max_rel_err(Bf[:, d, 0][:, fa], Bf_ref[:, d, 0][:, fa]) < 1e-12


def test_sod_initial_state_matches_oracle(ref_hydro):
    from fornaxamr_b200 import mesh, problems
    p = R.params_sod(nblocks_x=4)
    ref_hydro.setup(p)
    W_ref, _ = H.ref_state(ref_hydro)
    blocks = mesh.uniform_mesh((4, 1, 1), (0, 1, 0, 0.25, 0, 0.25))
    W = problems.sod(blocks)
    act = H.active_cells()
    assert np.array_equal(W[:, :, 0][..., act], W_ref[:, :, 0][..., act])


def _amr_product_state(p, gen, mhd=True):
    """Product mesh + initial state for an oracle preset, with the initial
    ghost fill of the driver's set-up (src/main.c:440-447) run through the
    compiled ghost program."""
    import fornaxamr_b200 as fx
    from fornaxamr_b200 import mesh
    coord = [p.xmin[0], p.xmax[0], p.xmin[1], p.xmax[1], p.xmin[2], p.xmax[2]]
    blocks = mesh.static_amr_mesh(list(p.root), coord, p.max_level,
                                  mesh.ball_refiner(list(p.center), list(p.refine_radius)[:p.max_level]))
    desc = mesh.to_desc(blocks)
    cfg = fx.make_config(mhd, p.gamma, coord)
    recs = fx.plan_export(cfg, desc, 3) if mhd else None
    out = gen(blocks, recs)
    W, Bf = out[0], out[1]
    H.apply_ghost_program(W, Bf, cfg, desc, 0)
    return blocks, desc, out


def test_amr_blast_mesh_and_initial_state_match_oracle(ref_mhd):
    from fornaxamr_b200 import mesh, problems
    p = R.params_amr_blast(root=3, radii=(0.25, 0.1))
    ref_mhd.setup(p)
    ints, geom, slots = ref_mhd.mesh_arrays()
    blocks, desc, (W, Bf) = _amr_product_state(p, lambda b, r: problems.amr_blast(b, r))
    mi, mg, ms = mesh.desc_to_arrays(desc)
    assert np.array_equal(mi[:, :3], ints[:, :3])
    assert np.array_equal(mg, geom)
    assert np.array_equal(ms, slots)
    W_ref, Bf_ref = H.ref_state(ref_mhd)
    assert np.array_equal(Bf, Bf_ref)
    assert np.array_equal(W, W_ref)


def test_collapse_mesh_and_initial_state_match_oracle(ref_mhd):
    from fornaxamr_b200 import mesh, problems
    p = R.params_collapse(root=4)
    ref_mhd.setup(p)
    ints, geom, slots = ref_mhd.mesh_arrays()
    blocks, desc, (W, Bf, grav) = _amr_product_state(p, lambda b, r: problems.collapse(b, r))
    mi, mg, ms = mesh.desc_to_arrays(desc)
    assert np.array_equal(ms, slots) and np.array_equal(mg, geom)
    W_ref, Bf_ref = H.ref_state(ref_mhd)
    act = np.nonzero(mi[:, 2] == 1)[0]
    # numpy's vector pow / arcsinh may differ from libm's in the last bit, so
    # the profile and gravity agree to round-off rather than bit for bit
    assert H.max_rel_err(W[act], W_ref[act]) <= 1e-14
    assert H.max_rel_err(Bf[act], Bf_ref[act]) <= 1e-14
    g_ref = np.stack([np.stack([ref_mhd.grav(b, d) for d in range(3)]) for b in act])
    assert H.max_rel_err(grav[act], g_ref) <= 1e-14
