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
