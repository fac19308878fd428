"""Reconstruction and integrator variants on the CPU: the restatement's
WENO-Z3 face value against the reference's (prj_reconstruct_weno3_face,
compiled from src/prj_reconstruct.h), and the eSSPRK10_4 time step factor of
prj_timeint_calc_dt."""
import numpy as np

from oracle import ref as R
from oracle import restate as RS


def test_weno3_restatement_matches_reference_bit_for_bit():
    r = R.Reference(True, "weno3")
    O = RS.Restatement()
    rng = np.random.default_rng(7)
    for _ in range(5000):
        q = rng.standard_normal(3) * 10.0 ** rng.uniform(-6, 6, 3)
        if rng.random() < 0.2:
            q[:] = q[0]
        if rng.random() < 0.1:
            q[rng.integers(3)] = q[1]
        for tgt in (0.5, -0.5):
            assert r.weno3_face(*q, tgt) == O.weno3_face(*q, tgt)


def test_essprk_time_step_is_six_rk2_steps():
    a = R.Reference(True)
    b = R.Reference(True, "ess")
    p = R.params_fourier(root=2)
    a.setup(p)
    b.setup(p)
    assert b.calc_dt() == a.calc_dt() * 6.0
