"""The resistive terms of the EMF update against the reference, through the
C ABI, in both forms.

Two cases, each run for several driver steps from the same initial state:

* a run-time resistivity (prj_mesh.mhd_eta != 0) on the Fourier-mode MHD
  state: every edge EMF gets eta * (curl B)_edge (src/prj_mhd.c:682-709);
* the artificial resistivity of dense, neutron-rich matter
  (src/prj_timeint.c:222-290): eta_cell = 1e12 ln(rho / 1e13) ln(Ye / 0.25)
  where both logarithms are positive, the edge taking the largest of its four
  cells.  The state is the Fourier-mode state mapped to rho = 1e13 (1 + 1e-3
  d) and Ye = 0.25 (1 + 0.2 d') with d, d' in [-1, 1], so that the mask is
  zero in some cells and positive in others, with pressure, velocity and
  field scaled so that the flow stays subsonic (Mach ~ 0.1, plasma beta
  ~ 200) and the explicit resistive update stable (eta dt / dx^2 ~ 0.05).

Tolerance: the ideal and run-time-eta arithmetic is bit for bit.  The
artificial mask evaluates `log`: CUDA's double `log` and the C library's may
differ in the last place, so that case asserts the required 1e-12 relative
bound on every block array and reports whether the state is also bit-equal.
"""
import warnings

import numpy as np
import pytest

import fornaxamr_b200 as fx
from oracle import ref as R
from tests import helpers as H

TOL = 1e-12
STEPS = 5


def dense_state(ref):
    """Rewrites the oracle's Fourier-mode state into the dense regime and
    refills ghosts and eos; returns the fraction of active cells whose
    artificial eta is positive."""
    W, Bf = H.ref_state(ref)
    g = 5.0 / 3.0
    rho, v1, eint = W[:, 0], W[:, 1], W[:, 4]
    d = (rho - 1.0) / np.abs(rho - 1.0).max()
    dv = v1 / np.abs(v1).max()
    p = (g - 1.0) * rho * eint
    rho_n = 1.0e13 * (1.0 + 1.0e-3 * d)
    p_n = p * 2.0 ** 109
    W[:, 0] = rho_n
    W[:, 1:4] *= 2.0 ** 33
    W[:, 4] = p_n / ((g - 1.0) * rho_n)
    W[:, 5] = 0.25 * (1.0 + 0.2 * dv)
    W[:, 6:9] *= 2.0 ** 53
    Bf *= 2.0 ** 53          # a power of two: the discrete divergence stays zero
    for b in range(W.shape[0]):
        ref.set_W(b, W[b].ravel())
        for dd in range(3):
            ref.set_Bf(b, dd, Bf[b, dd].ravel())
    ref.refill()
    act = H.active_cells()
    with np.errstate(divide="ignore", invalid="ignore"):
        eta = 1e12 * np.maximum(0.0, np.log(rho_n[:, 0][:, act] / 1e13)) * \
            np.maximum(0.0, np.log(W[:, 5, 0][:, act] / 0.25))
    return float(np.mean(eta > 0.0))


def make_ctx(ref, p, eta):
    desc = H.ref_desc(ref)
    coord = [p.xmin[0], p.xmax[0], p.xmin[1], p.xmax[1], p.xmin[2], p.xmax[2]]
    ctx = fx.Context(True, p.gamma, coord, mhd_eta=eta)
    ctx.set_mesh(desc)
    W, Bf = H.ref_state(ref)
    for b in range(W.shape[0]):
        ctx.upload_block(b, W[b].ravel(), [Bf[b, d].ravel() for d in range(3)])
    return ctx


def compare(ctx, ref, exact):
    W_ref, Bf_ref = H.ref_state(ref)
    W = np.empty_like(W_ref)
    Bf = np.empty_like(Bf_ref)
    ctx.download_all(W, Bf)
    errs = []
    for v in range(W.shape[1]):
        errs.append(H.max_rel_err(W[:, v], W_ref[:, v]))
    for d in range(3):
        errs.append(H.max_rel_err(Bf[:, d], Bf_ref[:, d]))
    same = np.array_equal(W, W_ref) and np.array_equal(Bf, Bf_ref)
    if exact:
        assert same
    return max(errs), same


def test_dense_state_has_artificial_eta_and_steps_on_the_reference(ref_mhd):
    """The dense state switches the artificial mask on in part of the mesh,
    and the reference steps it without reaching one of its exits."""
    p = R.params_fourier(root=2, nmodes=8, kmax=2)
    ref_mhd.setup(p)
    frac = dense_state(ref_mhd)
    assert 0.1 < frac < 0.9
    n, t, dt, st = ref_mhd.run(STEPS)
    assert n == STEPS and np.isfinite(t) and dt > 0.0


@pytest.mark.gpu
@pytest.mark.parametrize("form", [fx.FORM_PLAIN, fx.FORM_BATCHED])
def test_run_time_eta_matches_reference(ref_mhd, form):
    p = R.params_fourier(root=2, nmodes=8, kmax=2)
    ref_mhd.setup(p)
    eta = 2.0e-3
    ref_mhd.set_mhd_eta(eta)
    ctx = make_ctx(ref_mhd, p, eta)
    try:
        ref_st = ref_mhd.run(STEPS)
        st = ctx.run(form, STEPS, p.cfl, p.dt_factor, p.t_end, (0.0, 0.0, 0.0))
        assert st == ref_st[1:]
        err, _ = compare(ctx, ref_mhd, exact=True)
        assert err <= TOL
    finally:
        ref_mhd.set_mhd_eta(0.0)
        ctx.close()


@pytest.mark.gpu
@pytest.mark.parametrize("form", [fx.FORM_PLAIN, fx.FORM_BATCHED])
def test_artificial_eta_of_dense_matter_matches_reference(ref_mhd, form):
    p = R.params_fourier(root=2, nmodes=8, kmax=2)
    ref_mhd.setup(p)
    frac = dense_state(ref_mhd)
    assert frac > 0.1
    ctx = make_ctx(ref_mhd, p, 0.0)
    try:
        ref_st = ref_mhd.run(STEPS)
        st = ctx.run(form, STEPS, p.cfl, p.dt_factor, p.t_end, (0.0, 0.0, 0.0))
        assert st[2] == ref_st[3]
        assert abs(st[0] - ref_st[1]) <= TOL * abs(ref_st[1])
        err, same = compare(ctx, ref_mhd, exact=False)
        print(f"artificial eta ({frac:.2f} of cells), {STEPS} steps: max relative difference {err:.3e}, "
              f"bit-equal {same}")
        if not same:
            warnings.warn(f"artificial-eta state after {STEPS} steps differs from the reference in the last "
                          f"places (max relative {err:.3e}): CUDA log vs the C library's")
        assert err <= TOL
    finally:
        ctx.close()
