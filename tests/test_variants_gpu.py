"""The reference's other build variants on the device, against the same
variants of the reference compiled from its sources (oracle/Makefile
VARIANTS): WENO-Z3 reconstruction (PRJ_RECON_HYDRO = PRJ_RECON_WENO3) and
the eSSPRK10_4 integrator (TIME_INTEGRATION = eSSPRK10_4, the reference's
default: ten forward-Euler substeps of dt / 6, three stored states, block
arrays with 3 stage slots).  Both sides run the driver loop of src/main.c
with identical inputs; every block array (all stage slots) must agree bit
for bit.
"""
import numpy as np
import pytest

import fornaxamr_b200 as fx
from oracle import ref as R
from tests import helpers as H

pytestmark = pytest.mark.gpu

VARIANTS = {
    "weno3": (fx.RECON_WENO3, fx.INT_RK2),
    "ess": (fx.RECON_MC, fx.INT_ESSPRK10_4),
    "ess_weno3": (fx.RECON_WENO3, fx.INT_ESSPRK10_4),
}


def make_ctx(ref, p, mhd, variant):
    recon, integ = VARIANTS[variant]
    desc = H.ref_desc(ref)
    coord = [p.xmin[0], p.xmax[0], p.xmin[1], p.xmax[1], p.xmin[2], p.xmax[2]]
    ctx = fx.Context(mhd, p.gamma, coord, bc=tuple(p.bc), recon=recon, integrator=integ)
    ctx.set_mesh(desc)
    W, Bf = H.ref_state(ref)
    for b in range(W.shape[0]):
        ctx.upload_block(b, W[b].ravel(), None if Bf is None else [Bf[b, d].ravel() for d in range(3)])
    return ctx


def assert_state_equal(ctx, ref, mhd, active_only=False):
    W_ref, Bf_ref = H.ref_state(ref)
    nb, nv, ns = W_ref.shape[0], W_ref.shape[1], W_ref.shape[2]
    W = np.empty((nb, nv, ns, H.NCELLS))
    Bf = np.empty((nb, 3, ns, H.NFACES)) if mhd else None
    ctx.download_all(W, Bf)
    sel = slice(None)
    if active_only:
        ints, _, _ = ref.mesh_arrays()
        sel = ints[:, 2] == 1
    assert H.same_values(W[sel], W_ref[sel])
    if mhd:
        assert H.same_values(Bf[sel], Bf_ref[sel])


@pytest.mark.parametrize("variant", sorted(VARIANTS))
@pytest.mark.parametrize("form", [fx.FORM_PLAIN, fx.FORM_BATCHED])
def test_fourier_mhd_variant_matches_reference(variant, form):
    if not R.available(True, variant):
        pytest.fail(f"oracle variant {variant} missing: run make -C oracle")
    ref = R.Reference(True, variant)
    p = R.params_fourier(root=2)
    ref.setup(p)
    ctx = make_ctx(ref, p, True, variant)
    assert ctx.calc_dt(p.cfl) == ref.calc_dt()
    n, t_ref, dt_ref, st_ref = ref.run(3)
    t, dt, st = ctx.run(form, 3, p.cfl, p.dt_factor, p.t_end, (0.0, 0.0, 0.0))
    assert (t, dt, st) == (t_ref, dt_ref, st_ref)
    assert_state_equal(ctx, ref, True)
    ctx.close()


def test_amr_blast_ess_weno3_matches_reference():
    ref = R.Reference(True, "ess_weno3")
    p = R.params_amr_blast(root=2, max_level=1, radii=(0.4,))
    ref.setup(p)
    ctx = make_ctx(ref, p, True, "ess_weno3")
    n, t_ref, dt_ref, st_ref = ref.run(2)
    t, dt, st = ctx.run(fx.FORM_BATCHED, 2, p.cfl, p.dt_factor, p.t_end, (0.0, 0.0, 0.0))
    assert (t, dt, st) == (t_ref, dt_ref, st_ref)
    assert_state_equal(ctx, ref, True)
    ctx.close()


def test_sod_hydro_ess_weno3_matches_reference():
    ref = R.Reference(False, "ess_weno3")
    p = R.params_sod(nblocks_x=8)
    ref.setup(p)
    ctx = make_ctx(ref, p, False, "ess_weno3")
    n, t_ref, dt_ref, st_ref = ref.run(4)
    t, dt, st = ctx.run(fx.FORM_BATCHED, 4, p.cfl, p.dt_factor, p.t_end, (0.0, 0.0, 0.0))
    assert (t, dt, st) == (t_ref, dt_ref, st_ref)
    assert_state_equal(ctx, ref, False)
    ctx.close()


def test_dynamic_amr_with_ess_matches_reference():
    """adapts with three stage slots: new children start from zeroed slots"""
    ref = R.Reference(True, "ess")
    p = R.params_amr_blast(root=2, max_level=1, radii=(0.4,))
    ref.setup(p)
    ctx = make_ctx(ref, p, True, "ess")
    crit = [dict(estimator=R.EST_LOEHNER, refine=0.3, derefine=0.1, lohner_var=R.LOHNER_PRESSURE)]
    ref.amr_configure(R.amr_params(2, crit))
    ctx.amr_configure(fx.amr_config((2, 2, 2), 2, [dict(estimator=fx.AMR_LOEHNER, refine=0.3, derefine=0.1,
                                                         var=fx.AMR_VAR_PRESSURE)]))
    n, t_ref, dt_ref, st_ref, changes = ref.run_amr(2, 1)
    state, mine = ctx.run_amr(fx.FORM_BATCHED, 2, 1, p.cfl, p.dt_factor, p.t_end, (0.0, 0.0, 0.0))
    assert mine == changes and changes >= 1
    assert state == (t_ref, dt_ref, st_ref)
    assert_state_equal(ctx, ref, True, active_only=True)
    ctx.close()


def test_weno3_every_launch_shape_matches_reference():
    """the autotuner's six launch shapes of the WENO-Z3 face kernel give the
    same bits"""
    ref = R.Reference(True, "weno3")
    p = R.params_fourier(root=2, nmodes=16, kmax=3, amp_rho=0.3)
    ref.setup(p)
    ctxs = []
    for v in range(6):
        ctx = make_ctx(ref, p, True, "weno3")
        ctx.set_flux_shape(v)
        ctxs.append(ctx)
    n, t_ref, dt_ref, st_ref = ref.run(2)
    for ctx in ctxs:
        t, dt, st = ctx.run(fx.FORM_BATCHED, 2, p.cfl, p.dt_factor, p.t_end, (0.0, 0.0, 0.0))
        assert (t, dt, st) == (t_ref, dt_ref, st_ref)
        assert_state_equal(ctx, ref, True)
        ctx.close()
