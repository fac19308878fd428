"""Parity of the CUDA path with the reference CPU path (the oracle), through
the C ABI.  Identical inputs: the oracle builds the workload with the
reference's own code, the state is uploaded to the device, both sides step
with the same dt sequence, and every block array is compared.

Tolerance: the kernels evaluate the reference's double operations in the
same order with no contraction, so agreement is expected to be bit for bit;
the asserted bound is the required 1e-12 relative (per array, relative to
its max magnitude), and bit equality is asserted where it holds by design.
"""
import numpy as np
import pytest

import fornaxamr_b200 as fx
from oracle import ref as R
from tests import helpers as H

pytestmark = pytest.mark.gpu

TOL = 1e-12


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


def device_state(ctx, nb, nv, mhd):
    W = np.empty((nb, nv, 2, H.NCELLS))
    Bf = np.empty((nb, 3, 2, H.NFACES)) if mhd else None
    ctx.download_all(W, Bf)
    return W, Bf


def assert_state_equal(ctx, ref, mhd, exact=True):
    W_ref, Bf_ref = H.ref_state(ref)
    W, Bf = device_state(ctx, W_ref.shape[0], W_ref.shape[1], mhd)
    assert H.max_rel_err(W, W_ref) <= TOL
    if mhd:
        assert H.max_rel_err(Bf, Bf_ref) <= TOL
    if exact:
        assert np.array_equal(W, W_ref)
        if mhd:
            assert np.array_equal(Bf, Bf_ref)


@pytest.mark.parametrize("form", [fx.FORM_PLAIN, fx.FORM_BATCHED])
def test_fourier_mhd_steps_match_reference(ref_mhd, form):
    p = R.params_fourier(root=2, nmodes=8, kmax=2)
    ref_mhd.setup(p)
    ctx = make_ctx(ref_mhd, p, True)
    assert ctx.calc_dt(p.cfl) == ref_mhd.calc_dt()
    n, t_ref, dt_ref, st_ref = ref_mhd.run(3)
    t, dt, st = ctx.run(form, 3, p.cfl, p.dt_factor, p.t_end, (0.0, 0.0, 0.0))
    assert (t, dt, st) == (t_ref, dt_ref, st_ref)
    assert_state_equal(ctx, ref_mhd, True)
    ctx.close()


def test_single_stage_and_intermediates_match_reference(ref_mhd):
    p = R.params_fourier(root=2, nmodes=6, kmax=2)
    ref_mhd.setup(p)
    ctx = make_ctx(ref_mhd, p, True)
    dt = ref_mhd.calc_dt()
    ref_src = ref_mhd.stage(1, dt)
    src = ctx.stage(fx.FORM_PLAIN, 1, dt)
    assert src == ref_src
    # compare the entries the reference computes (its scratch elsewhere is
    # uninitialised heap memory)
    for b in range(ref_mhd.nblocks()):
        for d in range(3):
            fp = H.flux_positions(d, 9, True)
            assert np.array_equal(ctx.download_array(b, fx.ARR_FLUX, d)[fp], ref_mhd.flux(b, d)[fp])
            vp = H.vr_positions(d, True)
            assert np.array_equal(ctx.download_array(b, fx.ARR_VRIEMANN, d)[vp], ref_mhd.vriemann(b, d)[vp])
            bp = H.bv_positions(d)
            bv1, bv2 = ref_mhd.Bv(b, d)
            assert np.array_equal(ctx.download_array(b, fx.ARR_BV1, d)[bp], bv1[bp])
            assert np.array_equal(ctx.download_array(b, fx.ARR_BV2, d)[bp], bv2[bp])
            ep = H.emf_positions(d)
            assert np.array_equal(ctx.download_array(b, fx.ARR_EMF, d)[ep], ref_mhd.emf(b, d)[ep])
        assert np.array_equal(ctx.download_array(b, fx.ARR_EOSVAR), ref_mhd.eosvar(b))
    assert_state_equal(ctx, ref_mhd, True)
    ctx.close()


@pytest.mark.parametrize("form", [fx.FORM_PLAIN, fx.FORM_BATCHED])
def test_sod_hydro_matches_reference(ref_hydro, form):
    p = R.params_sod(nblocks_x=8, t_end=0.2)
    ref_hydro.setup(p)
    ctx = make_ctx(ref_hydro, p, False)
    n, t_ref, dt_ref, st_ref = ref_hydro.run(25)
    t, dt, st = ctx.run(form, 25, p.cfl, p.dt_factor, p.t_end, (0.0, 0.0, 0.0))
    assert (t, dt, st) == (t_ref, dt_ref, st_ref)
    assert_state_equal(ctx, ref_hydro, False, True)
    ctx.close()


def test_divergence_free_at_roundoff(ref_mhd):
    p = R.params_fourier(root=2, nmodes=8, kmax=3)
    ref_mhd.setup(p)
    ctx = make_ctx(ref_mhd, p, True)
    ctx.run(fx.FORM_BATCHED, 5, p.cfl, p.dt_factor, p.t_end, (0.0, 0.0, 0.0))
    nb = ref_mhd.nblocks()
    W, Bf = device_state(ctx, nb, 9, True)
    r = np.arange(16)
    i, j, k = np.meshgrid(r, r, r, indexing="ij")
    for b in range(nb):
        _, g = ref_mhd.block_geom(b)
        dx = g[6:9]
        f = Bf[b, :, 0]
        div = ((f[0][H.face_idx(0, i + 1, j, k)] - f[0][H.face_idx(0, i, j, k)]) / dx[0]
               + (f[1][H.face_idx(1, i, j + 1, k)] - f[1][H.face_idx(1, i, j, k)]) / dx[1]
               + (f[2][H.face_idx(2, i, j, k + 1)] - f[2][H.face_idx(2, i, j, k)]) / dx[2])
        bmax = max(np.abs(f[d][H.active_faces(d)]).max() for d in range(3))
        assert np.abs(div).max() * dx.min() / bmax <= 1e-13
    ctx.close()


# static AMR: levels 0-2 with level-1 blocks both coarse and fine neighbours
AMR3 = dict(root=3, radii=(0.25, 0.1))


@pytest.mark.parametrize("form", [fx.FORM_PLAIN, fx.FORM_BATCHED])
def test_amr_blast_mhd_steps_match_reference(ref_mhd, form):
    p = R.params_amr_blast(**AMR3)
    ref_mhd.setup(p)
    ctx = make_ctx(ref_mhd, p, True)
    assert ctx.calc_dt(p.cfl) == ref_mhd.calc_dt()
    n, t_ref, dt_ref, st_ref = ref_mhd.run(2)
    t, dt, st = ctx.run(form, 2, p.cfl, p.dt_factor, p.t_end, (0.0, 0.0, 0.0))
    assert (t, dt, st) == (t_ref, dt_ref, st_ref)
    assert_state_equal(ctx, ref_mhd, True)
    ctx.close()


def test_amr_stage_corrections_match_reference(ref_mhd):
    """One stage on the AMR mesh: fluxes after prj_riemann_flux_send and EMFs
    after prj_mhd_emf_send, at the entries the reference computes."""
    p = R.params_amr_blast(**AMR3)
    ref_mhd.setup(p)
    ctx = make_ctx(ref_mhd, p, True)
    dt = ref_mhd.calc_dt()
    assert ctx.stage(fx.FORM_PLAIN, 1, dt) == ref_mhd.stage(1, dt)
    ints, _, _ = ref_mhd.mesh_arrays()
    for b in np.nonzero(ints[:, 2] == 1)[0]:
        for d in range(3):
            fp = H.flux_positions(d, 9, True)
            assert np.array_equal(ctx.download_array(b, fx.ARR_FLUX, d)[fp], ref_mhd.flux(b, d)[fp])
            ep = H.emf_positions(d)
            assert np.array_equal(ctx.download_array(b, fx.ARR_EMF, d)[ep], ref_mhd.emf(b, d)[ep])
    assert_state_equal(ctx, ref_mhd, True)
    ctx.close()


@pytest.mark.parametrize("form", [fx.FORM_PLAIN, fx.FORM_BATCHED])
def test_amr_hydro_steps_match_reference(ref_hydro, form):
    p = R.params_amr_blast(root=2, radii=(0.3, 0.1))
    ref_hydro.setup(p)
    ctx = make_ctx(ref_hydro, p, False)
    n, t_ref, dt_ref, st_ref = ref_hydro.run(3)
    t, dt, st = ctx.run(form, 3, p.cfl, p.dt_factor, p.t_end, (0.0, 0.0, 0.0))
    assert (t, dt, st) == (t_ref, dt_ref, st_ref)
    assert_state_equal(ctx, ref_hydro, False, True)
    ctx.close()


def test_amr_divergence_free_at_roundoff(ref_mhd):
    p = R.params_amr_blast(**AMR3)
    ref_mhd.setup(p)
    ctx = make_ctx(ref_mhd, p, True)
    ctx.run(fx.FORM_BATCHED, 4, p.cfl, p.dt_factor, p.t_end, (0.0, 0.0, 0.0))
    nb = ref_mhd.nblocks()
    W, Bf = device_state(ctx, nb, 9, True)
    ints, geom, _ = ref_mhd.mesh_arrays()
    r = np.arange(16)
    i, j, k = np.meshgrid(r, r, r, indexing="ij")
    bmax = max(np.abs(Bf[b, d, 0][H.active_faces(d)]).max() for b in range(nb) if ints[b, 2] == 1 for d in range(3))
    for b in np.nonzero(ints[:, 2] == 1)[0]:
        dx = geom[b, 6:9]
        f = Bf[b, :, 0]
        div = ((f[0][H.face_idx(0, i + 1, j, k)] - f[0][H.face_idx(0, i, j, k)]) / dx[0]
               + (f[1][H.face_idx(1, i, j + 1, k)] - f[1][H.face_idx(1, i, j, k)]) / dx[1]
               + (f[2][H.face_idx(2, i, j, k + 1)] - f[2][H.face_idx(2, i, j, k)]) / dx[2])
        assert np.abs(div).max() * dx.min() / bmax <= 1e-13
    ctx.close()


@pytest.mark.parametrize("form", [fx.FORM_PLAIN, fx.FORM_BATCHED])
def test_collapse_gravity_steps_match_reference(ref_mhd, form):
    """4-level collapse with the static gravity source: momentum and energy
    source terms and the dt_src clamp of the driver (src/main.c:555-560)."""
    p = R.params_collapse(root=4)
    ref_mhd.setup(p)
    ctx = make_ctx(ref_mhd, p, True, gravity=True)
    n, t_ref, dt_ref, st_ref = ref_mhd.run(2)
    t, dt, st = ctx.run(form, 2, p.cfl, p.dt_factor, p.t_end, (0.0, 0.0, 0.0))
    assert (t, dt, st) == (t_ref, dt_ref, st_ref)
    assert_state_equal(ctx, ref_mhd, True)
    ctx.close()


@pytest.mark.parametrize("form", [fx.FORM_PLAIN, fx.FORM_BATCHED])
def test_sod_hydro_reflect_and_user_boundaries_match_reference(ref_hydro, form):
    """Sod tube between reflecting walls in x, and with a user band at x1
    inner plus reflecting walls elsewhere; 4 x 2 x 2 blocks, 25 driver
    steps."""
    for bc in ((1, 1, 0, 0, 0, 0), (2, 1, 1, 1, 0, 0)):
        p = R.params_sod(nblocks_x=4)
        p.root[:] = [4, 2, 2]
        p.xmax[:] = [1.0, 0.5, 0.5]
        p.bc[:] = list(bc)
        ref_hydro.setup(p)
        ctx = make_ctx(ref_hydro, p, False)
        n, t_ref, dt_ref, st_ref = ref_hydro.run(25)
        t, dt, st = ctx.run(form, 25, p.cfl, p.dt_factor, p.t_end, (0.0, 0.0, 0.0))
        assert (t, dt, st) == (t_ref, dt_ref, st_ref)
        assert_state_equal(ctx, ref_hydro, False, True)
        ctx.close()


@pytest.mark.parametrize("shape", range(6))
def test_every_face_kernel_shape_is_bit_identical(ref_mhd, shape):
    """Every launch shape the autotuner chooses among reproduces the
    reference."""
    p = R.params_fourier(root=2, nmodes=8, kmax=2)
    ref_mhd.setup(p)
    ctx = make_ctx(ref_mhd, p, True)
    ctx.set_flux_shape(shape)
    n, t_ref, dt_ref, st_ref = ref_mhd.run(2)
    t, dt, st = ctx.run(fx.FORM_BATCHED, 2, p.cfl, p.dt_factor, p.t_end, (0.0, 0.0, 0.0))
    assert (t, dt, st) == (t_ref, dt_ref, st_ref)
    assert_state_equal(ctx, ref_mhd, True)
    ctx.close()
