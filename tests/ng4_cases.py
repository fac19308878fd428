"""Four-ghost-layer build (FX_NGHOST=4: libfornax_b200_ng4.so, 24^3 block
arrays) against the reference compiled with PRJ_NGHOST=4: MC reconstruction
(oracle variant *_ng4) and WENO-Z7 (PRJ_RECON_HYDRO = PRJ_RECON_WENO7, which
selects four ghost layers itself).  Both sides run the driver loop of
src/main.c from identical inputs; every block array (both stage slots) must
agree bit for bit.

The layout is fixed per process, so this module runs in a child process
with FX_NGHOST=4 (tests/test_ng4.py starts it); it is not collected by a
plain `pytest tests`.
"""
import numpy as np
import pytest

import fornaxamr_b200 as fx
from oracle import ref as R
from tests import helpers as H

assert fx.NG == 4 and R.NG == 4, "run with FX_NGHOST=4"


def make_ctx(ref, p, mhd, recon):
    desc = H.ref_desc(ref)
    coord = [p.xmin[0], p.xmax[0], p.xmin[1], p.xmax[1], p.xmin[2], p.xmax[2]]
    ctx = fx.Context(mhd, p.gamma, coord, bc=tuple(p.bc), recon=recon)
    ctx.set_mesh(desc)
    W, Bf = H.ref_state(ref)
    for b in range(W.shape[0]):
        ctx.upload_block(b, W[b].ravel(), None if Bf is None else [Bf[b, d].ravel() for d in range(3)])
    return ctx


def assert_state_equal(ctx, ref, mhd, active_only=False):
    W_ref, Bf_ref = H.ref_state(ref)
    nb, nv, ns = W_ref.shape[:3]
    W = np.empty((nb, nv, ns, H.NCELLS))
    Bf = np.empty((nb, 3, ns, H.NFACES)) if mhd else None
    ctx.download_all(W, Bf)
    sel = slice(None)
    if active_only:
        sel = ref.mesh_arrays()[0][:, 2] == 1
    assert H.same_values(W[sel], W_ref[sel])
    if mhd:
        assert H.same_values(Bf[sel], Bf_ref[sel])


def run_case(ref, p, mhd, recon, form, nsteps, active_only=False):
    ctx = make_ctx(ref, p, mhd, recon)
    assert ctx.calc_dt(p.cfl) == ref.calc_dt()
    n, t_ref, dt_ref, st_ref = ref.run(nsteps)
    t, dt, st = ctx.run(form, nsteps, p.cfl, p.dt_factor, p.t_end, (0.0, 0.0, 0.0))
    assert (t, dt, st) == (t_ref, dt_ref, st_ref)
    assert_state_equal(ctx, ref, mhd, active_only)
    ctx.close()


def test_layout_constants():
    assert (H.PBS, H.NCELLS, H.NFACES, H.NEDGES) == (24, 13824, 14400, 15000)
    assert fx.library().fx_ghost_layers() == 4


@pytest.mark.gpu
@pytest.mark.parametrize("form", [fx.FORM_PLAIN, fx.FORM_BATCHED])
def test_fourier_mhd_mc_four_ghosts_matches_reference(form):
    ref = R.Reference(True)
    p = R.params_fourier(root=2)
    ref.setup(p)
    run_case(ref, p, True, fx.RECON_MC, form, 3)


@pytest.mark.gpu
@pytest.mark.parametrize("form", [fx.FORM_PLAIN, fx.FORM_BATCHED])
def test_fourier_mhd_weno7_matches_reference(form):
    ref = R.Reference(True, "weno7")
    p = R.params_fourier(root=2)
    ref.setup(p)
    run_case(ref, p, True, fx.RECON_WENO7, form, 3)


@pytest.mark.gpu
def test_sod_hydro_weno7_matches_reference():
    ref = R.Reference(False, "weno7")
    p = R.params_sod(nblocks_x=8)
    ref.setup(p)
    run_case(ref, p, False, fx.RECON_WENO7, fx.FORM_BATCHED, 4)


@pytest.mark.gpu
def test_amr_blast_weno7_matches_reference():
    """3 static levels: restriction, limited prolongation and the Toth-Roe
    face groups over four ghost layers, coarse/fine flux and EMF records"""
    ref = R.Reference(True, "weno7")
    p = R.params_amr_blast(root=3, radii=(0.25, 0.1))
    ref.setup(p)
    run_case(ref, p, True, fx.RECON_WENO7, fx.FORM_BATCHED, 2, active_only=False)


@pytest.mark.gpu
def test_weno7_face_value_matches_reference_on_random_stencils():
    """The face kernel's WENO-Z7 against the reference's, through full
    steps of a rough state: random Fourier amplitudes large enough that the
    nonlinear weights move away from the linear ones"""
    ref = R.Reference(True, "weno7")
    p = R.params_fourier(root=2, nmodes=32, kmax=4, amp_rho=0.4, amp_v=0.3, amp_A=0.1)
    ref.setup(p)
    run_case(ref, p, True, fx.RECON_WENO7, fx.FORM_BATCHED, 2)


def test_weno7_context_needs_four_ghosts_build():
    cfg = fx.make_config(True, 5.0 / 3.0, (0, 1, 0, 1, 0, 1), recon=fx.RECON_WENO7)
    assert cfg.recon == fx.RECON_WENO7


@pytest.mark.gpu
def test_weno7_every_launch_shape_matches_reference():
    """the autotuner's six launch shapes of the WENO-Z7 face kernel (register
    caps from 80 to 128, some with spills) give the same bits"""
    ref = R.Reference(True, "weno7")
    p = R.params_fourier(root=2, nmodes=16, kmax=3, amp_rho=0.3)
    ref.setup(p)
    ctxs = []
    for v in range(6):
        ctx = make_ctx(ref, p, True, fx.RECON_WENO7)
        ctx.set_flux_shape(v)
        ctxs.append(ctx)
    n, t_ref, dt_ref, st_ref = ref.run(2)
    for ctx in ctxs:
        t, dt, st = ctx.run(fx.FORM_BATCHED, 2, p.cfl, p.dt_factor, p.t_end, (0.0, 0.0, 0.0))
        assert (t, dt, st) == (t_ref, dt_ref, st_ref)
        assert_state_equal(ctx, ref, True)
        ctx.close()


def _amr(ctx, ref, p, crit, max_level):
    ctx.amr_configure(fx.amr_config(tuple(p.root), max_level, [crit]))
    ref.amr_configure(R.amr_params(max_level, [dict(estimator=crit["estimator"], refine=crit["refine"],
                                                    derefine=crit["derefine"], lohner_var=crit.get("var", 1),
                                                    jump_var=min(crit.get("var", 1), 1),
                                                    eps=crit.get("eps", 0.1))]))


def _mesh_equal(ctx, ref):
    from fornaxamr_b200 import mesh
    i2, g2, s2 = ref.mesh_arrays()
    mi, mg, ms = mesh.desc_to_arrays(ctx.get_mesh())
    assert np.array_equal(i2, mi) and np.array_equal(g2, mg) and np.array_equal(s2, ms)


@pytest.mark.gpu
def test_dynamic_amr_weno7_matches_reference():
    """prj_amr_adapt on the four-ghost layout: device tag votes, host remesh
    (slot boxes of four ghost layers), prolongation and restriction of cells
    and faces, recompiled fill; refine, step, then coarsen"""
    ref = R.Reference(True, "weno7")
    p = R.params_amr_blast(root=2, max_level=1, radii=(0.4,))
    ref.setup(p)
    _, t0, dt0, st0 = ref.run(2)
    ctx = make_ctx(ref, p, True, fx.RECON_WENO7)
    _amr(ctx, ref, p, dict(estimator=fx.AMR_LOEHNER, refine=0.3, derefine=0.1, var=1), 2)
    assert np.array_equal(ctx.amr_tag(), ref.amr_tag())
    assert ctx.amr_adapt() == bool(ref.amr_adapt()) is True
    _mesh_equal(ctx, ref)
    assert_state_equal(ctx, ref, True, active_only=True)
    n, t_ref, dt_ref, st_ref = ref.run(1)
    t, dt, st = ctx.run(fx.FORM_BATCHED, 1, p.cfl, p.dt_factor, p.t_end, (t0, dt0, st0))
    assert (t, dt, st) == (t_ref, dt_ref, st_ref)
    _amr(ctx, ref, p, dict(estimator=fx.AMR_LOEHNER, refine=100.0, derefine=100.0, var=1), 2)
    assert ctx.amr_adapt() == bool(ref.amr_adapt()) is True
    _mesh_equal(ctx, ref)
    assert_state_equal(ctx, ref, True, active_only=True)
    ctx.close()


@pytest.mark.gpu
def test_essprk_weno7_matches_reference():
    """the reference's default integrator (eSSPRK10_4, three stage slots)
    with WENO-Z7, both forms' batched path on the Fourier workload"""
    ref = R.Reference(True, "ess_weno7")
    p = R.params_fourier(root=2)
    ref.setup(p)
    desc = H.ref_desc(ref)
    coord = [p.xmin[0], p.xmax[0], p.xmin[1], p.xmax[1], p.xmin[2], p.xmax[2]]
    ctx = fx.Context(True, p.gamma, coord, bc=tuple(p.bc), recon=fx.RECON_WENO7, integrator=fx.INT_ESSPRK10_4)
    ctx.set_mesh(desc)
    W, Bf = H.ref_state(ref)
    for b in range(W.shape[0]):
        ctx.upload_block(b, W[b].ravel(), [Bf[b, d].ravel() for d in range(3)])
    assert ctx.calc_dt(p.cfl) == ref.calc_dt()
    n, t_ref, dt_ref, st_ref = ref.run(2)
    t, dt, st = ctx.run(fx.FORM_BATCHED, 2, p.cfl, p.dt_factor, p.t_end, (0.0, 0.0, 0.0))
    assert (t, dt, st) == (t_ref, dt_ref, st_ref)
    assert_state_equal(ctx, ref, True)
    ctx.close()


@pytest.mark.gpu
def test_sharded_weno7_on_emulated_ranks_matches_reference():
    """a mesh sharded over three ranks (contexts of one process on one GPU)
    on the four-ghost layout with WENO-Z7: halo exchanges of four ghost
    layers and the wider stencil"""
    import threading
    ref = R.Reference(True, "weno7")
    p = R.params_amr_blast(root=3, radii=(0.25, 0.1))
    ref.setup(p)
    desc = H.ref_desc(ref)
    nranks = 3
    owner = fx.morton_owner(desc, nranks)
    coord = [p.xmin[0], p.xmax[0], p.xmin[1], p.xmax[1], p.xmin[2], p.xmax[2]]
    W, Bf = H.ref_state(ref)
    group = fx.ShardGroup(nranks)
    ctxs = []
    for r in range(nranks):
        ctx = fx.Context(True, p.gamma, coord, bc=tuple(p.bc), recon=fx.RECON_WENO7)
        ctx.shard_set_mesh(desc, owner, nranks, r)
        ctx.attach_group(group)
        for b in np.nonzero(owner == r)[0]:
            ctx.upload_block(int(b), W[b].ravel(), [Bf[b, d].ravel() for d in range(3)])
        ctxs.append(ctx)
    out, err = [None] * nranks, []

    def work(r):
        try:
            out[r] = ctxs[r].run(fx.FORM_BATCHED, 2, p.cfl, p.dt_factor, p.t_end, (0.0, 0.0, 0.0))
        except Exception as e:
            err.append(e)
    threads = [threading.Thread(target=work, args=(r,)) for r in range(nranks)]
    for t in threads:
        t.start()
    for t in threads:
        t.join(timeout=600)
    assert not err, err
    n, t_ref, dt_ref, st_ref = ref.run(2)
    assert out == [(t_ref, dt_ref, st_ref)] * nranks
    W_ref, Bf_ref = H.ref_state(ref)
    for r, ctx in enumerate(ctxs):
        for b in np.nonzero(owner == r)[0]:
            Wd, _, Bd = ctx.download_block(int(b))
            assert np.array_equal(Wd, W_ref[b].ravel()), (r, b)
            for d in range(3):
                assert np.array_equal(Bd[d], Bf_ref[b, d].ravel()), (r, b, d)
        ctx.close()
    group.close()
