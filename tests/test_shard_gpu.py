"""Sharded meshes on the device: ranks emulated by contexts of one process on
one GPU (fx_shard_group: device-to-device copies between the contexts'
exchange buffers, host barriers, no kernel waiting on another rank), each
driven from its own host thread.  After the driver steps, every rank's owned
blocks (full W and Bf arrays, both stage slots) and the driver state must
equal the single-process reference bit for bit: the decomposition changes
where operations run, not what they compute.
"""
import threading

import numpy as np
import pytest

import fornaxamr_b200 as fx
from oracle import ref as R
from tests import helpers as H

pytestmark = pytest.mark.gpu


def shard_contexts(ref, p, mhd, nranks, gravity=False):
    desc = H.ref_desc(ref)
    owner = fx.morton_owner(desc, nranks)
    coord = [p.xmin[0], p.xmax[0], p.xmin[1], p.xmax[1], p.xmin[2], p.xmax[2]]
    W, Bf = H.ref_state(ref)
    group = fx.ShardGroup(nranks)
    ctxs = []
    for r in range(nranks):
        ctx = fx.Context(mhd, p.gamma, coord, bc=tuple(p.bc), gravity=gravity)
        ctx.shard_set_mesh(desc, owner, nranks, r)
        ctx.attach_group(group)
        for b in np.nonzero(owner == r)[0]:
            grav = [ref.grav(int(b), d) for d in range(3)] if gravity else None
            ctx.upload_block(int(b), W[b].ravel(), None if Bf is None else [Bf[b, d].ravel() for d in range(3)],
                             grav)
        ctxs.append(ctx)
    return ctxs, owner, group


def on_all_ranks(ctxs, fn):
    """fn(ctx) on one host thread per rank; results in rank order"""
    out = [None] * len(ctxs)
    err = []

    def work(r):
        try:
            out[r] = fn(ctxs[r])
        except Exception as e:  # re-raised below
            err.append(e)
    threads = [threading.Thread(target=work, args=(r,)) for r in range(len(ctxs))]
    for t in threads:
        t.start()
    for t in threads:
        t.join(timeout=600)
    if err:
        raise err[0]
    return out


def assert_owned_equal(ctxs, owner, ref, mhd):
    W_ref, Bf_ref = H.ref_state(ref)
    for r, ctx in enumerate(ctxs):
        for b in np.nonzero(owner == r)[0]:
            W, _, Bf = ctx.download_block(int(b))
            assert np.array_equal(W, W_ref[b].ravel()), (r, b)
            if mhd:
                for d in range(3):
                    assert np.array_equal(Bf[d], Bf_ref[b, d].ravel()), (r, b, d)


def run_and_compare(ref, p, mhd, nranks, nsteps, gravity=False):
    ctxs, owner, group = shard_contexts(ref, p, mhd, nranks, gravity)
    dts = on_all_ranks(ctxs, lambda c: c.calc_dt(p.cfl))
    assert dts == [ref.calc_dt()] * nranks
    states = on_all_ranks(ctxs, lambda c: c.run(fx.FORM_BATCHED, nsteps, p.cfl, p.dt_factor, p.t_end,
                                                (0.0, 0.0, 0.0)))
    n, t_ref, dt_ref, st_ref = ref.run(nsteps)
    assert states == [(t_ref, dt_ref, st_ref)] * nranks
    assert_owned_equal(ctxs, owner, ref, mhd)
    info = [c.shard_info() for c in ctxs]
    assert sum(i[0] for i in info) == int((owner >= 0).sum())
    for c in ctxs:
        c.close()
    group.close()
    return info


@pytest.mark.parametrize("nranks", [2, 3])
def test_fourier_mhd_on_ranks_matches_reference(ref_mhd, nranks):
    p = R.params_fourier(root=2, nmodes=8, kmax=2)
    ref_mhd.setup(p)
    info = run_and_compare(ref_mhd, p, True, nranks, 3)
    assert all(i[2] > 0 for i in info)  # halo cells and faces cross ranks


@pytest.mark.parametrize("nranks", [2, 4])
def test_amr_blast_on_ranks_matches_reference(ref_mhd, nranks):
    """3 levels: coarse/fine flux and EMF records whose fine blocks sit on
    other ranks, prolongation and restriction across ranks"""
    p = R.params_amr_blast(root=3, radii=(0.25, 0.1))
    ref_mhd.setup(p)
    run_and_compare(ref_mhd, p, True, nranks, 2)


def test_sod_hydro_on_ranks_matches_reference(ref_hydro):
    p = R.params_sod(nblocks_x=8)
    ref_hydro.setup(p)
    run_and_compare(ref_hydro, p, False, 3, 4)


def test_collapse_gravity_on_ranks_matches_reference(ref_mhd):
    p = R.params_collapse(root=4)
    ref_mhd.setup(p)
    run_and_compare(ref_mhd, p, True, 2, 2, gravity=True)


def test_steps_with_fixed_dt_on_ranks(ref_mhd):
    """fx_step with a given dt: the dt_src minimum is taken over the ranks"""
    p = R.params_amr_blast(root=2, max_level=1, radii=(0.4,))
    ref_mhd.setup(p)
    ctxs, owner, group = shard_contexts(ref_mhd, p, True, 2)
    dt = ref_mhd.calc_dt()
    src = on_all_ranks(ctxs, lambda c: c.step(fx.FORM_BATCHED, dt))
    ref_src = ref_mhd.step(dt)
    assert src == [ref_src, ref_src]
    assert_owned_equal(ctxs, owner, ref_mhd, True)
    for c in ctxs:
        c.close()
    group.close()


def test_sharded_context_rejects_what_it_does_not_run(ref_mhd):
    p = R.params_fourier(root=2, nmodes=4, kmax=1)
    ref_mhd.setup(p)
    ctxs, owner, group = shard_contexts(ref_mhd, p, True, 2)
    c = ctxs[0]
    other = int(np.nonzero(owner == 1)[0][0])
    with pytest.raises(fx.FxError):
        c.download_block(other)
    with pytest.raises(fx.FxError):
        c.step(fx.FORM_PLAIN, 1e-3)
    with pytest.raises(fx.FxError):
        c.flux_update(0, 0, 0)
    for c in ctxs:
        c.close()
    group.close()


def test_nccl_transport_attaches_on_one_rank(ref_mhd):
    """one-rank NCCL communicator on the sharded path (the exchanges of a
    single rank are empty; several ranks need one GPU each)"""
    p = R.params_fourier(root=2, nmodes=4, kmax=1)
    ref_mhd.setup(p)
    desc = H.ref_desc(ref_mhd)
    owner = fx.morton_owner(desc, 1)
    coord = [p.xmin[0], p.xmax[0], p.xmin[1], p.xmax[1], p.xmin[2], p.xmax[2]]
    ctx = fx.Context(True, p.gamma, coord, bc=tuple(p.bc))
    ctx.shard_set_mesh(desc, owner, 1, 0)
    ctx.attach_nccl(fx.nccl_unique_id())
    W, Bf = H.ref_state(ref_mhd)
    for b in range(len(desc)):
        ctx.upload_block(b, W[b].ravel(), [Bf[b, d].ravel() for d in range(3)])
    state = ctx.run(fx.FORM_BATCHED, 2, p.cfl, p.dt_factor, p.t_end, (0.0, 0.0, 0.0))
    n, t_ref, dt_ref, st_ref = ref_mhd.run(2)
    assert state == (t_ref, dt_ref, st_ref)
    assert_owned_equal([ctx], owner, ref_mhd, True)
    ctx.close()


def test_ghost_fill_on_ranks_matches_reference(ref_mhd):
    """fx_boundary_fill_ghosts_and_bf on a sharded mesh, from ghost zones
    scrambled on both sides (3-level blast, 3 ranks)"""
    p = R.params_amr_blast(root=3, radii=(0.25, 0.1))
    ref_mhd.setup(p)
    W, Bf = H.ref_state(ref_mhd)
    rng = np.random.default_rng(3)
    ghost = np.ones(H.NCELLS, bool)
    ghost[H.active_cells()] = False
    active = ref_mhd.mesh_arrays()[0][:, 2] == 1
    for b in np.nonzero(active)[0]:
        W[b][:, :, ghost] = rng.uniform(0.5, 1.5, (W.shape[1], W.shape[2], int(ghost.sum())))
        ref_mhd.set_W(int(b), W[b].ravel())
    ctxs, owner, group = shard_contexts(ref_mhd, p, True, 3)
    on_all_ranks(ctxs, lambda c: c.boundary_fill(1, 0))
    ref_mhd.fill_ghosts(1, 0)
    W_ref, Bf_ref = H.ref_state(ref_mhd)
    for r, ctx in enumerate(ctxs):
        for b in np.nonzero(owner == r)[0]:
            Wd, _, Bd = ctx.download_block(int(b))
            assert np.array_equal(Wd.reshape(W_ref[b].shape)[:, 0], W_ref[b][:, 0]), (r, b)
            for d in range(3):
                assert np.array_equal(Bd[d].reshape(2, -1)[0], Bf_ref[b, d, 0]), (r, b, d)
    for c in ctxs:
        c.close()
    group.close()
