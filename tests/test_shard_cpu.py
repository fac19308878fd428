"""Sharding over ranks on the CPU: each rank's part of the ghost fill and of
the coarse/fine corrections (fx_shard_export), run with the numpy
interpreter of the compiled programs after the exchange its lists describe,
must leave every owned block exactly as the single-device programs leave it.

The reference decomposes the block list over MPI ranks and exchanges ghost
zones and correction records (src/prj_boundary.c:1184-1222,
src/prj_mpi.c:4601); these tests check the decomposition against the
single-device compiled fill, which the other tests pin to the reference.
Halo storage starts as NaN, so a value a rank reads without receiving it
shows up as a mismatch.  One test moves the messages between two gloo
processes with torch.distributed.
"""
import socket

import numpy as np
import pytest

import fornaxamr_b200 as fx
from fornaxamr_b200 import mesh
from tests import helpers as H

COORD = (-0.7, 0.7, -0.7, 0.7, -0.7, 0.7)


def build(levels, mhd, use_bj=False):
    if levels == 0:
        blocks = mesh.uniform_mesh((2, 2, 2), COORD)
    else:
        blocks = mesh.static_amr_mesh((2, 2, 2), COORD, levels,
                                      mesh.ball_refiner((0.1, 0.05, 0.0), (0.4, 0.2)[:levels]))
    return fx.make_config(mhd, 5.0 / 3.0, COORD, use_bj=use_bj), mesh.to_desc(blocks)


def morton_owner(desc, nranks):
    return fx.morton_owner(desc, nranks)


def seeded_state(nb, mhd, seed=5):
    rng = np.random.default_rng(seed)
    W = rng.standard_normal((nb, 9 if mhd else 6, 2, H.NCELLS))
    Bf = rng.standard_normal((nb, 3, 2, H.NFACES)) if mhd else None
    return W, Bf


class Part:
    """One rank's local arrays: owned blocks from the global state, halo NaN."""

    def __init__(self, cfg, desc, owner, nranks, rank, W0, Bf0):
        self.ex = lambda which: fx.shard_export(cfg, desc, owner, nranks, rank, which)
        self.l2g, self.nown = self.ex(7)
        nl = len(self.l2g)
        self.W = np.full((nl,) + W0.shape[1:], np.nan)
        self.W[: self.nown] = W0[self.l2g[: self.nown]]
        self.Bf = None
        if Bf0 is not None:
            self.Bf = np.full((nl,) + Bf0.shape[1:], np.nan)
            self.Bf[: self.nown] = Bf0[self.l2g[: self.nown]]

    def pack(self, peer, slot):
        cl, cb = self.ex(8)
        c = cl[cb[peer]:cb[peer + 1]]
        parts = [self.W[c[:, 0], :6, slot, c[:, 1]].ravel()]
        if self.Bf is not None:
            fl, fb = self.ex(9)
            f = fl[fb[peer]:fb[peer + 1]]
            parts.append(self.Bf[f[:, 0], f[:, 1] // H.NFACES, slot, f[:, 1] % H.NFACES])
        return np.concatenate(parts)

    def recv_size(self, peer):
        cl, cb = self.ex(12)
        n = 6 * (cb[peer + 1] - cb[peer])
        if self.Bf is not None:
            fl, fb = self.ex(13)
            n += fb[peer + 1] - fb[peer]
        return int(n)

    def unpack(self, peer, slot, msg):
        cl, cb = self.ex(12)
        c = cl[cb[peer]:cb[peer + 1]]
        nc = 6 * len(c)
        self.W[c[:, 0], :6, slot, c[:, 1]] = msg[:nc].reshape(len(c), 6)
        if self.Bf is not None:
            fl, fb = self.ex(13)
            f = fl[fb[peer]:fb[peer + 1]]
            self.Bf[f[:, 0], f[:, 1] // H.NFACES, slot, f[:, 1] % H.NFACES] = msg[nc:]

    def fill(self, cfg, desc, slot):
        H.apply_ghost_program(self.W, self.Bf, cfg, desc, slot, export=self.ex, blocks=self.l2g)

    def matches(self, Wg, Bg, slot):
        own = self.l2g[: self.nown]
        ok = H.same_values(self.W[: self.nown, :, slot], Wg[own, :, slot])
        if Bg is not None:
            ok = ok and H.same_values(self.Bf[: self.nown, :, slot], Bg[own, :, slot])
        return ok


@pytest.mark.parametrize("levels,mhd,nranks,use_bj", [(0, True, 2, False), (1, True, 3, False), (1, False, 4, False),
                                                     (2, True, 3, False), (2, True, 3, True), (1, False, 4, True)])
def test_rank_parts_reproduce_the_single_device_fill(levels, mhd, nranks, use_bj):
    """use_bj: the Barth-Jespersen prolongations read the coarse cells' edge
    and corner neighbours too, so the halo exchange must carry them."""
    cfg, desc = build(levels, mhd, use_bj)
    owner = morton_owner(desc, nranks)
    W0, Bf0 = seeded_state(len(desc), mhd)
    slot = 1
    Wg, Bg = W0.copy(), None if Bf0 is None else Bf0.copy()
    H.apply_ghost_program(Wg, Bg, cfg, desc, slot)
    parts = [Part(cfg, desc, owner, nranks, r, W0, Bf0) for r in range(nranks)]
    for r, p in enumerate(parts):
        for s, q in enumerate(parts):
            if s == r:
                continue
            msg = q.pack(r, slot)
            assert len(msg) == p.recv_size(s)
            p.unpack(s, slot, msg)
    for p in parts:
        assert p.nown > 0
        p.fill(cfg, desc, slot)
        assert p.matches(Wg, Bg, slot)


def test_send_and_receive_lists_pair_up():
    cfg, desc = build(2, True)
    nranks = 3
    owner = morton_owner(desc, nranks)
    maps = [fx.shard_export(cfg, desc, owner, nranks, r, 7)[0] for r in range(nranks)]
    for k in range(4):
        for r in range(nranks):
            rl, rb = fx.shard_export(cfg, desc, owner, nranks, r, 12 + k)
            assert rb[r + 1] == rb[r]  # nothing from itself
            for s in range(nranks):
                if s == r:
                    continue
                sl, sb = fx.shard_export(cfg, desc, owner, nranks, s, 8 + k)
                a, b = rl[rb[s]:rb[s + 1]], sl[sb[r]:sb[r + 1]]
                assert np.array_equal(maps[r][a[:, 0]], maps[s][b[:, 0]])
                assert np.array_equal(a[:, 1], b[:, 1])
                assert np.all(owner[maps[r][a[:, 0]]] == s)


@pytest.mark.parametrize("levels,mhd,nranks", [(2, True, 3), (2, False, 4)])
def test_rank_parts_reproduce_the_single_device_corrections(levels, mhd, nranks):
    cfg, desc = build(levels, mhd)
    owner = morton_owner(desc, nranks)
    nb, nv = len(desc), 9 if mhd else 6
    rng = np.random.default_rng(7)
    kinds = [("flux", 2, (nb, 3, nv * H.NCELLS), nv)] + ([("emf", 3, (nb, 3, 8820), 1)] if mhd else [])
    nrec = 0
    for kind, which, shape, ncomp in kinds:
        A0 = rng.standard_normal(shape)
        Ag = A0.copy()
        recs, waves = fx.plan_export(cfg, desc, which)
        nrec += len(recs)
        H.apply_corrections(Ag, recs, waves, kind, nv)
        for r in range(nranks):
            l2g, nown = fx.shard_export(cfg, desc, owner, nranks, r, 7)
            A = np.full((len(l2g),) + shape[1:], np.nan)
            A[:nown] = A0[l2g[:nown]]
            rl, rb = fx.shard_export(cfg, desc, owner, nranks, r, 12 + which)
            flat, flat0 = A.reshape(len(l2g), -1), A0.reshape(nb, -1)
            for v in range(ncomp):
                flat[rl[:, 0], rl[:, 1] + 4 * v] = flat0[l2g[rl[:, 0]], rl[:, 1] + 4 * v]
            lr, lw = fx.shard_export(cfg, desc, owner, nranks, r, which)
            H.apply_corrections(A, lr, lw, kind, nv)
            assert H.same_values(A[:nown], Ag[l2g[:nown]])
    assert nrec > 0


def test_one_rank_is_the_single_device_plan():
    cfg, desc = build(1, True)
    owner = np.zeros(len(desc), np.int32)
    l2g, nown = fx.shard_export(cfg, desc, owner, 1, 0, 7)
    assert nown == len(l2g) == sum(d.active == 1 for d in desc)

    def glob(k, shift):  # local block key -> global block key
        return (l2g[k >> shift] << shift) | (k & ((1 << shift) - 1))
    for which, cols in ((0, ((0, 13), (1, 13))), (1, ((0, 15), (1, 15))),
                        (4, ((0, 13),) + tuple((q, 15) for q in range(1, 7))), (6, ((0, 0), (1, 0)))):
        a, aw = fx.plan_export(cfg, desc, which)
        b, bw = fx.shard_export(cfg, desc, owner, 1, 0, which)
        b = b.copy()
        for col, shift in cols:
            b[:, col] = glob(b[:, col], shift)
        assert np.array_equal(a, b) and np.array_equal(aw, bw)


def test_bad_ownership_is_rejected():
    cfg, desc = build(0, True)
    owner = morton_owner(desc, 2)
    with pytest.raises(fx.FxError):
        fx.shard_export(cfg, desc, owner, 17, 0, 7)
    bad = owner.copy()
    bad[0] = 5
    with pytest.raises(fx.FxError):
        fx.shard_export(cfg, desc, bad, 2, 0, 7)


def _gloo_rank(rank, port, q):
    import torch
    import torch.distributed as dist
    try:
        dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=2)
        cfg, desc = build(1, True)
        owner = morton_owner(desc, 2)
        W0, Bf0 = seeded_state(len(desc), True, seed=11)
        slot = 0
        part = Part(cfg, desc, owner, 2, rank, W0, Bf0)
        peer = 1 - rank
        out = torch.from_numpy(part.pack(peer, slot))
        inc = torch.empty(part.recv_size(peer), dtype=torch.float64)
        reqs = [dist.isend(out, peer), dist.irecv(inc, peer)]
        for r in reqs:
            r.wait()
        part.unpack(peer, slot, inc.numpy())
        part.fill(cfg, desc, slot)
        Wg, Bg = W0.copy(), Bf0.copy()
        H.apply_ghost_program(Wg, Bg, cfg, desc, slot)
        ok = part.matches(Wg, Bg, slot)
        dist.barrier()
        dist.destroy_process_group()
        q.put((rank, bool(ok), int(part.nown)))
    except Exception as e:  # reported to the parent
        q.put((rank, repr(e), 0))


def test_two_gloo_ranks_exchange_and_fill():
    import torch.multiprocessing as tmp
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    ctx = tmp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_gloo_rank, args=(r, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=600) for _ in procs)
    for p in procs:
        p.join(timeout=60)
    assert [r[1] for r in res] == [True, True], res
    assert all(r[2] > 0 for r in res)


def test_weak_scaling_mesh_gives_each_rank_one_cube():
    """bench.py --shard: a (8 N) x 8 x 8 root mesh over [0, N] x [0, 1]^2 cut
    into N runs of the mesh order gives every rank the 512 blocks of one
    unit cube, so each GPU holds a 128^3 sub-domain"""
    for nranks in (2, 3):
        coord = (0.0, float(nranks), 0.0, 1.0, 0.0, 1.0)
        desc = mesh.to_desc(mesh.uniform_mesh((8 * nranks, 8, 8), coord))
        owner = fx.morton_owner(desc, nranks)
        for r in range(nranks):
            mine = np.nonzero(owner == r)[0]
            assert len(mine) == 512
            xs = np.array([desc[b].xmin[0] for b in mine])
            assert xs.min() >= r - 1e-12 and xs.max() < r + 1 - 1e-12
