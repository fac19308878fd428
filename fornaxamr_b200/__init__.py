"""fornaxamr_b200: B200-native per-block Godunov MHD update of FornaxAMR.

The compute path is the native library libfornax_b200.so (hand-written
sm_100a CUDA behind the C ABI in include/fornax_b200.h).  This package is a
thin host-side front-end: ctypes bindings, mesh descriptions and workload
generators.  It never computes the update itself; without the native library
the import fails.
"""
from __future__ import annotations

import ctypes as C
from typing import Optional, Sequence

import numpy as np

from . import _lib
from ._lib import (ARR_BF, ARR_BV1, ARR_BV2, ARR_EMF, ARR_EOSVAR, ARR_FLUX, ARR_GRAV, ARR_RHS,
                   ARR_VRIEMANN, ARR_W, BC_OUTFLOW, BC_PERIODIC, BC_REFLECT, BC_USER, FORM_BATCHED,
                   FORM_PLAIN, PHASE_CELLS, PHASE_CT, PHASE_EMF, PHASE_FLUX, PHASE_GHOST, PHASE_STEP,
                   AMR_FRACTIONAL_JUMP, AMR_LOEHNER, AMR_PRESSURE_SCALE_HEIGHT, AMR_VAR_DENSITY,
                   AMR_VAR_PRESSURE, AMR_VAR_TEMPERATURE, AMR_VELOCITY, INT_ESSPRK10_4, INT_RK2,
                   RECON_MC, RECON_WENO3, RECON_WENO7, FxAmrConfig, FxBlockDesc, FxConfig)

__all__ = ["Context", "FxError", "FORM_PLAIN", "FORM_BATCHED", "NCELLS", "NFACES", "NEDGES",
           "library", "plan_export", "amr_config", "amr_remesh_host"]

from .layout import NCELLS, NEDGES, NFACES, NG  # noqa: E402  (sizes of the loaded build)
NSTAGES = 2

_L: Optional[C.CDLL] = None


def library() -> C.CDLL:
    global _L
    if _L is None:
        _L = _lib.load()
    return _L


class FxError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"fornax_b200 error {code}: {msg}")
        self.code = code


def _dp(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def make_config(mhd: bool, gamma: float, coord: Sequence[float], bc: Sequence[int] = (0,) * 6,
                gravity: bool = False, mhd_eta: float = 0.0, recon: int = RECON_MC,
                integrator: int = INT_RK2, use_bj: bool = False) -> FxConfig:
    cfg = FxConfig()
    cfg.use_bj = 1 if use_bj else 0
    cfg.recon = int(recon)
    cfg.integrator = int(integrator)
    cfg.mhd = 1 if mhd else 0
    cfg.gravity = 1 if gravity else 0
    cfg.gamma = float(gamma)
    for n in range(6):
        cfg.coord[n] = float(coord[n])
        cfg.bc[n] = int(bc[n])
    cfg.mhd_eta = float(mhd_eta)
    return cfg


def amr_config(root_nx: Sequence[int], max_level: int, criteria: Sequence[dict] = (),
               max_blocks: int = 65535, min_dx: float = 0.0, reach_density: float = -1.0,
               E_floor: float = -1.0) -> FxAmrConfig:
    """fx_amr_config from up to four criteria, each a dict with keys
    estimator (AMR_*), refine, derefine and optionally var (Loehner or jump
    variable, AMR_VAR_*) and eps; unset fields take the reference's defaults
    (src/prj_io.c:341-355: thresholds 0.5 / 0.2, pressure, eps 0.1)."""
    a = FxAmrConfig()
    for d in range(3):
        a.root_nx[d] = int(root_nx[d])
    a.max_level = int(max_level)
    a.max_blocks = int(max_blocks)
    a.min_dx = float(min_dx)
    a.reach_density = float(reach_density)
    a.E_floor = float(E_floor)
    for n in range(_lib.AMR_N):
        k = a.crit[n]
        k.set = 0
        k.estimator = AMR_LOEHNER
        k.lohner_var = AMR_VAR_PRESSURE
        k.jump_var = AMR_VAR_PRESSURE
        k.refine_thresh = 0.5
        k.derefine_thresh = 0.2
        k.lohner_eps = 0.1
    for n, c in enumerate(criteria):
        k = a.crit[n]
        k.set = 1
        k.estimator = int(c["estimator"])
        k.refine_thresh = float(c.get("refine", 0.5))
        k.derefine_thresh = float(c.get("derefine", 0.2))
        var = int(c.get("var", AMR_VAR_PRESSURE))
        k.lohner_var = var
        k.jump_var = min(var, 1)
        k.lohner_eps = float(c.get("eps", 0.1))
    return a


def amr_remesh_host(cfg: FxConfig, amr: FxAmrConfig, desc, votes: np.ndarray, capacity: int = 0):
    """Host-only block-tree half of prj_amr_adapt for given pass-1 votes
    (int32 [nblocks, 3]): returns (flags after the tag caps, new desc)."""
    L = library()
    nb = len(desc)
    cap = capacity or max(4 * nb, nb + 64)
    out = (FxBlockDesc * cap)()
    flags = np.zeros(nb, dtype=np.int32)
    v = np.ascontiguousarray(votes, dtype=np.int32).reshape(-1)
    nout = C.c_int(0)
    ip = C.POINTER(C.c_int32)
    rc = L.fx_amr_remesh_host(C.byref(cfg), C.byref(amr), nb, desc, v.ctypes.data_as(ip),
                              flags.ctypes.data_as(ip), cap, out, C.byref(nout))
    if rc != 0:
        raise FxError(rc, "fx_amr_remesh_host failed")
    res = (FxBlockDesc * nout.value)()
    C.memmove(res, out, C.sizeof(FxBlockDesc) * nout.value)
    return flags, res


def dump_metadata(desc) -> np.ndarray:
    """fx_dump_metadata: the MetaData rows of prj_io_write_dump."""
    out = np.zeros((len(desc), _lib.DUMP_METADATA_SIZE))
    rc = library().fx_dump_metadata(len(desc), desc, out.ctypes.data)
    if rc != 0:
        raise FxError(rc, "fx_dump_metadata failed")
    return out


def plan_export(cfg: FxConfig, desc, which: int):
    """Host-only dump of the compiled ghost fill: which = 0 cell ops, 1 face
    ops, 4 cell-field ops, 6 face-prolongation groups -> (ops [n, 4 or 8]
    int32, wave_begin); 2/3 the flux/EMF correction records with their wave
    offsets; 5 compiler statistics (emitted cell ops, emitted face ops,
    rewired copies, dead writes)."""
    L = library()
    nops = C.c_int(0)
    nwaves = C.c_int(0)
    rc = L.fx_plan_export(C.byref(cfg), len(desc), desc, which, None, C.byref(nops), None, C.byref(nwaves))
    if rc != 0:
        raise FxError(rc, "fx_plan_export failed")
    width = 4 if which in (0, 1) else 1 if which == 5 else 8
    ops = np.zeros((max(nops.value, 1), width), dtype=np.int32)
    waves = np.zeros(nwaves.value + 1, dtype=np.int32)
    rc = L.fx_plan_export(C.byref(cfg), len(desc), desc, which,
                          ops.ctypes.data_as(C.POINTER(C.c_int32)), C.byref(nops),
                          waves.ctypes.data_as(C.POINTER(C.c_int32)), C.byref(nwaves))
    if rc != 0:
        raise FxError(rc, "fx_plan_export failed")
    return ops[: nops.value], waves


def shard_export(cfg: FxConfig, desc, owner, nranks: int, rank: int, which: int):
    """Host-only dump of rank `rank`'s part of a sharded mesh
    (fx_shard_export): which 0, 1, 4, 6 -> (ops, wave_begin) as plan_export
    in the rank's local block numbering; 2 / 3 the correction records; 7 ->
    (local-to-global block map, owned block count); 8 + k / 12 + k -> the send
    / receive list of exchange k (0 cells, 1 faces, 2 flux, 3 EMF) as
    ((local block, index) pairs [n, 2], per-peer offsets [nranks + 1])."""
    L = library()
    own = np.ascontiguousarray(owner, dtype=np.int32)
    ip = C.POINTER(C.c_int32)
    nops = C.c_int(0)
    nwaves = C.c_int(0)
    rc = L.fx_shard_export(C.byref(cfg), len(desc), desc, own.ctypes.data_as(ip), nranks, rank, which,
                           None, C.byref(nops), None, C.byref(nwaves))
    if rc != 0:
        raise FxError(rc, "fx_shard_export failed")
    width = 4 if which in (0, 1) else 1 if which == 7 else 2 if which >= 8 else 8
    ops = np.zeros((max(nops.value, 1), width), dtype=np.int32)
    waves = np.zeros(nwaves.value + 1, dtype=np.int32)
    rc = L.fx_shard_export(C.byref(cfg), len(desc), desc, own.ctypes.data_as(ip), nranks, rank, which,
                           ops.ctypes.data_as(ip), C.byref(nops), waves.ctypes.data_as(ip), C.byref(nwaves))
    if rc != 0:
        raise FxError(rc, "fx_shard_export failed")
    if which == 7:
        return ops[: nops.value, 0].copy(), nwaves.value
    return ops[: nops.value], waves


class ShardGroup:
    """Ranks of a sharded mesh emulated inside one process
    (fx_shard_group_create): one context per rank, each driven from its own
    host thread; every rank makes the same calls in the same order."""

    def __init__(self, nranks: int):
        self.L = library()
        self._g = self.L.fx_shard_group_create(int(nranks))
        if not self._g:
            raise FxError(1, "fx_shard_group_create: nranks outside [1, 16]")
        self.nranks = int(nranks)

    def close(self) -> None:
        if self._g:
            self.L.fx_shard_group_destroy(self._g)
            self._g = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def nccl_unique_id() -> bytes:
    """fx_nccl_unique_id: the 128-byte id rank 0 shares with the other
    ranks before fx_shard_attach_nccl."""
    buf = (C.c_ubyte * 128)()
    rc = library().fx_nccl_unique_id(buf)
    if rc != 0:
        raise FxError(rc, "fx_nccl_unique_id failed (libnccl.so.2 not loadable?)")
    return bytes(buf)


def morton_owner(desc, nranks: int) -> np.ndarray:
    """owner[b] for fx_shard_set_mesh: the active blocks in mesh order (the
    reference's Morton order) cut into nranks contiguous runs of equal size,
    the unweighted form of prj_mpi_decompose (src/prj_mpi.c:375-470);
    inactive entries get -1."""
    active = [b for b in range(len(desc)) if desc[b].active == 1]
    owner = np.full(len(desc), -1, np.int32)
    for q, b in enumerate(active):
        owner[b] = q * nranks // len(active)
    return owner


class Context:
    """One device context (fx_ctx) with a mesh mirror."""

    def __init__(self, mhd: bool, gamma: float, coord: Sequence[float], bc: Sequence[int] = (0,) * 6,
                 gravity: bool = False, mhd_eta: float = 0.0, device: int = 0, recon: int = RECON_MC,
                 integrator: int = INT_RK2, use_bj: bool = False):
        self.L = library()
        self.mhd = bool(mhd)
        self.nv = 9 if mhd else 6
        # stage slots of the block W / Bf arrays: 2 (RK2) or 3 (eSSPRK10_4)
        self.ns = 3 if integrator == INT_ESSPRK10_4 else 2
        self.cfg = make_config(mhd, gamma, coord, bc, gravity, mhd_eta, recon, integrator, use_bj)
        self._h = C.c_void_p()
        rc = self.L.fx_create(device, C.byref(self.cfg), C.byref(self._h))
        if rc != 0:
            raise FxError(rc, "fx_create failed (is a GPU present?)")
        self.nblocks = 0

    # -- plumbing ---------------------------------------------------------------
    def _check(self, rc: int) -> None:
        if rc != 0:
            buf = C.create_string_buffer(512)
            self.L.fx_last_error(self._h, buf, 512)
            raise FxError(rc, buf.value.decode())

    def close(self) -> None:
        if self._h:
            self.L.fx_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def sync(self) -> None:
        self._check(self.L.fx_sync(self._h))

    def stream(self) -> int:
        p = C.c_void_p()
        self._check(self.L.fx_stream(self._h, C.byref(p)))
        return p.value or 0

    # -- mesh and data ------------------------------------------------------------
    def set_mesh(self, desc) -> None:
        self._check(self.L.fx_set_mesh(self._h, len(desc), desc))
        self.nblocks = len(desc)

    def shard_set_mesh(self, desc, owner, nranks: int, rank: int) -> None:
        """fx_shard_set_mesh: this context becomes rank `rank` of the mesh;
        blocks are then addressed by their mesh index (owned ones only)."""
        own = np.ascontiguousarray(owner, dtype=np.int32)
        self._check(self.L.fx_shard_set_mesh(self._h, len(desc), desc, own.ctypes.data_as(C.POINTER(C.c_int32)),
                                             int(nranks), int(rank)))
        self.nblocks = len(desc)
        self._group = None

    def attach_group(self, group: "ShardGroup") -> None:
        self._check(self.L.fx_shard_attach_group(self._h, group._g))
        self._group = group  # the group outlives the context's use of it

    def attach_nccl(self, uid: bytes) -> None:
        buf = (C.c_ubyte * 128).from_buffer_copy(uid)
        self._check(self.L.fx_shard_attach_nccl(self._h, buf))

    def shard_info(self):
        """(owned blocks, local blocks incl. halo, doubles sent per step)"""
        a, b, n = C.c_int(0), C.c_int(0), C.c_longlong(0)
        self._check(self.L.fx_shard_info(self._h, C.byref(a), C.byref(b), C.byref(n)))
        return a.value, b.value, n.value

    def upload_block(self, b: int, W: np.ndarray, Bf=None, grav=None) -> None:
        W = np.ascontiguousarray(W, dtype=np.float64)
        keep = [W]
        bfp = None
        if Bf is not None:
            arrs = [np.ascontiguousarray(x, dtype=np.float64) for x in Bf]
            keep += arrs
            bfp = (C.POINTER(C.c_double) * 3)(*[_dp(x) for x in arrs])
        gp = None
        if grav is not None:
            arrs = [np.ascontiguousarray(x, dtype=np.float64) for x in grav]
            keep += arrs
            gp = (C.POINTER(C.c_double) * 3)(*[_dp(x) for x in arrs])
        self._check(self.L.fx_upload_block(self._h, b, _dp(W), bfp, gp))

    def download_block(self, b: int):
        W = np.empty(self.nv * self.ns * NCELLS)
        eos = np.empty(3 * NCELLS)
        bfp = None
        Bf = None
        if self.mhd:
            Bf = [np.empty(self.ns * NFACES) for _ in range(3)]
            bfp = (C.POINTER(C.c_double) * 3)(*[_dp(x) for x in Bf])
        self._check(self.L.fx_download_block(self._h, b, _dp(W), _dp(eos), bfp))
        return W, eos, Bf

    def upload_all(self, W_all: Optional[np.ndarray], Bf_all: Optional[np.ndarray]) -> None:
        w = None if W_all is None else _dp(W_all)
        f = None if Bf_all is None else _dp(Bf_all)
        self._check(self.L.fx_upload_all(self._h, w, f))

    def download_all(self, W_all: Optional[np.ndarray], Bf_all: Optional[np.ndarray]) -> None:
        w = None if W_all is None else _dp(W_all)
        f = None if Bf_all is None else _dp(Bf_all)
        self._check(self.L.fx_download_all(self._h, w, f))

    def upload_state(self, W_all: Optional[np.ndarray], Bf_all: Optional[np.ndarray]) -> None:
        """Stage slot 0 only (the layout of upload_all, ns slots per block)."""
        Wc = None if W_all is None else np.ascontiguousarray(W_all, dtype=np.float64)
        Bc = None if Bf_all is None else np.ascontiguousarray(Bf_all, dtype=np.float64)
        self._check(self.L.fx_upload_state(self._h, None if Wc is None else _dp(Wc),
                                           None if Bc is None else _dp(Bc)))
        self.sync()  # the host arrays must outlive the copies

    def download_state(self, W_all: Optional[np.ndarray], Bf_all: Optional[np.ndarray]) -> None:
        w = None if W_all is None else _dp(W_all)
        f = None if Bf_all is None else _dp(Bf_all)
        self._check(self.L.fx_download_state(self._h, w, f))
        self.sync()

    def upload_state_active(self, W_all: np.ndarray, Bf_all: Optional[np.ndarray]) -> None:
        """fx_upload_state_active: slot 0 of the active cells and faces from
        page-locked host arrays (e.g. torch pin_memory), then the ghost fill."""
        self._check(self.L.fx_upload_state_active(self._h, W_all.ctypes.data,
                                                  None if Bf_all is None else Bf_all.ctypes.data))

    def download_state_active(self, W_all: np.ndarray, Bf_all: Optional[np.ndarray]) -> None:
        self._check(self.L.fx_download_state_active(self._h, W_all.ctypes.data,
                                                    None if Bf_all is None else Bf_all.ctypes.data))

    def dump_gather(self, bf: bool = False):
        """fx_dump_gather: the Data, Eos (and Bf) dataset contents of
        prj_io_write_dump; rows of non-active entries stay zero."""
        nb = self.nblocks
        data = np.zeros((nb, self.nv, 16 ** 3))
        eos = np.zeros((nb, 3, 16 ** 3))
        bfa = np.zeros((nb, 3, NFACES)) if (bf and self.mhd) else None
        self._check(self.L.fx_dump_gather(self._h, data.ctypes.data, eos.ctypes.data,
                                          None if bfa is None else bfa.ctypes.data))
        return data, eos, bfa

    def download_array(self, b: int, which: int, dir_: int = 0) -> np.ndarray:
        sizes = {ARR_W: self.nv * self.ns * NCELLS, ARR_EOSVAR: 3 * NCELLS, ARR_RHS: self.nv * NCELLS,
                 ARR_FLUX: self.nv * NCELLS, ARR_VRIEMANN: 3 * NCELLS, ARR_GRAV: NCELLS,
                 ARR_BF: self.ns * NFACES, ARR_BV1: NCELLS, ARR_BV2: NCELLS, ARR_EMF: NEDGES}
        out = np.empty(sizes[which])
        self._check(self.L.fx_download_array(self._h, b, which, dir_, _dp(out)))
        return out

    # -- reference entry points ----------------------------------------------------
    def flux_update(self, b: int, w_slot: int, use_bf1: int) -> None:
        self._check(self.L.fx_flux_update(self._h, b, w_slot, use_bf1))

    def mhd_update_emf(self, b: int, stage: int) -> None:
        self._check(self.L.fx_mhd_update_emf(self._h, b, stage))

    def mhd_update_bf(self, b: int, stage: int, dt: float) -> None:
        self._check(self.L.fx_mhd_update_bf(self._h, b, stage, dt))

    def update_cells(self, b: int, stage: int, dt: float) -> float:
        v = C.c_double(1.0e100)
        self._check(self.L.fx_update_cells(self._h, b, stage, dt, C.byref(v)))
        return v.value

    def eos_fill_active_cells(self, stage: int) -> None:
        self._check(self.L.fx_eos_fill_active_cells(self._h, stage))

    def eos_fill_mesh(self, stage: int) -> None:
        self._check(self.L.fx_eos_fill_mesh(self._h, stage))

    def boundary_fill(self, stage: int, use_bf1: int) -> None:
        self._check(self.L.fx_boundary_fill_ghosts_and_bf(self._h, stage, use_bf1))

    def riemann_flux_send(self) -> None:
        self._check(self.L.fx_riemann_flux_send(self._h))

    def mhd_emf_send(self) -> None:
        self._check(self.L.fx_mhd_emf_send(self._h))

    # -- time integration -------------------------------------------------------------
    def calc_dt(self, cfl: float) -> float:
        v = C.c_double(0.0)
        self._check(self.L.fx_calc_dt(self._h, cfl, C.byref(v)))
        return v.value

    def stage(self, form: int, stage: int, dt: float) -> float:
        v = C.c_double(0.0)
        self._check(self.L.fx_stage(self._h, form, stage, dt, C.byref(v)))
        return v.value

    def step(self, form: int, dt: float, want_dt_src: bool = True) -> Optional[float]:
        if want_dt_src:
            v = C.c_double(0.0)
            self._check(self.L.fx_step(self._h, form, dt, C.byref(v)))
            return v.value
        self._check(self.L.fx_step(self._h, form, dt, None))
        return None

    def run(self, form: int, nsteps: int, cfl: float, dt_factor: float, t_end: float, state):
        st = (C.c_double * 3)(*state)
        self._check(self.L.fx_run(self._h, form, nsteps, cfl, dt_factor, t_end, st))
        return st[0], st[1], int(st[2])

    # -- measurement --------------------------------------------------------------------
    def time_phase(self, phase: int, reps: int, dt: float = 0.0) -> float:
        v = C.c_double(0.0)
        self._check(self.L.fx_time_phase(self._h, phase, reps, dt, C.byref(v)))
        return v.value

    def autotune(self):
        """(chosen shape, per-shape face-kernel times in ms)."""
        times = np.zeros(16)
        choice = C.c_int(0)
        self._check(self.L.fx_autotune(self._h, _dp(times), 16, C.byref(choice)))
        return choice.value, times

    def branch_record(self, max_stages: int) -> None:
        """fx_branch_trace(RECORD): the next plain-form stages record their decisions."""
        self._check(self.L.fx_branch_trace(self._h, _lib.BRANCH_RECORD, int(max_stages), None))

    def branch_replay(self) -> None:
        """fx_branch_trace(REPLAY): the next plain-form stages replay them."""
        self._check(self.L.fx_branch_trace(self._h, _lib.BRANCH_REPLAY, 0, None))

    def branch_off(self) -> int:
        """fx_branch_trace(OFF); returns the decisions the last replay overrode."""
        v = C.c_ulonglong(0)
        self._check(self.L.fx_branch_trace(self._h, _lib.BRANCH_OFF, 0, C.byref(v)))
        return v.value

    def set_flux_shape(self, variant: int) -> None:
        """Force a face-kernel launch shape (see fx_set_flux_shape)."""
        self._check(self.L.fx_set_flux_shape(self._h, variant))

    def info(self, what: int) -> int:
        v = C.c_longlong(0)
        self._check(self.L.fx_info(self._h, what, C.byref(v)))
        return v.value

    # ---- discrete adjoint ------------------------------------------------------
    # -- dynamic AMR ------------------------------------------------------------------
    def amr_configure(self, amr: FxAmrConfig) -> None:
        self._check(self.L.fx_amr_configure(self._h, C.byref(amr)))

    def amr_tag(self) -> np.ndarray:
        """prj_amr_tag's refine_flag per block entry (after the caps)."""
        out = np.zeros(self.nblocks, dtype=np.int32)
        self._check(self.L.fx_amr_tag(self._h, out.ctypes.data_as(C.POINTER(C.c_int32))))
        return out

    def amr_adapt(self) -> bool:
        """prj_amr_adapt plus the driver's refill; True if the mesh changed."""
        ch = C.c_int(0)
        self._check(self.L.fx_amr_adapt(self._h, C.byref(ch)))
        if ch.value:
            self.nblocks = self.mesh_size()
        return bool(ch.value)

    def mesh_size(self) -> int:
        n = C.c_int(0)
        self._check(self.L.fx_get_mesh(self._h, 0, None, C.byref(n)))
        return n.value

    def get_mesh(self):
        """The mirrored mesh as a ctypes fx_block_desc array."""
        n = self.mesh_size()
        out = (FxBlockDesc * n)()
        m = C.c_int(0)
        self._check(self.L.fx_get_mesh(self._h, n, out, C.byref(m)))
        return out

    def amr_timings(self) -> dict:
        """Host wall time (ms) of the phases of the last amr_adapt."""
        ms = (C.c_double * 6)()
        self._check(self.L.fx_amr_timings(self._h, ms))
        return dict(zip(("tag", "remesh", "data", "compile", "refill", "total"), ms[:]))

    def run_amr(self, form: int, nsteps: int, interval: int, cfl: float, dt_factor: float, t_end: float,
                state):
        """The driver loop of src/main.c:485-607 with prj_amr_adapt every
        `interval` steps (by the global step number in state[2]); returns
        (state, number of adapts that changed the mesh)."""
        changes = 0
        done = 0
        while done < nsteps:
            step = int(state[2])
            n = min(nsteps - done, interval - step % interval) if interval > 0 else nsteps - done
            state = self.run(form, n, cfl, dt_factor, t_end, state)
            done += n
            if state[2] == step:  # t_end reached
                break
            if interval > 0 and int(state[2]) % interval == 0:
                changes += int(self.amr_adapt())
        return state, changes

    def amr_energy_injected(self) -> float:
        e = C.c_double(0.0)
        self._check(self.L.fx_amr_energy_injected(self._h, C.byref(e)))
        return e.value

    def adjoint_forward(self, nsteps: int, dt: float) -> None:
        """nsteps batched RK2 steps with fixed dt, storing every stage."""
        self._check(self.L.fx_adjoint_forward(self._h, nsteps, dt))

    def adjoint_backward(self, W_bar: np.ndarray, Bf_bar: Optional[np.ndarray] = None,
                         initial_fill: bool = False):
        """(W_bar_out, Bf_bar_out) = d J / d (state at adjoint_forward's
        entry) from d J / d (final state); layouts of upload_all."""
        W_bar = np.ascontiguousarray(W_bar, dtype=np.float64)
        Wo = np.empty_like(W_bar)
        nb = W_bar.size // (self.nv * NSTAGES * NCELLS)
        Bo = np.empty(nb * 3 * NSTAGES * NFACES)
        bp = None
        if Bf_bar is not None:
            Bf_bar = np.ascontiguousarray(Bf_bar, dtype=np.float64)
            bp = _dp(Bf_bar)
        self._check(self.L.fx_adjoint_backward(self._h, _dp(W_bar), bp, _dp(Wo), _dp(Bo),
                                               1 if initial_fill else 0))
        return Wo, Bo

    def adjoint_ms(self) -> float:
        """Device time of the last reverse sweep (ms)."""
        v = C.c_double(0.0)
        self._check(self.L.fx_adjoint_time(self._h, C.byref(v)))
        return v.value
