"""ctypes front-end for the oracle libraries built by oracle/Makefile.

TEST INFRASTRUCTURE ONLY: imported by tests/, the smoke check and the CPU
baseline leg of bench.py.  The libraries wrap the reference FornaxAMR C core
(compiled unmodified from its own sources) plus oracle/ref_harness.c, so every
number produced here is the reference's CPU path.

Block arrays are returned as numpy copies in the reference's own per-block
layout (src/prj_defs.h:383-453 of the reference): W is [var][stage][cell] with
cell = LIDX, eosvar/flux/v_riemann are AoSoA with 4-wide k lanes, Bf is
[stage][FACE_IDX], emf is [EDGE_IDX].
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(HERE, "_ref")

# the process's ghost layers (FX_NGHOST, 2 or 4) select the reference builds
# with the same PRJ_NGHOST
NG = int(os.environ.get("FX_NGHOST", "2"))
BS = 16
PBS = BS + 2 * NG
NCELLS = PBS ** 3
NFACES = (PBS + 1) * PBS * PBS
NEDGES = (PBS + 1) * (PBS + 1) * PBS
NSTAGES = 2

ARR_W, ARR_EOSVAR, ARR_U, ARR_RHS, ARR_FLUX, ARR_VRIEMANN, ARR_GRAV, ARR_BF, ARR_BV1, ARR_BV2, ARR_EMF = range(11)

CFG_SOD, CFG_FOURIER_MHD, CFG_AMR_BLAST, CFG_COLLAPSE = 1, 2, 3, 4


class RhParams(C.Structure):
    _fields_ = [
        ("config", C.c_int),
        ("root", C.c_int * 3),
        ("max_level", C.c_int),
        ("max_blocks", C.c_int),
        ("xmin", C.c_double * 3),
        ("xmax", C.c_double * 3),
        ("gamma", C.c_double),
        ("cfl", C.c_double),
        ("dt_factor", C.c_double),
        ("t_end", C.c_double),
        ("nmodes", C.c_int),
        ("kmax", C.c_int),
        ("amp_rho", C.c_double),
        ("amp_v", C.c_double),
        ("amp_A", C.c_double),
        ("seed_rho", C.c_ulonglong),
        ("seed_v", C.c_ulonglong),
        ("seed_A", C.c_ulonglong),
        ("center", C.c_double * 3),
        ("refine_radius", C.c_double * 4),
        ("p_in", C.c_double),
        ("p_out", C.c_double),
        ("r_in", C.c_double),
        ("B0", C.c_double * 3),
        ("rho_c", C.c_double),
        ("r0", C.c_double),
        ("K", C.c_double),
        ("beta", C.c_double),
        ("gm_point", C.c_double),
        ("bc", C.c_int * 6),
    ]


AMR_N = 4
EST_LOEHNER, EST_VELOCITY, EST_PRESSURE_SCALE_HEIGHT, EST_FRACTIONAL_JUMP = 0, 1, 2, 3
LOHNER_DENSITY, LOHNER_PRESSURE, LOHNER_TEMPERATURE = 0, 1, 2
JUMP_DENSITY, JUMP_PRESSURE = 0, 1


class RhAmr(C.Structure):
    """Dynamic-AMR parameters of prj_mesh (src/prj_types.h:465-503)."""
    _fields_ = [
        ("max_level", C.c_int),
        ("min_dx", C.c_double),
        ("reach_density", C.c_double),
        ("E_floor", C.c_double),
        ("set", C.c_int * AMR_N),
        ("estimator", C.c_int * AMR_N),
        ("lohner_var", C.c_int * AMR_N),
        ("jump_var", C.c_int * AMR_N),
        ("refine_thresh", C.c_double * AMR_N),
        ("derefine_thresh", C.c_double * AMR_N),
        ("lohner_eps", C.c_double * AMR_N),
    ]


def amr_params(max_level: int, criteria, min_dx: float = 0.0, reach_density: float = -1.0,
               E_floor: float = -1.0) -> RhAmr:
    """criteria: up to four dicts with keys estimator, refine, derefine and
    optionally lohner_var, jump_var, eps (defaults of src/prj_io.c:341-355)."""
    a = RhAmr()
    a.max_level = max_level
    a.min_dx = min_dx
    a.reach_density = reach_density
    a.E_floor = E_floor
    for n in range(AMR_N):
        a.set[n] = 0
        a.estimator[n] = EST_LOEHNER
        a.lohner_var[n] = LOHNER_PRESSURE
        a.jump_var[n] = JUMP_PRESSURE
        a.refine_thresh[n] = 0.5
        a.derefine_thresh[n] = 0.2
        a.lohner_eps[n] = 0.1
    for n, c in enumerate(criteria):
        a.set[n] = 1
        a.estimator[n] = c["estimator"]
        a.refine_thresh[n] = c.get("refine", 0.5)
        a.derefine_thresh[n] = c.get("derefine", 0.2)
        a.lohner_var[n] = c.get("lohner_var", LOHNER_PRESSURE)
        a.jump_var[n] = c.get("jump_var", JUMP_PRESSURE)
        a.lohner_eps[n] = c.get("eps", 0.1)
    return a


def lib_path(mhd: bool, variant: str = "") -> str:
    """variant: "" (RK2, MC), "weno3", "ess" (eSSPRK10_4), "ess_weno3"; with
    four ghost layers "" (MC, PRJ_NGHOST=4), "weno7" (WENO-Z7) or "ess_weno7".
    "fx": the RK2 / MC build with the drop-in binding linked in its place
    (prj_timeint_step and prj_timeint_calc_dt reach the device through
    fornaxamr_b200/dropin/prj_fx.c)."""
    if NG == 4 and variant == "fx":
        raise ValueError("the drop-in build links the two-ghost-layer library")
    if NG == 4 and variant not in ("", "weno7", "ess_weno7"):
        raise ValueError(f"no four-ghost-layer reference build for variant {variant!r}")
    if NG == 2 and variant.endswith("weno7"):
        raise ValueError("WENO-Z7 needs four ghost layers (FX_NGHOST=4)")
    if NG == 4 and not variant:
        variant = "ng4"
    name = ("mhd" if mhd else "hydro") + ("_" + variant if variant else "")
    return os.path.join(REF_DIR, f"libprjref_{name}.so")


def available(mhd: bool = True, variant: str = "") -> bool:
    return os.path.exists(lib_path(mhd, variant))


class Reference:
    """One loaded copy of the reference core (one build variant)."""

    def __init__(self, mhd: bool = True, variant: str = ""):
        path = lib_path(mhd, variant)
        if not os.path.exists(path):
            raise FileNotFoundError(f"oracle library missing: {path} (run make -C oracle)")
        self.mhd = mhd
        self.lib = L = C.CDLL(path, mode=C.RTLD_LOCAL)
        dp = C.POINTER(C.c_double)
        ip = C.POINTER(C.c_int)
        L.rh_setup.argtypes = [C.POINTER(RhParams)]
        L.rh_setup.restype = C.c_int
        L.rh_calc_dt.restype = C.c_double
        L.rh_step.argtypes = [C.c_double, dp]
        L.rh_stage.argtypes = [C.c_int, C.c_double, dp]
        L.rh_run.argtypes = [C.c_int, dp]
        L.rh_run.restype = C.c_int
        L.rh_time_steps.argtypes = [C.c_int, C.c_double]
        L.rh_time_steps.restype = C.c_double
        L.rh_block_geom.argtypes = [C.c_int, ip, dp]
        L.rh_block_slots.argtypes = [C.c_int, ip]
        L.rh_block_array.argtypes = [C.c_int, C.c_int, C.c_int]
        L.rh_block_array.restype = dp
        L.rh_mc_slope.argtypes = [C.c_double] * 3
        L.rh_mc_slope.restype = C.c_double
        L.rh_hllc.argtypes = [dp, dp] + [C.c_double] * 7 + [dp]
        L.rh_prim2cons.argtypes = [dp, dp]
        L.rh_cons2prim.argtypes = [dp, dp]
        L.rh_eos_rey.argtypes = [C.c_double] * 3 + [dp]
        L.rh_set_gamma.argtypes = [C.c_double]
        L.rh_flux_update.argtypes = [C.c_int, C.c_int, C.c_int]
        L.rh_fill_ghosts.argtypes = [C.c_int, C.c_int]
        L.rh_sim_time.restype = C.c_double
        L.rh_amr_configure.argtypes = [C.POINTER(RhAmr)]
        L.rh_amr_tag.argtypes = [ip]
        L.rh_amr_adapt.restype = C.c_int
        L.rh_run_amr.argtypes = [C.c_int, C.c_int, dp]
        L.rh_run_amr.restype = C.c_int
        L.rh_block_tree.argtypes = [C.c_int, ip]
        L.rh_E_injected.restype = C.c_double
        L.rh_weno3_face.argtypes = [C.c_double] * 4
        L.rh_weno3_face.restype = C.c_double
        L.rh_sim_dt.restype = C.c_double
        L.rh_set_mhd_eta.argtypes = [C.c_double]
        L.rh_set_use_bj.argtypes = [C.c_int]
        if mhd:
            L.rh_hlld.argtypes = [dp, dp] + [C.c_double] * 5 + [dp]
            L.rh_emf_upwind.argtypes = [dp, dp, dp]
            L.rh_emf_upwind.restype = C.c_double
        if variant == "fx":
            L.prj_fx_configure.argtypes = [C.c_int, C.c_int]
            L.prj_fx_active.restype = C.c_int
        self.variant = variant
        self.nhydro = L.rh_nhydro()
        self.nstages = L.rh_nstages()
        if L.rh_nghost() != NG:
            raise RuntimeError(f"{path}: PRJ_NGHOST {L.rh_nghost()}, FX_NGHOST {NG}")

    # -- set-up and stepping ------------------------------------------------
    def setup(self, params: RhParams) -> None:
        rc = self.lib.rh_setup(C.byref(params))
        if rc != 0:
            raise RuntimeError(f"rh_setup failed with {rc}")

    def calc_dt(self) -> float:
        return self.lib.rh_calc_dt()

    def step(self, dt: float) -> float:
        out = C.c_double(0.0)
        self.lib.rh_step(dt, C.byref(out))
        return out.value

    def stage(self, which: int, dt: float) -> float:
        out = C.c_double(0.0)
        self.lib.rh_stage(which, dt, C.byref(out))
        return out.value

    def run(self, nsteps: int):
        st = (C.c_double * 3)()
        n = self.lib.rh_run(nsteps, st)
        return n, st[0], st[1], int(st[2])

    def time_steps(self, nsteps: int, dt: float) -> float:
        return self.lib.rh_time_steps(nsteps, dt)

    # -- the drop-in build ("fx") ----------------------------------------------
    DROPIN_MIRROR, DROPIN_RESIDENT = 0, 1

    def dropin_configure(self, form: int, mode: int) -> None:
        """prj_fx_configure: the device form and where the state lives."""
        self.lib.prj_fx_configure(form, mode)

    def dropin_release(self) -> None:
        self.lib.prj_fx_release()

    def dropin_active(self) -> bool:
        return bool(self.lib.prj_fx_active())

    def dropin_to_host(self) -> None:
        """prj_fx_to_host on the harness's mesh (resident mode)."""
        self.lib.rh_dropin_to_host()

    def set_mhd_eta(self, eta: float) -> None:
        """Run-time resistivity (prj_mesh.mhd_eta)."""
        self.lib.rh_set_mhd_eta(eta)

    def set_use_bj(self, on: bool) -> None:
        """Barth-Jespersen prolongation limiter (prj_mesh.use_BJ); rh_setup
        resets it to off."""
        self.lib.rh_set_use_bj(1 if on else 0)

    def refill(self) -> None:
        """The driver's set-up refill (eos, ghost fill, eos) after stage-0
        cells or faces were rewritten with set_W / set_Bf."""
        self.lib.rh_refill()

    # -- dynamic AMR ------------------------------------------------------------
    def amr_configure(self, a: RhAmr) -> None:
        self.lib.rh_amr_configure(C.byref(a))

    def amr_tag(self) -> np.ndarray:
        """refine_flag of every block after prj_amr_tag (before 2:1 balance)."""
        out = (C.c_int * self.nblocks())()
        self.lib.rh_amr_tag(out)
        return np.array(out[:], dtype=np.int32)

    def amr_adapt(self) -> int:
        return self.lib.rh_amr_adapt()

    def run_amr(self, nsteps: int, interval: int):
        st = (C.c_double * 4)()
        n = self.lib.rh_run_amr(nsteps, interval, st)
        return n, st[0], st[1], int(st[2]), int(st[3])

    def block_tree(self, b: int) -> np.ndarray:
        """parent, children[8], refine_flag, can_refine"""
        out = (C.c_int * 11)()
        self.lib.rh_block_tree(b, out)
        return np.array(out[:], dtype=np.int32)

    def tree_arrays(self) -> np.ndarray:
        return np.stack([self.block_tree(b) for b in range(self.nblocks())])

    def E_injected(self) -> float:
        return self.lib.rh_E_injected()

    # -- mesh description -----------------------------------------------------
    def nblocks(self) -> int:
        return self.lib.rh_nblocks()

    def block_geom(self, b: int):
        ints = (C.c_int * 4)()
        dbl = (C.c_double * 13)()
        self.lib.rh_block_geom(b, ints, dbl)
        return list(ints), np.array(dbl[:], dtype=np.float64)

    def block_slots(self, b: int) -> np.ndarray:
        out = (C.c_int * (56 * 15))()
        self.lib.rh_block_slots(b, out)
        return np.array(out[:], dtype=np.int32).reshape(56, 15)

    # -- block arrays ---------------------------------------------------------
    def _arr(self, b: int, which: int, dir_: int, count: int) -> np.ndarray:
        p = self.lib.rh_block_array(b, which, dir_)
        if not p:
            raise ValueError("array not present in this build")
        return np.ctypeslib.as_array(p, shape=(count,)).copy()

    def _set(self, b: int, which: int, dir_: int, data: np.ndarray) -> None:
        p = self.lib.rh_block_array(b, which, dir_)
        if not p:
            raise ValueError("array not present in this build")
        dst = np.ctypeslib.as_array(p, shape=(data.size,))
        dst[:] = data.ravel()

    def W(self, b: int) -> np.ndarray:
        return self._arr(b, ARR_W, 0, self.nhydro * self.nstages * NCELLS)

    def set_W(self, b: int, data: np.ndarray) -> None:
        self._set(b, ARR_W, 0, data)

    def eosvar(self, b: int) -> np.ndarray:
        return self._arr(b, ARR_EOSVAR, 0, 3 * NCELLS)

    def flux(self, b: int, d: int) -> np.ndarray:
        return self._arr(b, ARR_FLUX, d, self.nhydro * NCELLS)

    def vriemann(self, b: int, d: int) -> np.ndarray:
        return self._arr(b, ARR_VRIEMANN, d, 3 * NCELLS)

    def grav(self, b: int, d: int) -> np.ndarray:
        return self._arr(b, ARR_GRAV, d, NCELLS)

    def rhs(self, b: int) -> np.ndarray:
        return self._arr(b, ARR_RHS, 0, self.nhydro * NCELLS)

    def Bf(self, b: int, d: int) -> np.ndarray:
        return self._arr(b, ARR_BF, d, self.nstages * NFACES)

    def set_Bf(self, b: int, d: int, data: np.ndarray) -> None:
        self._set(b, ARR_BF, d, data)

    def Bv(self, b: int, d: int):
        return self._arr(b, ARR_BV1, d, NCELLS), self._arr(b, ARR_BV2, d, NCELLS)

    def emf(self, b: int, d: int) -> np.ndarray:
        return self._arr(b, ARR_EMF, d, NEDGES)

    def flux_update(self, b: int, w_slot: int, use_bf1: int) -> None:
        self.lib.rh_flux_update(b, w_slot, use_bf1)

    def fill_ghosts(self, stage: int, use_bf1: int) -> None:
        self.lib.rh_fill_ghosts(stage, use_bf1)

    def flux_send(self) -> None:
        """prj_riemann_flux_send on the current flux arrays."""
        self.lib.rh_flux_send()

    def emf_send(self) -> None:
        """prj_mhd_emf_send on the current emf arrays (no-op for hydro)."""
        self.lib.rh_emf_send()

    def set_flux(self, b: int, d: int, data: np.ndarray) -> None:
        self._set(b, ARR_FLUX, d, data)

    def set_emf(self, b: int, d: int, data: np.ndarray) -> None:
        self._set(b, ARR_EMF, d, data)

    def mesh_arrays(self):
        """(ints [n,4], geom [n,13], slots [n,56,15]) of the current mesh."""
        nb = self.nblocks()
        ints = np.zeros((nb, 4), dtype=np.int64)
        geom = np.zeros((nb, 13), dtype=np.float64)
        slots = np.zeros((nb, 56, 15), dtype=np.int64)
        for b in range(nb):
            i, g = self.block_geom(b)
            ints[b] = i
            geom[b] = g
            slots[b] = self.block_slots(b)
        return ints, geom, slots

    # -- single kernels -------------------------------------------------------
    def mc_slope(self, qm, q0, qp) -> float:
        return self.lib.rh_mc_slope(qm, q0, qp)

    def weno3_face(self, qm, q0, qp, target) -> float:
        return self.lib.rh_weno3_face(qm, q0, qp, target)

    def hlld(self, WL, WR, pL, pR, gL, gR, bn) -> np.ndarray:
        wl = np.ascontiguousarray(WL, dtype=np.float64)
        wr = np.ascontiguousarray(WR, dtype=np.float64)
        out = np.zeros(14)
        dp = C.POINTER(C.c_double)
        self.lib.rh_hlld(wl.ctypes.data_as(dp), wr.ctypes.data_as(dp), pL, pR, gL, gR, bn,
                         out.ctypes.data_as(dp))
        return out

    def hllc(self, WL, WR, pL, pR, gL, gR, du, dv, dw) -> np.ndarray:
        wl = np.ascontiguousarray(WL, dtype=np.float64)
        wr = np.ascontiguousarray(WR, dtype=np.float64)
        out = np.zeros(self.nhydro + 3)
        dp = C.POINTER(C.c_double)
        self.lib.rh_hllc(wl.ctypes.data_as(dp), wr.ctypes.data_as(dp), pL, pR, gL, gR,
                         du, dv, dw, out.ctypes.data_as(dp))
        return out

    def emf_upwind(self, face, cell, vn) -> float:
        dp = C.POINTER(C.c_double)
        f = np.ascontiguousarray(face, dtype=np.float64)
        c = np.ascontiguousarray(cell, dtype=np.float64)
        v = np.ascontiguousarray(vn, dtype=np.float64)
        return self.lib.rh_emf_upwind(f.ctypes.data_as(dp), c.ctypes.data_as(dp), v.ctypes.data_as(dp))

    def prim2cons(self, w) -> np.ndarray:
        dp = C.POINTER(C.c_double)
        w = np.ascontiguousarray(w, dtype=np.float64)
        u = np.zeros(self.nhydro)
        self.lib.rh_prim2cons(w.ctypes.data_as(dp), u.ctypes.data_as(dp))
        return u

    def cons2prim(self, u) -> np.ndarray:
        dp = C.POINTER(C.c_double)
        u = np.ascontiguousarray(u, dtype=np.float64)
        w = np.zeros(self.nhydro)
        self.lib.rh_cons2prim(u.ctypes.data_as(dp), w.ctypes.data_as(dp))
        return w

    def eos_rey(self, rho, eint, ye) -> np.ndarray:
        dp = C.POINTER(C.c_double)
        out = np.zeros(3)
        self.lib.rh_eos_rey(rho, eint, ye, out.ctypes.data_as(dp))
        return out

    def set_gamma(self, g: float) -> None:
        self.lib.rh_set_gamma(g)


# ---------------------------------------------------------------------------
# Workload presets (the same recipes the product's own generators implement)
# ---------------------------------------------------------------------------

def params_sod(nblocks_x: int = 64, gamma: float = 1.4, t_end: float = 0.2) -> RhParams:
    """1-D Sod tube run as a 3-D pencil of nblocks_x blocks of 16^3 cells on
    x in [0,1] (transverse extent one block, dx equal on all axes)."""
    p = RhParams()
    p.config = CFG_SOD
    p.root[:] = [nblocks_x, 1, 1]
    p.max_level = 0
    p.xmin[:] = [0.0, 0.0, 0.0]
    p.xmax[:] = [1.0, 1.0 / nblocks_x, 1.0 / nblocks_x]
    p.gamma = gamma
    p.cfl = 0.4
    p.dt_factor = 1.2
    p.t_end = t_end
    return p


def params_fourier(root: int = 8, nmodes: int = 32, kmax: int = 4, amp_rho: float = 0.1,
                   amp_v: float = 0.1, amp_A: float = 0.05, gamma: float = 5.0 / 3.0,
                   seeds=(1, 2, 3)) -> RhParams:
    """Seeded Fourier-mode ideal MHD on [0,1]^3 with root^3 blocks of 16^3."""
    p = RhParams()
    p.config = CFG_FOURIER_MHD
    p.root[:] = [root, root, root]
    p.max_level = 0
    p.xmin[:] = [0.0, 0.0, 0.0]
    p.xmax[:] = [1.0, 1.0, 1.0]
    p.gamma = gamma
    p.cfl = 0.4
    p.dt_factor = 1.2
    p.t_end = 1.0e30
    p.nmodes = nmodes
    p.kmax = kmax
    p.amp_rho = amp_rho
    p.amp_v = amp_v
    p.amp_A = amp_A
    p.seed_rho, p.seed_v, p.seed_A = seeds
    return p


def params_amr_blast(root: int = 8, half_width: float = 0.7, max_level: int = 2,
                     radii=(0.4, 0.2, 0.1), gamma: float = 5.0 / 3.0) -> RhParams:
    """Magnetised blast on a static AMR hierarchy: rho = 1, p = 0.1 outside and
    10 inside r < 0.05 about (0.1, 0.05, 0), B = (1, 1, 0) / sqrt(2) /
    sqrt(4 pi) through A = (0, 0, Bx y - By x).  Blocks of level l that
    overlap the ball of radius radii[l] about the same centre are refined
    (the block-overlaps-ball rule of problems/prj_problem_sedov.c), then the
    reference's 2:1 balance runs."""
    p = RhParams()
    p.config = CFG_AMR_BLAST
    p.root[:] = [root, root, root]
    p.max_level = max_level
    p.max_blocks = 200000
    p.xmin[:] = [-half_width] * 3
    p.xmax[:] = [half_width] * 3
    p.gamma = gamma
    p.cfl = 0.4
    p.dt_factor = 1.2
    p.t_end = 1.0e30
    p.center[:] = [0.1, 0.05, 0.0]
    p.refine_radius[:] = list(radii) + [0.0] * (4 - len(radii))
    p.p_in, p.p_out, p.r_in = 10.0, 0.1, 0.05
    b = 1.0 / np.sqrt(2.0) / np.sqrt(4.0 * np.pi)
    p.B0[:] = [b, b, 0.0]
    return p


def params_collapse(root: int = 12, half_width: float = 1.0, max_level: int = 3,
                    radii=(0.4, 0.2, 0.1), rho_c: float = 1.0e10, K: float = 4.6e5,
                    beta: float = 1.0e4, gm_point: float = 0.0) -> RhParams:
    """Collapse-like MHD with a static gravity field: rho = rho_c (1 +
    (r/r0)^2)^-1.5 with r0 = 0.05 of the domain length, p = K rho^gamma
    (gamma 4/3), v_r = -0.1 c_s r / (r + r0), a dipole-like loop field whose
    central strength gives plasma beta `beta`, and g = -(gm_point +
    M(<r)) x / r^3 written once into the blocks' grav arrays.  Blocks of
    level l that overlap the ball of radius radii[l] about the origin are
    refined, then 2:1 balanced."""
    p = RhParams()
    p.config = CFG_COLLAPSE
    p.root[:] = [root, root, root]
    p.max_level = max_level
    p.max_blocks = 400000
    p.xmin[:] = [-half_width] * 3
    p.xmax[:] = [half_width] * 3
    p.gamma = 4.0 / 3.0
    p.cfl = 0.4
    p.dt_factor = 1.2
    p.t_end = 1.0e30
    p.center[:] = [0.0, 0.0, 0.0]
    p.refine_radius[:] = list(radii) + [0.0] * (4 - len(radii))
    p.rho_c = rho_c
    p.r0 = 0.05 * 2.0 * half_width
    p.K = K
    p.beta = beta
    p.gm_point = gm_point
    # central field 2 B0 (A_phi = B0 r0^3 R / (r^2 + r0^2)^1.5); beta = 2 p / B^2
    p_c = K * rho_c ** p.gamma
    p.B0[:] = [0.5 * np.sqrt(2.0 * p_c / beta), 0.0, 0.0]
    return p
