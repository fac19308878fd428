"""ctypes front-end of the plain-C restatement oracle/fx_oracle.c
(oracle/_ref/libfxoracle.so).  TEST INFRASTRUCTURE ONLY."""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
PATH = os.path.join(HERE, "_ref", "libfxoracle.so")

_dp = C.POINTER(C.c_double)


class AmrCrit(C.Structure):
    """fxo_amr_crit: one refinement criterion."""
    _fields_ = [
        ("set", C.c_int),
        ("estimator", C.c_int),
        ("lohner_var", C.c_int),
        ("jump_var", C.c_int),
        ("refine_thresh", C.c_double),
        ("derefine_thresh", C.c_double),
        ("lohner_eps", C.c_double),
    ]


def available() -> bool:
    return os.path.exists(PATH)


class Restatement:
    def __init__(self):
        if not available():
            raise FileNotFoundError(f"{PATH} missing (run make -C oracle)")
        L = self.lib = C.CDLL(PATH, mode=C.RTLD_LOCAL)
        L.fxo_mc_slope.argtypes = [C.c_double] * 3
        L.fxo_mc_slope.restype = C.c_double
        L.fxo_weno3_face.argtypes = [C.c_double] * 4
        L.fxo_weno3_face.restype = C.c_double
        L.fxo_hlld.argtypes = [_dp, _dp] + [C.c_double] * 5 + [_dp]
        L.fxo_hlld.restype = C.c_int
        L.fxo_hllc.argtypes = [_dp, _dp] + [C.c_double] * 7 + [_dp]
        L.fxo_emf_upwind.argtypes = [_dp, _dp, _dp]
        L.fxo_emf_upwind.restype = C.c_double
        L.fxo_prim2cons.argtypes = [C.c_int, _dp, _dp]
        L.fxo_cons2prim.argtypes = [C.c_int, _dp, _dp]
        L.fxo_eos_rey.argtypes = [C.c_double] * 3 + [_dp]
        L.fxo_eos_rty.argtypes = [C.c_double] * 3 + [_dp, _dp]
        L.fxo_calc_dt.argtypes = [C.c_int, C.c_double, _dp, _dp, C.c_double]
        L.fxo_calc_dt.restype = C.c_double
        L.fxo_step_block.argtypes = [C.c_int, C.c_double, _dp, _dp, _dp, C.c_double]
        L.fxo_step_block.restype = C.c_double
        L.fxo_amr_vote.argtypes = [C.c_int, C.c_double, _dp, _dp, _dp, C.c_int, C.POINTER(AmrCrit), C.c_int,
                                   C.c_double, C.POINTER(C.c_int)]

    @staticmethod
    def _p(a):
        return a.ctypes.data_as(_dp)

    def mc_slope(self, qm, q0, qp):
        return self.lib.fxo_mc_slope(qm, q0, qp)

    def weno3_face(self, qm, q0, qp, target):
        return self.lib.fxo_weno3_face(qm, q0, qp, target)

    def hlld(self, WL, WR, pL, pR, gL, gR, bn):
        wl = np.ascontiguousarray(WL, np.float64).copy()
        wr = np.ascontiguousarray(WR, np.float64).copy()
        wl[6] = bn
        wr[6] = bn
        out = np.zeros(14)
        fail = self.lib.fxo_hlld(self._p(wl), self._p(wr), pL, pR, gL, gR, bn, self._p(out))
        return out, fail

    def hllc(self, WL, WR, pL, pR, gL, gR, du, dv, dw):
        wl = np.ascontiguousarray(WL, np.float64)
        wr = np.ascontiguousarray(WR, np.float64)
        out = np.zeros(9)
        self.lib.fxo_hllc(self._p(wl), self._p(wr), pL, pR, gL, gR, du, dv, dw, self._p(out))
        return out

    def emf_upwind(self, f, c, vn):
        f, c, vn = (np.ascontiguousarray(x, np.float64) for x in (f, c, vn))
        return self.lib.fxo_emf_upwind(self._p(f), self._p(c), self._p(vn))

    def prim2cons(self, nv, w):
        w = np.ascontiguousarray(w, np.float64)
        u = np.zeros(nv)
        self.lib.fxo_prim2cons(nv, self._p(w), self._p(u))
        return u

    def cons2prim(self, nv, u):
        u = np.ascontiguousarray(u, np.float64)
        w = np.zeros(nv)
        self.lib.fxo_cons2prim(nv, self._p(u), self._p(w))
        return w

    def eos_rey(self, g, rho, eint):
        out = np.zeros(3)
        self.lib.fxo_eos_rey(g, rho, eint, self._p(out))
        return out

    def eos_rty(self, g, rho, T):
        e = C.c_double()
        p = C.c_double()
        self.lib.fxo_eos_rty(g, rho, T, C.byref(e), C.byref(p))
        return e.value, p.value

    def calc_dt(self, nv, gamma, dx, W, cfl):
        dx = np.ascontiguousarray(dx, np.float64)
        return self.lib.fxo_calc_dt(nv, gamma, self._p(dx), self._p(W), cfl)

    def step_block(self, nv, gamma, dx, W, Bf, dt):
        """In place on W (nv*2*8000) and Bf (3*2*8400 or None); returns dt_src."""
        dx = np.ascontiguousarray(dx, np.float64)
        bp = self._p(Bf) if Bf is not None else None
        return self.lib.fxo_step_block(nv, gamma, self._p(dx), self._p(W), bp, dt)

    def amr_votes(self, nv, gamma, W, grav, dx, active, parent, crits, reach=-1.0):
        """Pass 1 of prj_amr_tag for every block: int32 [nb, 3] (refine vote,
        derefine vote, boundary mask; zeros for inactive entries).  W is
        [nb, nv, 2, 8000]; grav [nb, 3, 8000] or None; crits a list of dicts
        (estimator, refine, derefine, var, eps)."""
        arr = (AmrCrit * max(len(crits), 1))()
        for n, c in enumerate(crits):
            arr[n].set = 1
            arr[n].estimator = int(c["estimator"])
            var = int(c.get("var", 1))
            arr[n].lohner_var = var
            arr[n].jump_var = min(var, 1)
            arr[n].refine_thresh = float(c.get("refine", 0.5))
            arr[n].derefine_thresh = float(c.get("derefine", 0.2))
            arr[n].lohner_eps = float(c.get("eps", 0.1))
        nb = W.shape[0]
        out = np.zeros((nb, 3), dtype=np.int32)
        o = (C.c_int * 3)()
        for b in range(nb):
            if not active[b]:
                continue
            w = np.ascontiguousarray(W[b], np.float64)
            g = None if grav is None else self._p(np.ascontiguousarray(grav[b], np.float64))
            d = np.ascontiguousarray(dx[b], np.float64)
            self.lib.fxo_amr_vote(nv, gamma, self._p(w), g, self._p(d), 1 if parent[b] >= 0 else 0,
                                  arr, len(crits), reach, o)
            out[b] = o[:]
        return out
