"""ctypes front-end of the plain-C restatement oracle/fx_oracle.c
(oracle/_ref/libfxoracle.so).  TEST INFRASTRUCTURE ONLY."""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
PATH = os.path.join(HERE, "_ref", "libfxoracle.so")

_dp = C.POINTER(C.c_double)


def available() -> bool:
    return os.path.exists(PATH)


class Restatement:
    def __init__(self):
        if not available():
            raise FileNotFoundError(f"{PATH} missing (run make -C oracle)")
        L = self.lib = C.CDLL(PATH, mode=C.RTLD_LOCAL)
        L.fxo_mc_slope.argtypes = [C.c_double] * 3
        L.fxo_mc_slope.restype = C.c_double
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

    @staticmethod
    def _p(a):
        return a.ctypes.data_as(_dp)

    def mc_slope(self, qm, q0, qp):
        return self.lib.fxo_mc_slope(qm, q0, qp)

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
