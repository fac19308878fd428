"""The discrete adjoint's hardest building block -- the vector-Jacobian
product of one face (MC reconstruction of the 4-cell stencil + HLLD) -- against
central finite differences of the same face evaluated on the host, in every
region of the Riemann fan: left/right supersonic, single and double star on
either side of the contact, strong field, bn = 0 and the HLL fallback.

Tolerance: 1e-5 relative on the directional derivative (central differences
with eps = 1e-6 are accurate to about 1e-9 here); samples where the
difference quotients at eps and eps/10 disagree lie within eps of a limiter
or fan-region switch and are skipped.
"""
import ctypes as C

import numpy as np
import pytest

import fornaxamr_b200 as fx

DP = C.POINTER(C.c_double)
GAMMA = 5.0 / 3.0


def _eval(L, w4, bn):
    out = np.zeros(14)
    assert L.fx_face_eval_host(w4.ctypes.data_as(DP), bn, GAMMA, out.ctypes.data_as(DP)) == 0
    return out


def _vjp(L, w4, bn, ob):
    wb = np.zeros(36)
    bnb = C.c_double(0.0)
    assert L.fx_face_vjp_host(w4.ctypes.data_as(DP), bn, GAMMA, ob.ctypes.data_as(DP),
                              wb.ctypes.data_as(DP), C.byref(bnb)) == 0
    return wb, bnb.value


def _state(rng, kind):
    w = np.zeros((4, 9))
    rho0 = rng.uniform(0.5, 2.0)
    e0 = rng.uniform(0.5, 3.0)
    vn = {"supersonic_right": 4.0, "supersonic_left": -4.0, "contact_left": -0.3}.get(kind, 0.1)
    for n in range(4):
        w[n, 0] = rho0 * (1 + 0.05 * rng.normal())
        w[n, 1] = vn + 0.05 * rng.normal()
        w[n, 2:4] = 0.2 * rng.normal(size=2)
        w[n, 4] = e0 * (1 + 0.05 * rng.normal())
        w[n, 5] = 0.1 + 0.01 * rng.normal()
        w[n, 7] = rng.normal() * (2.0 if kind == "strong_field" else 0.5)
        w[n, 8] = 0.5 * rng.normal()
    if kind == "hll_fallback":  # strong expansion: negative star total pressure
        w[:2, 1] = -6.0 + 0.05 * rng.normal(size=2)
        w[2:, 1] = 6.0 + 0.05 * rng.normal(size=2)
    bn = {"bn_zero": 0.0, "strong_field": 2.0}.get(kind, 0.7 * rng.normal())
    return w.ravel(), bn


@pytest.mark.parametrize("kind", ["double_star", "contact_left", "strong_field", "bn_zero",
                                  "supersonic_right", "supersonic_left", "hll_fallback"])
def test_face_vjp_matches_finite_differences(kind):
    L = fx.library()
    rng = np.random.default_rng(sum(ord(ch) for ch in kind))
    checked = 0
    for _ in range(40):
        w4, bn = _state(rng, kind)
        ob = rng.normal(size=14)
        d = rng.normal(size=36)
        d[6::9] = 0.0
        dbn = 0.0 if kind == "bn_zero" else rng.normal()
        wb, bnb = _vjp(L, w4, bn, ob)
        ad = wb @ d + bnb * dbn
        fd = []
        for eps in (1e-6, 1e-7):
            fp = _eval(L, w4 + eps * d, bn + eps * dbn)
            fm = _eval(L, w4 - eps * d, bn - eps * dbn)
            fd.append(ob @ (fp - fm) / (2 * eps))
        if abs(fd[0] - fd[1]) > 1e-5 * max(1.0, abs(fd[0])):
            continue
        checked += 1
        assert abs(ad - fd[0]) <= 1e-5 * max(1e-8, abs(fd[0]))
    assert checked >= 30
