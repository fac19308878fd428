"""Generates the golden vectors in tests/golden/ from the reference itself.

Run (where the oracle libraries are built from the reference sources):
    python tests/golden/make_golden.py

Every output is produced by the compiled reference core
(oracle/_ref/libprjref_*.so: prj_riemann_hlld, prj_riemann_hllc,
prj_reconstruct_mc_face_slope, prj_mhd_emf_upwind, prj_eos_prim2cons /
cons2prim / rey, prj_timeint_step).  Inputs are seeded synthetic states that
exercise every branch of the solvers.  Cases are screened with the
restatement first so that no case reaches one of the reference's exit(1)
paths.
"""
from __future__ import annotations

import hashlib
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import ref as R  # noqa: E402
from oracle.restate import Restatement  # noqa: E402


def prim_state(rng, nv, vx, bscale, lowp=False):
    g = 5.0 / 3.0 if nv == 9 else 1.4
    rho = rng.uniform(0.1, 2.0)
    p = rng.uniform(0.005, 0.02) if lowp else rng.uniform(0.05, 2.0)
    w = np.zeros(nv)
    w[0] = rho
    w[1] = vx
    w[2:4] = rng.normal(0.0, 0.5, 2)
    w[4] = p / ((g - 1.0) * rho)
    w[5] = rng.uniform(0.05, 0.5)
    if nv == 9:
        w[6:9] = rng.normal(0.0, bscale, 3)
    return w, p, g


def hlld_cases(ref, rs, rng, per_kind=60):
    X, Y, K = [], [], []
    kinds = ["subsonic", "left_supersonic", "right_supersonic", "rarefaction", "bn_zero", "strong_field"]
    for kind in kinds:
        made = 0
        while made < per_kind:
            if kind == "left_supersonic":
                vxl = vxr = rng.uniform(4.0, 8.0)
            elif kind == "right_supersonic":
                vxl = vxr = -rng.uniform(4.0, 8.0)
            elif kind == "rarefaction":
                vxl, vxr = -rng.uniform(3.0, 6.0), rng.uniform(3.0, 6.0)
            else:
                vxl, vxr = rng.normal(0.0, 0.5, 2)
            bscale = 3.0 if kind == "strong_field" else 0.7
            wl, pl, g = prim_state(rng, 9, vxl, bscale, lowp=kind == "rarefaction")
            wr, pr, _ = prim_state(rng, 9, vxr, bscale, lowp=kind == "rarefaction")
            bn = 0.0 if kind == "bn_zero" else rng.normal(0.0, bscale)
            if kind == "bn_zero":
                wl[7:9] *= 1e-6
            _, fail = rs.hlld(wl, wr, pl, pr, g, g, bn)
            if fail:
                continue
            out = ref.hlld(wl, wr, pl, pr, g, g, bn)
            X.append(np.concatenate([wl, wr, [pl, pr, g, g, bn]]))
            Y.append(out)
            K.append(kinds.index(kind))
            made += 1
    return np.array(X), np.array(Y), np.array(K)


def hllc_cases(ref, rng, n=240):
    X, Y = [], []
    for q in range(n):
        kind = q % 4
        if kind == 1:
            vxl = vxr = rng.uniform(3.0, 6.0)
        elif kind == 2:
            vxl = vxr = -rng.uniform(3.0, 6.0)
        else:
            vxl, vxr = rng.normal(0.0, 0.6, 2)
        wl, pl, g = prim_state(rng, 6, vxl, 0.0)
        wr, pr, _ = prim_state(rng, 6, vxr, 0.0)
        d = rng.normal(0.0, 0.3, 3)
        out = ref.hllc(wl, wr, pl, pr, g, g, d[0], d[1], d[2])
        X.append(np.concatenate([wl, wr, [pl, pr, g, g], d]))
        Y.append(out)
    return np.array(X), np.array(Y)


def digest(*arrays) -> str:
    h = hashlib.sha256()
    for a in arrays:
        h.update(np.ascontiguousarray(a, dtype=np.float64).tobytes())
    return h.hexdigest()


def main():
    rng = np.random.default_rng(20260101)
    rs = Restatement()
    mhd = R.Reference(True)
    hyd = R.Reference(False)
    mhd.setup(R.params_fourier(root=1, nmodes=2, kmax=1))
    hyd.setup(R.params_sod(nblocks_x=1))

    out = {}
    X, Y, K = hlld_cases(mhd, rs, rng)
    out.update(hlld_in=X, hlld_out=Y, hlld_kind=K)
    X, Y = hllc_cases(hyd, rng)
    out.update(hllc_in=X, hllc_out=Y)

    q = rng.normal(0.0, 1.0, (400, 3))
    q[:40, 1] = q[:40, 0]                       # flat left
    q[40:80, 2] = q[40:80, 1]                   # flat right
    q[80:120] = 0.0                             # all zero
    q[120:160, 1] = 0.5 * (q[120:160, 0] + q[120:160, 2])   # linear
    out["mc_in"] = q
    out["mc_out"] = np.array([mhd.mc_slope(*r) for r in q])

    f = rng.normal(0.0, 1.0, (300, 4))
    c = rng.normal(0.0, 1.0, (300, 4))
    vn = rng.normal(0.0, 1.0, (300, 4))
    vn[rng.random((300, 4)) < 0.3] = 0.0
    out.update(emf_f=f, emf_c=c, emf_vn=vn,
               emf_out=np.array([mhd.emf_upwind(f[n], c[n], vn[n]) for n in range(300)]))

    w9 = np.array([prim_state(rng, 9, rng.normal(), 1.0)[0] for _ in range(100)])
    u9 = np.array([mhd.prim2cons(w) for w in w9])
    w6 = np.array([prim_state(rng, 6, rng.normal(), 0.0)[0] for _ in range(100)])
    u6 = np.array([hyd.prim2cons(w) for w in w6])
    out.update(p2c9_in=w9, p2c9_out=u9, c2p9_out=np.array([mhd.cons2prim(u) for u in u9]),
               p2c6_in=w6, p2c6_out=u6, c2p6_out=np.array([hyd.cons2prim(u) for u in u6]))
    mhd.set_gamma(5.0 / 3.0)
    re = rng.uniform(0.1, 5.0, (100, 2))
    out.update(eos_in=re, eos_out=np.array([mhd.eos_rey(r[0], r[1], 0.1) for r in re]))

    # whole RK2 steps of the reference (state checksums after 3 steps)
    for name, lib, p in (("mhd_block1", mhd, R.params_fourier(root=1, nmodes=8, kmax=2)),
                         ("mhd_block8", mhd, R.params_fourier(root=2, nmodes=8, kmax=2)),
                         ("hydro_sod4", hyd, R.params_sod(nblocks_x=4))):
        lib.setup(p)
        n, t, dt, st = lib.run(3)
        arrays = [lib.W(b) for b in range(lib.nblocks())]
        if lib.mhd:
            arrays += [lib.Bf(b, d) for b in range(lib.nblocks()) for d in range(3)]
        out[f"{name}_state"] = np.array([t, dt, st])
        out[f"{name}_sha256"] = np.array(digest(*arrays))
        out[f"{name}_W0_center"] = lib.W(0)[::977].copy()

    np.savez_compressed(os.path.join(HERE, "reference_vectors.npz"), **out)
    print("wrote", os.path.join(HERE, "reference_vectors.npz"),
          {k: v.shape for k, v in out.items()})


if __name__ == "__main__":
    main()
