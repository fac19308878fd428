"""The four benchmark configurations at their stated sizes, through the C ABI,
in both forms, against digests of the reference's own final state.

Sod tube (1024 cells, hydro, run to t = 0.2, about 2.4k steps), Fourier MHD
on 128^3 (512 blocks, 32 modes, 20 steps), the 3-level magnetised blast (8^3
roots, 2122 active blocks, 50 steps) and the 4-level gravity collapse (12^3
roots, 4584 active blocks, 100 steps).  The oracle builds the initial state
(the reference's own set-up code), the device runs the driver loop
(fx_run: calc_dt, dt limits, both RK2 stages, dt_src clamp), and the final
state of every active block is digested as in tests/config_cases.py and
compared with the digests the compiled reference produced from the same
initial state (tests/golden/make_config_digests.py).

Tolerance: agreement is expected bit for bit (same operations in the same
order, no contraction).  If a block's digest differs, the test measures the
stored sample of cells and faces instead and passes (with a warning naming
the blocks) only if its relative error is within the required 1e-12
(relative to the largest magnitude of each variable).
(t, dt, step) must be equal exactly, and div B of every active block must be
at round-off (<= 1e-13 relative to max |B| / dx).
"""
import os
import warnings

import numpy as np
import pytest

import fornaxamr_b200 as fx
from tests import config_cases as CC
from tests import helpers as H

pytestmark = pytest.mark.gpu

TOL = 1e-12
HERE = os.path.dirname(os.path.abspath(__file__))
FORMS = (("plain", fx.FORM_PLAIN), ("batched", fx.FORM_BATCHED))
_LAST_SETUP = {}


def _golden(name):
    path = os.path.join(HERE, "golden", f"config_{name}.npz")
    if not os.path.exists(path):
        pytest.fail(f"missing fixture {path}: run tests/golden/make_config_digests.py {name}")
    return dict(np.load(path))


def _setup(ref, case):
    """The oracle's initial state; the device run never steps the oracle, so a
    case set up by the previous test of this module is reused."""
    if _LAST_SETUP.get(case.mhd) != case.name:
        ref.setup(case.params())
        _LAST_SETUP[case.mhd] = case.name
    return case.params()


def _divb_rel(Bf_blocks, dx_blocks):
    """max over blocks of |div B| dx_min / max |B| (max over the mesh)."""
    r = np.arange(16)
    i, j, k = np.meshgrid(r, r, r, indexing="ij")
    f0 = [H.face_idx(0, i, j, k), H.face_idx(0, i + 1, j, k)]
    f1 = [H.face_idx(1, i, j, k), H.face_idx(1, i, j + 1, k)]
    f2 = [H.face_idx(2, i, j, k), H.face_idx(2, i, j, k + 1)]
    bmax = max(np.abs(f[d][H.active_faces(d)]).max() for f in Bf_blocks for d in range(3))
    worst = 0.0
    for f, dx in zip(Bf_blocks, dx_blocks):
        div = ((f[0][f0[1]] - f[0][f0[0]]) / dx[0] + (f[1][f1[1]] - f[1][f1[0]]) / dx[1]
               + (f[2][f2[1]] - f[2][f2[0]]) / dx[2])
        worst = max(worst, float(np.abs(div).max() * dx.min() / bmax))
    return worst


CASE_FORMS = [(n, f) for n in CC.CASES for f, _ in FORMS]


@pytest.mark.parametrize("name,form", CASE_FORMS, ids=[f"{n}-{f}" for n, f in CASE_FORMS])
def test_config_at_stated_size_matches_reference(request, name, form):
    case = CC.CASES[name]
    g = _golden(name)
    ref = request.getfixturevalue("ref_mhd" if case.mhd else "ref_hydro")
    p = _setup(ref, case)
    desc = H.ref_desc(ref)
    ints, geom, _ = ref.mesh_arrays()
    active = np.nonzero(ints[:, 2] == 1)[0]
    assert np.array_equal(active, g["active"])
    coord = [p.xmin[0], p.xmax[0], p.xmin[1], p.xmax[1], p.xmin[2], p.xmax[2]]
    ctx = fx.Context(case.mhd, p.gamma, coord, bc=tuple(p.bc), gravity=case.gravity)
    try:
        ctx.set_mesh(desc)
        for b in range(ref.nblocks()):
            try:
                W = ref.W(b)
            except ValueError:
                continue
            Bf = [ref.Bf(b, d) for d in range(3)] if case.mhd else None
            grav = [ref.grav(b, d) for d in range(3)] if case.gravity else None
            ctx.upload_block(b, W, Bf, grav)
        nsteps = int(g["steps_requested"])
        t, dt, st = ctx.run(dict(FORMS)[form], nsteps, p.cfl, p.dt_factor, p.t_end, (0.0, 0.0, 0.0))
        assert (t, dt, st) == (float(g["t"]), float(g["dt"]), int(g["step"]))
        md = CC.MeshDigest(active, ctx.nv, H.NCELLS, H.NFACES, case.mhd)
        Bf_act = []
        for b in active:
            W, _, Bf = ctx.download_block(int(b))
            md.add(b, W, Bf)
            if case.mhd:
                Bf_act.append([x[:H.NFACES] for x in Bf])
        got = md.arrays()
        bad = np.nonzero(np.any(got["block_digests"] != g["block_digests"], axis=1))[0]
        if len(bad):
            errs = []
            for v in range(ctx.nv):
                scale = max(np.abs(g["cell_vals"][:, v]).max(), 1e-300)
                errs.append(np.abs(got["cell_vals"][:, v] - g["cell_vals"][:, v]).max() / scale)
            if case.mhd:
                for d in range(3):
                    scale = max(np.abs(g["face_vals"][d]).max(), 1e-300)
                    errs.append(np.abs(got["face_vals"][d] - g["face_vals"][d]).max() / scale)
            worst = float(max(errs))
            msg = (f"{name}/{form}: {len(bad)} of {len(active)} block digests differ "
                   f"(first blocks {active[bad[:8]].tolist()}); sampled max relative error {worst:.3e}")
            assert worst <= TOL, msg
            warnings.warn(msg + " (within 1e-12 on the sample, but not bit-equal)")
        if case.mhd:
            dx = geom[active, 6:9]
            assert _divb_rel(Bf_act, dx) <= 1e-13
    finally:
        ctx.close()
