"""fx_calc_dt_noalloc, the allocation-free timestep over caller-owned device
state, against the context's fx_calc_dt on the same blocks.

Some hosts cannot call cudaMalloc while they step (their device memory is a
fixed pool carved up at start-up, or the step runs where allocation is not
allowed), so this entry point keeps its scratch in a static device array.
The caller's device buffers here are torch tensors (the test is the caller;
the entry point itself allocates nothing).  Tolerance: 1e-12 relative, the
same bound as the other parity tests; both paths evaluate the same per-cell
operations in the same order, so equality is expected.  Cases: MHD and
hydro with RK2, MHD with eSSPRK10_4 (three stage slots, dt x 6), a list with
an index outside the state (NaN result), each called twice in a row; and
the same tests again in a child process on the four-ghost-layer library.
"""
import ctypes
import os
import subprocess
import sys

import numpy as np
import pytest

import fornaxamr_b200 as fx
from fornaxamr_b200 import _lib
from oracle import ref as R
from tests import helpers as H

TOL = 1e-12
HERE = os.path.dirname(os.path.abspath(__file__))


def test_capacity_and_arguments_rejected_before_device_work():
    L = fx.library()
    fake = ctypes.c_void_p(256)  # never dereferenced: the checks come first
    too_many = _lib.NOALLOC_MAX_BLOCKS + 1
    rk2, ess = fx.INT_RK2, fx.INT_ESSPRK10_4
    assert L.fx_calc_dt_noalloc(fake, 1, rk2, fake, 8, None, too_many, 5.0 / 3.0, 0.4, None, fake) == _lib.FX_ETOOBIG
    assert L.fx_calc_dt_noalloc(fake, 1, rk2, fake, 8, None, 0, 5.0 / 3.0, 0.4, None, fake) == _lib.FX_EINVAL
    assert L.fx_calc_dt_noalloc(fake, 1, ess, fake, 0, None, 8, 5.0 / 3.0, 0.4, None, fake) == _lib.FX_EINVAL
    assert L.fx_calc_dt_noalloc(None, 1, rk2, fake, 8, None, 8, 5.0 / 3.0, 0.4, None, fake) == _lib.FX_EINVAL
    assert L.fx_calc_dt_noalloc(fake, 2, rk2, fake, 8, None, 8, 5.0 / 3.0, 0.4, None, fake) == _lib.FX_EINVAL
    assert L.fx_calc_dt_noalloc(fake, 1, 7, fake, 8, None, 8, 5.0 / 3.0, 0.4, None, fake) == _lib.FX_EINVAL


def _context_dt(ref, p, mhd, integrator):
    desc = H.ref_desc(ref)
    coord = [p.xmin[0], p.xmax[0], p.xmin[1], p.xmax[1], p.xmin[2], p.xmax[2]]
    ctx = fx.Context(mhd, p.gamma, coord, integrator=integrator)
    ctx.set_mesh(desc)
    nb = ref.nblocks()
    W = np.stack([ref.W(b) for b in range(nb)])
    for b in range(nb):
        ctx.upload_block(b, W[b], [ref.Bf(b, d) for d in range(3)] if mhd else None)
    dt = ctx.calc_dt(p.cfl)
    ctx.close()
    return dt, W


CASES = [("mhd_rk2", 1, fx.INT_RK2), ("hydro_rk2", 0, fx.INT_RK2), ("mhd_essprk10_4", 1, fx.INT_ESSPRK10_4)]


@pytest.mark.gpu
@pytest.mark.parametrize("name,mhd,integrator", CASES, ids=[c[0] for c in CASES])
def test_noalloc_dt_matches_context_dt_twice(name, mhd, integrator):
    import torch
    # the eSSPRK10_4 reference build of this library's ghost layers (the
    # four-layer one is built with WENO-Z7; the timestep does not depend on it)
    variant = ("ess" if fx.NG == 2 else "ess_weno7") if integrator == fx.INT_ESSPRK10_4 else ""
    ref = R.Reference(bool(mhd), variant)
    p = R.params_fourier(root=2, nmodes=8, kmax=2) if mhd else R.params_sod(nblocks_x=8)
    ref.setup(p)
    dt_ctx, W = _context_dt(ref, p, bool(mhd), integrator)
    assert dt_ctx == ref.calc_dt()

    nb = W.shape[0]
    dev = torch.device("cuda:0")
    Wd = torch.from_numpy(np.ascontiguousarray(W)).to(dev)
    dx = torch.tensor(np.stack([ref.block_geom(b)[1][6:9] for b in range(nb)]), dtype=torch.float64, device=dev)
    blocks = torch.arange(nb - 1, -1, -1, dtype=torch.int32, device=dev)  # every block, listed backwards
    outside = torch.tensor([0, nb, 1], dtype=torch.int32, device=dev)     # one index past the state
    out = torch.full((6,), float("nan"), dtype=torch.float64, device=dev)
    stream = ctypes.c_void_p(torch.cuda.current_stream(dev).cuda_stream)
    L = fx.library()
    for n, (blist, nlist) in enumerate(((None, nb), (None, nb), (blocks, nb), (blocks, nb),
                                        (outside, 3), (outside, 3))):
        out[n] = 0.0
        rc = L.fx_calc_dt_noalloc(ctypes.c_void_p(Wd.data_ptr()), mhd, integrator, ctypes.c_void_p(dx.data_ptr()),
                                  nb, None if blist is None else ctypes.c_void_p(blist.data_ptr()), nlist,
                                  p.gamma, p.cfl, stream, ctypes.c_void_p(out.data_ptr() + 8 * n))
        assert rc == _lib.FX_SUCCESS
    torch.cuda.synchronize(dev)
    got = out.cpu().numpy()
    assert np.all(np.abs(got[:4] - dt_ctx) <= TOL * abs(dt_ctx))
    assert got[0] == got[1] and got[2] == got[3]
    assert np.isnan(got[4]) and np.isnan(got[5])


@pytest.mark.gpu
@pytest.mark.skipif(fx.NG == 4, reason="already the four-ghost-layer library")
def test_noalloc_on_four_ghost_layer_library():
    """The same GPU tests in a child process with FX_NGHOST=4
    (libfornax_b200_ng4.so, 24^3 cells per block)."""
    env = dict(os.environ, FX_NGHOST="4")
    r = subprocess.run([sys.executable, "-m", "pytest", "-q", "-p", "no:cacheprovider", "-m", "gpu",
                        os.path.join(HERE, "test_zz_no_alloc.py"), "-k", "matches_context"],
                       cwd=os.path.dirname(HERE), env=env, capture_output=True, text=True, timeout=900)
    assert r.returncode == 0, r.stdout[-4000:] + r.stderr[-2000:]
    assert "3 passed" in r.stdout
