"""fx_calc_dt_noalloc, the allocation-free timestep over caller-owned device
state, against the context's fx_calc_dt on the same blocks.

The caller's device buffers are torch tensors (the test is the caller; the
entry point itself allocates nothing).  Tolerance: 1e-12 relative, the same
bound as the other parity tests; both paths evaluate the same per-cell
operations in the same order, so equality is expected.
"""
import ctypes

import numpy as np
import pytest

import fornaxamr_b200 as fx
from fornaxamr_b200 import _lib
from oracle import ref as R
from tests import helpers as H

TOL = 1e-12


def test_capacity_and_arguments_rejected_before_device_work():
    L = fx.library()
    fake = ctypes.c_void_p(256)  # never dereferenced: the checks come first
    too_many = _lib.NOALLOC_MAX_BLOCKS + 1
    assert L.fx_calc_dt_noalloc(fake, 1, fake, None, too_many, 5.0 / 3.0, 0.4, None, fake) == _lib.FX_ETOOBIG
    assert L.fx_calc_dt_noalloc(fake, 1, fake, None, 0, 5.0 / 3.0, 0.4, None, fake) == _lib.FX_EINVAL
    assert L.fx_calc_dt_noalloc(None, 1, fake, None, 8, 5.0 / 3.0, 0.4, None, fake) == _lib.FX_EINVAL
    assert L.fx_calc_dt_noalloc(fake, 2, fake, None, 8, 5.0 / 3.0, 0.4, None, fake) == _lib.FX_EINVAL


def _context_dt(ref, p, mhd):
    desc = H.ref_desc(ref)
    coord = [p.xmin[0], p.xmax[0], p.xmin[1], p.xmax[1], p.xmin[2], p.xmax[2]]
    ctx = fx.Context(mhd, p.gamma, coord)
    ctx.set_mesh(desc)
    W, Bf = H.ref_state(ref)
    for b in range(W.shape[0]):
        ctx.upload_block(b, W[b].ravel(), None if Bf is None else [Bf[b, d].ravel() for d in range(3)])
    dt = ctx.calc_dt(p.cfl)
    ctx.close()
    return dt, W


@pytest.mark.gpu
@pytest.mark.parametrize("mhd", [1, 0])
def test_noalloc_dt_matches_context_dt_twice(ref_mhd, ref_hydro, mhd):
    import torch
    if mhd:
        ref, p = ref_mhd, R.params_fourier(root=2, nmodes=8, kmax=2)
    else:
        ref, p = ref_hydro, R.params_sod(nblocks_x=8)
    ref.setup(p)
    dt_ctx, W = _context_dt(ref, p, bool(mhd))
    assert dt_ctx == ref.calc_dt()

    nb = W.shape[0]
    dev = torch.device("cuda:0")
    Wd = torch.from_numpy(np.ascontiguousarray(W)).to(dev)
    dx = torch.tensor(np.stack([ref.block_geom(b)[1][6:9] for b in range(nb)]), dtype=torch.float64, device=dev)
    blocks = torch.arange(nb - 1, -1, -1, dtype=torch.int32, device=dev)  # every block, listed backwards
    out = torch.full((4,), float("nan"), dtype=torch.float64, device=dev)
    stream = ctypes.c_void_p(torch.cuda.current_stream(dev).cuda_stream)
    L = fx.library()
    for n, blist in enumerate((None, None, blocks, blocks)):
        rc = L.fx_calc_dt_noalloc(ctypes.c_void_p(Wd.data_ptr()), mhd, ctypes.c_void_p(dx.data_ptr()),
                                  None if blist is None else ctypes.c_void_p(blist.data_ptr()), nb,
                                  p.gamma, p.cfl, stream, ctypes.c_void_p(out.data_ptr() + 8 * n))
        assert rc == _lib.FX_SUCCESS
    torch.cuda.synchronize(dev)
    got = out.cpu().numpy()
    assert np.all(np.abs(got - dt_ctx) <= TOL * abs(dt_ctx))
    assert got[0] == got[1] and got[2] == got[3]
