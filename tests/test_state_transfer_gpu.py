"""fx_upload_state_active / fx_download_state_active: the state through its
active region only, read and written by kernels straight from page-locked
host arrays, against the full-array transfers.

After an active-only upload the library runs the slot-0 ghost fill, so the
device state must equal the one a full upload of a host state whose ghosts
came from that fill gives, bit for bit (every ghost entry of slot 0 starts
as NaN on the device, so one the fill missed would show), and stay equal
after a step; an
active-only download must reproduce the active entries of a full download
and leave every other host entry untouched.  Pageable host memory is
rejected.
"""
import numpy as np
import pytest

import fornaxamr_b200 as fx
from oracle import ref as R
from tests import helpers as H

pytestmark = pytest.mark.gpu


def _pinned(shape):
    import torch
    return torch.empty(int(np.prod(shape)), dtype=torch.float64, pin_memory=True).numpy().reshape(shape)


def _ctx(ref, p, mhd):
    coord = [p.xmin[0], p.xmax[0], p.xmin[1], p.xmax[1], p.xmin[2], p.xmax[2]]
    ctx = fx.Context(mhd, p.gamma, coord, bc=tuple(p.bc))
    ctx.set_mesh(H.ref_desc(ref))
    return ctx


@pytest.mark.parametrize("mhd", [True, False])
def test_active_state_transfers_match_full_transfers(ref_mhd, ref_hydro, mhd):
    ref = ref_mhd if mhd else ref_hydro
    p = R.params_fourier(root=2, nmodes=8, kmax=2) if mhd else R.params_sod(nblocks_x=8)
    ref.setup(p)
    W, Bf = H.ref_state(ref)          # after the reference's set-up fill
    a = _ctx(ref, p, mhd)
    b = _ctx(ref, p, mhd)
    try:
        a.upload_all(np.ascontiguousarray(W), None if Bf is None else np.ascontiguousarray(Bf))
        # b starts with slot 0 scrambled (NaN) and slot 1 as a's
        Ws = W.copy()
        Ws[:, :, 0] = np.nan
        Bs = None
        if mhd:
            Bs = Bf.copy()
            Bs[:, :, 0] = np.nan
        b.upload_all(Ws, Bs)
        # the host copy holds the active entries of slot 0 only
        act = H.active_cells()
        Wp = _pinned(W.shape)
        Wp[...] = np.nan
        Wp[:, :, 0, act] = W[:, :, 0, act]
        Bp = None
        if mhd:
            Bp = _pinned(Bf.shape)
            Bp[...] = np.nan
            for d in range(3):
                fa = H.active_faces(d)
                Bp[:, d, 0, fa] = Bf[:, d, 0, fa]
        b.upload_state_active(Wp, Bp)
        Wa, Wb = np.empty_like(W), np.empty_like(W)
        Ba = np.empty_like(Bf) if mhd else None
        Bb = np.empty_like(Bf) if mhd else None
        a.download_all(Wa, Ba)
        b.download_all(Wb, Bb)
        assert np.array_equal(Wa[:, :, 0], Wb[:, :, 0])
        if mhd:
            assert np.array_equal(Ba[:, :, 0], Bb[:, :, 0])

        dt = a.calc_dt(p.cfl)
        assert b.calc_dt(p.cfl) == dt
        a.step(fx.FORM_BATCHED, dt)
        b.step(fx.FORM_BATCHED, dt)
        a.download_all(Wa, Ba)
        b.download_all(Wb, Bb)
        assert np.array_equal(Wa, Wb)
        if mhd:
            assert np.array_equal(Ba, Bb)

        Wp[...] = np.nan
        if mhd:
            Bp[...] = np.nan
        b.download_state_active(Wp, Bp)
        assert np.array_equal(Wp[:, :, 0][..., act], Wa[:, :, 0][..., act])
        rest = np.ones(H.NCELLS, bool)
        rest[act] = False
        assert np.isnan(Wp[:, :, 0][..., rest]).all() and np.isnan(Wp[:, :, 1]).all()
        if mhd:
            for d in range(3):
                fa = H.active_faces(d)
                assert np.array_equal(Bp[:, d, 0][:, fa], Ba[:, d, 0][:, fa])
                rest = np.ones(H.NFACES, bool)
                rest[fa] = False
                assert np.isnan(Bp[:, d, 0][:, rest]).all()

        with pytest.raises(fx.FxError):
            b.upload_state_active(np.ascontiguousarray(W), None if Bf is None else np.ascontiguousarray(Bf))
    finally:
        a.close()
        b.close()
