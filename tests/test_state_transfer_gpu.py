"""fx_upload_state_active / fx_download_state_active: the state through its
active region, against the full-array transfers.

Both copy the rows of the active region (the active (i, j) range, every k)
with the copy engines.  The upload then sets the cell field from the faces
and runs the slot-0 ghost fill, so after one full upload (the contract: a
few outermost ghost entries are written by no fill and keep their set-up
values) the device state must return to the host's state bit for bit even
after the device has stepped away from it, and stay equal to a fresh full
upload through a step.  The download must reproduce those rows of a full
download and leave every other host entry untouched.
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
        b.upload_all(np.ascontiguousarray(W), None if Bf is None else np.ascontiguousarray(Bf))
        dt = a.calc_dt(p.cfl)
        b.step(fx.FORM_BATCHED, dt)       # b moves away from the host state
        Wp = _pinned(W.shape)
        Wp[...] = W
        Bp = None
        if mhd:
            Bp = _pinned(Bf.shape)
            Bp[...] = Bf
        b.upload_state_active(Wp, Bp)
        Wa, Wb = np.empty_like(W), np.empty_like(W)
        Ba = np.empty_like(Bf) if mhd else None
        Bb = np.empty_like(Bf) if mhd else None
        a.download_all(Wa, Ba)
        b.download_all(Wb, Bb)
        assert np.array_equal(Wa[:, :, 0], Wb[:, :, 0])
        if mhd:
            assert np.array_equal(Ba[:, :, 0], Bb[:, :, 0])

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
        r = np.arange(-H.NG, 16 + H.NG)
        i, j, k = np.meshgrid(r, r, r, indexing="ij")
        rows = ((i >= 0) & (i < 16) & (j >= 0) & (j < 16)).ravel()
        cells = H.lidx(i, j, k).ravel()
        span = np.zeros(H.NCELLS, bool)
        span[cells[rows]] = True
        assert np.array_equal(Wp[:, :, 0][..., span], Wa[:, :, 0][..., span])
        assert np.isnan(Wp[:, :, 0][..., ~span]).all() and np.isnan(Wp[:, :, 1]).all()
        if mhd:
            for d in range(3):
                e = [np.arange(-H.NG, 16 + H.NG + (1 if a == d else 0)) for a in range(3)]
                fi, fj, fk = np.meshgrid(*e, indexing="ij")
                top = [16 if d == 0 else 15, 16 if d == 1 else 15]
                sel = ((fi >= 0) & (fi <= top[0]) & (fj >= 0) & (fj <= top[1])).ravel()
                faces = H.face_idx(d, fi, fj, fk).ravel()
                fspan = np.zeros(H.NFACES, bool)
                fspan[faces[sel]] = True
                assert np.array_equal(Bp[:, d, 0][:, fspan], Ba[:, d, 0][:, fspan])
                assert np.isnan(Bp[:, d, 0][:, ~fspan]).all()
    finally:
        a.close()
        b.close()
