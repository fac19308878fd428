"""The dump payloads of prj_io_write_dump (src/prj_io.c:1994-2330, dump format
version 4): fx_dump_metadata's MetaData rows and fx_dump_gather's Data, Eos
and Bf rows against a numpy restatement of the reference's packing applied
to the reference's own block arrays and mesh (the oracle).  The HDF5
container itself is not written here (no HDF5 library in this image)."""
import numpy as np
import pytest

import fornaxamr_b200 as fx
from oracle import ref as R
from tests import helpers as H

AMR3 = dict(root=3, radii=(0.25, 0.1))


def metadata_restated(ref):
    """prj_io_fill_metadata (src/prj_io.c:1133-1165) over the reference's
    blocks; a slot's xmin / xmax / dx are its neighbour's (prj_add_neighbor,
    src/prj_amr.c:540-565, no periodic shift), zero for a free slot."""
    ints, geom, slots = ref.mesh_arrays()
    tree = ref.tree_arrays()
    nb = len(ints)
    m = np.zeros((nb, 639))
    m[:, 0] = ints[:, 0]
    m[:, 2] = ints[:, 1]
    m[:, 3] = ints[:, 2]
    m[:, 4:13] = geom[:, 0:9]
    m[:, 13] = tree[:, 0]
    m[:, 15:23] = tree[:, 1:9]
    for b in range(nb):
        idx = 23
        for n in range(56):
            nid = int(slots[b, n, 0])
            m[b, idx] = nid
            if 0 <= nid < nb:
                m[b, idx + 2:idx + 11] = geom[nid, 0:9]
            idx += 11
    return m


def dump_restated(ref, mhd):
    """the Data / Eos / Bf loops of prj_io_write_dump: active blocks only,
    stage slot 0, cell = (i 16 + j) 16 + k"""
    ints, _, _ = ref.mesh_arrays()
    nb = len(ints)
    nv = ref.nhydro
    data = np.zeros((nb, nv, 4096))
    eos = np.zeros((nb, 3, 4096))
    bf = np.zeros((nb, 3, H.NFACES)) if mhd else None
    r = np.arange(16)
    i, j, k = np.meshgrid(r, r, r, indexing="ij")
    cells = H.lidx(i, j, k).ravel()
    eidx = [H.bidx(3, v, i, j, k).ravel() for v in range(3)]
    for b in np.nonzero(ints[:, 2] == 1)[0]:
        W = ref.W(b).reshape(nv, ref.nstages, H.NCELLS)
        data[b] = W[:, 0, cells]
        ev = ref.eosvar(b)
        for v in range(3):
            eos[b, v] = ev[eidx[v]]
        if mhd:
            for d in range(3):
                bf[b, d] = ref.Bf(b, d)[:H.NFACES]
    return data, eos, bf


def test_metadata_rows_match_the_reference_packing(ref_mhd):
    p = R.params_amr_blast(**AMR3)
    ref_mhd.setup(p)
    got = fx.dump_metadata(H.ref_desc(ref_mhd))
    assert np.array_equal(got, metadata_restated(ref_mhd))


@pytest.mark.gpu
@pytest.mark.parametrize("case", ["fourier", "blast", "sod"])
def test_dump_payloads_match_the_reference_packing(ref_mhd, ref_hydro, case):
    mhd = case != "sod"
    ref = ref_mhd if mhd else ref_hydro
    p = {"fourier": lambda: R.params_fourier(root=2, nmodes=8, kmax=2),
         "blast": lambda: R.params_amr_blast(**AMR3),
         "sod": lambda: R.params_sod(nblocks_x=8)}[case]()
    ref.setup(p)
    coord = [p.xmin[0], p.xmax[0], p.xmin[1], p.xmax[1], p.xmin[2], p.xmax[2]]
    ctx = fx.Context(mhd, p.gamma, coord, bc=tuple(p.bc))
    try:
        ctx.set_mesh(H.ref_desc(ref))
        W, Bf = H.ref_state(ref)
        for b in range(W.shape[0]):
            ctx.upload_block(b, W[b].ravel(), None if Bf is None else [Bf[b, d].ravel() for d in range(3)])
        assert ctx.run(fx.FORM_BATCHED, 2, p.cfl, p.dt_factor, p.t_end, (0.0, 0.0, 0.0)) == ref.run(2)[1:]
        data, eos, bf = ctx.dump_gather(bf=True)
        rd, re, rb = dump_restated(ref, mhd)
        assert np.array_equal(data, rd)
        assert np.array_equal(eos, re)
        if mhd:
            assert np.array_equal(bf, rb)
    finally:
        ctx.close()
