"""CPU checks of the host side against the reference:
  - the product's mesh builder reproduces prj_mesh_init's blocks and
    neighbour slots (src/prj_mesh.c:1438-1686, 46-243);
  - the compiled ghost-fill programs, interpreted in numpy, reproduce
    prj_boundary_fill_ghosts_and_bf (src/prj_boundary.c:1150-1241) bit for bit
    on a state whose ghost zones were scrambled first.
"""
import numpy as np
import pytest

from oracle import ref as R
from tests import helpers as H


def _desc_and_cfg(ref, p, mhd, use_bj=False):
    import fornaxamr_b200 as fx
    desc = H.ref_desc(ref)
    coord = [p.xmin[0], p.xmax[0], p.xmin[1], p.xmax[1], p.xmin[2], p.xmax[2]]
    return desc, fx.make_config(mhd, p.gamma, coord, bc=tuple(p.bc), use_bj=use_bj)


@pytest.mark.parametrize("root", [(2, 2, 2), (3, 2, 1), (1, 1, 1)])
def test_uniform_mesh_matches_reference(ref_mhd, root):
    from fornaxamr_b200 import mesh
    p = R.params_fourier(root=1)
    p.root[:] = list(root)
    p.xmax[:] = [1.0, 0.75, 0.5]
    ref_mhd.setup(p)
    ints, geom, slots = ref_mhd.mesh_arrays()
    blocks = mesh.uniform_mesh(root, (0.0, 1.0, 0.0, 0.75, 0.0, 0.5))
    mi, mg, ms = mesh.desc_to_arrays(mesh.to_desc(blocks))
    assert np.array_equal(mi[:, :3], ints[:, :3])
    assert np.array_equal(mg, geom)
    # unused slots: the reference leaves id -1 and zero boxes
    assert np.array_equal(ms, slots)


def _scrambled_fill_check(ref, p, mhd, seed, use_bj=False):
    ref.setup(p)
    ref.set_use_bj(use_bj)
    desc, cfg = _desc_and_cfg(ref, p, mhd, use_bj)
    W, Bf = H.ref_state(ref)
    nb = W.shape[0]
    rng = np.random.default_rng(seed)
    ghost = np.ones(H.NCELLS, bool)
    ghost[H.active_cells()] = False
    for b in range(nb):
        W[b, :, 0, ghost] = rng.uniform(0.5, 2.0, size=(ghost.sum(), W.shape[1]))
        ref.set_W(b, W[b].ravel())
        if mhd:
            for d in range(3):
                gf = np.ones(H.NFACES, bool)
                gf[H.active_faces(d)] = False
                Bf[b, d, 0, gf] = rng.uniform(-1.0, 1.0, size=gf.sum())
                ref.set_Bf(b, d, Bf[b, d].ravel())
    ref.fill_ghosts(1, 0)
    W_ref, Bf_ref = H.ref_state(ref)
    ref.set_use_bj(False)

    Wm = W.copy()
    Bm = Bf.copy() if mhd else None
    nw = H.apply_ghost_program(Wm, Bm, cfg, desc, 0)
    if mhd:
        assert np.array_equal(Bm[:, :, 0], Bf_ref[:, :, 0])
    assert np.array_equal(Wm[:, :, 0], W_ref[:, :, 0])
    return nw


@pytest.mark.parametrize("root", [(2, 2, 2), (3, 3, 2), (1, 1, 1)])
def test_mhd_ghost_program_matches_reference(ref_mhd, root):
    p = R.params_fourier(root=1, nmodes=4, kmax=2)
    p.root[:] = list(root)
    nw = _scrambled_fill_check(ref_mhd, p, True, seed=sum(root))
    # single-level meshes collapse to one wave after copy propagation
    assert nw == 1


def test_hydro_ghost_program_matches_reference(ref_hydro):
    p = R.params_sod(nblocks_x=4)
    _scrambled_fill_check(ref_hydro, p, False, seed=7)


def test_ghost_program_waves_are_conflict_free(ref_mhd):
    import fornaxamr_b200 as fx
    p = R.params_fourier(root=2, nmodes=2, kmax=1)
    ref_mhd.setup(p)
    desc, cfg = _desc_and_cfg(ref_mhd, p, True)
    cops, cw = fx.plan_export(cfg, desc, 0)
    fops, fw = fx.plan_export(cfg, desc, 1)
    bops, bw = fx.plan_export(cfg, desc, 4)
    for w in range(len(cw) - 1):
        c = cops[cw[w]:cw[w + 1]]
        cdst = c[:, 0].astype(np.int64)
        assert len(np.unique(cdst)) == len(cdst)
        assert not np.intersect1d(cdst, c[:, 1]).size
        f = fops[fw[w]:fw[w + 1]]
        fdst = f[:, 0].astype(np.int64) * 4 + (f[:, 2] & 3)
        assert len(np.unique(fdst)) == len(fdst)
        assert not np.intersect1d(fdst, f[:, 1].astype(np.int64) * 4 + (f[:, 2] & 3)).size
        b = bops[bw[w]:bw[w + 1]]
        assert len(np.unique(b[:, 0])) == len(b)
        for d in range(3):
            reads = np.concatenate([b[:, 1 + 2 * d], b[:, 2 + 2 * d]]).astype(np.int64) * 4 + d
            assert not np.intersect1d(fdst, reads).size


def test_ghost_compiler_statistics(ref_mhd):
    """Copy propagation and dead-write elimination remove the reference's
    repeated boundary passes: fewer operations than writes that land, and
    exactly one destination per ghost element."""
    import fornaxamr_b200 as fx
    p = R.params_fourier(root=2, nmodes=2, kmax=1)
    ref_mhd.setup(p)
    desc, cfg = _desc_and_cfg(ref_mhd, p, True)
    stats, _ = fx.plan_export(cfg, desc, 5)
    emitted_cells, emitted_faces, rewired, dead = (int(x) for x in stats[:, 0])
    cops, _ = fx.plan_export(cfg, desc, 0)
    fops, _ = fx.plan_export(cfg, desc, 1)
    bops, _ = fx.plan_export(cfg, desc, 4)
    assert rewired > 0 and dead > 0
    assert len(cops) + len(fops) == emitted_cells + emitted_faces - dead
    # every ghost cell of every block written once (8 blocks x (PBS^3 - 16^3))
    assert len(np.unique(cops[:, 0])) == len(cops) == 8 * (H.PBS ** 3 - 16 ** 3)
    assert len(bops) == 8 * (H.PBS ** 3 - 16 ** 3)


# static AMR hierarchies of the magnetised blast: (root, radii) -> per-level
# active blocks [0, 60, 32] (levels 1-2) and [9, 140, 32] (levels 0-2, with
# level-1 blocks that are coarse for one neighbour and fine for another)
AMR_CASES = [(2, (0.3, 0.1)), (3, (0.25, 0.1))]


@pytest.mark.parametrize("root,radii", AMR_CASES)
def test_amr_ghost_program_matches_reference(ref_mhd, root, radii):
    p = R.params_amr_blast(root=root, radii=radii)
    nw = _scrambled_fill_check(ref_mhd, p, True, seed=root)
    assert nw >= 2


def test_amr_hydro_ghost_program_matches_reference(ref_hydro):
    p = R.params_amr_blast(root=2, radii=(0.3, 0.1))
    _scrambled_fill_check(ref_hydro, p, False, seed=11)


@pytest.mark.parametrize("root,radii", AMR_CASES)
def test_amr_ghost_program_with_barth_jespersen_matches_reference(ref_mhd, root, radii):
    """use_BJ = 1: the cell prolongations read all 27 coarse cells and the
    outer faces of the Toth-Roe groups the 3x3 tangential face stencil
    (src/prj_reconstruct.h:145-195, 248-290)."""
    import fornaxamr_b200 as fx
    p = R.params_amr_blast(root=root, radii=radii)
    nw = _scrambled_fill_check(ref_mhd, p, True, seed=root + 5, use_bj=True)
    assert nw >= 2
    desc, cfg = _desc_and_cfg(ref_mhd, p, True, use_bj=True)
    cops, _ = fx.plan_export(cfg, desc, 0)
    pops, _ = fx.plan_export(cfg, desc, 6)
    assert (cops[:, 3] == H.GOP_PROLONG_BJ).sum() > 0 and (cops[:, 3] == H.GOP_PROLONG).sum() == 0
    assert len(pops) > 0 and np.all(pops[:, 6] & 1)


def test_amr_hydro_ghost_program_with_barth_jespersen_matches_reference(ref_hydro):
    p = R.params_amr_blast(root=2, radii=(0.3, 0.1))
    _scrambled_fill_check(ref_hydro, p, False, seed=13, use_bj=True)


@pytest.mark.parametrize("root,radii", AMR_CASES)
def test_amr_corrections_match_reference(ref_mhd, root, radii):
    """prj_riemann_flux_send and prj_mhd_emf_send on scrambled flux / EMF
    arrays against the compiled correction records."""
    import fornaxamr_b200 as fx
    p = R.params_amr_blast(root=root, radii=radii)
    ref_mhd.setup(p)
    desc, cfg = _desc_and_cfg(ref_mhd, p, True)
    nb = ref_mhd.nblocks()
    rng = np.random.default_rng(root)
    flux = rng.uniform(-1.0, 1.0, size=(nb, 3, 9 * H.NCELLS))
    emf = rng.uniform(-1.0, 1.0, size=(nb, 3, H.NEDGES))
    emf[rng.uniform(size=emf.shape) < 0.05] = -0.0
    for b in range(nb):
        for d in range(3):
            ref_mhd.set_flux(b, d, flux[b, d])
            ref_mhd.set_emf(b, d, emf[b, d])
    ref_mhd.flux_send()
    ref_mhd.emf_send()
    frec, fw = fx.plan_export(cfg, desc, 2)
    erec, ew = fx.plan_export(cfg, desc, 3)
    assert len(frec) > 0 and len(erec) > 0
    H.apply_corrections(flux, frec, fw, "flux")
    H.apply_corrections(emf, erec, ew, "emf")
    for b in range(nb):
        for d in range(3):
            assert np.array_equal(flux[b, d], ref_mhd.flux(b, d))
            assert np.array_equal(emf[b, d].view(np.int64), ref_mhd.emf(b, d).view(np.int64))


@pytest.mark.parametrize("bc", [(1, 1, 0, 0, 0, 0), (2, 0, 1, 1, 0, 0), (1, 2, 0, 0, 1, 1)])
def test_hydro_reflect_and_user_boundaries_match_reference(ref_hydro, bc):
    """Reflecting (normal velocity negated) and user (v1 set) boundary bands,
    src/prj_boundary.c:413-530, on a 4 x 2 x 2 hydro mesh."""
    p = R.params_sod(nblocks_x=4)
    p.root[:] = [4, 2, 2]
    p.xmax[:] = [1.0, 0.5, 0.5]
    p.bc[:] = list(bc)
    _scrambled_fill_check(ref_hydro, p, False, seed=sum(bc))
