"""Shared test helpers: numpy views of the reference layout and a numpy
interpreter of the compiled ghost-fill programs (used to check the ghost-fill
compiler against the reference on the CPU)."""
from __future__ import annotations

import numpy as np

BS, NG, PBS = 16, 2, 20
NCELLS = PBS ** 3
NFACES = 21 * 20 * 20
NEDGES = 21 * 21 * 20

GOP_COPY, GOP_COPY_NEG, GOP_COPY_USER, GOP_RESTRICT, GOP_PROLONG = 0, 1, 2, 3, 4
FOP_COPY, FOP_RESTRICT, FOP_PROLONG = 8, 9, 10


def lidx(i, j, k):
    return ((np.asarray(i) + NG) * PBS + (np.asarray(j) + NG)) * PBS + (np.asarray(k) + NG)


def face_idx(d, i, j, k):
    i, j, k = (np.asarray(x) + NG for x in (i, j, k))
    if d == 0:
        return i * PBS * PBS + j * PBS + k
    if d == 1:
        return i * (PBS + 1) * PBS + j * PBS + k
    return i * PBS * (PBS + 1) + j * (PBS + 1) + k


def active_cells():
    r = np.arange(BS)
    i, j, k = np.meshgrid(r, r, r, indexing="ij")
    return lidx(i, j, k).ravel()


def active_faces(d):
    ri = np.arange(BS + 1 if d == 0 else BS)
    rj = np.arange(BS + 1 if d == 1 else BS)
    rk = np.arange(BS + 1 if d == 2 else BS)
    i, j, k = np.meshgrid(ri, rj, rk, indexing="ij")
    return face_idx(d, i, j, k).ravel()


def bidx(nc, v, i, j, k):
    """AoSoA index (4-wide k lanes) of component v of an nc-component buffer."""
    i, j, k = (np.asarray(x) + NG for x in (i, j, k))
    return ((((i * PBS + j) * (PBS // 4) + k // 4) * nc + v) * 4 + k % 4)


def computed_faces(d, mhd):
    """(i, j, k) of the faces prj_flux_update computes in direction d: normal
    index [0, 16], transverse [-1, 16] for MHD, [0, 15] for hydro."""
    rngs = []
    for a in range(3):
        if a == d:
            rngs.append(np.arange(0, BS + 1))
        else:
            rngs.append(np.arange(-1, BS + 1) if mhd else np.arange(0, BS))
    i, j, k = np.meshgrid(*rngs, indexing="ij")
    return i.ravel(), j.ravel(), k.ravel()


def flux_positions(d, nv, mhd):
    i, j, k = computed_faces(d, mhd)
    return np.concatenate([bidx(nv, v, i, j, k) for v in range(nv)])


def vr_positions(d, mhd):
    i, j, k = computed_faces(d, mhd)
    return np.concatenate([bidx(3, v, i, j, k) for v in range(3)])


def bv_positions(d):
    i, j, k = computed_faces(d, True)
    return lidx(i, j, k)


def edge_idx(d, i, j, k):
    i, j, k = (np.asarray(x) + NG for x in (i, j, k))
    if d == 0:
        return i * (PBS + 1) * (PBS + 1) + j * (PBS + 1) + k
    if d == 1:
        return i * PBS * (PBS + 1) + j * (PBS + 1) + k
    return i * (PBS + 1) * PBS + j * PBS + k


def emf_positions(d):
    """edges prj_timeint_mhd_update_emf computes: [0,15] along d, [0,16] across"""
    rngs = [np.arange(0, BS) if a == d else np.arange(0, BS + 1) for a in range(3)]
    i, j, k = np.meshgrid(*rngs, indexing="ij")
    return edge_idx(d, i.ravel(), j.ravel(), k.ravel())


def apply_cell_program(W, ops, waves, slot, nvg):
    """W: [nb, nv, 2, NCELLS] (modified in place)."""
    for w in range(len(waves) - 1):
        o = ops[waves[w]:waves[w + 1]]
        for t in np.unique(o[:, 3]):
            s = o[o[:, 3] == t]
            db, dc = s[:, 0] >> 13, s[:, 0] & 8191
            sb, sc = s[:, 1] >> 13, s[:, 1] & 8191
            if t in (GOP_COPY, GOP_COPY_NEG, GOP_COPY_USER):
                vals = W[sb, :nvg, slot, sc].copy()
                if t == GOP_COPY_NEG:
                    for n in range(len(s)):
                        vals[n, s[n, 2]] = -vals[n, s[n, 2]]
                if t == GOP_COPY_USER:
                    vals[s[:, 2] != 0, 1] = 5.0
                W[db, :nvg, slot, dc] = vals
            elif t == GOP_RESTRICT:
                acc = None
                for off in (0, 1, 20, 21, 400, 401, 420, 421):
                    v = W[sb, :nvg, slot, sc + off]
                    acc = v if acc is None else acc + v
                W[db, :nvg, slot, dc] = 0.125 * acc
            else:
                raise NotImplementedError(f"op type {t}")


def apply_face_program(Bf, ops, waves, slot):
    """Bf: [nb, 3, 2, NFACES] (modified in place)."""
    for w in range(len(waves) - 1):
        o = ops[waves[w]:waves[w + 1]]
        for t in np.unique(o[:, 3]):
            s = o[o[:, 3] == t]
            db, df = s[:, 0] >> 15, s[:, 0] & 32767
            sb, sf = s[:, 1] >> 15, s[:, 1] & 32767
            d = s[:, 2] & 3
            if t == FOP_COPY:
                Bf[db, d, slot, df] = Bf[sb, d, slot, sf]
            elif t == FOP_RESTRICT:
                o1 = (s[:, 2] >> 2) & 1023
                o0 = (s[:, 2] >> 12) & 1023
                Bf[db, d, slot, df] = 0.25 * (Bf[sb, d, slot, sf] + Bf[sb, d, slot, sf + o1]
                                              + Bf[sb, d, slot, sf + o0] + Bf[sb, d, slot, sf + o0 + o1])
            else:
                raise NotImplementedError(f"face op type {t}")


def apply_b_ops(W, Bf, bops, slot):
    """cell-field operations: W[6+d] of dst = 0.5 (f[2d] + f[2d+1])."""
    if len(bops) == 0:
        return
    db, dc = bops[:, 0] >> 13, bops[:, 0] & 8191
    for d in range(3):
        k0, k1 = bops[:, 1 + 2 * d], bops[:, 2 + 2 * d]
        W[db, 6 + d, slot, dc] = 0.5 * (Bf[k0 >> 15, d, slot, k0 & 32767] + Bf[k1 >> 15, d, slot, k1 & 32767])


def apply_ghost_program(W, Bf, cfg, desc, slot):
    """Runs the compiled ghost fill (fx_plan_export) in numpy, wave by wave."""
    import fornaxamr_b200 as fx
    cops, cw = fx.plan_export(cfg, desc, 0)
    nw = len(cw) - 1
    if Bf is not None:
        fops, fw = fx.plan_export(cfg, desc, 1)
        bops, bw = fx.plan_export(cfg, desc, 4)
    for w in range(nw):
        apply_cell_program(W, cops[cw[w]:cw[w + 1]], [0, cw[w + 1] - cw[w]], slot, 6)
        if Bf is not None:
            apply_face_program(Bf, fops[fw[w]:fw[w + 1]], [0, fw[w + 1] - fw[w]], slot)
            apply_b_ops(W, Bf, bops[bw[w]:bw[w + 1]], slot)
    return nw


def bf2bc(W, Bf, slot):
    r = np.arange(-NG, BS + NG)
    i, j, k = np.meshgrid(r, r, r, indexing="ij")
    c = lidx(i, j, k).ravel()
    i, j, k = i.ravel(), j.ravel(), k.ravel()
    W[:, 6, slot, c] = 0.5 * (Bf[:, 0, slot, face_idx(0, i, j, k)] + Bf[:, 0, slot, face_idx(0, i + 1, j, k)])
    W[:, 7, slot, c] = 0.5 * (Bf[:, 1, slot, face_idx(1, i, j, k)] + Bf[:, 1, slot, face_idx(1, i, j + 1, k)])
    W[:, 8, slot, c] = 0.5 * (Bf[:, 2, slot, face_idx(2, i, j, k)] + Bf[:, 2, slot, face_idx(2, i, j, k + 1)])


def ref_state(ref):
    nb = ref.nblocks()
    W = np.stack([ref.W(b).reshape(ref.nhydro, 2, NCELLS) for b in range(nb)])
    Bf = None
    if ref.mhd:
        Bf = np.stack([np.stack([ref.Bf(b, d).reshape(2, NFACES) for d in range(3)]) for b in range(nb)])
    return W, Bf


def ref_desc(ref):
    from fornaxamr_b200 import mesh
    ints, geom, slots = ref.mesh_arrays()
    return mesh.desc_from_arrays(ints, geom, slots)


def max_rel_err(a, b, floor=1e-300):
    a = np.asarray(a)
    b = np.asarray(b)
    scale = np.maximum(np.abs(b).max(), floor)
    return float(np.abs(a - b).max() / scale)
