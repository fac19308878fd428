"""Seeded synthetic workloads (host-side initial conditions).

The measured workloads use the recipes below; the same recipes are
implemented independently in the oracle harness so tests can compare the two
initial states.  Initial data are written for every cell and face of a
block, ghosts included, the way the reference's problem initialisers do
(e.g. problems/prj_problem_shock1d.c:38-62); the ghost zones are then
refilled on the device by the ghost fill.

Fourier-mode ideal MHD: rho = 1 + sum of n seeded modes, v = sum of n modes
times unit directions, p = 1, A = sum of n modes on cell edges and
B = curl A on faces with the discrete curl of the reference
(src/prj_mhd.c:106-142), so div B = 0 to round-off.  Each mode is
(amp/n) cos(2 pi k.x + phi) with integer k, 1 <= |k|_inf <= kmax, drawn from
splitmix64 (the generator of src/prj_perturbation.c:5-20).
"""
from __future__ import annotations

import math
from typing import List, Sequence, Tuple

import numpy as np

from .mesh import BS, NG, Block

PBS = BS + 2 * NG
NCELLS = PBS ** 3
NFACES = (PBS + 1) * PBS * PBS
MASK = (1 << 64) - 1


class SplitMix64:
    def __init__(self, seed: int):
        self.state = seed & MASK

    def next(self) -> int:
        self.state = (self.state + 0x9E3779B97F4A7C15) & MASK
        z = self.state
        z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & MASK
        z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & MASK
        return z ^ (z >> 31)

    def uniform01(self) -> float:
        return float(self.next() >> 11) * (1.0 / 9007199254740992.0)


def draw_modes(n: int, kmax: int, amp_total: float, seed: int):
    """(k [n,3], phase [n], dir [n,3], amp) -- same draw order as the oracle."""
    rng = SplitMix64(seed)
    k = np.zeros((n, 3))
    phase = np.zeros(n)
    dirs = np.zeros((n, 3))
    for q in range(n):
        while True:
            kk = [int(rng.next() % (2 * kmax + 1)) - kmax for _ in range(3)]
            if any(kk):
                break
        k[q] = kk
        phase[q] = 2.0 * math.pi * rng.uniform01()
        while True:
            d = [rng.uniform01() - 0.5 for _ in range(3)]
            dn = math.sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2])
            if dn >= 1.0e-3:
                break
        dirs[q] = [d[0] / dn, d[1] / dn, d[2] / dn]
    return k, phase, dirs, (amp_total / n if n > 0 else 0.0)


def _mode_sum(modes, x, y, z, vector: bool):
    k, phase, dirs, amp = modes
    out = np.zeros(x.shape + ((3,) if vector else ()))
    for q in range(k.shape[0]):
        arg = 2.0 * math.pi * (k[q, 0] * x + k[q, 1] * y + k[q, 2] * z) + phase[q]
        c = amp * np.cos(arg)
        if vector:
            out += c[..., None] * dirs[q]
        else:
            out += c
    return out


def _centers(b: Block, axis: int) -> np.ndarray:
    return b.xmin[axis] + (np.arange(-NG, BS + NG) + 0.5) * b.dx[axis]


def _edges(b: Block, axis: int, comp: int) -> np.ndarray:
    off = 0.5 if axis == comp else 0.0
    return b.xmin[axis] + (np.arange(-NG, BS + NG) + off) * b.dx[axis]


def _face_index(d: int, i, j, k):
    i, j, k = i + NG, j + NG, k + NG
    if d == 0:
        return (i * PBS + j) * PBS + k
    if d == 1:
        return (i * (PBS + 1) + j) * PBS + k
    return (i * PBS + j) * (PBS + 1) + k


def bf2bc_all(W: np.ndarray, Bf: np.ndarray, slot: int) -> None:
    """Cell B = face averages over all 20^3 cells (src/prj_mhd.c:555-603)."""
    r = np.arange(-NG, BS + NG)
    i, j, k = np.meshgrid(r, r, r, indexing="ij")
    W[6, slot] = (0.5 * (Bf[0, slot][_face_index(0, i, j, k)] + Bf[0, slot][_face_index(0, i + 1, j, k)])).ravel()
    W[7, slot] = (0.5 * (Bf[1, slot][_face_index(1, i, j, k)] + Bf[1, slot][_face_index(1, i, j + 1, k)])).ravel()
    W[8, slot] = (0.5 * (Bf[2, slot][_face_index(2, i, j, k)] + Bf[2, slot][_face_index(2, i, j, k + 1)])).ravel()


def fourier_mhd(blocks: Sequence[Block], nmodes: int = 32, kmax: int = 4, amp_rho: float = 0.1,
                amp_v: float = 0.1, amp_A: float = 0.05, gamma: float = 5.0 / 3.0,
                seeds: Tuple[int, int, int] = (1, 2, 3)):
    """Initial W [nb, 9, 2, 8000] and Bf [nb, 3, 2, 8400] of the Fourier-mode
    MHD workload on a single-level mesh."""
    m_rho = draw_modes(nmodes, kmax, amp_rho, seeds[0])
    m_v = draw_modes(nmodes, kmax, amp_v, seeds[1])
    m_A = draw_modes(nmodes, kmax, amp_A, seeds[2])
    nb = len(blocks)
    W = np.zeros((nb, 9, 2, NCELLS))
    Bf = np.zeros((nb, 3, 2, NFACES))
    r = np.arange(-NG, BS + NG)
    for n, b in enumerate(blocks):
        x, y, z = np.meshgrid(_centers(b, 0), _centers(b, 1), _centers(b, 2), indexing="ij")
        rho = 1.0 + _mode_sum(m_rho, x, y, z, False)
        v = _mode_sum(m_v, x, y, z, True)
        for s in range(2):
            W[n, 0, s] = rho.ravel()
            W[n, 1, s] = v[..., 0].ravel()
            W[n, 2, s] = v[..., 1].ravel()
            W[n, 3, s] = v[..., 2].ravel()
            W[n, 4, s] = (1.0 / ((gamma - 1.0) * rho)).ravel()
            W[n, 5, s] = 0.1
        # vector potential on edges: component d at edge (i, j, k)
        A = []
        for d in range(3):
            ex, ey, ez = np.meshgrid(_edges(b, 0, d), _edges(b, 1, d), _edges(b, 2, d), indexing="ij")
            A.append(_mode_sum(m_A, ex, ey, ez, True)[..., d])
        # discrete curl on faces i, j, k in [-2, 16] (src/prj_mhd.c:106-142);
        # A[d][i+2, j+2, k+2] holds edge (i, j, k)
        s = slice(0, PBS - 1)
        sp = slice(1, PBS)
        B1 = (A[2][s, sp, s] - A[2][s, s, s]) / b.dx[1] - (A[1][s, s, sp] - A[1][s, s, s]) / b.dx[2]
        B2 = (A[0][s, s, sp] - A[0][s, s, s]) / b.dx[2] - (A[2][sp, s, s] - A[2][s, s, s]) / b.dx[0]
        B3 = (A[1][sp, s, s] - A[1][s, s, s]) / b.dx[0] - (A[0][s, sp, s] - A[0][s, s, s]) / b.dx[1]
        fi, fj, fk = np.meshgrid(r[:-1], r[:-1], r[:-1], indexing="ij")
        for d, Bd in enumerate((B1, B2, B3)):
            Bf[n, d, 0][_face_index(d, fi, fj, fk)] = Bd
            Bf[n, d, 1] = Bf[n, d, 0]
        bf2bc_all(W[n], Bf[n], 0)
        bf2bc_all(W[n], Bf[n], 1)
    return W, Bf


def sod(blocks: Sequence[Block], gamma: float = 1.4):
    """Sod shock tube along x: (rho, p) = (1, 1) for x < 0.5, (0.125, 0.1)
    otherwise, v = 0, Ye = 0.1 (hydro: W [nb, 6, 2, 8000])."""
    nb = len(blocks)
    W = np.zeros((nb, 6, 2, NCELLS))
    for n, b in enumerate(blocks):
        x, _, _ = np.meshgrid(_centers(b, 0), _centers(b, 1), _centers(b, 2), indexing="ij")
        rho = np.where(x < 0.5, 1.0, 0.125)
        p = np.where(x < 0.5, 1.0, 0.1)
        for s in range(2):
            W[n, 0, s] = rho.ravel()
            W[n, 4, s] = (p / ((gamma - 1.0) * rho)).ravel()
            W[n, 5, s] = 0.1
    return W


# ---- static-AMR workloads ------------------------------------------------------

NEDGES = (PBS + 1) * (PBS + 1) * PBS


def _edge_index(d: int, i, j, k):
    """EDGE_IDX of the reference layout (src/prj_defs.h)."""
    i, j, k = i + NG, j + NG, k + NG
    if d == 0:
        return (i * (PBS + 1) + j) * (PBS + 1) + k
    if d == 1:
        return (i * PBS + j) * (PBS + 1) + k
    return (i * (PBS + 1) + j) * PBS + k


def _bfield_from_potential(blocks: Sequence[Block], apot, emf_records) -> np.ndarray:
    """Bf [nb, 3, 2, NFACES] = discrete curl of A (src/prj_mhd.c:106-142).  A
    is sampled at the edge centres of every live block, the coarse copies of
    edges shared with finer blocks are replaced by the average of the two
    fine edges (the EMF restriction records of prj_mhd_emf_send, given as
    (records, wave offsets) from fx_plan_export), then differenced."""
    nb = len(blocks)
    E = np.zeros((nb, 3, NEDGES))
    r = np.arange(-NG, BS + NG)
    ei, ej, ek = np.meshgrid(r, r, r, indexing="ij")
    for n, b in enumerate(blocks):
        if b.id < 0 or b.active != 1:
            continue
        for d in range(3):
            ex, ey, ez = np.meshgrid(_edges(b, 0, d), _edges(b, 1, d), _edges(b, 2, d), indexing="ij")
            E[n, d][_edge_index(d, ei, ej, ek)] = apot(ex, ey, ez)[d]
    recs, waves = emf_records
    flat = E.reshape(nb, 3 * NEDGES)
    for w in range(len(waves) - 1):
        rr = recs[waves[w]:waves[w + 1]].astype(np.int64)
        if len(rr):
            # value = 0; value += e0; value += e1; value *= 0.5
            flat[rr[:, 0], rr[:, 1]] = ((0.0 + flat[rr[:, 2], rr[:, 3]]) + flat[rr[:, 2], rr[:, 4]]) * 0.5
    Bf = np.zeros((nb, 3, 2, NFACES))
    f = np.arange(-NG, BS + NG - 1)
    fi, fj, fk = np.meshgrid(f, f, f, indexing="ij")
    for n, b in enumerate(blocks):
        if b.id < 0 or b.active != 1:
            continue
        e1, e2, e3 = E[n, 0], E[n, 1], E[n, 2]
        B1 = (e3[_edge_index(2, fi, fj + 1, fk)] - e3[_edge_index(2, fi, fj, fk)]) / b.dx[1] - \
            (e2[_edge_index(1, fi, fj, fk + 1)] - e2[_edge_index(1, fi, fj, fk)]) / b.dx[2]
        B2 = (e1[_edge_index(0, fi, fj, fk + 1)] - e1[_edge_index(0, fi, fj, fk)]) / b.dx[2] - \
            (e3[_edge_index(2, fi + 1, fj, fk)] - e3[_edge_index(2, fi, fj, fk)]) / b.dx[0]
        B3 = (e2[_edge_index(1, fi + 1, fj, fk)] - e2[_edge_index(1, fi, fj, fk)]) / b.dx[0] - \
            (e1[_edge_index(0, fi, fj + 1, fk)] - e1[_edge_index(0, fi, fj, fk)]) / b.dx[1]
        for d, Bd in enumerate((B1, B2, B3)):
            Bf[n, d, 0][_face_index(d, fi, fj, fk)] = Bd
            Bf[n, d, 1] = Bf[n, d, 0]
    return Bf


def _prim_cells(blocks: Sequence[Block], cell, nv: int) -> np.ndarray:
    """W [nb, nv, 2, NCELLS] with both stage slots set from cell(x, y, z) ->
    dict of variable arrays over the 20^3 cell centres of each live block."""
    nb = len(blocks)
    W = np.zeros((nb, nv, 2, NCELLS))
    for n, b in enumerate(blocks):
        if b.id < 0 or b.active != 1:
            continue
        x, y, z = np.meshgrid(_centers(b, 0), _centers(b, 1), _centers(b, 2), indexing="ij")
        w = cell(x, y, z)
        for v, a in w.items():
            for s in range(2):
                W[n, v, s] = np.broadcast_to(a, x.shape).ravel()
    return W


def amr_blast(blocks: Sequence[Block], emf_records=None, mhd: bool = True, gamma: float = 5.0 / 3.0,
              center=(0.1, 0.05, 0.0), p_in: float = 10.0, p_out: float = 0.1, r_in: float = 0.05,
              B0=None):
    """Magnetised blast: rho = 1, p = p_in for r < r_in about center, p_out
    elsewhere, v = 0, Ye = 0.1, B = (B0x, B0y, 0) through A = (0, 0,
    B0x y - B0y x) (default B0 = (1, 1) / sqrt(2) / sqrt(4 pi)).  Returns W and,
    for MHD, Bf; the ghost zones still need the ghost fill."""
    if B0 is None:
        b = 1.0 / math.sqrt(2.0) / math.sqrt(4.0 * math.pi)
        B0 = (b, b, 0.0)

    def cell(x, y, z):
        dx, dy, dz = x - center[0], y - center[1], z - center[2]
        r = np.sqrt(dx * dx + dy * dy + dz * dz)
        p = np.where(r < r_in, p_in, p_out)
        return {0: 1.0, 4: p / ((gamma - 1.0) * 1.0), 5: 0.1}

    W = _prim_cells(blocks, cell, 9 if mhd else 6)
    if not mhd:
        return W, None

    def apot(x, y, z):
        return (np.zeros_like(x), np.zeros_like(x), B0[0] * y - B0[1] * x)

    Bf = _bfield_from_potential(blocks, apot, emf_records)
    for n in range(len(blocks)):
        if blocks[n].active == 1:
            bf2bc_all(W[n], Bf[n], 0)
            bf2bc_all(W[n], Bf[n], 1)
    return W, Bf


def collapse(blocks: Sequence[Block], emf_records=None, half_width: float = 1.0, rho_c: float = 1.0e10,
             K: float = 4.6e5, beta: float = 1.0e4, gm_point: float = 0.0, gamma: float = 4.0 / 3.0):
    """Collapse-like MHD: rho = rho_c (1 + (r/r0)^2)^-1.5 with r0 = 0.05 of
    the domain length, p = K rho^gamma, v_r = -0.1 c_s r / (r + r0), Ye = 0.1,
    a dipole-like loop A_phi = B0 r0^3 R / (r^2 + r0^2)^1.5 with central field
    2 B0 at plasma beta `beta`, and the static acceleration g = -(gm_point +
    M(<r)) x / r^3 of the profile's enclosed mass.  Returns W, Bf and grav
    [nb, 3, NCELLS] (all 20^3 cells)."""
    r0 = 0.05 * 2.0 * half_width
    p_c = K * rho_c ** gamma
    B0 = 0.5 * math.sqrt(2.0 * p_c / beta)

    def cell(x, y, z):
        r = np.sqrt(x * x + y * y + z * z)
        q = r / r0
        s = 1.0 + q * q
        rho = rho_c / (s * np.sqrt(s))
        p = K * np.power(rho, gamma)
        cs = np.sqrt(gamma * p / rho)
        vr = -0.1 * cs * r / (r + r0)
        with np.errstate(divide="ignore"):
            inv_r = np.where(r > 0.0, 1.0 / r, 0.0)
        return {0: rho, 1: vr * x * inv_r, 2: vr * y * inv_r, 3: vr * z * inv_r,
                4: p / ((gamma - 1.0) * rho), 5: 0.1}

    W = _prim_cells(blocks, cell, 9)

    def apot(x, y, z):
        r2 = x * x + y * y + z * z
        s = r2 + r0 * r0
        f = B0 * r0 * r0 * r0 / (s * np.sqrt(s))
        return (-y * f, x * f, np.zeros_like(x))

    Bf = _bfield_from_potential(blocks, apot, emf_records)
    nb = len(blocks)
    grav = np.zeros((nb, 3, NCELLS))
    for n, b in enumerate(blocks):
        if b.id < 0 or b.active != 1:
            continue
        bf2bc_all(W[n], Bf[n], 0)
        bf2bc_all(W[n], Bf[n], 1)
        x, y, z = np.meshgrid(_centers(b, 0), _centers(b, 1), _centers(b, 2), indexing="ij")
        r = np.sqrt(x * x + y * y + z * z)
        a = r / r0
        menc = 4.0 * math.pi * rho_c * r0 * r0 * r0 * (np.arcsinh(a) - a / np.sqrt(1.0 + a * a))
        with np.errstate(divide="ignore", invalid="ignore"):
            gmag = np.where(r > 0.0, -(gm_point + menc) / (r * r * r), 0.0)
        grav[n, 0] = (gmag * x).ravel()
        grav[n, 1] = (gmag * y).ravel()
        grav[n, 2] = (gmag * z).ravel()
    return W, Bf, grav
