"""Mesh descriptions for the device mirror.

A FornaxAMR mesh is a list of blocks (geometry, level, 56 neighbour slots).
This module builds that description for uniform root grids the way
prj_mesh_init does (reference src/prj_mesh.c:1438-1686): blocks ordered
i-major over the root grid, 16^3 cells each, and neighbour slots from the
26 adjacent root blocks with the send/recv boxes of
prj_neighbor_compute_geometry (src/prj_mesh.c:46-243).  The slot table is an
interface the drop-in must reproduce exactly, so the box rules are restated
here with the same meaning.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field
from typing import List, Sequence

import numpy as np

from ._lib import FxBlockDesc

BS = 16
NG = 2

NEIGHBOR_NONE, NEIGHBOR_FACE, NEIGHBOR_EDGE, NEIGHBOR_CORNER = 0, 1, 2, 3


@dataclass
class Slot:
    id: int = -1
    rel_level: int = 0
    type: int = NEIGHBOR_NONE
    send_start: List[int] = field(default_factory=lambda: [0, 0, 0])
    send_end: List[int] = field(default_factory=lambda: [0, 0, 0])
    recv_start: List[int] = field(default_factory=lambda: [0, 0, 0])
    recv_end: List[int] = field(default_factory=lambda: [0, 0, 0])


@dataclass
class Block:
    id: int
    level: int
    xmin: List[float]
    xmax: List[float]
    dx: List[float]
    active: int = 1
    slots: List[Slot] = field(default_factory=lambda: [Slot() for _ in range(56)])

    @property
    def vol(self) -> float:
        return self.dx[0] * self.dx[1] * self.dx[2]

    @property
    def area(self) -> List[float]:
        # prj_block_setup_geometry, src/prj_mesh.c:675-687
        return [self.dx[1] * self.dx[2], self.dx[0] * self.dx[2], self.dx[0] * self.dx[1]]


def slot_index(ox: int, oy: int, oz: int) -> int:
    """prj_neighbor_slot_index (src/prj_mesh.c:19-35)."""
    if ox == 0 and oy == 0 and oz == 0:
        return -1
    index = (ox + 1) * 9 + (oy + 1) * 3 + (oz + 1)
    return index - 1 if index > 13 else index


def compute_geometry(a: Block, b: Block, slot: Slot) -> None:
    """Send/recv boxes of neighbour b as seen from block a (the slot lives in
    a; send boxes are in a's cells, recv boxes in b's cells)."""
    axisrel = [0, 0, 0]
    touching = 0
    for d in range(3):
        tol = 1.0e-2 * min(a.dx[d], b.dx[d])
        if abs(a.xmax[d] - b.xmin[d]) < tol:
            axisrel[d] = 1
            touching += 1
        elif abs(b.xmax[d] - a.xmin[d]) < tol:
            axisrel[d] = -1
            touching += 1
    slot.type = [NEIGHBOR_NONE, NEIGHBOR_FACE, NEIGHBOR_EDGE, NEIGHBOR_CORNER][touching]
    slot.rel_level = b.level - a.level
    for d in range(3):
        if slot.rel_level == 0:
            if axisrel[d] == 1:
                rs, re, ss, se = -NG, 0, BS - NG, BS
            elif axisrel[d] == -1:
                rs, re, ss, se = BS, BS + NG, 0, NG
            else:
                rs, re, ss, se = 0, BS, 0, BS
        elif slot.rel_level == -1:
            if axisrel[d] == 1:
                rs, re, ss, se = -NG, 0, BS - 2 * NG, BS
            elif axisrel[d] == -1:
                rs, re, ss, se = BS, BS + NG, 0, 2 * NG
            else:
                if (b.xmin[d] + b.xmax[d]) > (a.xmin[d] + a.xmax[d]):
                    rs, re = 0, BS // 2
                else:
                    rs, re = BS // 2, BS
                ss, se = 0, BS
        elif slot.rel_level == 1:
            if axisrel[d] == 1:
                rs, re, ss, se = -NG, 0, BS - NG // 2, BS
            elif axisrel[d] == -1:
                rs, re, ss, se = BS, BS + NG, 0, NG // 2
            else:
                if (b.xmin[d] + b.xmax[d]) > (a.xmin[d] + a.xmax[d]):
                    rs, re, ss, se = -NG, BS, BS // 2 - NG // 2, BS
                else:
                    rs, re, ss, se = 0, BS + NG, 0, BS // 2 + NG // 2
        else:
            raise ValueError("neighbour geometry error: level jump larger than one")
        slot.recv_start[d], slot.recv_end[d] = rs, re
        slot.send_start[d], slot.send_end[d] = ss, se


def uniform_mesh(root: Sequence[int], coord: Sequence[float]) -> List[Block]:
    """Root grid of root[0] x root[1] x root[2] blocks on the box
    coord = (x1min, x1max, x2min, x2max, x3min, x3max), non-periodic."""
    nx, ny, nz = root
    bdx = [(coord[1] - coord[0]) / nx, (coord[3] - coord[2]) / ny, (coord[5] - coord[4]) / nz]
    lo = [coord[0], coord[2], coord[4]]
    blocks: List[Block] = []
    for i in range(nx):
        for j in range(ny):
            for k in range(nz):
                idx = (i, j, k)
                xmin = [lo[a] + float(idx[a]) * bdx[a] for a in range(3)]
                xmax = [xmin[a] + bdx[a] for a in range(3)]
                dx = [bdx[a] / float(BS) for a in range(3)]
                blocks.append(Block(id=len(blocks), level=0, xmin=xmin, xmax=xmax, dx=dx))
    for i in range(nx):
        for j in range(ny):
            for k in range(nz):
                b = blocks[(i * ny + j) * nz + k]
                for ox in (-1, 0, 1):
                    for oy in (-1, 0, 1):
                        for oz in (-1, 0, 1):
                            s = slot_index(ox, oy, oz)
                            if s < 0:
                                continue
                            n = (i + ox, j + oy, k + oz)
                            if not (0 <= n[0] < nx and 0 <= n[1] < ny and 0 <= n[2] < nz):
                                continue
                            nid = (n[0] * ny + n[1]) * nz + n[2]
                            b.slots[s].id = nid
                            compute_geometry(b, blocks[nid], b.slots[s])
    return blocks


def to_desc(blocks: Sequence[Block]) -> "C.Array":
    """ctypes array of fx_block_desc for fx_set_mesh."""
    arr = (FxBlockDesc * len(blocks))()
    for n, b in enumerate(blocks):
        d = arr[n]
        d.id = b.id
        d.level = b.level
        d.active = b.active
        d.rank = 0
        for a in range(3):
            d.xmin[a] = b.xmin[a]
            d.xmax[a] = b.xmax[a]
            d.dx[a] = b.dx[a]
        d.vol = b.vol
        area = b.area
        for a in range(3):
            d.area[a] = area[a]
        for s, sl in enumerate(b.slots):
            ds = d.slot[s]
            ds.id = sl.id
            ds.rel_level = sl.rel_level
            ds.type = sl.type
            for a in range(3):
                ds.send_loc_start[a] = sl.send_start[a]
                ds.send_loc_end[a] = sl.send_end[a]
                ds.recv_loc_start[a] = sl.recv_start[a]
                ds.recv_loc_end[a] = sl.recv_end[a]
    return arr


def desc_from_arrays(ints: np.ndarray, geom: np.ndarray, slots: np.ndarray) -> "C.Array":
    """fx_block_desc array from packed arrays: ints[n] = (id, level, active,
    rank), geom[n] = (xmin3, xmax3, dx3, vol, area3), slots[n] = 56 x 15
    (id, rel_level, type, send_start3, send_end3, recv_start3, recv_end3)."""
    nb = ints.shape[0]
    arr = (FxBlockDesc * nb)()
    for n in range(nb):
        d = arr[n]
        d.id, d.level, d.active, d.rank = (int(x) for x in ints[n, :4])
        for a in range(3):
            d.xmin[a] = float(geom[n, a])
            d.xmax[a] = float(geom[n, 3 + a])
            d.dx[a] = float(geom[n, 6 + a])
            d.area[a] = float(geom[n, 10 + a])
        d.vol = float(geom[n, 9])
        for s in range(56):
            row = slots[n, s]
            ds = d.slot[s]
            ds.id, ds.rel_level, ds.type = int(row[0]), int(row[1]), int(row[2])
            for a in range(3):
                ds.send_loc_start[a] = int(row[3 + a])
                ds.send_loc_end[a] = int(row[6 + a])
                ds.recv_loc_start[a] = int(row[9 + a])
                ds.recv_loc_end[a] = int(row[12 + a])
    return arr


def desc_to_arrays(arr) -> tuple:
    """Inverse of desc_from_arrays (for comparisons)."""
    nb = len(arr)
    ints = np.zeros((nb, 4), dtype=np.int64)
    geom = np.zeros((nb, 13), dtype=np.float64)
    slots = np.zeros((nb, 56, 15), dtype=np.int64)
    for n in range(nb):
        d = arr[n]
        ints[n] = (d.id, d.level, d.active, d.rank)
        geom[n, 0:3] = d.xmin[:]
        geom[n, 3:6] = d.xmax[:]
        geom[n, 6:9] = d.dx[:]
        geom[n, 9] = d.vol
        geom[n, 10:13] = d.area[:]
        for s in range(56):
            ds = d.slot[s]
            slots[n, s] = ([ds.id, ds.rel_level, ds.type] + list(ds.send_loc_start) + list(ds.send_loc_end)
                           + list(ds.recv_loc_start) + list(ds.recv_loc_end))
    return ints, geom, slots
