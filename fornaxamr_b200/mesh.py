"""Mesh descriptions for the device mirror.

A FornaxAMR mesh is a list of blocks (geometry, level, 56 neighbour slots).
This module builds that description for uniform root grids the way
prj_mesh_init does (reference src/prj_mesh.c:1438-1686): blocks ordered
i-major over the root grid, 16^3 cells each, and neighbour slots from the
26 adjacent root blocks.  The builders here decide which block sits in which
slot (the reference's probe and first-free-slot order); the slot's type,
relative level and send/recv boxes (prj_neighbor_compute_geometry,
src/prj_mesh.c:46-243) are filled by the native library
(fx_mesh_slot_geometry) when the description is made, so the box rules exist
once, in the library the dynamic-AMR remesh uses too.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field
from typing import List, Sequence

import numpy as np

from ._lib import FxBlockDesc

from .layout import BS, NG  # noqa: E402  (block size, ghost layers of the loaded build)

NEIGHBOR_NONE, NEIGHBOR_FACE, NEIGHBOR_EDGE, NEIGHBOR_CORNER = 0, 1, 2, 3


@dataclass
class Slot:
    id: int = -1   # neighbour block index, -1 if the slot is free


@dataclass
class Block:
    id: int
    level: int
    xmin: List[float]
    xmax: List[float]
    dx: List[float]
    active: int = 1
    slots: List[Slot] = field(default_factory=lambda: [Slot() for _ in range(56)])
    refine_flag: int = 0
    parent: int = -1
    children: List[int] = field(default_factory=lambda: [-1] * 8)

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
    return blocks


# ---- static refinement ------------------------------------------------------


def _touch_face_edge_corner(a: Block, b: Block) -> bool:
    """prj_boxes_touch_face_edge_corner (src/prj_amr.c:398-425)."""
    tol = 1.0e-12
    touches = 0
    for ax in range(3):
        if not (min(a.xmax[ax], b.xmax[ax]) >= max(a.xmin[ax], b.xmin[ax]) - tol):
            return False
        if abs(a.xmax[ax] - b.xmin[ax]) < tol or abs(b.xmax[ax] - a.xmin[ax]) < tol:
            touches += 1
    if touches == 0:
        return False
    if all(abs(a.xmin[ax] - b.xmin[ax]) < tol and abs(a.xmax[ax] - b.xmax[ax]) < tol for ax in range(3)):
        return False
    return True


def _add_neighbor(a: Block, b: Block) -> None:
    """prj_add_neighbor (src/prj_amr.c:540-573): first free slot."""
    if any(sl.id == b.id for sl in a.slots):
        return
    for sl in a.slots:
        if sl.id < 0:
            sl.id = b.id
            return
    raise ValueError("more than 56 neighbours")


def _logical_coords(b: Block, root: Sequence[int], coord: Sequence[float]):
    """prj_mesh_block_logical_coords (src/prj_mesh.c:1250-1288)."""
    out = []
    for ax in range(3):
        lo, hi = coord[2 * ax], coord[2 * ax + 1]
        count = float(root[ax]) * 2.0 ** b.level
        scaled = (b.xmin[ax] - lo) * (count / (hi - lo))
        out.append(int(scaled + 0.5))
    return tuple(out)


def init_neighbors(blocks: List[Block], root: Sequence[int], coord: Sequence[float]) -> None:
    """prj_amr_init_neighbors, Morton path (src/prj_amr.c:1551-1579,
    575-711): clear every slot list, then for each active block in index
    order probe the candidate boxes of levels l-1, l, l+1 and register every
    touching pair both ways in the first free slots."""
    import math
    for b in blocks:
        if b.id >= 0:
            b.slots = [Slot() for _ in range(56)]
    lookup = {}
    for b in blocks:
        if b.id >= 0 and b.active == 1:
            lookup[(b.level,) + _logical_coords(b, root, coord)] = b.id
    for a in blocks:
        if a.id < 0 or a.active != 1:
            continue
        for lev in (a.level - 1, a.level, a.level + 1):
            if lev < 0:
                continue
            rng = []
            for ax in range(3):
                lo_c, hi_c = coord[2 * ax], coord[2 * ax + 1]
                scale = (float(root[ax]) * 2.0 ** lev) / (hi_c - lo_c)
                lo = (a.xmin[ax] - lo_c) * scale
                hi = (a.xmax[ax] - lo_c) * scale
                rng.append(range(int(math.floor(lo)) - 1, int(math.ceil(hi)) + 1))
            for ix in rng[0]:
                for iy in rng[1]:
                    for iz in rng[2]:
                        if ix < 0 or iy < 0 or iz < 0:
                            continue
                        nid = lookup.get((lev, ix, iy, iz), -1)
                        if nid < 0 or nid == a.id:
                            continue
                        b = blocks[nid]
                        if _touch_face_edge_corner(a, b):
                            _add_neighbor(a, b)
                            _add_neighbor(b, a)


def _refine_block(blocks: List[Block], i: int, max_level: int) -> None:
    """prj_amr_refine_block (src/prj_amr.c:2389-2497): eight children
    appended in octant order (x fastest), the parent made inactive."""
    p = blocks[i]
    if p.active != 1 or p.level >= max_level:
        return
    xmid = [0.5 * (p.xmin[a] + p.xmax[a]) for a in range(3)]
    for oct_ in range(8):
        bits = (oct_ & 1, (oct_ >> 1) & 1, (oct_ >> 2) & 1)
        xmin = [p.xmin[a] if bits[a] == 0 else xmid[a] for a in range(3)]
        xmax = [xmid[a] if bits[a] == 0 else p.xmax[a] for a in range(3)]
        child = Block(id=len(blocks), level=p.level + 1, xmin=xmin, xmax=xmax,
                      dx=[p.dx[a] * 0.5 for a in range(3)], parent=p.id)
        blocks.append(child)
        p.children[oct_] = child.id
    p.active = 0
    p.refine_flag = 0


def _enforce_two_to_one(blocks: List[Block]) -> None:
    """prj_amr_enforce_two_to_one (src/prj_amr.c:1471-1499)."""
    changed = True
    while changed:
        changed = False
        for b in blocks:
            if b.id < 0 or b.active != 1 or b.refine_flag <= 0:
                continue
            for sl in b.slots:
                nb = blocks[sl.id] if 0 <= sl.id < len(blocks) else None
                if nb is not None and nb.id >= 0 and nb.active == 1 and nb.level < b.level:
                    if nb.refine_flag != 1:
                        nb.refine_flag = 1
                        changed = True


def static_amr_mesh(root: Sequence[int], coord: Sequence[float], max_level: int, refine) -> List[Block]:
    """A static AMR hierarchy built the way a problem's initial refinement
    does it (the loop of problems/prj_problem_sedov.c:139-181): for each
    level in turn, flag the active blocks of that level for which
    refine(block, level) holds, enforce 2:1 balance, refine every flagged
    block, and rebuild the neighbour slots.  Block order, child order and
    slot order follow the reference, so the description is identical to the
    reference mesh for the same rule."""
    blocks = uniform_mesh(root, coord)
    for level in range(max_level):
        any_flag = False
        for b in blocks:
            if b.id < 0 or b.active != 1 or b.level != level:
                continue
            b.refine_flag = 0
            if refine(b, level):
                b.refine_flag = 1
                any_flag = True
        if not any_flag:
            break
        _enforce_two_to_one(blocks)
        changed = False
        i = 0
        while i < len(blocks):
            b = blocks[i]
            if b.id >= 0 and b.active == 1 and b.refine_flag > 0:
                _refine_block(blocks, i, max_level)
                changed = changed or blocks[i].active == 0
            i += 1
        if not changed:
            break
        init_neighbors(blocks, root, coord)
    return blocks


def ball_refiner(center: Sequence[float], radii: Sequence[float]):
    """Refine a level-l block when it overlaps the ball of radius radii[l]
    about center (the block-overlaps-ball rule of problems/prj_problem_sedov.c:20-44)."""
    def refine(b: Block, level: int) -> bool:
        if level >= len(radii):
            return False
        d2 = 0.0
        for a in range(3):
            if b.xmin[a] > center[a]:
                d = b.xmin[a] - center[a]
            elif b.xmax[a] < center[a]:
                d = center[a] - b.xmax[a]
            else:
                d = 0.0
            d2 += d * d
        return d2 < radii[level] * radii[level]
    return refine


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
        d.parent = b.parent
        for o in range(8):
            d.children[o] = b.children[o]
        d.can_refine = 1
        for s, sl in enumerate(b.slots):
            d.slot[s].id = sl.id
    from . import library
    rc = library().fx_mesh_slot_geometry(len(blocks), arr)
    if rc != 0:
        raise ValueError(f"fx_mesh_slot_geometry failed ({rc}): a slot id outside the mesh or a level jump > 1")
    return arr


def desc_from_arrays(ints: np.ndarray, geom: np.ndarray, slots: np.ndarray, tree=None) -> "C.Array":
    """fx_block_desc array from packed arrays: ints[n] = (id, level, active,
    rank), geom[n] = (xmin3, xmax3, dx3, vol, area3), slots[n] = 56 x 15
    (id, rel_level, type, send_start3, send_end3, recv_start3, recv_end3),
    tree[n] (optional) = (parent, children8[, refine_flag, can_refine])."""
    nb = ints.shape[0]
    arr = (FxBlockDesc * nb)()
    for n in range(nb):
        d = arr[n]
        d.id, d.level, d.active, d.rank = (int(x) for x in ints[n, :4])
        if tree is not None:
            d.parent = int(tree[n, 0])
            for o in range(8):
                d.children[o] = int(tree[n, 1 + o])
            d.can_refine = int(tree[n, 10]) if tree.shape[1] > 10 else 1
        else:
            d.parent = -1
            for o in range(8):
                d.children[o] = -1
            d.can_refine = 1
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


def desc_tree(arr) -> np.ndarray:
    """(parent, children8, can_refine) per entry, int64 [n, 10]."""
    out = np.zeros((len(arr), 10), dtype=np.int64)
    for n in range(len(arr)):
        d = arr[n]
        out[n, 0] = d.parent
        out[n, 1:9] = d.children[:]
        out[n, 9] = d.can_refine
    return out


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
