"""torch.autograd bridge to the discrete adjoint of the RK2 MHD step.

The step and its reverse pass run in the library (fx_adjoint_forward /
fx_adjoint_backward, hand-written sm_100a kernels); this module only moves
arrays.  `Steps.apply(W0, Bf0, ctx, nsteps, dt)` returns the state after
`nsteps` RK2 steps with fixed dt, starting from (W0, Bf0) followed by the
driver's initial ghost fill; its backward is the library's reverse pass
(including the adjoint of that initial fill).

`initial_state` builds (W0, Bf0) from cell-centred density and velocity and
an edge vector potential with torch operations, so a scalar objective of the
final state back-propagates to (rho0, v0, A0).
"""
from __future__ import annotations

import numpy as np
import torch

from .mesh import BS, NG
from .problems import NCELLS, NFACES, PBS, _edge_index, _face_index

NSTAGES = 2


class Steps(torch.autograd.Function):
    @staticmethod
    def forward(fctx, W0, Bf0, ctx, nsteps: int, dt: float):
        nb = W0.shape[0]
        ctx.upload_all(np.ascontiguousarray(W0.detach().cpu().numpy().reshape(-1)),
                       np.ascontiguousarray(Bf0.detach().cpu().numpy().reshape(-1)))
        ctx.boundary_fill(1, 0)
        ctx.adjoint_forward(nsteps, dt)
        W = np.empty(W0.numel())
        Bf = np.empty(Bf0.numel())
        ctx.download_all(W, Bf)
        fctx.ctx = ctx
        fctx.shapes = (W0.shape, Bf0.shape, W0.device)
        return (torch.from_numpy(W).reshape(W0.shape).to(W0.device),
                torch.from_numpy(Bf).reshape(Bf0.shape).to(W0.device))

    @staticmethod
    def backward(fctx, gW, gBf):
        ws, bs, dev = fctx.shapes
        gW = np.zeros(int(np.prod(ws))) if gW is None else gW.detach().cpu().numpy().reshape(-1)
        gBf = None if gBf is None else gBf.detach().cpu().numpy().reshape(-1)
        Wo, Bo = fctx.ctx.adjoint_backward(gW, gBf, initial_fill=True)
        return (torch.from_numpy(Wo).reshape(ws).to(dev), torch.from_numpy(Bo).reshape(bs).to(dev),
                None, None, None)


def _index_arrays():
    r = np.arange(-NG, BS + NG)
    i, j, k = np.meshgrid(r, r, r, indexing="ij")
    f = np.arange(-NG, BS + NG - 1)
    fi, fj, fk = np.meshgrid(f, f, f, indexing="ij")
    return i, j, k, fi, fj, fk


def initial_state(rho0: torch.Tensor, v0: torch.Tensor, A0: torch.Tensor, gamma: float, dx,
                  p0: float = 1.0, ye: float = 0.1):
    """(W0 [nb, 9, 2, 8000], Bf0 [nb, 3, 2, 8400]) from rho0 [nb, 16, 16, 16],
    v0 [nb, 3, 16, 16, 16] (active cells; ghost cells are refilled by the
    initial ghost fill), A0 [nb, 3, 20, 20, 20] (edge (i, j, k) of component
    d at [d, i + 2, j + 2, k + 2], i, j, k in [-2, 17]) and the cell widths
    dx [nb, 3]: p = p0, B = curl A on the faces in [-2, 16] (the reference's
    discrete curl, src/prj_mhd.c:106-142) and cell B the face averages."""
    nb = rho0.shape[0]
    dt_ = rho0.dtype
    dev = rho0.device
    i, j, k, fi, fj, fk = _index_arrays()
    act = torch.as_tensor(((i >= 0) & (i < BS) & (j >= 0) & (j < BS) & (k >= 0) & (k < BS)).ravel(), device=dev)
    rho = torch.ones(nb, NCELLS, dtype=dt_, device=dev)
    rho = rho.masked_scatter(act.expand(nb, -1), rho0.reshape(nb, -1))
    vel = [torch.zeros(nb, NCELLS, dtype=dt_, device=dev).masked_scatter(act.expand(nb, -1), v0[:, a].reshape(nb, -1))
           for a in range(3)]
    dxt = torch.as_tensor(np.asarray(dx, dtype=np.float64), device=dev)
    s = slice(0, PBS - 1)
    sp = slice(1, PBS)
    A = A0
    B1 = (A[:, 2][:, s, sp, s] - A[:, 2][:, s, s, s]) / dxt[:, 1, None, None, None] - \
        (A[:, 1][:, s, s, sp] - A[:, 1][:, s, s, s]) / dxt[:, 2, None, None, None]
    B2 = (A[:, 0][:, s, s, sp] - A[:, 0][:, s, s, s]) / dxt[:, 2, None, None, None] - \
        (A[:, 2][:, sp, s, s] - A[:, 2][:, s, s, s]) / dxt[:, 0, None, None, None]
    B3 = (A[:, 1][:, sp, s, s] - A[:, 1][:, s, s, s]) / dxt[:, 0, None, None, None] - \
        (A[:, 0][:, s, sp, s] - A[:, 0][:, s, s, s]) / dxt[:, 1, None, None, None]
    faces = []
    for d, Bd in enumerate((B1, B2, B3)):
        idx = torch.as_tensor(_face_index(d, fi, fj, fk).ravel(), device=dev)
        f = torch.zeros(nb, NFACES, dtype=dt_, device=dev).index_copy(1, idx, Bd.reshape(nb, -1))
        faces.append(f)
    cellB = []
    for d in range(3):
        lo = torch.as_tensor(_face_index(d, i, j, k).ravel(), device=dev)
        hi = torch.as_tensor(_face_index(d, i + (d == 0), j + (d == 1), k + (d == 2)).ravel(), device=dev)
        cellB.append(0.5 * (faces[d][:, lo] + faces[d][:, hi]))
    eint = p0 / ((gamma - 1.0) * rho)
    yev = torch.full_like(rho, ye)
    per_var = [rho, vel[0], vel[1], vel[2], eint, yev, cellB[0], cellB[1], cellB[2]]
    W0 = torch.stack([torch.stack([x, x], dim=1) for x in per_var], dim=1)
    Bf0 = torch.stack([torch.stack([f, f], dim=1) for f in faces], dim=1)
    return W0, Bf0


def kinetic_energy_in_ball(W: torch.Tensor, blocks, center, radius: float) -> torch.Tensor:
    """J = sum over active cells with |x - center| < radius of
    0.5 rho |v|^2 dV, from W slot 0."""
    i, j, k, _, _, _ = _index_arrays()
    act = ((i >= 0) & (i < BS) & (j >= 0) & (j < BS) & (k >= 0) & (k < BS)).ravel()
    J = W.new_zeros(())
    for n, b in enumerate(blocks):
        if b.active != 1:
            continue
        x = b.xmin[0] + (i.ravel() + 0.5) * b.dx[0] - center[0]
        y = b.xmin[1] + (j.ravel() + 0.5) * b.dx[1] - center[1]
        z = b.xmin[2] + (k.ravel() + 0.5) * b.dx[2] - center[2]
        sel = act & (x * x + y * y + z * z < radius * radius)
        if not sel.any():
            continue
        idx = torch.as_tensor(np.nonzero(sel)[0], device=W.device)
        rho = W[n, 0, 0, idx]
        v2 = W[n, 1, 0, idx] ** 2 + W[n, 2, 0, idx] ** 2 + W[n, 3, 0, idx] ** 2
        J = J + (0.5 * rho * v2).sum() * (b.dx[0] * b.dx[1] * b.dx[2])
    return J


__all__ = ["Steps", "initial_state", "kinetic_energy_in_ball", "_edge_index"]
