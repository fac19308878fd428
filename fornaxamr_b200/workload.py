"""Run the Fourier-mode MHD workload on the device.

    python -m fornaxamr_b200.workload [--root R] [--steps N] [--form batched|plain]

Builds a uniform root^3 mesh of 16^3 blocks on [0,1]^3, generates the
seeded Fourier-mode initial state (fornaxamr_b200.problems.fourier_mhd), runs
the driver's initial ghost fill and N driver steps (calc_dt + RK2 step), and
prints the device time per step.  Used as the small, self-contained case for
kernel profiles.
"""
from __future__ import annotations

import argparse
import time

import numpy as np


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--root", type=int, default=4)
    ap.add_argument("--steps", type=int, default=2)
    ap.add_argument("--form", default="batched", choices=["batched", "plain"])
    ap.add_argument("--modes", type=int, default=32)
    args = ap.parse_args()

    import fornaxamr_b200 as fx
    from fornaxamr_b200 import mesh, problems

    coord = (0.0, 1.0, 0.0, 1.0, 0.0, 1.0)
    blocks = mesh.uniform_mesh((args.root,) * 3, coord)
    W, Bf = problems.fourier_mhd(blocks, nmodes=args.modes)
    ctx = fx.Context(True, 5.0 / 3.0, coord)
    ctx.set_mesh(mesh.to_desc(blocks))
    ctx.upload_all(np.ascontiguousarray(W), np.ascontiguousarray(Bf))
    ctx.boundary_fill(1, 0)
    ctx.sync()
    form = fx.FORM_BATCHED if args.form == "batched" else fx.FORM_PLAIN
    t0 = time.perf_counter()
    state = ctx.run(form, args.steps, 0.4, 1.2, 1.0e30, (0.0, 0.0, 0))
    ctx.sync()
    dt = time.perf_counter() - t0
    zones = len(blocks) * 4096
    print(f"{len(blocks)} blocks, {args.steps} steps ({args.form}): t={state[0]:.6e} "
          f"wall {1e3 * dt / max(args.steps, 1):.3f} ms/step, {zones * args.steps / dt:.3e} zone-updates/s")
    ctx.close()


if __name__ == "__main__":
    main()
