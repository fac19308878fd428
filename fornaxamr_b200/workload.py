"""Run one of the measured workloads on the device (the small, self-contained
cases the kernel profiles are taken on).

    python -m fornaxamr_b200.workload [--problem fourier|blast|collapse]
        [--root R] [--steps N] [--form batched|plain] [--adjoint N] [--shape S]
        [--amr-interval K [--max-level L]] [--variant rk2|weno3|ess|ess_weno3|weno7]

fourier: uniform root^3 mesh of 16^3 blocks on [0,1]^3 with the seeded
Fourier-mode MHD state (fornaxamr_b200.problems.fourier_mhd).
blast: static AMR magnetised blast, root^3 roots on [-0.7, 0.7]^3, levels
refined inside r < 0.4 and 0.2 about (0.1, 0.05, 0).
collapse: static AMR gravity collapse, root^3 roots on [-1, 1]^3, spheres
0.4 / 0.2 / 0.1 about the origin.

Runs the driver's initial ghost fill and N driver steps (calc_dt + RK2 step)
and prints the time per step.  With --amr-interval K the mesh adapts every K
steps (prj_amr_adapt with a Loehner pressure criterion, refine 0.3 /
derefine 0.1, up to level L, default 3) and the adapt phases are printed.
--variant selects the reference build variant: WENO-Z3 reconstruction
(weno3), the eSSPRK10_4 integrator (ess) or both (ess_weno3), or WENO-Z7
(weno7; run the process with FX_NGHOST=4, the four-ghost-layer build).  With --adjoint N (fourier only, amplitude
0.01, |k| <= 3) it runs N fixed-dt steps storing every stage, then one
reverse sweep, and prints the reverse sweep's device time per step.
"""
from __future__ import annotations

import argparse
import time

import numpy as np


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--problem", default="fourier", choices=["fourier", "blast", "collapse"])
    ap.add_argument("--root", type=int, default=4)
    ap.add_argument("--steps", type=int, default=2)
    ap.add_argument("--form", default="batched", choices=["batched", "plain"])
    ap.add_argument("--modes", type=int, default=32)
    ap.add_argument("--adjoint", type=int, default=0)
    ap.add_argument("--shape", type=int, default=-1, help="force a face-kernel launch shape (fx_set_flux_shape)")
    ap.add_argument("--amr-interval", type=int, default=0)
    ap.add_argument("--variant", default="rk2", choices=["rk2", "weno3", "ess", "ess_weno3", "weno7"])
    ap.add_argument("--max-level", type=int, default=3)
    args = ap.parse_args()
    if args.variant != "rk2" and args.problem == "collapse":
        ap.error("--variant applies to the fourier and blast problems")

    import fornaxamr_b200 as fx
    from fornaxamr_b200 import mesh, problems

    grav = None
    gamma = 5.0 / 3.0
    gravity = False
    if args.problem == "fourier":
        coord = (0.0, 1.0, 0.0, 1.0, 0.0, 1.0)
        blocks = mesh.uniform_mesh((args.root,) * 3, coord)
        if args.adjoint:
            W, Bf = problems.fourier_mhd(blocks, nmodes=args.modes, kmax=3, amp_rho=0.01, amp_v=0.01, amp_A=0.005)
        else:
            W, Bf = problems.fourier_mhd(blocks, nmodes=args.modes)
    else:
        hw = 0.7 if args.problem == "blast" else 1.0
        coord = (-hw, hw, -hw, hw, -hw, hw)
        if args.problem == "blast":
            blocks = mesh.static_amr_mesh((args.root,) * 3, coord, 2,
                                          mesh.ball_refiner((0.1, 0.05, 0.0), (0.4, 0.2)))
        else:
            blocks = mesh.static_amr_mesh((args.root,) * 3, coord, 3,
                                          mesh.ball_refiner((0.0, 0.0, 0.0), (0.4, 0.2, 0.1)))
        recs = fx.plan_export(fx.make_config(True, gamma, coord), mesh.to_desc(blocks), 3)
        if args.problem == "blast":
            W, Bf = problems.amr_blast(blocks, recs)
        else:
            gamma = 4.0 / 3.0
            gravity = True
            W, Bf, grav = problems.collapse(blocks, recs, half_width=hw)
    recon = fx.RECON_WENO3 if "weno3" in args.variant else fx.RECON_WENO7 if args.variant == "weno7" \
        else fx.RECON_MC
    integ = fx.INT_ESSPRK10_4 if args.variant.startswith("ess") else fx.INT_RK2
    ctx = fx.Context(True, gamma, coord, gravity=gravity, recon=recon, integrator=integ)
    ctx.set_mesh(mesh.to_desc(blocks))
    if ctx.ns == 2:
        ctx.upload_all(np.ascontiguousarray(W), np.ascontiguousarray(Bf))
    else:
        W3 = np.zeros(W.shape[:2] + (3,) + W.shape[3:])
        B3 = np.zeros(Bf.shape[:2] + (3,) + Bf.shape[3:])
        W3[:, :, 0] = W[:, :, 0]
        B3[:, :, 0] = Bf[:, :, 0]
        ctx.upload_state(W3, B3)
    if grav is not None:
        for b in range(len(blocks)):
            if blocks[b].active == 1:
                ctx.upload_block(b, W[b].ravel(), [Bf[b, d].ravel() for d in range(3)],
                                 [grav[b, d] for d in range(3)])
    ctx.boundary_fill(1, 0)
    ctx.sync()
    if args.shape >= 0:
        ctx.set_flux_shape(args.shape)
    zones = sum(1 for b in blocks if b.active == 1) * 4096
    if args.adjoint:
        dt = ctx.calc_dt(0.4)
        ctx.adjoint_forward(args.adjoint, dt)
        ctx.adjoint_backward(np.full(W.size, 1.0e-3))
        print(f"{len(blocks)} blocks, adjoint of {args.adjoint} steps: "
              f"{ctx.adjoint_ms() / args.adjoint:.3f} ms/step (reverse sweep, device)")
        ctx.close()
        return
    form = fx.FORM_BATCHED if args.form == "batched" else fx.FORM_PLAIN
    if args.amr_interval > 0:
        ctx.amr_configure(fx.amr_config((args.root,) * 3, args.max_level, [
            dict(estimator=fx.AMR_LOEHNER, refine=0.3, derefine=0.1, var=fx.AMR_VAR_PRESSURE)]))
        state = (0.0, 0.0, 0)
        t0 = time.perf_counter()
        for _ in range(max(args.steps // args.amr_interval, 1)):
            state = ctx.run(form, args.amr_interval, 0.4, 1.2, 1.0e30, state)
            changed = ctx.amr_adapt()
            t = ctx.amr_timings()
            print(f"step {int(state[2])}: adapt changed={changed} blocks={ctx.nblocks} " +
                  " ".join(f"{k}={v:.1f}ms" for k, v in t.items()), flush=True)
        ctx.sync()
        dt = time.perf_counter() - t0
        print(f"{int(state[2])} steps with adapts every {args.amr_interval}: wall {1e3 * dt / max(int(state[2]), 1):.3f} ms/step")
        ctx.close()
        return
    t0 = time.perf_counter()
    state = ctx.run(form, args.steps, 0.4, 1.2, 1.0e30, (0.0, 0.0, 0))
    ctx.sync()
    dt = time.perf_counter() - t0
    print(f"{len(blocks)} blocks ({zones // 4096} active), {args.steps} steps ({args.form}): t={state[0]:.6e} "
          f"wall {1e3 * dt / max(args.steps, 1):.3f} ms/step, {zones * args.steps / dt:.3e} zone-updates/s")
    ctx.close()


if __name__ == "__main__":
    main()
