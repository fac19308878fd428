"""Discrete adjoint of 10 RK2 MHD steps (64^3 = 4^3 blocks of 16^3, outflow,
gamma 5/3, seeded Fourier modes with amplitude 0.01 and |k|_inf <= 3) through
the torch.autograd bridge, checked against central finite differences of
the plain per-block forward along 64 seeded smooth random unit directions
in (rho0, v0, A0) (each a sum of 8 Fourier modes per field, so the
perturbation is smooth like the data).

Objective J = sum over cells with |x - (0.5, 0.5, 0.5)| < 0.25 of
0.5 rho |v|^2 dV after the steps; dt is fixed (taken from the initial state).
The discrete map is piecewise smooth: the MC limiter's candidate, the HLLD
fan and the upwind direction switch at kinks, and with 2.5e5 cells every
probe direction crosses some of them even at eps = 1e-8 (the decision
replay below counts them; most are ties at round-off, such as the limiter
choices on the initially uniform pressure, whose noise-level differences
the perturbation reshuffles).  So the adjoint is checked two ways:

* against the branch-frozen map, the map the discrete adjoint
  differentiates: the forward at the unperturbed state records every face's
  and edge's decisions (fx_branch_trace), the perturbed forwards replay them,
  and every one of the 64 directions must agree to 1e-6 relative at
  eps = 1e-6;
* against the map as it stands, whose difference quotients carry the kink
  crossings: median relative error below 1e-7 at eps = 1e-7 (1e-6 at
  eps = 1e-6), 90 % of the directions below 1e-6 at eps = 1e-7 and none
  above 1e-5.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

NSTEPS = 10
CENTER = (0.5, 0.5, 0.5)
RADIUS = 0.25
GAMMA = 5.0 / 3.0


def _setup():
    import torch

    import fornaxamr_b200 as fx
    from fornaxamr_b200 import mesh, problems
    coord = (0.0, 1.0, 0.0, 1.0, 0.0, 1.0)
    blocks = mesh.uniform_mesh((4, 4, 4), coord)
    ctx = fx.Context(True, GAMMA, coord)
    ctx.set_mesh(mesh.to_desc(blocks))
    nb = len(blocks)
    m_rho = problems.draw_modes(32, 3, 0.01, 11)
    m_v = problems.draw_modes(32, 3, 0.01, 12)
    m_A = problems.draw_modes(32, 3, 0.005, 13)
    rho0 = np.zeros((nb, 16, 16, 16))
    v0 = np.zeros((nb, 3, 16, 16, 16))
    A0 = np.zeros((nb, 3, 20, 20, 20))
    r = np.arange(16)
    for n, b in enumerate(blocks):
        x, y, z = np.meshgrid(*[b.xmin[a] + (r + 0.5) * b.dx[a] for a in range(3)], indexing="ij")
        rho0[n] = 1.0 + problems._mode_sum(m_rho, x, y, z, False)
        v = problems._mode_sum(m_v, x, y, z, True)
        v0[n] = np.moveaxis(v, -1, 0)
        for d in range(3):
            ex, ey, ez = np.meshgrid(problems._edges(b, 0, d), problems._edges(b, 1, d),
                                     problems._edges(b, 2, d), indexing="ij")
            A0[n, d] = problems._mode_sum(m_A, ex, ey, ez, True)[..., d]
    dx = np.array([b.dx for b in blocks])
    t = lambda a: torch.tensor(a, dtype=torch.float64)
    return fx, ctx, blocks, dx, t(rho0), t(v0), t(A0)


def _J_plain(fx, ctx, blocks, dx, rho0, v0, A0, dt, branches=None):
    """J after NSTEPS plain-form steps; branches: None (the solver as it
    stands), "record" or "replay" (fx_branch_trace).  Returns (J, decisions
    the replay overrode)."""
    import torch

    from fornaxamr_b200 import autograd as ag
    with torch.no_grad():
        W0, Bf0 = ag.initial_state(rho0, v0, A0, GAMMA, dx)
    ctx.upload_all(np.ascontiguousarray(W0.numpy().reshape(-1)), np.ascontiguousarray(Bf0.numpy().reshape(-1)))
    ctx.boundary_fill(1, 0)
    if branches == "record":
        ctx.branch_record(2 * NSTEPS)
    elif branches == "replay":
        ctx.branch_replay()
    for _ in range(NSTEPS):
        ctx.step(fx.FORM_PLAIN, dt, want_dt_src=False)
    flips = ctx.branch_off() if branches else 0
    W = np.empty(W0.numel())
    ctx.download_all(W, None)
    J = float(ag.kinetic_energy_in_ball(torch.from_numpy(W).reshape(W0.shape), blocks, CENTER, RADIUS))
    return J, flips


def _smooth_direction(blocks, shapes, seed):
    """A seeded smooth random direction in (rho0, v0, A0): 8 Fourier modes
    (|k|_inf <= 3) per field, unit 2-norm overall."""
    from fornaxamr_b200 import problems
    m_r = problems.draw_modes(8, 3, 1.0, 1000 + 3 * seed)
    m_v = problems.draw_modes(8, 3, 1.0, 1001 + 3 * seed)
    m_a = problems.draw_modes(8, 3, 1.0, 1002 + 3 * seed)
    dr, dv, da = (np.zeros(s) for s in shapes)
    r = np.arange(16)
    for n, b in enumerate(blocks):
        x, y, z = np.meshgrid(*[b.xmin[a] + (r + 0.5) * b.dx[a] for a in range(3)], indexing="ij")
        dr[n] = problems._mode_sum(m_r, x, y, z, False)
        dv[n] = np.moveaxis(problems._mode_sum(m_v, x, y, z, True), -1, 0)
        for d in range(3):
            ex, ey, ez = np.meshgrid(problems._edges(b, 0, d), problems._edges(b, 1, d),
                                     problems._edges(b, 2, d), indexing="ij")
            da[n, d] = problems._mode_sum(m_a, ex, ey, ez, True)[..., d]
    nrm = np.sqrt((dr ** 2).sum() + (dv ** 2).sum() + (da ** 2).sum())
    return [dr / nrm, dv / nrm, da / nrm]


def test_adjoint_gradient_matches_finite_differences_of_plain_forward():
    import torch

    from fornaxamr_b200 import autograd as ag
    fx, ctx, blocks, dx, rho0, v0, A0 = _setup()
    with torch.no_grad():
        W0, Bf0 = ag.initial_state(rho0, v0, A0, GAMMA, dx)
    ctx.upload_all(np.ascontiguousarray(W0.numpy().reshape(-1)), np.ascontiguousarray(Bf0.numpy().reshape(-1)))
    ctx.boundary_fill(1, 0)
    dt = ctx.calc_dt(0.4)

    xs = [rho0.clone().requires_grad_(True), v0.clone().requires_grad_(True), A0.clone().requires_grad_(True)]
    W0, Bf0 = ag.initial_state(xs[0], xs[1], xs[2], GAMMA, dx)
    W, Bf = ag.Steps.apply(W0, Bf0, ctx, NSTEPS, dt)
    J = ag.kinetic_energy_in_ball(W, blocks, CENTER, RADIUS)
    J.backward()
    grads = [x.grad.numpy() for x in xs]
    J_rec, _ = _J_plain(fx, ctx, blocks, dx, rho0, v0, A0, dt, "record")
    assert float(J.detach()) == pytest.approx(J_rec, rel=1e-13)

    frozen, flips = [], []
    errs = {1e-6: [], 1e-7: []}
    for seed in range(64):
        dirs = _smooth_direction(blocks, [g.shape for g in grads], seed)
        ad = sum(float((g * q).sum()) for g, q in zip(grads, dirs))
        qs = [torch.from_numpy(q) for q in dirs]
        xp = [x.detach() + 1e-6 * q for x, q in zip(xs, qs)]
        xm = [x.detach() - 1e-6 * q for x, q in zip(xs, qs)]
        Jp, fp = _J_plain(fx, ctx, blocks, dx, *xp, dt, "replay")
        Jm, fm = _J_plain(fx, ctx, blocks, dx, *xm, dt, "replay")
        fd = (Jp - Jm) / 2e-6
        frozen.append(abs(ad - fd) / abs(fd))
        flips.append(fp + fm)
        for eps in errs:
            Jp, _ = _J_plain(fx, ctx, blocks, dx, *[x.detach() + eps * q for x, q in zip(xs, qs)], dt)
            Jm, _ = _J_plain(fx, ctx, blocks, dx, *[x.detach() - eps * q for x, q in zip(xs, qs)], dt)
            fd = (Jp - Jm) / (2 * eps)
            errs[eps].append(abs(ad - fd) / abs(fd))
    frozen = np.array(frozen)
    e6 = np.array(errs[1e-6])
    e7 = np.array(errs[1e-7])
    print("adjoint vs central FD of the branch-frozen map (eps 1e-6): median %.2e max %.2e; decisions the "
          "perturbed states would take otherwise: median %d, max %d per direction"
          % (np.median(frozen), frozen.max(), int(np.median(flips)), max(flips)))
    print("adjoint vs central FD of the map as it stands: eps 1e-6 median %.2e max %.2e; eps 1e-7 median %.2e "
          "max %.2e" % (np.median(e6), e6.max(), np.median(e7), e7.max()))
    assert frozen.max() <= 1e-6
    assert np.median(e6) <= 1e-6 and np.median(e7) <= 1e-7
    assert (e7 <= 1e-6).mean() >= 0.9 and e7.max() <= 1e-5
    ctx.close()


def test_adjoint_costs_at_most_four_forward_steps():
    import torch

    from fornaxamr_b200 import autograd as ag
    fx, ctx, blocks, dx, rho0, v0, A0 = _setup()
    with torch.no_grad():
        W0, Bf0 = ag.initial_state(rho0, v0, A0, GAMMA, dx)
    ctx.upload_all(np.ascontiguousarray(W0.numpy().reshape(-1)), np.ascontiguousarray(Bf0.numpy().reshape(-1)))
    ctx.boundary_fill(1, 0)
    dt = ctx.calc_dt(0.4)
    nb = len(blocks)
    ctx.adjoint_forward(NSTEPS, dt)
    seed = np.zeros(W0.numel())
    seed[:] = 1e-3
    for _ in range(2):
        ctx.adjoint_backward(seed)
    ms_adj = ctx.adjoint_ms() / NSTEPS
    ms_fwd = ctx.time_phase(fx.PHASE_STEP, 10, dt)
    assert ms_adj <= 4.0 * ms_fwd, (ms_adj, ms_fwd)
    ctx.close()
