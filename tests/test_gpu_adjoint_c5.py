"""The differentiation workload at its configured size: 1024 worlds of 16-box stacks (box half-extent
0.1 m, lateral jitter +-1 cm, per-world friction mu ~ U[0.4, 0.8], initial body velocities ~ N(0, 0.1)),
64 substeps at dt = 1/600 s with 8 iterations, checkpoints every 16 substeps.  The loss of a world is
the squared distance of its stack's final centre of mass from a target (the initial centre of mass
moved by N(0, 2 cm) along x and y).

The worlds never interact, so one pair of rollouts with every world perturbed at once gives every
world's own central difference: 1024 independent checks per quantity.

A substep is piecewise smooth: in every iteration a contact is active or not (depth < 0), friction is
inside its cone or clamped to it, a body's speed is above the 1e-4 rest threshold or zeroed.  Resting
stacks sit on these seams (a contact at rest hovers at depth 0 from one iteration to the next), so a
free-running difference crosses many of them and does not converge as eps shrinks (printed).  The
adjoint is the derivative on the piece the rollout is on.  The check replays, on both sides of each
difference, the nominal rollout's contacts and branches (``SubstepAdjoint.forward(..., branches,
replay=True)``: the contacts the adjoint holds fixed, as the reference's tape does through its narrow
phase, and the same branches), so the difference is taken on that piece.  In FP32 a difference still
carries rounding noise (which grows as eps shrinks) and truncation error (which grows with eps), so
each difference is paired with the difference at a second eps and their gap serves as its error
estimate:

* the configured check -- 64 substeps, eps = 1e-4, over the full set: the derivative of the total loss
  along a random direction of all initial velocities, and along the adjoint's own friction gradient
  (scaled to a largest entry of 1; a wrong gradient shows as a smaller difference), agree with the
  differences to 5 % plus twice the gap to the differences at eps = 3e-4;
* per world, over one checkpoint segment (16 substeps) at eps = 1e-3: d loss / d mu_w and the
  derivative along a random direction of the world's initial velocities agree with the difference to
  5 % plus twice the gap to the difference at eps = 3e-4 on at least 95 % of the worlds (per-world
  differences over 64 substeps are dominated by FP32 noise at every eps: printed, not asserted).
"""

import json

import numpy as np
import pytest
import torch

from newton_custom_contact_b200 import CollisionPipeline, SolverXPBD, scenes
from newton_custom_contact_b200.adjoint import SubstepAdjoint, simulate

pytestmark = pytest.mark.gpu

DEV = torch.device("cuda")
EPS = 1e-4
EPS2 = 3e-4  # the second eps of the differences' error estimate
CHECK_EPS = 1e-3
REPLAY_EPS = (EPS, EPS2, CHECK_EPS)
DIR_RTOL = 0.05
HEIGHT = 16
RTOL, ATOL = 0.05, 1e-6


def _agreement(an, fd, fd_other=None):
    """fraction of worlds where the adjoint agrees with the difference: to RTOL (+ ATOL), or, given the
    difference at a second eps, to RTOL plus twice the two differences' gap (the difference's own error
    estimate: rounding noise shrinks and truncation grows with eps)"""
    tol = RTOL * np.abs(fd) + ATOL
    if fd_other is not None:
        tol = tol + 2.0 * np.abs(fd - fd_other)
    return float(np.mean(np.abs(an - fd) <= tol))


def _relerr(an, fd):
    e = np.abs(an - fd) / np.maximum(np.abs(fd), 1e-12)
    return {f"p{q}": float(np.percentile(e, q)) for q in (50, 90, 99)}


def test_c5_friction_and_velocity_gradients_1024_worlds(cuda):
    m, info = scenes.scene_c5(worlds=1024, device=DEV)
    dt, n_sub = info["dt"], info["substeps"]
    pipe = CollisionPipeline(m)
    solver = SolverXPBD(m, iterations=info["iterations"])
    B, W = m.body_count, m.world_count
    world = torch.repeat_interleave(torch.arange(W, device=DEV), HEIGHT)
    s0 = m.state()
    q0, qd0 = s0.body_q.clone(), s0.body_qd.clone()
    f = torch.zeros(B, 6, device=DEV)
    base_mu = m.shape_material_mu.clone()
    # shape 0 is the ground plane; shapes 1.. are the boxes, HEIGHT per world in world order
    mu_w0 = base_mu[1::HEIGHT].double().clone()

    def shape_mu_of(mu_w):
        return torch.cat([base_mu[:1].to(mu_w.dtype), torch.repeat_interleave(mu_w, HEIGHT)])

    def com_of(q):
        com = torch.zeros(W, 3, dtype=torch.float64, device=DEV)
        com.index_add_(0, world, q[:, :3].double())
        return com / HEIGHT

    gen = torch.Generator().manual_seed(5)
    target = com_of(q0)
    target[:, :2] += 0.02 * torch.randn(W, 2, generator=gen, dtype=torch.float64).to(DEV)
    v = torch.randn(B, 6, generator=gen).to(DEV)

    def world_loss(q):
        return ((com_of(q) - target) ** 2).sum(1)

    # the nominal rollout through the adjoint's forward pass, recording each substep's contacts and branches
    fwd = SubstepAdjoint(solver)
    c = pipe.contacts()
    a = m.state()
    q, qd = q0.clone(), qd0.clone()
    recs, branches = [], []
    for _ in range(n_sub):
        a.body_q.copy_(q)
        pipe.collide(a, c)
        recs.append({k: c._seg[k].clone() for k in ("rec", "world_base", "world_count")})
        br = fwd.branch_buffers(c)
        qn, qdn = torch.empty_like(q), torch.empty_like(qd)
        fwd.forward(c, q, qd, f, dt, qn, qdn, branches=br)
        branches.append(br)
        q, qd = qn, qdn

    def rollout(n, mu, qd_init, replay):
        m.shape_material_mu.copy_(shape_mu_of(mu).float())
        q, qd = q0.clone(), qd_init.clone()
        b_state = m.state()
        for r, br in zip(recs[:n], branches[:n]):
            for k, t in r.items():
                c._seg[k].copy_(t)
            c._seg_valid = True
            qn, qdn = torch.empty_like(q), torch.empty_like(qd)
            if replay:
                fwd.forward(c, q, qd, f, dt, qn, qdn, branches=br, replay=True)
            else:
                a.body_q.copy_(q)
                a.body_qd.copy_(qd)
                a.body_f.copy_(f)
                solver.step(a, b_state, None, c, dt)
                qn, qdn = b_state.body_q.clone(), b_state.body_qd.clone()
            q, qd = qn, qdn
        m.shape_material_mu.copy_(base_mu)
        return q

    stats = {"worlds": W}
    results = {}
    for n in (16, n_sub):
        # analytic gradients through the checkpointed rollout (every 16 substeps)
        mu_w = mu_w0.clone().requires_grad_(True)
        qdv = qd0.clone().requires_grad_(True)
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
        ev[0].record()
        q1, _ = simulate(pipe, solver, q0.clone(), qdv, f, substeps=n, dt=dt, checkpoint_every=16,
                         shape_mu=shape_mu_of(mu_w))
        ev[1].record()
        world_loss(q1).sum().backward()
        ev[2].record()
        torch.cuda.synchronize()
        m.shape_material_mu.copy_(base_mu)
        # the recorded forward equals the solver's rollout bit for bit
        torch.testing.assert_close(rollout(n, mu_w0, qd0, True), q1.detach(), rtol=0, atol=0)
        g_mu = mu_w.grad.detach()
        g_v = torch.zeros(W, dtype=torch.float64, device=DEV)
        g_v.index_add_(0, world, (qdv.grad.double() * v.double()).sum(1))
        an = {"friction": g_mu.cpu().numpy(), "velocity": g_v.cpu().numpy()}
        # directions: the initial velocities along v (every world), the frictions along the adjoint's own
        # gradient scaled to a largest entry of 1 (the direction of largest change; a wrong gradient
        # shows as a smaller difference)
        dmu = g_mu / g_mu.abs().max()
        an_dir = {"friction": float((g_mu * dmu).sum()), "velocity": float(g_v.sum())}
        st = {"median_abs_grad": {k: float(np.median(np.abs(x))) for k, x in an.items()}, "adjoint_direction": an_dir,
              "ms": {"forward": ev[0].elapsed_time(ev[1]), "backward": ev[1].elapsed_time(ev[2])}}
        for h in REPLAY_EPS:
            loss = lambda mu, qd: world_loss(rollout(n, mu, qd, True)).cpu().numpy()  # noqa: E731
            fd = {"friction": (loss(mu_w0 + h, qd0) - loss(mu_w0 - h, qd0)) / (2 * h),
                  "velocity": (loss(mu_w0, qd0 + h * v) - loss(mu_w0, qd0 - h * v)) / (2 * h)}
            fdir = {"friction": float((loss(mu_w0 + h * dmu, qd0).sum() - loss(mu_w0 - h * dmu, qd0).sum()) / (2 * h)),
                    "velocity": float(fd["velocity"].sum())}
            results[(n, h)] = (an, fd, an_dir, fdir)
            st[f"replayed eps={h:g}"] = {k: {"agrees": _agreement(an[k], fd[k]), "relerr": _relerr(an[k], fd[k]),
                                             "direction": fdir[k]} for k in an}
            if (n, EPS2) in results and h == CHECK_EPS:
                other = results[(n, EPS2)][1]
                for k in an:
                    st[f"replayed eps={h:g}"][k]["agrees_within_own_error"] = _agreement(an[k], fd[k], other[k])
        for h in (EPS, 1e-3):
            loss = lambda mu, qd: world_loss(rollout(n, mu, qd, False)).cpu().numpy()  # noqa: E731
            fv = (loss(mu_w0, qd0 + h * v) - loss(mu_w0, qd0 - h * v)) / (2 * h)
            st[f"free eps={h:g}"] = {"velocity_agrees": _agreement(an["velocity"], fv),
                                     "velocity_direction": float(fv.sum())}
        stats[f"{n} substeps"] = st
    print("C5 gradient check:", json.dumps(stats))

    # the configured check: 64 substeps, eps = 1e-4, directional derivatives over the full set
    an, fd, an_dir, fdir = results[(n_sub, EPS)]
    _, _, _, fdir3 = results[(n_sub, EPS2)]
    for k in ("friction", "velocity"):
        assert np.isfinite(an[k]).all() and np.abs(an[k]).max() > 0.0
        assert abs(an_dir[k] - fdir[k]) <= DIR_RTOL * abs(fdir[k]) + 2.0 * abs(fdir[k] - fdir3[k]), stats
    # per world, over one checkpoint segment (16 substeps), at eps = 1e-3 with the error estimate from 3e-4
    an16, fd16, _, _ = results[(16, CHECK_EPS)]
    _, fd16b, _, _ = results[(16, EPS2)]
    for k in ("friction", "velocity"):
        assert _agreement(an16[k], fd16[k], fd16b[k]) >= 0.95, stats
