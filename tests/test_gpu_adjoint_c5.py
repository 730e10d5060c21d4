"""The differentiation workload at its configured size: 1024 worlds of 16-box stacks (box half-extent
0.1 m, lateral jitter +-1 cm, per-world friction mu ~ U[0.4, 0.8], initial body velocities ~ N(0, 0.1)),
64 substeps at dt = 1/600 s with 8 iterations, checkpoints every 16 substeps.  The loss of a world is
the squared distance of its stack's final centre of mass from a target (the initial centre of mass
moved by N(0, 2 cm) along x and y).

The worlds never interact, so one pair of rollouts with every world perturbed at once gives every
world's own central difference: 1024 independent checks per quantity, at eps = 1e-4.

A substep is piecewise smooth: in every iteration a contact is active or not (depth < 0), friction is
inside its cone or clamped to it, a body's speed is above the 1e-4 rest threshold or zeroed.  Resting
stacks sit on these seams (a contact at rest hovers at depth 0 from one iteration to the next), so a
difference at eps = 1e-4 crosses many of them, and its value depends on eps (the free-running
statistics below, printed, show how much).  The adjoint is the derivative on the piece the rollout is
on.  The check that pins it replays, on both sides of each difference, the nominal rollout's contacts
and branches (``SubstepAdjoint.forward(..., branches, replay=True)``: the same contacts the adjoint
holds fixed, as the reference's tape does through its narrow phase, and the same branches), so the
difference is taken on that piece:

* d loss / d mu_w (per-world friction through the shapes' coefficients) and the derivative of each
  world's loss along a random direction of its initial body velocities: the adjoint agrees with the
  difference to 5 % (plus 1e-6 absolute) on at least 95 % of the worlds;
* over the full set, the derivative of the total loss along a random direction of all per-world
  frictions, and along a random direction of all initial velocities: to 1 %.
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
HEIGHT = 16
RTOL, ATOL = 0.05, 1e-6


def _agreement(an, fd):
    """fraction of worlds where the adjoint agrees with the difference"""
    return float(np.mean(np.abs(an - fd) <= RTOL * np.abs(fd) + ATOL))


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

    def world_loss(q):
        return ((com_of(q) - target) ** 2).sum(1)

    # analytic gradients through the checkpointed rollout (every 16 substeps)
    mu_w = mu_w0.clone().requires_grad_(True)
    qdv = qd0.clone().requires_grad_(True)
    q1, _ = simulate(pipe, solver, q0.clone(), qdv, f, substeps=n_sub, dt=dt, checkpoint_every=16,
                     shape_mu=shape_mu_of(mu_w))
    world_loss(q1).sum().backward()
    g_mu = mu_w.grad.detach().cpu().numpy()
    v = torch.randn(B, 6, generator=gen).to(DEV)
    g_v = torch.zeros(W, dtype=torch.float64, device=DEV)
    g_v.index_add_(0, world, (qdv.grad.double() * v.double()).sum(1))
    g_v = g_v.cpu().numpy()
    dmu = torch.randn(W, generator=gen, dtype=torch.float64).to(DEV)
    an_dir_mu = float((mu_w.grad * dmu).sum())
    an_dir_v = float(g_v.sum())

    # the nominal rollout through the adjoint's forward pass, recording each substep's contacts and branches
    m.shape_material_mu.copy_(base_mu)
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
    torch.testing.assert_close(q, q1.detach(), rtol=0, atol=0)

    def rollout(mu, qd_init, replay):
        m.shape_material_mu.copy_(shape_mu_of(mu).float())
        q, qd = q0.clone(), qd_init.clone()
        b_state = m.state()
        for r, br in zip(recs, branches):
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
        return world_loss(q).cpu().numpy()

    def differences(replay, h):
        fd_mu = (rollout(mu_w0 + h, qd0, replay) - rollout(mu_w0 - h, qd0, replay)) / (2 * h)
        fd_v = (rollout(mu_w0, qd0 + h * v, replay) - rollout(mu_w0, qd0 - h * v, replay)) / (2 * h)
        fd_dir_mu = float((rollout(mu_w0 + h * dmu, qd0, replay).sum()
                           - rollout(mu_w0 - h * dmu, qd0, replay).sum()) / (2 * h))
        return fd_mu, fd_v, fd_dir_mu

    fz_mu, fz_v, fz_dir_mu = differences(True, EPS)
    stats = {
        "worlds": W,
        "median_abs_grad": {"friction": float(np.median(np.abs(g_mu))), "velocity": float(np.median(np.abs(g_v)))},
        "branches_replayed": {
            "friction_agrees": _agreement(g_mu, fz_mu), "friction_relerr": _relerr(g_mu, fz_mu),
            "velocity_agrees": _agreement(g_v, fz_v), "velocity_relerr": _relerr(g_v, fz_v),
            "friction_direction": [an_dir_mu, fz_dir_mu], "velocity_direction": [an_dir_v, float(fz_v.sum())]},
    }
    # the same differences free-running (branches evaluated): how far the seams move them, at three eps
    free = {}
    for h in (EPS, 1e-3, 1e-2):
        fm, fv, fdir = differences(False, h)
        free[str(h)] = {"friction_agrees": _agreement(g_mu, fm), "velocity_agrees": _agreement(g_v, fv),
                        "friction_direction": fdir, "velocity_direction": float(fv.sum())}
    stats["free_running"] = free
    print("C5 gradient check:", json.dumps(stats))

    assert np.isfinite(g_mu).all() and np.isfinite(g_v).all()
    assert np.abs(g_mu).max() > 0.0 and np.abs(g_v).max() > 0.0
    assert stats["branches_replayed"]["friction_agrees"] >= 0.95, stats
    assert stats["branches_replayed"]["velocity_agrees"] >= 0.95, stats
    assert abs(an_dir_mu - fz_dir_mu) <= 0.01 * abs(fz_dir_mu), stats
    assert abs(an_dir_v - float(fz_v.sum())) <= 0.01 * abs(float(fz_v.sum())), stats
