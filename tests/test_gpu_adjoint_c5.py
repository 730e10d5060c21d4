"""The differentiation workload at its configured size: 1024 worlds of 16-box stacks (box half-extent
0.1 m, lateral jitter +-1 cm, per-world friction mu ~ U[0.4, 0.8], initial twists ~ N(0, 0.1)),
64 substeps at dt = 1/600 s with 8 iterations, checkpoints every 16 substeps.

The loss is a sum of per-world terms and the worlds never interact, so one pair of rollouts with
every world perturbed at once gives every world's own central difference: 1024 independent checks
per quantity.  Central differences use eps = 1e-4 and replay the nominal rollout's contacts (the
adjoint holds each substep's contact set and geometry fixed, as the reference's tape does through
its narrow phase).  Checked:

* d loss / d mu_w (per-world friction, through the shapes' coefficients): on the worlds where the
  differences at eps = 1e-4 and 2e-4 agree to 5 % (the rollout is smooth there at that scale;
  stacks stick and slip, so some worlds sit on a kink), the adjoint agrees with the difference to
  5 % + 1e-4 for at least 95 % of them, and such worlds are at least half of all;
* the directional derivative of each world's loss along a random direction of its initial twists:
  the same criterion;
* over the full set, the derivative of the total loss along a random direction of all per-world
  frictions against its central difference, to 5 %.
"""

import json

import numpy as np
import pytest
import torch

from newton_custom_contact_b200 import CollisionPipeline, SolverXPBD, scenes
from newton_custom_contact_b200.adjoint import simulate

pytestmark = pytest.mark.gpu

DEV = torch.device("cuda")
EPS = 1e-4
HEIGHT = 16


def _replay(solver, m, c, recs, q, qd, f, dt):
    a, b = m.state(), m.state()
    a.body_q.copy_(q)
    a.body_qd.copy_(qd)
    for r in recs:
        a.body_f.copy_(f)
        for k, v in r.items():
            c._seg[k].copy_(v)
        c._seg_valid = True
        solver.step(a, b, None, c, dt)
        a, b = b, a
    return a.body_q


def _agreement(an, fd1, fd2):
    """(fraction of worlds whose differences agree, fraction of those where the adjoint agrees)"""
    smooth = np.abs(fd1 - fd2) <= 0.05 * np.maximum(np.abs(fd1), np.abs(fd2)) + 1e-6
    ok = np.abs(an - fd1) <= 0.05 * np.abs(fd1) + 1e-4
    return float(smooth.mean()), float(ok[smooth].mean()) if smooth.any() else 0.0


def test_c5_friction_and_twist_gradients_1024_worlds(cuda):
    m, info = scenes.scene_c5(worlds=1024, device=DEV)
    dt, n_sub = info["dt"], info["substeps"]
    pipe = CollisionPipeline(m)
    solver = SolverXPBD(m, iterations=info["iterations"])
    B, W, S = m.body_count, m.world_count, m.shape_count
    world = torch.repeat_interleave(torch.arange(W, device=DEV), HEIGHT)
    s0 = m.state()
    q0, qd0 = s0.body_q.clone(), s0.body_qd.clone()
    f = torch.zeros(B, 6, device=DEV)
    base_mu = m.shape_material_mu.clone()
    # shape 0 is the ground plane; shapes 1.. are the boxes, HEIGHT per world in world order
    mu_w0 = base_mu[1::HEIGHT].double().clone()

    def shape_mu_of(mu_w):
        return torch.cat([base_mu[:1].to(mu_w.dtype), torch.repeat_interleave(mu_w, HEIGHT)])

    gen = torch.Generator().manual_seed(5)
    cw = torch.randn(W, 3, generator=gen, dtype=torch.float64).to(DEV)
    cw[:, 2] = 0.0  # lateral COM: what friction moves

    def world_loss(q):
        com = torch.zeros(W, 3, dtype=torch.float64, device=DEV)
        com.index_add_(0, world, q[:, :3].double())
        return (com / HEIGHT * cw).sum(1)  # one linear term per world

    # analytic gradients through the checkpointed rollout (every 16 substeps)
    mu_w = mu_w0.clone().requires_grad_(True)
    qdv = qd0.clone().requires_grad_(True)
    q1, _ = simulate(pipe, solver, q0.clone(), qdv, f, substeps=n_sub, dt=dt, checkpoint_every=16,
                     shape_mu=shape_mu_of(mu_w))
    world_loss(q1).sum().backward()
    g_mu = mu_w.grad.detach().cpu().numpy()
    v = torch.randn(B, 6, generator=gen).to(DEV)
    g_tw = torch.zeros(W, dtype=torch.float64, device=DEV)
    g_tw.index_add_(0, world, (qdv.grad.double() * v.double()).sum(1))
    g_tw = g_tw.cpu().numpy()

    # the nominal rollout's contacts, replayed by the differences
    m.shape_material_mu.copy_(base_mu)
    a, b = m.state(), m.state()
    c = pipe.contacts()
    a.body_q.copy_(q0)
    a.body_qd.copy_(qd0)
    recs = []
    for _ in range(n_sub):
        a.body_f.zero_()
        pipe.collide(a, c)
        recs.append({k: c._seg[k].clone() for k in ("rec", "world_base", "world_count")})
        solver.step(a, b, None, c, dt)
        a, b = b, a
    torch.testing.assert_close(a.body_q, q1.detach(), rtol=0, atol=0)

    def losses(mu=None, qd=None):
        m.shape_material_mu.copy_(shape_mu_of(mu0 if mu is None else mu).float())
        qq = _replay(solver, m, c, recs, q0, qd0 if qd is None else qd, f, dt)
        return world_loss(qq).cpu().numpy()

    mu0 = mu_w0
    fd_mu = {h: (losses(mu=mu0 + h) - losses(mu=mu0 - h)) / (2 * h) for h in (EPS, 2 * EPS)}
    fd_tw = {h: (losses(qd=qd0 + h * v) - losses(qd=qd0 - h * v)) / (2 * h) for h in (EPS, 2 * EPS)}
    # full set: all frictions along one random direction
    dmu = torch.randn(W, generator=gen, dtype=torch.float64).to(DEV)
    an_dir = float((mu_w.grad * dmu).sum())
    fd_dir = float((losses(mu=mu0 + EPS * dmu).sum() - losses(mu=mu0 - EPS * dmu).sum()) / (2 * EPS))
    m.shape_material_mu.copy_(base_mu)

    smooth_mu, ok_mu = _agreement(g_mu, fd_mu[EPS], fd_mu[2 * EPS])
    smooth_tw, ok_tw = _agreement(g_tw, fd_tw[EPS], fd_tw[2 * EPS])
    stats = {"worlds": W, "friction": {"smooth_fraction": smooth_mu, "adjoint_agrees": ok_mu,
                                       "median_abs_grad": float(np.median(np.abs(g_mu)))},
             "twist": {"smooth_fraction": smooth_tw, "adjoint_agrees": ok_tw,
                       "median_abs_grad": float(np.median(np.abs(g_tw)))},
             "friction_direction": {"adjoint": an_dir, "central_difference": fd_dir}}
    print("C5 gradient check:", json.dumps(stats))
    assert np.isfinite(g_mu).all() and np.isfinite(g_tw).all()
    assert np.abs(g_mu).max() > 0.0
    assert smooth_mu >= 0.5 and ok_mu >= 0.95, stats
    assert smooth_tw >= 0.5 and ok_tw >= 0.95, stats
    assert abs(an_dir - fd_dir) <= 0.05 * abs(fd_dir), stats
