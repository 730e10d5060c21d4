"""Hand-written adjoint of the XPBD substep (nb_xpbd_step_adjoint) on the GPU.

* its recomputed forward state equals the solver step's output;
* one substep: gradients of a random linear loss of (body_q, body_qd) with
  respect to every component of body_q, body_qd and body_f against central
  finite differences of the solver step with the same contacts (relative
  3e-2, absolute 5e-3 at one iteration, 8e-2 / 2e-2 at four, against the
  best of three step sizes: large steps cross the kinks of the contact set,
  small ones drown in FP32 rounding);
* a 20-substep rollout through torch.autograd (checkpoints every 8 substeps)
  against central differences of rollouts that replay the nominal rollout's
  contacts; checkpoint spacing does not change the gradients;
* restitution is refused.

The reference's own gradient (wp.Tape over its Warp kernels) cannot be
computed here: Warp is not installed.
"""

import numpy as np
import pytest
import torch

from newton_custom_contact_b200 import CollisionPipeline, SolverXPBD, scenes
from newton_custom_contact_b200._abi import GeoType
from newton_custom_contact_b200.adjoint import Rollout, SubstepAdjoint, simulate

pytestmark = pytest.mark.gpu

DEV = torch.device("cuda")
DT = 1.0 / 480.0


def _quat_x(a):
    return [np.sin(a / 2), 0.0, 0.0, np.cos(a / 2)]


def _scene(iterations=4):
    """Three worlds: a sliding, spinning sphere; a tilted box landing on an edge; two stacked spheres.
    Contacts are held fixed by the adjoint, so a finite difference must hold them fixed too."""
    types = [GeoType.SPHERE, GeoType.BOX, GeoType.SPHERE, GeoType.SPHERE]
    scales = [[0.1, 0, 0], [0.1, 0.08, 0.05], [0.08, 0, 0], [0.06, 0, 0]]
    # worlds do not interact: all at the origin, where FP32 positions carry the most digits
    poses = [[0.0, 0.0, 0.097] + [0, 0, 0, 1],
             [0.0, 0.0, 0.0584] + _quat_x(0.15),  # one edge 3 mm deep, the other 21 mm clear
             [0.0, 0.0, 0.077] + [0, 0, 0, 1],
             [0.0, 0.0, 0.077 + 0.08 + 0.06 - 0.003] + [0, 0, 0, 1]]
    # every contact slides by millimetres per substep and its bodies turn relative to each other both about
    # and across the normal: friction, torsional and rolling friction stay on one side of their
    # non-differentiable points (zero slip, the friction cone's edge) under the finite-difference steps
    qd = [[1.5, 0.8, 0.0, 3.0, -2.0, 2.5],
          [1.2, -0.9, -0.1, 2.0, 1.5, -2.0],
          [0.9, 0.5, 0.0, 2.5, -3.0, 1.5],
          [-0.8, 1.1, 0.0, -2.0, 3.5, -1.0]]
    m = scenes.assemble_free_bodies(np.array([0, 1, 2, 2]), np.array([int(t) for t in types]), np.array(scales),
                                    np.array(poses), np.full(4, 0.6), 3, qd=np.array(qd), device=DEV)
    pipe = CollisionPipeline(m)
    solver = SolverXPBD(m, iterations=iterations)
    return m, pipe, solver


def _loss_weights(B, seed=0):
    g = torch.Generator().manual_seed(seed)
    return (torch.randn(B, 7, generator=g).to(DEV), torch.randn(B, 6, generator=g).to(DEV))


def _step(solver, m, c, q, qd, f):
    a, b = m.state(), m.state()
    a.body_q.copy_(q)
    a.body_qd.copy_(qd)
    a.body_f.copy_(f)
    solver.step(a, b, None, c, DT)
    return b.body_q, b.body_qd


def test_adjoint_forward_matches_step():
    m, pipe, solver = _scene()
    a = m.state()
    c = pipe.contacts()
    pipe.collide(a, c)
    assert int(c.rigid_contact_count.item()) > 0
    q1, qd1 = _step(solver, m, c, a.body_q, a.body_qd, a.body_f)
    fq, fqd = torch.empty_like(q1), torch.empty_like(qd1)
    adj = SubstepAdjoint(solver)
    adj(c, a.body_q, a.body_qd, a.body_f, torch.zeros_like(q1), torch.zeros_like(qd1), DT, forward_out=(fq, fqd))
    torch.cuda.synchronize()
    assert adj.status() == 0
    torch.testing.assert_close(fq, q1, rtol=1e-6, atol=1e-6)
    torch.testing.assert_close(fqd, qd1, rtol=1e-5, atol=1e-5)


@pytest.mark.parametrize("iterations", [1, 4])
def test_substep_gradient_matches_finite_differences(iterations):
    m, pipe, solver = _scene(iterations)
    a = m.state()
    c = pipe.contacts()
    pipe.collide(a, c)
    B = m.body_count
    wq, wqd = _loss_weights(B)
    f = torch.zeros(B, 6, device=DEV)
    f[:, :3] = torch.tensor([1.0, -2.0, 0.5], device=DEV)
    q0, qd0 = a.body_q.clone(), a.body_qd.clone()
    adj = SubstepAdjoint(solver)
    gq, gqd, gf = adj(c, q0, qd0, f, wq, wqd, DT)
    torch.cuda.synchronize()

    def loss(q, qd, ff):
        q1, qd1 = _step(solver, m, c, q, qd, ff)
        return float((q1.double() * wq.double()).sum() + (qd1.double() * wqd.double()).sum())

    # with several iterations the per-iteration kinks compose: central differences of some entries then
    # vary by 10 % or more between step sizes, so the tolerance is wider there
    rel, abs_ = (3e-2, 5e-3) if iterations == 1 else (8e-2, 2e-2)
    bad = _fd_mismatches(loss, {"q": q0, "qd": qd0, "f": f}, {"q": gq, "qd": gqd, "f": gf},
                         [(n, i, k) for n, w in (("q", 7), ("qd", 6), ("f", 6)) for i in range(B) for k in range(w)],
                         rel=rel, abs_=abs_)
    assert not bad, bad


FD_STEPS = {"q": (1e-3, 1e-4, 1e-5), "qd": (1e-3, 1e-4, 1e-5), "f": (1e-1, 1e-2, 1e-3)}


def _fd_mismatches(loss, base, grads, entries, rel=3e-2, abs_=5e-3):
    """Entries whose analytic derivative matches no central difference of `loss` among FD_STEPS: the
    large steps are limited by the contact set's kinks (a contact turning active), the small ones by
    FP32 rounding of the step's outputs."""
    bad = []
    for name, i, k in entries:
        an = float(grads[name][i, k])
        fds = []
        for h in FD_STEPS[name]:
            xp, xm = base[name].clone(), base[name].clone()
            xp[i, k] += h
            xm[i, k] -= h
            lp = loss(*[xp if n == name else base[n] for n in ("q", "qd", "f")])
            lm = loss(*[xm if n == name else base[n] for n in ("q", "qd", "f")])
            fds.append((lp - lm) / (2 * h))
        if not any(abs(fd - an) <= abs_ + rel * max(abs(fd), abs(an)) for fd in fds):
            bad.append((name, i, k, an, fds))
    return bad


def _record_contacts(pipe, solver, m, q, qd, f, substeps):
    """Nominal rollout; per substep a copy of the solver records the step used."""
    a, b = m.state(), m.state()
    c = pipe.contacts()
    a.body_q.copy_(q)
    a.body_qd.copy_(qd)
    recs = []
    for _ in range(substeps):
        a.body_f.copy_(f)
        pipe.collide(a, c)
        recs.append({k: c._seg[k].clone() for k in ("rec", "world_base", "world_count")})
        solver.step(a, b, None, c, DT)
        a, b = b, a
    return c, recs


def _replay(solver, m, c, recs, q, qd, f):
    a, b = m.state(), m.state()
    a.body_q.copy_(q)
    a.body_qd.copy_(qd)
    for r in recs:
        a.body_f.copy_(f)
        for k, v in r.items():
            c._seg[k].copy_(v)
        c._seg_valid = True
        solver.step(a, b, None, c, DT)
        a, b = b, a
    return a.body_q, a.body_qd


def test_rollout_gradient_matches_finite_differences():
    m, pipe, solver = _scene(iterations=4)
    B = m.body_count
    s0 = m.state()
    q0, qd0 = s0.body_q.clone(), s0.body_qd.clone()
    f = torch.zeros(B, 6, device=DEV)
    wq, wqd = _loss_weights(B, seed=1)
    qv, qdv, fv = q0.clone().requires_grad_(True), qd0.clone().requires_grad_(True), f.clone().requires_grad_(True)
    q1, qd1 = simulate(pipe, solver, qv, qdv, fv, substeps=20, dt=DT, checkpoint_every=8)
    ((q1 * wq).sum() + (qd1 * wqd).sum()).backward()
    c, recs = _record_contacts(pipe, solver, m, q0, qd0, f, 20)
    qn, qdn = _replay(solver, m, c, recs, q0, qd0, f)
    torch.testing.assert_close(qn, q1.detach(), rtol=0, atol=0)  # the replay is the nominal rollout

    def loss(q, qd, ff):
        a, b = _replay(solver, m, c, recs, q, qd, ff)
        return float((a.double() * wq.double()).sum() + (b.double() * wqd.double()).sum())

    checks = [("qd", 0, 0), ("qd", 1, 5), ("qd", 3, 3), ("qd", 2, 1), ("q", 0, 2), ("q", 1, 1), ("q", 2, 0),
              ("q", 3, 6), ("f", 0, 0), ("f", 1, 2), ("f", 3, 4), ("f", 2, 5)]
    bad = _fd_mismatches(loss, {"q": q0, "qd": qd0, "f": f}, {"q": qv.grad, "qd": qdv.grad, "f": fv.grad}, checks,
                         rel=5e-2, abs_=1e-2)
    assert not bad, bad


def test_checkpoint_spacing_does_not_change_gradients():
    m, pipe, solver = _scene(iterations=2)
    B = m.body_count
    s0 = m.state()
    wq, wqd = _loss_weights(B, seed=2)
    out = []
    for every in (3, 16):
        qv, qdv = s0.body_q.clone().requires_grad_(True), s0.body_qd.clone().requires_grad_(True)
        fv = torch.zeros(B, 6, device=DEV, requires_grad=True)
        q1, qd1 = simulate(pipe, solver, qv, qdv, fv, substeps=12, dt=DT, checkpoint_every=every)
        ((q1 * wq).sum() + (qd1 * wqd).sum()).backward()
        out.append((qv.grad.clone(), qdv.grad.clone(), fv.grad.clone()))
    for x, y in zip(out[0], out[1]):
        torch.testing.assert_close(x, y, rtol=1e-5, atol=1e-6)


def test_restitution_is_refused():
    m, pipe, solver = _scene()
    solver.enable_restitution = True
    a = m.state()
    c = pipe.contacts()
    pipe.collide(a, c)
    z = torch.zeros_like
    with pytest.raises(NotImplementedError):
        SubstepAdjoint(solver)(c, a.body_q, a.body_qd, a.body_f, z(a.body_q), z(a.body_qd), DT)
    with pytest.raises(NotImplementedError):
        Rollout(CollisionPipeline(m, contact_matching="latest"), SolverXPBD(m), DT)


def test_c5_stack_com_gradient():
    """The differentiation workload: 16-box stacks, 64 substeps at dt = 1/600 with 8 iterations,
    loss = sum over worlds of |COM_final - target|^2, gradient with respect to the initial state
    through the checkpointed rollout (every 16 substeps).  Per-component central differences of a
    64-substep stack drown in FP32 rounding, so the check is directional: for a random direction v of
    the initial twists, the derivative of a linear COM loss along v against central differences of
    rollouts that replay the nominal rollout's contacts (same sign, within a factor of 4)."""
    m, info = scenes.scene_c5(worlds=3, device=DEV)
    pipe = CollisionPipeline(m)
    solver = SolverXPBD(m, iterations=info["iterations"])
    dt, n_sub = info["dt"], info["substeps"]
    B, W = m.body_count, m.world_count
    s0 = m.state()
    q0, qd0 = s0.body_q.clone(), s0.body_qd.clone()
    f = torch.zeros(B, 6, device=DEV)
    world = torch.repeat_interleave(torch.arange(W, device=DEV), B // W)

    def com(q):
        c = torch.zeros(W, 3, dtype=q.dtype, device=DEV)
        c.index_add_(0, world, q[:, :3])
        return c / (B // W)

    target = com(q0) + torch.tensor([0.05, -0.02, 0.0], device=DEV)
    # the workload's loss: a finite, non-zero gradient
    qv, qdv = q0.clone().requires_grad_(True), qd0.clone().requires_grad_(True)
    q1, _ = simulate(pipe, solver, qv, qdv, f, substeps=n_sub, dt=dt, checkpoint_every=16)
    ((com(q1) - target) ** 2).sum().backward()
    assert bool(torch.isfinite(qdv.grad).all()) and float(qdv.grad.abs().max()) > 0.0
    # directional check with a linear loss
    gen = torch.Generator().manual_seed(11)
    cw = torch.randn(W, 3, generator=gen).to(DEV)
    v = torch.randn(B, 6, generator=gen).to(DEV)
    qdv2 = qd0.clone().requires_grad_(True)
    q1b, _ = simulate(pipe, solver, q0.clone(), qdv2, f, substeps=n_sub, dt=dt, checkpoint_every=16)
    (com(q1b) * cw).sum().backward()
    an = float((qdv2.grad * v).sum())

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

    def loss(qd):
        qq, _ = _replay_dt(solver, m, c, recs, q0, qd, f, dt)
        return float((com(qq.double()) * cw.double()).sum())

    # A 64-substep stack is piecewise smooth at a fine scale (contacts turn on and off, friction
    # sticks and slips every few substeps): central differences along v vary by 2x between step
    # sizes (measured: 0.061 / 0.027 / 0.037 at h = 1e-2 / 3e-3 / 1e-3 against 0.111 analytic), so
    # only sign and magnitude are checked here; the tight checks run on the smoother scenes above.
    fds = [(loss(qd0 + h * v) - loss(qd0 - h * v)) / (2 * h) for h in (1e-2, 3e-3, 1e-3)]
    assert all(fd * an > 0.0 for fd in fds), (an, fds)
    assert any(0.25 <= an / fd <= 4.0 for fd in fds), (an, fds)


def _replay_dt(solver, m, c, recs, q, qd, f, dt):
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
    return a.body_q, a.body_qd
