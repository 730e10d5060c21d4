"""Learned warm start on the GPU: tensor-core inference, training kernels, and the solver pass.

* ``nb_ws_infer`` (tcgen05, BF16 operands, FP32 accumulation) against a CPU
  fp32 evaluation of the same network with the same BF16 rounding points and
  the same output map (prior ratio, inverse mass, friction cone); tolerance
  2e-2 relative + 3e-2 x out_scale x prior / w absolute (accumulation order
  and a BF16 rounding flip of a hidden activation are the only differences);
* ``nb_ws_grads`` against torch autograd on the CPU (fp32, straight-through
  BF16 rounding), relative 1e-3; one ``nb_ws_adam`` step against the formula;
* the solver: a network that predicts zero leaves the step bit-identical to
  the plain one; predictions that deepen every world's penetration fall back
  in every world, again bit-identical to the plain step; predictions that
  lift every contact are kept and reported in the contact impulse.
"""

import numpy as np
import pytest
import torch

from newton_custom_contact_b200 import CollisionPipeline, SolverXPBD, scenes
from newton_custom_contact_b200.warmstart import N_FEAT, N_HID, N_IN, N_OUT, WarmStart, WarmStartNet

pytestmark = pytest.mark.gpu

DEV = torch.device("cuda")


def _bf(x):
    return x.to(torch.bfloat16).to(torch.float32)


def _random_net(seed=3):
    net = WarmStartNet(device=DEV, seed=seed)
    g = torch.Generator().manual_seed(seed + 1)
    for k in ("b1", "b2", "b3"):
        net.params[k] = (torch.randn(net.params[k].shape, generator=g) * 0.2).to(DEV)
    net.params["w3"] = (torch.randn(N_OUT, N_HID, generator=g) / np.sqrt(N_HID)).to(DEV)
    net.in_mean = (torch.randn(N_IN, generator=g) * 0.5).to(DEV)
    net.in_inv_std = (torch.rand(N_IN, generator=g) * 2 + 0.5).to(DEV)
    net.out_scale = torch.tensor([0.5, 2.0, 3.0], device=DEV)
    net._packed = None
    return net


def _ref_forward(net, x):
    """Corrections c of network inputs x [R, 24]."""
    p = {k: v.detach().cpu() for k, v in net.params.items()}
    xn = _bf((x.cpu() - net.in_mean.cpu()) * net.in_inv_std.cpu())
    h1 = _bf(torch.nn.functional.silu(xn @ _bf(p["w1"]).T + p["b1"]))
    h2 = _bf(torch.nn.functional.silu(h1 @ _bf(p["w2"]).T + p["b2"]))
    return (h2 @ _bf(p["w3"]).T + p["b3"]) * net.out_scale.cpu()


def _ref_lambda(net, feat):
    """lambda of feature rows [R, 27] on the CPU: y = MLP(inputs), c = prior * y, lambda = c / w,
    lambda_n >= 0, |lambda_t| <= mu lambda_n, zero without a prior."""
    y = _ref_forward(net, feat[:, :N_IN])
    wn, wt, prior, mu = feat[:, N_IN], feat[:, N_IN + 1], feat[:, N_IN + 2], feat[:, 17]
    ok = (prior > 0) & (wn > 0) & (wt > 0)
    safe = lambda w: torch.where(w > 0, w, torch.ones_like(w))
    ln = y[:, 0].clamp_min(0.0) * prior / safe(wn)
    l1 = y[:, 1] * prior / safe(wt)
    l2 = y[:, 2] * prior / safe(wt)
    lt = torch.sqrt(l1 * l1 + l2 * l2)
    cap = mu * ln
    sc = torch.where(lt > cap, torch.where(lt > 0, cap / torch.where(lt > 0, lt, torch.ones_like(lt)), 0.0), 1.0)
    lam = torch.stack([ln, l1 * sc, l2 * sc], 1)
    return torch.where(ok[:, None], lam, torch.zeros_like(lam))


def _random_features(n, seed):
    g = torch.Generator().manual_seed(seed)
    x = torch.randn(n, N_FEAT, generator=g) * 1.5
    x[:, 17] = torch.rand(n, generator=g)  # friction coefficient
    x[:, N_IN:N_IN + 2] = torch.rand(n, 2, generator=g) * 4.0 + 0.25  # inverse masses
    x[:, N_IN + 2] = torch.rand(n, generator=g) * 2.0 + 0.01  # prior
    x[::7, N_IN + 2] = 0.0  # no prior: lambda = 0
    x[3::11, N_IN] = 0.0  # immovable along the normal: lambda = 0
    return x


@pytest.mark.parametrize("cap,count", [(1000, 1000), (1000, 300), (1000, 5000), (129, 0), (90001, 90001)])
def test_infer_matches_cpu_reference(cap, count):
    net = _random_net()
    x = _random_features(cap, cap)
    feat = x.to(DEV)
    out = torch.full((cap, N_OUT), 7.25, device=DEV)
    status = torch.zeros(1, dtype=torch.int32, device=DEV)
    net.infer(feat, torch.tensor([count], dtype=torch.int32, device=DEV), out, status)
    torch.cuda.synchronize()
    assert int(status.item()) == 0
    n = min(cap, count)
    got = out.cpu()
    if n:
        ref = _ref_lambda(net, x[:n])
        w = x[:n][:, [N_IN, N_IN + 1, N_IN + 1]]
        scale = float(net.out_scale.max()) * x[:n, N_IN + 2:N_IN + 3] / torch.where(w > 0, w, torch.ones_like(w))
        tol = 2e-2 * ref.abs() + 3e-2 * scale + 1e-6
        err = (got[:n] - ref).abs()
        assert bool((err <= tol).all()), f"max err {float(err.max())}"
        assert bool((got[:n][x[:n, N_IN + 2] == 0] == 0).all())
        assert bool((got[:n, 0] >= 0).all())
    assert bool((got[n:] == 7.25).all())  # rows beyond the count are not written


def _torch_grads(net, x, t):
    p = {k: v.detach().cpu().clone().requires_grad_(True) for k, v in net.params.items()}

    def q(w):  # straight-through BF16 rounding
        return w + (_bf(w) - w).detach()

    xn = _bf((x - net.in_mean.cpu()) * net.in_inv_std.cpu())
    h1 = q(torch.nn.functional.silu(xn @ q(p["w1"]).T + p["b1"]))
    h2 = q(torch.nn.functional.silu(h1 @ q(p["w2"]).T + p["b2"]))
    y = h2 @ q(p["w3"]).T + p["b3"]
    loss = ((y - t / net.out_scale.cpu()) ** 2).sum(1).mean()
    loss.backward()
    return {k: v.grad for k, v in p.items()}, float(loss.detach())


@pytest.mark.parametrize("rows", [1, 300, 4096])
def test_grads_match_autograd(rows):
    net = _random_net(seed=rows)
    g = torch.Generator().manual_seed(rows)
    x = torch.randn(rows, N_IN, generator=g)
    t = torch.randn(rows, N_OUT, generator=g) * net.out_scale.cpu()
    grads, loss = net.grads(x.to(DEV), t.to(DEV))
    ref, ref_loss = _torch_grads(net, x, t)
    assert abs(loss - ref_loss) <= 1e-4 * max(1.0, abs(ref_loss))
    for k in ref:
        a, b = grads[k].cpu(), ref[k]
        scale = float(b.abs().max()) + 1e-12
        assert float((a - b).abs().max()) <= 1e-3 * scale, k


def test_adam_step():
    from newton_custom_contact_b200 import _lib
    import ctypes as C

    from newton_custom_contact_b200._abi import ptr

    g = torch.Generator().manual_seed(0)
    w = torch.randn(1000, generator=g)
    gr = torch.randn(1000, generator=g)
    m1 = torch.randn(1000, generator=g) * 0.1
    m2 = torch.rand(1000, generator=g) * 0.1
    wd, m1d, m2d, gd = w.to(DEV), m1.to(DEV), m2.to(DEV), gr.to(DEV)
    lib = _lib.load()
    _lib.check("nb_ws_adam", lib.nb_ws_adam(C.c_void_p(ptr(wd)), C.c_void_p(ptr(gd)), C.c_void_p(ptr(m1d)),
                                            C.c_void_p(ptr(m2d)), 1000, 1e-2, 0.9, 0.999, 1e-8, 1e-4, 3,
                                            C.c_void_p(_lib.stream_handle(DEV))))
    e1 = 0.9 * m1 + 0.1 * gr
    e2 = 0.999 * m2 + 0.001 * gr * gr
    ew = w - 1e-2 * ((e1 / (1 - 0.9 ** 3)) / (torch.sqrt(e2 / (1 - 0.999 ** 3)) + 1e-8) + 1e-4 * w)
    # (1 - beta) is formed in fp32 on the device: a few ulp from the float64 constants here
    torch.testing.assert_close(m1d.cpu(), e1, rtol=1e-5, atol=1e-6)
    torch.testing.assert_close(m2d.cpu(), e2, rtol=1e-5, atol=1e-6)
    torch.testing.assert_close(wd.cpu(), ew, rtol=1e-5, atol=1e-6)


def _settled(iterations=4, substeps=48, matching="disabled"):
    m, _ = scenes.scene_c2(seed=1, worlds=64, nmin=8, nmax=32, device=DEV)
    pipe = CollisionPipeline(m, contact_matching=matching)
    solver = SolverXPBD(m, iterations=iterations)
    a, b = m.state(), m.state()
    c = pipe.contacts()
    dt = 1.0 / 480.0
    for _ in range(substeps):
        a.clear_forces()
        pipe.collide(a, c)
        solver.step(a, b, None, c, dt)
        a, b = b, a
    a.clear_forces()
    pipe.collide(a, c)
    return m, pipe, solver, a, c, dt


def _constant_net(b3):
    net = WarmStartNet(device=DEV)
    net.params["w3"] = torch.zeros(N_OUT, N_HID, device=DEV)
    net.params["b3"] = torch.tensor(b3, dtype=torch.float32, device=DEV)
    net._packed = None
    return net


def _step_pair(m, solver, a, c, dt, ws):
    plain, warm = m.state(), m.state()
    solver.warm_start = None
    solver.step(a, plain, None, c, dt)
    solver.warm_start = ws
    solver.step(a, warm, None, c, dt)
    solver.warm_start = None
    torch.cuda.synchronize()
    return plain, warm


def test_zero_prediction_is_plain_step():
    m, pipe, solver, a, c, dt = _settled()
    assert int(c.rigid_contact_count.item()) > 0
    ws = WarmStart(_constant_net([0.0, 0.0, 0.0]), iterations=None)
    plain, warm = _step_pair(m, solver, a, c, dt, ws)
    assert torch.equal(plain.body_q, warm.body_q)
    assert torch.equal(plain.body_qd, warm.body_qd)
    assert ws.fallback_count == 0


def _resting_spheres(worlds=96):
    """One sphere per world, 1 mm into the ground plane: exactly one contact per world."""
    from newton_custom_contact_b200._abi import GeoType

    types = np.full(worlds, int(GeoType.SPHERE))
    scales = np.zeros((worlds, 3))
    scales[:, 0] = np.linspace(0.05, 0.2, worlds)
    poses = np.zeros((worlds, 7))
    poses[:, 0] = np.arange(worlds) * 0.5
    poses[:, 2] = scales[:, 0] - 1e-3
    poses[:, 6] = 1.0
    m = scenes.assemble_free_bodies(np.arange(worlds), types, scales, poses, np.full(worlds, 0.5), worlds,
                                    device=DEV)
    pipe = CollisionPipeline(m)
    solver = SolverXPBD(m, iterations=4)
    a = m.state()
    c = pipe.contacts()
    a.clear_forces()
    pipe.collide(a, c)
    return m, pipe, solver, a, c, 1.0 / 480.0


class _ConstantLambda(WarmStart):
    """Feeds the step a fixed contact-frame lambda for every contact (bypasses the network's
    lambda_n >= 0 bound, so the solver's own fallback can be exercised)."""

    def __init__(self, lam):
        super().__init__(None, iterations=None)
        self.lam = lam

    def enabled(self):
        return True

    def predict(self, features, count, out, status):
        out.copy_(torch.tensor(self.lam, dtype=torch.float32, device=out.device).expand_as(out))


def test_deepening_prediction_falls_back_everywhere():
    m, pipe, solver, a, c, dt = _resting_spheres()
    n = int(c.rigid_contact_count.item())
    assert n == m.world_count
    # lambda_n < 0 pulls every sphere further into the ground: every world falls back to the plain step
    ws = _ConstantLambda([-0.05, 0.0, 0.0])
    plain, warm = _step_pair(m, solver, a, c, dt, ws)
    assert torch.equal(plain.body_q, warm.body_q)
    assert torch.equal(plain.body_qd, warm.body_qd)
    assert ws.fallback_count == m.world_count


def test_lifting_prediction_is_kept_and_reported():
    """lambda_n > 0 lifts every sphere out of the ground: kept in every world, and included in the
    contact's reported impulse."""
    m, pipe, solver, a, c, dt = _resting_spheres()
    ws = _ConstantLambda([1e-4, 0.0, 0.0])
    plain, warm = _step_pair(m, solver, a, c, dt, ws)
    assert ws.fallback_count == 0
    assert not torch.equal(plain.body_q, warm.body_q)
    # the warm start removed (part of) the 1 mm penetration before the plain iterations
    assert bool((warm.body_q[:, 2] >= plain.body_q[:, 2] - 1e-6).all())
    solved = ws._last[: m.world_count, 0]
    assert bool((solved >= 1e-4 * (1 - 1e-5)).all())


def test_features_and_targets_with_matching():
    """Features are finite, the previous-lambda columns follow match_index, targets are the solved impulses."""
    m, pipe, solver, a, c, dt = _settled(matching="latest")
    ws = WarmStart(None, iterations=None, record=True)
    solver.warm_start = ws
    b = m.state()
    for _ in range(3):
        solver.step(a, b, None, c, dt)
        a, b = b, a
        a.clear_forces()
        pipe.collide(a, c)
    solver.warm_start = None
    x, t = ws.samples()
    assert x.shape[1] == N_FEAT and t.shape[1] == N_OUT and x.shape[0] == t.shape[0] > 0
    assert bool(torch.isfinite(x).all()) and bool(torch.isfinite(t).all())
    assert float(t[:, 0].max()) > 0.0  # some contact pushed
    # second recorded substep: previous-lambda features gathered through the match index
    n0 = ws._records[0][1].shape[0]
    assert n0 > 0
    matched = ws._records[1][0][:, 0]  # contacts whose previous lambda was found through the match index
    assert float(matched.sum()) > 0.0
    prior = ws._records[1][0][:, N_IN + 2]
    assert bool((prior >= 0).all()) and float(prior.max()) > 0.0


def test_trained_network_gains_over_plain_solver():
    """The committed network (trained on plain 8-iteration rollouts of the uneven-worlds scene, seed 2)
    on an unseen scene (seed 1): with the same 2 iterations, the warm-started solver leaves about half
    the mean contact penetration of the plain one (plain 4 iterations: about the same as the warm start)."""
    import os

    from newton_custom_contact_b200.train_warmstart import make_scene, rollout

    path = os.path.join(os.path.dirname(__file__), "..", "newton_custom_contact_b200", "data", "warmstart_c2.npz")
    net = WarmStartNet.load(path, device=DEV)
    m, pipe = make_scene(1, 256, DEV)
    plain, _ = rollout(m, pipe, 2, 48, policy=None, warmup=48)
    ws = WarmStart(net, iterations=2)
    warm, _ = rollout(m, pipe, 2, 48, policy=ws, warmup=48)
    mean_plain = float(np.mean([p["mean"] for p in plain]))
    mean_warm = float(np.mean([p["mean"] for p in warm]))
    assert mean_warm < 0.75 * mean_plain, (mean_warm, mean_plain)
    assert ws.fallback_count < 0.5 * m.world_count * 96
