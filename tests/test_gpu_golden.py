"""The CUDA path against golden vectors produced by the reference's own code.

The fixtures (``tests/golden/*.npz``, written by ``tests/golden/make_golden.py``) hold the reference's
CollisionPipeline.collide (newton/_src/sim/collide.py:902-1124) and SolverXPBD.step
(newton/_src/solvers/xpbd/solver_xpbd.py:259-764) run through a CPU emulation of Warp on small C1 / C2 /
C3 scenes: the state before each of 16 substeps, the contacts of the first and the last substep, and
the reference's own spread under reordered float atomics.

* Parity build (``--fmad=false``): contacts bit for bit; every substep started from the reference's
  state bit for bit; a free-running 16-substep rollout bit for bit at every substep (joint scene:
  against the rollout that uses the library's own asin / acos).
* Product build (FMA contraction in the solver; contact generation is compiled unfused in both
  builds): contacts bit for bit; poses of every substep started from the reference's state within
  1e-5 relative / 1e-6 m absolute, or, where larger, four times the reference's own spread of that
  substep; velocities within the same bar carried through the velocity update -- XPBD derives a
  substep's velocities from its position change over dt (linear: dx / dt, angular: 2 dq / dt), so a
  pose difference at the bar b of a body is a velocity difference of b / dt (2 b / dt angular).
"""

import os
import sys

import numpy as np
import pytest
import torch

from newton_custom_contact_b200 import CollisionPipeline, SolverXPBD

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
GOLDEN = os.path.join(HERE, "golden")
SCENES = ("c2_small", "c2_small_landed", "c1", "c3_arm")
FIELDS = ("point0", "point1", "normal", "offset0", "offset1", "margin0", "margin1")
RTOL, ATOL = 1e-5, 1e-6


def _load(name):
    return dict(np.load(os.path.join(GOLDEN, f"{name}.npz")))


_MODELS = {}


def _model(name):
    if name not in _MODELS:
        if GOLDEN not in sys.path:
            sys.path.insert(0, GOLDEN)
        import make_golden

        _MODELS.update(make_golden.scenes(device="cuda"))
    return _MODELS[name]


def asin_suffix(fx):
    return "_library_asin" if "body_q_all_library_asin" in fx else ""


class Runner:
    """collide + one SolverXPBD.step of the library from a given state."""

    def __init__(self, name, fx):
        self.model, info = _model(name)
        self.pipe = CollisionPipeline(self.model)
        self.solver = SolverXPBD(self.model, iterations=int(fx["iterations"]))
        self.dt = float(fx["dt"])
        self.s0, self.s1 = self.model.state(), self.model.state()
        self.contacts = self.pipe.contacts()

    def substep(self, q, qd):
        self.s0.body_q.copy_(torch.from_numpy(np.ascontiguousarray(q)))
        self.s0.body_qd.copy_(torch.from_numpy(np.ascontiguousarray(qd)))
        self.s0.clear_forces()
        self.pipe.collide(self.s0, self.contacts)
        self.solver.step(self.s0, self.s1, None, self.contacts, self.dt)
        torch.cuda.synchronize()
        return self.s1.body_q.cpu().numpy(), self.s1.body_qd.cpu().numpy()

    def contacts_in_key_order(self):
        """Public contacts ordered by the reference's global key (shape0, shape1, sub key): ours are
        in key order within each world, and a shape pair belongs to one world, so a stable sort by
        the shape pair gives the global order."""
        c = self.contacts
        n = int(c.rigid_contact_count.item())
        out = {k: getattr(c, f"rigid_contact_{k}")[:n].cpu().numpy() for k in ("shape0", "shape1") + FIELDS}
        order = np.lexsort((out["shape1"], out["shape0"]))
        return {k: v[order] for k, v in out.items()}


def _bits(a):
    return np.ascontiguousarray(a, dtype=np.float32).view(np.uint32)


def _within(got, want, spread, atol=ATOL):
    tol = np.maximum(atol + RTOL * np.abs(want), 4.0 * float(spread))
    return bool(np.all(np.abs(got - want) <= tol))


def _velocity_within(got, want, q_want, spread, dt):
    """Velocities against the pose bar of each body carried through the velocity update."""
    pose_bar = ATOL + RTOL * np.abs(q_want).max(axis=1, keepdims=True)
    bar = np.concatenate([np.repeat(pose_bar, 3, axis=1), np.repeat(2.0 * pose_bar, 3, axis=1)], axis=1) / dt
    tol = np.maximum(bar, 4.0 * float(spread))
    return bool(np.all(np.abs(got - want) <= tol))


@pytest.mark.parametrize("name", SCENES)
def test_contacts_bit_exact_with_reference(cuda, name):
    fx = _load(name)
    run = Runner(name, fx)
    for k in (1, 16):
        run.substep(fx["body_q_all"][k - 1], fx["body_qd_all"][k - 1])
        got = run.contacts_in_key_order()
        assert len(got["shape0"]) == len(fx[f"contact_shape0_s{k}"]) > 0
        assert np.array_equal(got["shape0"], fx[f"contact_shape0_s{k}"])
        assert np.array_equal(got["shape1"], fx[f"contact_shape1_s{k}"])
        for f in FIELDS:
            assert np.array_equal(_bits(got[f]), _bits(fx[f"contact_{f}_s{k}"])), f"{f} of substep {k}"


@pytest.mark.parametrize("name", SCENES)
def test_substeps_bit_exact_with_reference(cuda, name):
    """Every substep from the reference's own state, and a free-running rollout, bit for bit."""
    fx = _load(name)
    sfx = asin_suffix(fx)
    run = Runner(name, fx)
    Q, QD = fx["body_q_all" + sfx], fx["body_qd_all" + sfx]
    for k in range(1, Q.shape[0]):
        q, qd = run.substep(Q[k - 1], QD[k - 1])
        assert np.array_equal(_bits(q), _bits(Q[k])), f"body_q of substep {k}"
        assert np.array_equal(_bits(qd), _bits(QD[k])), f"body_qd of substep {k}"
    q, qd = Q[0], QD[0]
    for k in range(1, Q.shape[0]):
        q, qd = run.substep(q, qd)
        assert np.array_equal(_bits(q), _bits(Q[k])), f"free-running body_q after {k} substeps"
        assert np.array_equal(_bits(qd), _bits(QD[k])), f"free-running body_qd after {k} substeps"


@pytest.mark.product_build
@pytest.mark.parametrize("name", SCENES)
def test_product_build_within_tolerance_of_reference(cuda, name):
    fx = _load(name)
    run = Runner(name, fx)
    for k in (1, 16):
        run.substep(fx["body_q_all"][k - 1], fx["body_qd_all"][k - 1])
        got = run.contacts_in_key_order()
        assert np.array_equal(got["shape0"], fx[f"contact_shape0_s{k}"])
        assert np.array_equal(got["shape1"], fx[f"contact_shape1_s{k}"])
        for f in FIELDS:
            assert np.array_equal(_bits(got[f]), _bits(fx[f"contact_{f}_s{k}"])), f"{f} of substep {k}"
    Q, QD = fx["body_q_all"], fx["body_qd_all"]
    for k in range(1, Q.shape[0]):
        q, qd = run.substep(Q[k - 1], QD[k - 1])
        assert _within(q, Q[k], fx["spread_q"][k]), f"body_q of substep {k}: {np.abs(q - Q[k]).max()}"
        assert _velocity_within(qd, QD[k], Q[k], fx["spread_qd"][k], float(fx["dt"])), \
            f"body_qd of substep {k}: {np.abs(qd - QD[k]).max()}"
