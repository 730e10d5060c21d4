"""The oracle against golden vectors produced by the reference's own code.

``tests/golden/*.npz`` were written by ``tests/golden/make_golden.py``, which runs the reference's
unmodified CollisionPipeline.collide (newton/_src/sim/collide.py:902-1124) and SolverXPBD.step
(newton/_src/solvers/xpbd/solver_xpbd.py:259-764) through a CPU emulation of the Warp kernel
language, with deterministic=True (contacts in key order before the solver).  Those fixtures pin the
oracle -- and through the bit-exact GPU tests, the CUDA kernels -- to the reference source rather
than to a restatement of it:

* contacts (shapes, body-frame points, offsets, normals, margins) of the first and the last of 16
  substeps match bit for bit;
* free-running rollouts of 16 substeps match bit for bit at every substep when the oracle sums
  per-body deltas in float in contact order, as the emulated reference does (joint scenes: against
  the rollout that uses the library's own asin / acos, the one function the two sides do not share);
* the CUDA kernels sum in that same order (bit-exact with the oracle's float mode), so the same
  holds for them; the fixtures' spread records how far the reference itself moves when its float
  atomics run in other orders, as they may on a GPU.
"""

import os

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
GOLDEN = os.path.join(HERE, "golden")
SCENES = ("c2_small", "c2_small_landed", "c1", "c3_arm")
FIELDS = ("point0", "point1", "normal", "offset0", "offset1", "margin0", "margin1")


def _scene(name):
    """The model a fixture was made from (the generator's scene list, rebuilt on the CPU)."""
    import sys

    if GOLDEN not in sys.path:
        sys.path.insert(0, GOLDEN)
    import make_golden

    model, info = make_golden.scenes()[name]
    return model, info


def _load(name):
    path = os.path.join(GOLDEN, f"{name}.npz")
    return dict(np.load(path))


def oracle_contacts(orc, model, layout, q):
    """Oracle contacts as a dict of arrays in the reference's deterministic key order."""
    segs = orc.collide(model, layout, q)
    tab = orc.contacts_table(model, layout, segs)
    keys = (tab[:, 1].astype(np.int64) << 43) | (tab[:, 2].astype(np.int64) << 23) | tab[:, 3].astype(np.int64)
    tab = tab[np.argsort(keys, kind="stable")]
    f32 = lambda a: np.ascontiguousarray(a, dtype=np.float32)  # noqa: E731
    return {"shape0": tab[:, 1].astype(np.int32), "shape1": tab[:, 2].astype(np.int32),
            "point0": f32(tab[:, 4:7]), "point1": f32(tab[:, 7:10]), "normal": f32(tab[:, 10:13]),
            "offset0": f32(tab[:, 13:16]), "offset1": f32(tab[:, 16:19]), "margin0": f32(tab[:, 19]),
            "margin1": f32(tab[:, 20])}


def rollout(orc, model, layout, fx, acc_mode, suffix=""):
    """Oracle rollout of the fixture's substeps from its first state; returns [(q, qd)] per substep."""
    from newton_custom_contact_b200 import SolverXPBD

    p = SolverXPBD(model, iterations=int(fx["iterations"])).params()
    dt = float(fx["dt"])
    q, qd = fx["body_q_all" + suffix][0], fx["body_qd_all" + suffix][0]
    f = np.zeros((model.body_count, 6), np.float32)
    out = []
    for _ in range(fx["body_q_all" + suffix].shape[0] - 1):
        segs = orc.collide(model, layout, q)
        q, qd, _ = orc.step(model, layout, p, q, qd, f, segs, dt, acc_mode=acc_mode,
                            joint_target_pos=model.host("joint_target_pos"),
                            joint_target_vel=model.host("joint_target_vel"))
        out.append((q.copy(), qd.copy()))
    return out


def one_substep(orc, model, layout, fx, k, acc_mode, suffix=""):
    """Oracle substep k started from the reference's state k - 1."""
    from newton_custom_contact_b200 import SolverXPBD

    p = SolverXPBD(model, iterations=int(fx["iterations"])).params()
    q, qd = fx["body_q_all" + suffix][k - 1], fx["body_qd_all" + suffix][k - 1]
    segs = orc.collide(model, layout, q)
    f = np.zeros((model.body_count, 6), np.float32)
    q, qd, _ = orc.step(model, layout, p, q, qd, f, segs, float(fx["dt"]), acc_mode=acc_mode,
                        joint_target_pos=model.host("joint_target_pos"),
                        joint_target_vel=model.host("joint_target_vel"))
    return q, qd


RTOL, ATOL = 1e-5, 1e-6


def within_reference(got, want, spread):
    """Element-wise |got - want| <= max(1e-6 + 1e-5 |want|, 4 x spread): the FP32 tolerance of the
    comparison (1e-5 relative, 1e-6 absolute), widened to four times the reference's own spread of
    that substep under reordered contacts where that is larger."""
    tol = np.maximum(ATOL + RTOL * np.abs(want), 4.0 * float(spread))
    return bool(np.all(np.abs(got - want) <= tol))


def asin_suffix(fx):
    """Fixture rollouts of joint scenes to compare bit for bit: the one with the library's asin/acos."""
    return "_library_asin" if "body_q_all_library_asin" in fx else ""


@pytest.fixture(scope="module")
def layouts():
    from newton_custom_contact_b200.collide import PairLayout

    out = {}
    for name in SCENES:
        model, info = _scene(name)
        out[name] = (model, PairLayout(model, model.host("shape_contact_pairs")))
    return out


@pytest.mark.parametrize("name", SCENES)
def test_fixture_is_the_generators_scene(name, layouts):
    fx = _load(name)
    model, _ = layouts[name]
    if name != "c2_small_landed":  # the landed fixture starts after 24 frames of the same scene
        assert np.array_equal(fx["body_q_all"][0], model.host("body_q").astype(np.float32))
    assert fx["body_q_all"].shape == (17, model.body_count, 7)


@pytest.mark.parametrize("name", SCENES)
@pytest.mark.parametrize("k", (1, 16))
def test_oracle_contacts_bit_exact_with_reference(orc, layouts, name, k):
    fx = _load(name)
    model, lay = layouts[name]
    got = oracle_contacts(orc, model, lay, fx["body_q_all"][k - 1])
    assert len(got["shape0"]) == len(fx[f"contact_shape0_s{k}"]) > 0
    assert np.array_equal(got["shape0"], fx[f"contact_shape0_s{k}"])
    assert np.array_equal(got["shape1"], fx[f"contact_shape1_s{k}"])
    for f in FIELDS:
        a, b = got[f], fx[f"contact_{f}_s{k}"].astype(np.float32)
        assert np.array_equal(a.view(np.uint32), b.view(np.uint32)), f


@pytest.mark.parametrize("name", SCENES)
def test_oracle_float_sums_bit_exact_with_reference(orc, layouts, name):
    fx = _load(name)
    model, lay = layouts[name]
    sfx = asin_suffix(fx)
    got = rollout(orc, model, lay, fx, orc.ACC_FLOAT, sfx)
    for k, (q, qd) in enumerate(got, start=1):
        rq, rqd = fx["body_q_all" + sfx][k], fx["body_qd_all" + sfx][k]
        assert np.array_equal(q.view(np.uint32), rq.view(np.uint32)), f"body_q after {k} substeps"
        assert np.array_equal(qd.view(np.uint32), rqd.view(np.uint32)), f"body_qd after {k} substeps"


def test_fixed_point_sums_leave_the_reference(orc, layouts):
    """Why the kernels sum in order instead of in exact fixed point: one substep of the joint scene
    with 2^-32 fixed-point sums lands beyond 1e-5 relative of the reference's velocities, further than
    any of the reference's own reorderings (bodies with one or two contributions sum order-free in
    float, and rounding each term to the fixed-point grid changes them)."""
    fx = _load("c3_arm")
    model, lay = layouts["c3_arm"]
    sfx = asin_suffix(fx)
    worst = 0.0
    for k in range(1, fx["body_q_all"].shape[0]):
        _, qd = one_substep(orc, model, lay, fx, k, orc.ACC_FIXED, sfx)
        ref = fx["body_qd_all" + sfx][k]
        excess = np.abs(qd - ref) - np.maximum(ATOL + RTOL * np.abs(ref), 4.0 * float(fx["spread_qd" + sfx][k]))
        worst = max(worst, float(excess.max()))
    assert worst > 0.0


def test_platform_asin_and_library_asin_rollouts_agree():
    """On the joint scene the only source of difference between the two reference rollouts is the
    asin / acos implementation (the platform's or the library's fp32 functions): over all 16 substeps
    they agree to a few fp32 ulps of the state."""
    fx = _load("c3_arm")
    for k in range(fx["body_q_all"].shape[0]):
        assert np.allclose(fx["body_q_all"][k], fx["body_q_all_library_asin"][k], rtol=1e-6, atol=1e-6)
        assert np.allclose(fx["body_qd_all"][k], fx["body_qd_all_library_asin"][k], rtol=1e-5, atol=1e-5)
