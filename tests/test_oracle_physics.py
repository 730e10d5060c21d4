"""Physical known-answer tests of the CPU oracle's solver extras.

Scenes and assertions are those of the reference's own tests:
  * restitution: newton/tests/test_physics_validation.py:644-723 (sphere dropped
    1 m, rebound height e^2 * h within 1 %, ratio of the two within 1 %), with
    SolverXPBD(iterations=10, angular_damping=0, enable_restitution=True)
    (:1662-1671).  The reference uses a Y-up builder; this one is Z-up, so the
    same drop runs along Z.
  * contact forces: newton/tests/test_solver_xpbd.py:469-656 (static
    equilibrium of a small sphere, a heavy sphere, a box and a three-cube
    pyramid; iterations=32, rigid_contact_con_weighting=True) and :658-726
    (zero force in free fall and for a pair inside the gap).
  * no bounce: newton/tests/test_shapes_no_bounce.py:21-226 (a grid of shapes
    dropped on the ground never rises above max(2 m, its start) in 200 frames),
    with the sphere / box / capsule shapes of the grid.
  * shapes at rest on a plane, a two-box drop and boxes / spheres / a capsule held on
    a ramp by an end wall: newton/tests/test_rigid_contact.py:28-227, 766-831 and
    230-503 with SolverXPBD(iterations=2) (:841).
  * head-on collisions of sphere / box / capsule pairs:
    newton/tests/test_collision_pipeline.py:46-262.
  * static and dynamic friction, free fall, projectile motion and momentum
    conservation: newton/tests/test_physics_validation.py:505-641, :21-80,
    :256-318, :413-498 with the XPBD settings those tests register; the
    revolute pendulum's period (:83-158, 20 iterations, dt 3e-4) and joint
    actuation by joint forces (:321-409).
The CUDA path is compared with the oracle bit for bit in test_gpu_solver_extras.py.
"""

import math

import numpy as np
import pytest

from newton_custom_contact_b200 import ModelBuilder, SolverXPBD
from newton_custom_contact_b200.collide import PairLayout


def _sim(orc, model, solver, dt, steps, on_step=None, want_impulse=False):
    lay = PairLayout(model, model.host("shape_contact_pairs"))
    p = solver.params()
    q = model.host("body_q").copy()
    qd = model.host("body_qd").copy()
    f = np.zeros((model.body_count, 6), np.float32)
    for i in range(steps):
        segs = orc.collide(model, lay, q)
        out = orc.step(model, lay, p, q, qd, f, segs, dt, want_impulse=want_impulse)
        q, qd = out[0], out[1]
        if on_step is not None:
            on_step(i, q, qd, segs, lay, out[3] if want_impulse else None)
    return q, qd


def _forces_by_contact(orc, model, lay, segs, imp, dt):
    """[(shape0, shape1, force6)] for every live contact (impulse / dt, kernels.py:2363-2393)."""
    tab = orc.contacts_table(model, lay, segs)
    cs = 5 * lay.world_pair_start.astype(np.int64)
    slots = np.concatenate([np.arange(cs[w], cs[w] + int(segs.world_count[w])) for w in range(model.world_count)])
    return tab[:, 1].astype(int), tab[:, 2].astype(int), imp[slots] * np.float32(1.0 / dt)


def test_oracle_restitution_bounce(orc):
    g, h_drop, radius = -10.0, 1.0, 0.05
    rebound = {}
    for e in (0.5, 0.8):
        cfg = ModelBuilder.ShapeConfig()
        cfg.mu = 0.0
        cfg.restitution = e
        cfg.margin = 0.001
        cfg.gap = 0.0
        b = ModelBuilder(gravity=g)
        b.add_ground_plane(cfg=cfg)
        body = b.add_body(xform=((0.0, 0.0, radius + h_drop), (0.0, 0.0, 0.0, 1.0)))
        b.add_shape_sphere(body, radius=radius, cfg=cfg)
        model = b.finalize(device="cpu")
        solver = SolverXPBD(model, iterations=10, angular_damping=0.0, enable_restitution=True)
        sim_dt = 1e-3
        steps = int(3.0 * np.sqrt(2.0 * h_drop / abs(g)) / sim_dt)
        z = []
        _sim(orc, model, solver, sim_dt, steps, on_step=lambda i, q, qd, s, l, im: z.append(float(q[0, 2])))
        z = np.array(z)
        assert z.min() > -0.01
        impact = next(i for i in range(1, len(z) - 1) if z[i] < z[i - 1] and z[i] <= z[i + 1])
        h = z[impact:].max() - radius
        assert abs(h - e * e * h_drop) <= 0.01 * e * e * h_drop, (e, h)
        rebound[e] = h
    ratio = rebound[0.8] / rebound[0.5]
    assert abs(ratio - 2.56) <= 0.01 * 2.56


def test_oracle_contact_force_static_equilibrium(orc):
    gravity = 9.81
    sr, sd = 0.25, 1000.0
    hr, hd = 0.5, 2000.0
    bh, cube_h = 0.5, 0.5
    sphere_m = sd * 4.0 / 3.0 * np.pi * sr ** 3
    heavy_m = hd * 4.0 / 3.0 * np.pi * hr ** 3
    box_m = 1000.0 * (2 * bh) ** 3
    cube_mg = 1000.0 * (2 * cube_h) ** 3 * gravity
    ident = (0.0, 0.0, 0.0, 1.0)
    b = ModelBuilder()
    b.add_ground_plane()
    b.default_shape_cfg.density = sd
    sphere = b.add_body(xform=((0.0, 0.0, sr), ident))
    b.add_shape_sphere(sphere, radius=sr)
    b.default_shape_cfg.density = hd
    heavy = b.add_body(xform=((10.0, 0.0, hr), ident))
    b.add_shape_sphere(heavy, radius=hr)
    b.default_shape_cfg.density = 1000.0
    box = b.add_body(xform=((20.0, 0.0, bh), ident))
    b.add_shape_box(box, hx=bh, hy=bh, hz=bh)
    left = b.add_body(xform=((30.0 - cube_h, 0.0, cube_h), ident))
    b.add_shape_box(left, hx=cube_h, hy=cube_h, hz=cube_h)
    right = b.add_body(xform=((30.0 + cube_h, 0.0, cube_h), ident))
    b.add_shape_box(right, hx=cube_h, hy=cube_h, hz=cube_h)
    top = b.add_body(xform=((30.0, 0.0, 3.0 * cube_h), ident))
    b.add_shape_box(top, hx=cube_h, hy=cube_h, hz=cube_h)
    model = b.finalize(device="cpu")
    solver = SolverXPBD(model, iterations=32, rigid_contact_con_weighting=True)
    shape_body = model.host("shape_body")
    sub_dt = 1.0 / 60.0 / 8
    settle, avg = 200, 60
    acc = {"sphere": np.zeros(3), "heavy": np.zeros(3), "box": np.zeros(3), "left": 0.0, "right": 0.0,
           "box_contacts": []}

    def on_step(i, q, qd, segs, lay, imp):
        if i < settle * 8 or (i + 1) % 8:
            return  # update_contacts after the last substep of every averaged frame
        s0, s1, f = _forces_by_contact(orc, model, lay, segs, imp, sub_dt)
        nbox = 0
        for a, c, fc in zip(s0, s1, f):
            if a == 0:
                other, fv = c, fc[:3]
            elif c == 0:
                other, fv = a, -fc[:3]
            else:
                continue
            ob = shape_body[other]
            if ob == sphere:
                acc["sphere"] += fv
            elif ob == heavy:
                acc["heavy"] += fv
            elif ob == box:
                acc["box"] += fv
                nbox += 1
            elif ob == left:
                acc["left"] += -fv[2]
            elif ob == right:
                acc["right"] += -fv[2]
        acc["box_contacts"].append(nbox)

    _sim(orc, model, solver, sub_dt, (settle + avg) * 8, on_step=on_step, want_impulse=True)
    assert min(acc["box_contacts"]) > 1
    sph, hv, bx = acc["sphere"] / avg, acc["heavy"] / avg, acc["box"] / avg
    np.testing.assert_allclose(sph[2], -sphere_m * gravity, rtol=0.05)
    np.testing.assert_allclose(sph[:2], 0.0, atol=0.5)
    np.testing.assert_allclose(hv[2], -heavy_m * gravity, rtol=0.05)
    np.testing.assert_allclose(hv[:2], 0.0, atol=0.5)
    np.testing.assert_allclose(bx[2], -box_m * gravity, rtol=0.10)
    np.testing.assert_allclose(bx[:2], 0.0, atol=1.0)
    np.testing.assert_allclose(acc["left"] / avg, 1.5 * cube_mg, rtol=0.15)
    np.testing.assert_allclose(acc["right"] / avg, 1.5 * cube_mg, rtol=0.15)


def test_oracle_contact_force_zero_free_fall_and_inside_gap(orc):
    ident = (0.0, 0.0, 0.0, 1.0)
    # free fall, no ground
    b = ModelBuilder()
    body = b.add_body(xform=((0.0, 0.0, 5.0), ident))
    b.add_shape_sphere(body, radius=0.25)
    model = b.finalize(device="cpu")
    seen = []
    _sim(orc, model, SolverXPBD(model, iterations=2), 1.0 / 60.0, 1, want_impulse=True,
         on_step=lambda i, q, qd, s, l, imp: seen.append(np.abs(imp).max()))
    assert seen[0] == 0.0
    # pair inside a 1 m gap, not touching, no gravity
    b = ModelBuilder(gravity=0.0)
    b.default_shape_cfg.gap = 1.0
    b.add_ground_plane()
    body = b.add_body(xform=((0.0, 0.0, 0.25 + 0.5), ident))
    b.add_shape_sphere(body, radius=0.25)
    model = b.finalize(device="cpu")
    out = {}

    def grab(i, q, qd, segs, lay, imp):
        out["n"] = int(segs.world_count.sum())
        out["f"] = _forces_by_contact(orc, model, lay, segs, imp, 1.0 / 60.0)[2]

    _sim(orc, model, SolverXPBD(model, iterations=2), 1.0 / 60.0, 1, want_impulse=True, on_step=grab)
    assert out["n"] > 0
    np.testing.assert_allclose(out["f"][:, :3], 0.0, atol=1e-6)


def test_shared_asin_acos_accuracy(orc):
    """The asin / acos used by the joint solve on both sides: within 2 ulp of float64 on [-1, 1]."""
    lib = orc.load()
    xs = np.concatenate([np.linspace(-1.0, 1.0, 20001, dtype=np.float32),
                         np.float32([0.0, -0.0, 1e-30, 1e-10, 1e-5, 0.4999999, 0.5, 0.5000001, 0.9999999])])
    for fn, ref in ((lib.orc_asin, np.arcsin), (lib.orc_acos, np.arccos)):
        got = np.array([fn(float(x)) for x in xs], np.float32)
        exact = ref(xs.astype(np.float64))
        ulp = np.spacing(np.abs(exact).astype(np.float32)).astype(np.float64)
        assert (np.abs(got.astype(np.float64) - exact) / ulp).max() <= 2.0
    assert lib.orc_asin(1.0) == np.float32(np.pi / 2) and lib.orc_acos(1.0) == 0.0


# ---- body_parent_f: newton/tests/test_solver_xpbd.py:752-1016 (single-body pendulums to world /
# kinematic parent with revolute, ball and fixed joints; a two-link chain; free body).  Bodies start
# at the pose the reference's eval_fk gives them (child 1 m below the anchor).

def _pendulum(kind, parent_kinematic, gravity=9.81):
    b = ModelBuilder(gravity=-gravity)
    b.request_state_attributes("body_parent_f")
    ident = (0.0, 0.0, 0.0, 1.0)
    parent = -1
    if parent_kinematic:
        parent = b.add_body(xform=((0.0, 0.0, 0.0), ident), is_kinematic=True)
        b.add_shape_box(parent, hx=0.05, hy=0.05, hz=0.05)
    child = b.add_link(xform=((0.0, 0.0, -1.0), ident))
    b.add_shape_box(child, hx=0.1, hy=0.1, hz=0.1)
    pxf, cxf = ((0.0, 0.0, 0.0), ident), ((0.0, 0.0, 1.0), ident)
    if kind == "revolute":
        b.add_joint_revolute(parent, child, parent_xform=pxf, child_xform=cxf, axis=(0.0, 1.0, 0.0))
    elif kind == "ball":
        b.add_joint_ball(parent, child, parent_xform=pxf, child_xform=cxf)
    else:
        b.add_joint_fixed(parent, child, parent_xform=pxf, child_xform=cxf)
    return b.finalize(device="cpu"), child


def _parent_f_average(orc, model, iterations, settle, avg, dt=1.0 / 60.0 / 8):
    lay = PairLayout(model, model.host("shape_contact_pairs"))
    p = SolverXPBD(model, iterations=iterations).params()
    q, qd = model.host("body_q").copy(), model.host("body_qd").copy()
    f = np.zeros((model.body_count, 6), np.float32)
    jt = model.host("joint_target_pos")
    acc = np.zeros((model.body_count, 6))
    for frame in range(settle + avg):
        for _ in range(8):
            q, qd, _, pf = orc.step(model, lay, p, q, qd, f, None, dt, joint_target_pos=jt,
                                    joint_target_vel=np.zeros_like(jt), joint_f=np.zeros_like(jt),
                                    want_parent_f=True)
        if frame >= settle:
            acc += pf
    return acc / avg


@pytest.mark.parametrize("kind", ["revolute", "ball", "fixed"])
@pytest.mark.parametrize("parent_kinematic", [False, True])
def test_oracle_parent_force_single_pendulum(orc, kind, parent_kinematic):
    model, child = _pendulum(kind, parent_kinematic)
    pf = _parent_f_average(orc, model, iterations=8, settle=60, avg=30)[child]
    weight = float(model.host("body_mass")[child]) * 9.81
    np.testing.assert_allclose(pf[2], weight, rtol=0.01)
    np.testing.assert_allclose(pf[:2], 0.0, atol=0.1)
    np.testing.assert_allclose(pf[3:6], 0.0, atol=0.1)


def test_oracle_parent_force_chain_weight_propagation(orc):
    b = ModelBuilder(gravity=-9.81)
    b.request_state_attributes("body_parent_f")
    ident = (0.0, 0.0, 0.0, 1.0)
    l0 = b.add_link(xform=((0.0, 0.0, -1.0), ident))
    b.add_shape_box(l0, hx=0.1, hy=0.1, hz=0.1)
    b.add_joint_revolute(-1, l0, parent_xform=((0.0, 0.0, 0.0), ident), child_xform=((0.0, 0.0, 1.0), ident),
                         axis=(0.0, 1.0, 0.0))
    l1 = b.add_link(xform=((0.0, 0.0, -3.0), ident))
    b.add_shape_box(l1, hx=0.1, hy=0.1, hz=0.1)
    b.add_joint_revolute(l0, l1, parent_xform=((0.0, 0.0, -1.0), ident), child_xform=((0.0, 0.0, 1.0), ident),
                         axis=(0.0, 1.0, 0.0))
    model = b.finalize(device="cpu")
    pf = _parent_f_average(orc, model, iterations=32, settle=120, avg=60)
    m = model.host("body_mass")
    np.testing.assert_allclose(pf[0, 2], float(m[0] + m[1]) * 9.81, rtol=0.10)
    np.testing.assert_allclose(pf[1, 2], float(m[1]) * 9.81, rtol=0.10)


def test_oracle_parent_force_zero_for_free_body(orc):
    b = ModelBuilder()
    b.request_state_attributes("body_parent_f")
    body = b.add_body(xform=((0.0, 0.0, 0.0), (0.0, 0.0, 0.0, 1.0)))
    b.add_shape_sphere(body, radius=0.1)
    model = b.finalize(device="cpu")
    pf = _parent_f_average(orc, model, iterations=2, settle=0, avg=1)
    np.testing.assert_allclose(pf[0], 0.0, atol=1e-6)


def test_oracle_shapes_never_exceed_initial_z(orc):
    """newton/tests/test_shapes_no_bounce.py:186-226 on the oracle: spheres, boxes and
    capsules dropped on a plane never rise above max(2 m, their initial z) over 200 frames
    at 100 fps with 10 substeps, XPBD with 2 iterations, relaxation 0.8, no angular
    damping; by the last frame every body has landed below its start."""
    from newton_custom_contact_b200 import scenes

    model, z0 = scenes.scene_falling_shapes(1, device="cpu")
    solver = SolverXPBD(model, iterations=2, rigid_contact_relaxation=0.8, angular_damping=0.0)
    limit = np.maximum(np.float32(2.0), z0)
    frames = {"n": 0, "contacts": 0}

    def check(i, q, qd, segs, lay, imp):
        frames["contacts"] = max(frames["contacts"], int(np.sum(segs.world_count)))
        if (i + 1) % 10 == 0:
            frames["n"] += 1
            assert np.all(q[:, 2] <= limit), f"frame {frames['n']}: max excess {float((q[:, 2] - limit).max()):.4f} m"

    q, _ = _sim(orc, model, solver, 1.0 / 100.0 / 10, 2000, on_step=check)
    assert frames["n"] == 200 and np.all(np.isfinite(q))
    assert frames["contacts"] >= 16 and np.all(q[:, 2] < z0)


def _frames(orc, model, solver, frame_dt, substeps, frames, on_frame=None):
    """`frames` frames of `substeps` substeps (collide + step each) on the oracle."""
    lay = PairLayout(model, model.host("shape_contact_pairs"))
    p = solver.params()
    q = model.host("body_q").copy()
    qd = model.host("body_qd").copy()
    f = np.zeros((model.body_count, 6), np.float32)
    dt = frame_dt / substeps
    for k in range(frames):
        for _ in range(substeps):
            segs = orc.collide(model, lay, q)
            q, qd = orc.step(model, lay, p, q, qd, f, segs, dt)[:2]
        if on_frame is not None:
            on_frame(k, q, qd)
    return q, qd


def test_oracle_shapes_on_plane(orc):
    """newton/tests/test_rigid_contact.py:28-227 with SolverXPBD(iterations=2) (:841):
    spheres (r 0.1 s), Y-lying capsules (r 0.1 s, half height 0.3 s) and boxes
    (0.2 s, 0.25 s, 0.3 s) for s in (0.5, 1) dropped from 0.5 m come to rest on the
    plane after 120 frames of 30 substeps at 60 fps: |v|, |w| < 0.2, positions within
    0.25 of resting on the plane, orientations within 0.1 of identity.  The reference's
    cylinder and mesh bodies are left out (shapes this solver does not collide)."""
    from newton_custom_contact_b200.builder import quat_from_axis_angle

    b = ModelBuilder()
    expected = []
    for i, s in enumerate((0.5, 1.0)):
        y = i * 1.5
        body = b.add_body(xform=[0.0, y, 0.5, 0.0, 0.0, 0.0, 1.0])
        b.add_shape_sphere(body, radius=0.1 * s)
        expected.append((0.0, y, 0.1 * s))
        body = b.add_body(xform=[2.0, y, 0.5, 0.0, 0.0, 0.0, 1.0])
        z_to_y = quat_from_axis_angle((1.0, 0.0, 0.0), -0.5 * np.pi)
        b.add_shape_capsule(body, xform=np.concatenate([[0.0, 0.0, 0.0], z_to_y]), radius=0.1 * s,
                            half_height=0.3 * s)
        expected.append((2.0, y, 0.1 * s))
        body = b.add_body(xform=[4.0, y, 0.5, 0.0, 0.0, 0.0, 1.0])
        b.add_shape_box(body, hx=0.2 * s, hy=0.25 * s, hz=0.3 * s)
        expected.append((4.0, y, 0.3 * s))
    b.add_ground_plane()
    model = b.finalize(device="cpu")
    solver = SolverXPBD(model, iterations=2)
    q, qd = _frames(orc, model, solver, 1.0 / 60.0, 30, 120)
    assert np.all(np.isfinite(q)) and np.all(np.isfinite(qd))
    assert np.abs(qd[:, :3]).max() < 0.2 and np.abs(qd[:, 3:]).max() < 0.2
    assert np.abs(q[:, :3] - np.asarray(expected)).max() < 0.25
    assert np.abs(q[:, 3:] - np.array([0.0, 0.0, 0.0, 1.0])).max() < 0.1


def test_oracle_box_drop(orc):
    """newton/tests/test_rigid_contact.py:766-831 with SolverXPBD(iterations=2): a box
    (half 0.5) resting 0.1 above the plane and a second one tilted 0.5 rad about x
    dropped from 2.1 m onto it; over 60 frames of 8 substeps the vertical speed never
    exceeds free fall from the drop height, and both end near the origin, above the
    ground and nearly at rest."""
    from newton_custom_contact_b200.builder import quat_from_axis_angle

    h = 0.5
    b = ModelBuilder()
    b.add_ground_plane()
    body = b.add_body(xform=[0.0, 0.0, h * 1.2, 0.0, 0.0, 0.0, 1.0])
    b.add_shape_box(body, hx=h, hy=h, hz=h)
    body = b.add_body(xform=np.concatenate([[0.0, 0.0, h * 4.2], quat_from_axis_angle((1.0, 0.0, 0.0), 0.5)]))
    b.add_shape_box(body, hx=h, hy=h, hz=h)
    model = b.finalize(device="cpu")
    solver = SolverXPBD(model, iterations=2)
    v_max = np.sqrt(2.0 * 9.81 * h * 3.2)
    seen = {"v": 0.0}

    def track(k, q, qd):
        seen["v"] = max(seen["v"], float(np.abs(qd[:, 2]).max()))

    q, qd = _frames(orc, model, solver, 1.0 / 60.0, 8, 60, on_frame=track)
    assert seen["v"] < v_max
    assert np.all(np.abs(q[:, 0]) < 1.0) and np.all(np.abs(q[:, 1]) < 1.0)
    assert np.all(q[:, 2] > 0.5 * h)
    assert np.all(np.linalg.norm(qd[:, :3], axis=1) < 1.0)


# ---- friction: newton/tests/test_physics_validation.py:505-563 (static) and :571-641
# (dynamic), SolverXPBD(iterations=10, angular_damping=0) (:1619-1622).  The reference's
# builder is Y-up; this one is Z-up, so the box rests along Z and slides along X.

def _friction_loop(orc, model, solver, dt, steps, force_fn=None, qd0=None):
    lay = PairLayout(model, model.host("shape_contact_pairs"))
    p = solver.params()
    q = model.host("body_q").copy()
    qd = model.host("body_qd").copy() if qd0 is None else np.asarray(qd0, np.float32).copy()
    zero = np.zeros((model.body_count, 6), np.float32)
    for i in range(steps):
        f = zero if force_fn is None else force_fn(i)
        segs = orc.collide(model, lay, q)
        q, qd = orc.step(model, lay, p, q, qd, f, segs, dt)[:2]
    return q, qd


def _box_on_ground(mu, boxes_x):
    cfg = ModelBuilder.ShapeConfig(mu=mu, gap=0.1)
    b = ModelBuilder(up_axis="Z", gravity=-10.0)
    b.add_ground_plane(cfg=cfg)
    h = 0.25
    for y in boxes_x:
        body = b.add_body(xform=[0.0, y, h + 0.001, 0.0, 0.0, 0.0, 1.0])
        b.add_shape_box(body, hx=h, hy=h, hz=h, cfg=cfg)
    return b.finalize(device="cpu"), h


def test_oracle_static_friction(orc):
    """A push of 0.3 mu m g leaves the box in place; 2 mu m g slides it (after 20 settling steps)."""
    mu = 0.5
    model, h = _box_on_ground(mu, [0.0, 5.0])
    mass = 1000.0 * (2 * h) ** 3
    push = np.zeros((2, 6), np.float32)
    push[0, 0] = 0.3 * mu * mass * 10.0
    push[1, 0] = 2.0 * mu * mass * 10.0
    zero = np.zeros_like(push)
    solver = SolverXPBD(model, iterations=10, angular_damping=0.0)
    q, _ = _friction_loop(orc, model, solver, 1e-3, 200, force_fn=lambda i: push if i > 20 else zero)
    assert abs(q[0, 0]) < 0.01 and q[0, 2] == pytest.approx(h, abs=0.01)
    assert q[1, 0] > 0.05 and q[1, 2] == pytest.approx(h, abs=0.01)


def test_oracle_dynamic_friction(orc):
    """A box sliding at 2 m/s stops after v0^2 / (2 mu g) = 0.5 m (within 1 %)."""
    mu, v0, g = 0.4, 2.0, 10.0
    model, h = _box_on_ground(mu, [0.0])
    qd0 = model.host("body_qd").copy()
    qd0[0, 0] = v0
    solver = SolverXPBD(model, iterations=10, angular_damping=0.0)
    t_stop = v0 / (mu * g)
    q, qd = _friction_loop(orc, model, solver, 1e-3, int(1.5 * t_stop / 1e-3), qd0=qd0)
    d_stop = v0 ** 2 / (2.0 * mu * g)
    assert q[0, 0] == pytest.approx(d_stop, abs=0.01 * d_stop)
    assert abs(qd[0, 0]) < 0.01 and q[0, 2] == pytest.approx(h, abs=0.01)


# ---- integration without contacts: newton/tests/test_physics_validation.py free fall
# :21-80, projectile :256-318, momentum conservation :413-498, with
# SolverXPBD(angular_damping=0) (:1509-1512).  Z-up here (the reference is Y-up).

def _free_loop(orc, model, dt, steps, qd0=None, on_step=None):
    solver = SolverXPBD(model, angular_damping=0.0)
    lay = PairLayout(model, model.host("shape_contact_pairs"))
    p = solver.params()
    q = model.host("body_q").copy()
    qd = model.host("body_qd").copy() if qd0 is None else np.asarray(qd0, np.float32).copy()
    f = np.zeros((model.body_count, 6), np.float32)
    for i in range(1, steps + 1):
        q, qd = orc.step(model, lay, p, q, qd, f, None, dt)[:2]
        if on_step is not None:
            on_step(i, q, qd)
    return q, qd


def _tolerances(g, dt, t):
    return max(2.0 * 0.5 * abs(g) * dt * t, 1e-3), max(abs(g) * dt, 1e-3)


def test_oracle_free_fall(orc):
    g, h0, dt = -10.0, 5.0, 1e-3
    b = ModelBuilder(up_axis="Z", gravity=g)
    b.add_shape_sphere(b.add_body(xform=[0.0, 0.0, h0, 0.0, 0.0, 0.0, 1.0]), radius=0.1)
    model = b.finalize(device="cpu")

    def check(i, q, qd):
        if i % 100 == 0:
            t = i * dt
            pos_tol, vel_tol = _tolerances(g, dt, t)
            assert q[0, 2] == pytest.approx(h0 + 0.5 * g * t * t, abs=pos_tol)
            assert qd[0, 2] == pytest.approx(g * t, abs=vel_tol)
            assert abs(q[0, 0]) < 1e-4 and abs(q[0, 1]) < 1e-4

    _free_loop(orc, model, dt, 500, on_step=check)


def test_oracle_projectile(orc):
    g, dt = -10.0, 1e-3
    p0, v0 = np.array([0.0, 0.0, 10.0]), np.array([5.0, 0.0, 10.0])
    b = ModelBuilder(up_axis="Z", gravity=g)
    b.add_shape_sphere(b.add_body(xform=list(p0) + [0.0, 0.0, 0.0, 1.0]), radius=0.1)
    model = b.finalize(device="cpu")
    qd0 = np.zeros((1, 6), np.float32)
    qd0[0, :3] = v0

    def check(i, q, qd):
        if i in (10, 20, 30, 50, 70, 100):
            t = i * dt
            pos_tol, vel_tol = _tolerances(g, dt, t)
            want_p = p0 + v0 * t + np.array([0.0, 0.0, 0.5 * g * t * t])
            want_v = v0 + np.array([0.0, 0.0, g * t])
            assert np.all(np.abs(q[0, :3] - want_p) <= pos_tol)
            assert np.all(np.abs(qd[0, :3] - want_v) <= vel_tol)

    _free_loop(orc, model, dt, 100, qd0=qd0, on_step=check)


def _rot(qxyzw):
    x, y, z, w = (float(v) for v in qxyzw)
    return np.array([[1 - 2 * (y * y + z * z), 2 * (x * y - z * w), 2 * (x * z + y * w)],
                     [2 * (x * y + z * w), 1 - 2 * (x * x + z * z), 2 * (y * z - x * w)],
                     [2 * (x * z - y * w), 2 * (y * z + x * w), 1 - 2 * (x * x + y * y)]])


def test_oracle_momentum_conservation(orc):
    """Four separated free boxes without gravity: linear and angular momentum drift below
    5e-4 (relative) over 1000 steps, and the bodies move."""
    pos = [(0.0, 0.0, 0.0), (100.0, 0.0, 0.0), (0.0, 100.0, 0.0), (0.0, 0.0, 100.0)]
    vel = [(1.0, 0.0, 0.0, 0.0, 0.0, 0.5), (0.0, -1.0, 0.0, 0.3, 0.0, 0.0), (0.0, 0.0, 1.5, 0.0, -0.2, 0.0),
           (-0.5, 0.5, -0.5, 0.0, 0.0, -0.3)]
    b = ModelBuilder(up_axis="Z", gravity=0.0)
    for p in pos:
        b.add_shape_box(b.add_body(xform=list(p) + [0.0, 0.0, 0.0, 1.0]), hx=0.5, hy=0.5, hz=0.5)
    model = b.finalize(device="cpu")
    m = model.host("body_mass")
    inertia = model.host("body_inertia").reshape(-1, 3, 3)

    def momenta(q, qd):
        p_tot, l_tot = np.zeros(3), np.zeros(3)
        for i in range(4):
            p_tot += m[i] * qd[i, :3]
            l_tot += np.cross(q[i, :3], m[i] * qd[i, :3])
            r = _rot(q[i, 3:7])
            l_tot += r @ inertia[i] @ r.T @ qd[i, 3:6]
        return p_tot, l_tot

    qd0 = np.asarray(vel, np.float32)
    q0 = model.host("body_q").copy()
    p_a, l_a = momenta(q0, qd0)
    q, qd = _free_loop(orc, model, 1e-3, 1000, qd0=qd0)
    p_b, l_b = momenta(q, qd)
    assert np.linalg.norm(p_b - p_a) / np.linalg.norm(p_a) < 5e-4
    assert np.linalg.norm(l_b - l_a) / np.linalg.norm(l_a) < 5e-4
    assert np.linalg.norm(q[:, :3] - np.asarray(pos)) > 0.1


def test_oracle_pendulum_period(orc):
    """newton/tests/test_physics_validation.py:83-158 with SolverXPBD(iterations=20,
    angular_damping=0) and dt 3e-4 (:1579-1591): a point-like sphere (r 0.01) on a 1 m
    revolute pendulum released at 0.05 rad follows theta0 cos(omega t) with
    T = 2 pi sqrt(I_pivot / (m g L)) within 1 % of the amplitude (mean error over 3.5
    periods).  Z-up here, swinging about y; the body starts at the pose forward
    kinematics gives the initial angle."""
    g, L, theta0, dt = 10.0, 1.0, 0.05, 3e-4
    b = ModelBuilder(gravity=-g)
    s, c = math.sin(theta0), math.cos(theta0)
    q_link = (0.0, math.sin(0.5 * theta0), 0.0, math.cos(0.5 * theta0))  # theta0 about +y
    link = b.add_link(xform=((-L * s, 0.0, -L * c), q_link))
    b.add_shape_sphere(link, radius=0.01)
    ident = (0.0, 0.0, 0.0, 1.0)
    b.add_joint_revolute(-1, link, parent_xform=((0.0, 0.0, 0.0), ident), child_xform=((0.0, 0.0, L), ident),
                         axis=(0.0, 1.0, 0.0))
    model = b.finalize(device="cpu")
    m = float(model.host("body_mass")[0])
    i_pivot = float(model.host("body_inertia").reshape(-1, 3, 3)[0, 1, 1]) + m * L * L
    period = 2.0 * math.pi * math.sqrt(i_pivot / (m * g * L))
    lay = PairLayout(model, model.host("shape_contact_pairs"))
    p = SolverXPBD(model, iterations=20, angular_damping=0.0).params()
    q, qd = model.host("body_q").copy(), model.host("body_qd").copy()
    f = np.zeros((1, 6), np.float32)
    jt = model.host("joint_target_pos")
    zeros = np.zeros_like(jt)
    steps = int(3.5 * period / dt)
    angles = np.empty(steps)
    for i in range(steps):
        q, qd = orc.step(model, lay, p, q, qd, f, None, dt, joint_target_pos=jt, joint_target_vel=zeros,
                         joint_f=zeros)[:2]
        angles[i] = math.atan2(-q[0, 0], -q[0, 2])  # +theta swings the body towards -x
    t = np.arange(1, steps + 1) * dt
    err = np.mean(np.abs(angles - theta0 * np.cos(2.0 * math.pi / period * t))) / theta0
    assert err < 0.01, err


def test_oracle_joint_actuation(orc):
    """newton/tests/test_physics_validation.py:321-409 with SolverXPBD(iterations=20,
    angular_damping=0): without gravity, a joint torque of 5 N m on a revolute link and a
    force of 5 N on a prismatic link accelerate them as tau / I and F / m over 300 steps
    of 1 ms.  Measured on the bodies' twists (the joint coordinates of the reference
    follow from them)."""
    tau, force, dt, steps = 5.0, 5.0, 1e-3, 300
    b = ModelBuilder(gravity=0.0)
    ident = (0.0, 0.0, 0.0, 1.0)
    rev = b.add_link(xform=((0.0, 0.0, 0.0), ident))
    b.add_shape_box(rev, hx=0.2, hy=0.2, hz=0.2)
    b.add_joint_revolute(-1, rev, parent_xform=((0.0, 0.0, 0.0), ident), child_xform=((0.0, 0.0, 0.0), ident),
                         axis=(0.0, 0.0, 1.0))
    pri = b.add_link(xform=((0.0, 0.0, 5.0), ident))
    b.add_shape_sphere(pri, radius=0.1)
    b.add_joint_prismatic(-1, pri, parent_xform=((0.0, 0.0, 5.0), ident), child_xform=((0.0, 0.0, 0.0), ident),
                          axis=(1.0, 0.0, 0.0))
    model = b.finalize(device="cpu")
    i_zz = float(model.host("body_inertia").reshape(-1, 3, 3)[rev, 2, 2])
    m_pri = float(model.host("body_mass")[pri])
    qd_start = model.host("joint_qd_start")
    jf = np.zeros(model.joint_dof_count, np.float32)
    jf[qd_start[0]] = tau
    jf[qd_start[1]] = force
    lay = PairLayout(model, model.host("shape_contact_pairs"))
    p = SolverXPBD(model, iterations=20, angular_damping=0.0).params()
    q, qd = model.host("body_q").copy(), model.host("body_qd").copy()
    f = np.zeros((model.body_count, 6), np.float32)
    zeros = np.zeros(model.joint_dof_count, np.float32)
    for _ in range(steps):
        q, qd = orc.step(model, lay, p, q, qd, f, None, dt, joint_target_pos=zeros, joint_target_vel=zeros,
                         joint_f=jf)[:2]
    t = steps * dt
    assert qd[rev, 5] == pytest.approx(tau * t / i_zz, abs=max(tau / i_zz * dt, 1e-3))
    assert qd[pri, 0] == pytest.approx(force * t / m_pri, abs=max(force / m_pri * dt, 1e-3))
    assert qd[rev, 5] > 0.0 and qd[pri, 0] > 0.0


def _qmul(a, b):
    ax, ay, az, aw = a
    bx, by, bz, bw = b
    return [aw * bx + ax * bw + ay * bz - az * by, aw * by - ax * bz + ay * bw + az * bx,
            aw * bz + ax * by - ay * bx + az * bw, aw * bw - ax * bx - ay * by - az * bz]


def test_oracle_ramp_multicontact_stays_put(orc):
    """newton/tests/test_rigid_contact.py:230-503 (a 30 degree ramp plane with guide walls
    and an end wall, XPBD with 2 iterations, 100 frames of 10 substeps at 60 fps): every
    body moves less than 0.15 cube sizes and turns less than 10 degrees.  The bodies are
    the reference's contiguous run of in-scope shapes from the wall up (two cubes, two
    spheres, the capsule); its cylinder, cones and convex hulls, which rest further up the
    run, are left out with everything behind them."""
    from newton_custom_contact_b200.builder import quat_from_axis_angle

    length, thick, angle, wall_h = 10.0, 0.5, np.radians(30.0), 2.0
    cube = 0.99
    width = cube * 2.01
    ramp_c = np.array([0.0, length / 2 * np.cos(angle), length / 2 * np.sin(angle)])
    rq = list(quat_from_axis_angle((1.0, 0.0, 0.0), float(angle)))
    r = _rot(rq)
    fwd, up, right = r @ [0.0, -1.0, 0.0], r @ [0.0, 0.0, 1.0], r @ [1.0, 0.0, 0.0]
    b = ModelBuilder()
    b.add_shape_plane(body=-1, xform=list(ramp_c) + rq, width=0.0, length=0.0)
    for side in (1.0, -1.0):
        c = ramp_c + side * (width / 2 + 0.05) * right + 0.15 * up
        b.add_shape_box(-1, xform=list(c) + rq, hx=0.05, hy=length / 2, hz=0.15)
    shift = 0.6 * length
    tmp = ramp_c + 0.5 * cube * (up + shift * fwd)
    b.add_shape_box(-1, xform=[0.0, tmp[1] - cube / 2 * 1.4 - thick / 2, tmp[2], 0.0, 0.0, 0.0, 1.0],
                    hx=width / 2, hy=thick / 2, hz=wall_h / 2)
    for side in (1.0, -1.0):
        p = ramp_c + 0.5 * cube * (up + side * right + shift * fwd)
        b.add_shape_box(b.add_body(xform=list(p) + rq), hx=cube / 2, hy=cube / 2, hz=cube / 2)
    for side in (1.0, -1.0):
        p = ramp_c + 0.5 * cube * (up + side * right + (shift - 2.01) * fwd)
        b.add_shape_sphere(b.add_body(xform=list(p) + rq), radius=cube / 2)
    p = ramp_c + 0.5 * cube * (up + (shift - 4.02) * fwd)
    z_to_x = [0.0, math.sin(math.pi / 4), 0.0, math.cos(math.pi / 4)]
    b.add_shape_capsule(b.add_body(xform=list(p) + _qmul(rq, z_to_x)), radius=cube / 2, half_height=cube / 2)
    b.add_ground_plane()
    model = b.finalize(device="cpu")
    q0 = model.host("body_q").copy()
    q, _ = _sim(orc, model, SolverXPBD(model, iterations=2), 1.0 / 60.0 / 10, 1000)
    for i in range(model.body_count):
        assert np.linalg.norm(q[i, :3] - q0[i, :3]) < 0.15 * cube, i
        dot = min(1.0, abs(float(np.dot(q[i, 3:], q0[i, 3:]))))
        assert 2.0 * math.acos(dot) < math.radians(10.0), i


# ---- newton/tests/test_collision_pipeline.py:46-262: body A (x = -1) thrown at 5 m/s
# into body B (x = +1) without gravity; contacts found once per frame and reused for its
# 10 substeps, XPBD defaults, 100 frames at 60 fps.  Afterwards A has no sideways
# velocity, and B moves forward (0.03 < vx <= 5) without sideways (and, where the
# reference asks, angular) velocity.  The pairs of shapes this solver collides:

_HEAD_ON = [("sphere", "sphere", True), ("sphere", "box", True), ("sphere", "capsule", True),
            ("box", "box", False), ("capsule", "capsule", False)]


def _add_default_shape(b, kind, body):
    if kind == "box":
        b.add_shape_box(body)            # builder defaults: half extents 0.5
    elif kind == "sphere":
        b.add_shape_sphere(body, radius=0.5)
    else:
        b.add_shape_capsule(body, radius=0.25, half_height=0.3)


@pytest.mark.parametrize("kind_a,kind_b,strict_b", _HEAD_ON)
def test_oracle_head_on_collision(orc, kind_a, kind_b, strict_b):
    b = ModelBuilder(gravity=0.0)
    b.rigid_gap = 0.005
    _add_default_shape(b, kind_a, b.add_body(xform=[-1.0, 0.0, 0.0, 0.0, 0.0, 0.0, 1.0]))
    _add_default_shape(b, kind_b, b.add_body(xform=[1.0, 0.0, 0.0, 0.0, 0.0, 0.0, 1.0]))
    model = b.finalize(device="cpu")
    lay = PairLayout(model, model.host("shape_contact_pairs"))
    p = SolverXPBD(model).params()
    q = model.host("body_q").copy()
    qd = model.host("body_qd").copy()
    qd[0, 0] = 5.0
    f = np.zeros((2, 6), np.float32)
    dt = 1.0 / 60.0 / 10
    for _ in range(100):
        segs = orc.collide(model, lay, q)
        for _ in range(10):
            q, qd = orc.step(model, lay, p, q, qd, f, segs, dt)[:2]
    tol = 3e-3
    assert abs(qd[0, 1]) < tol and abs(qd[0, 2]) < tol
    assert 0.03 < qd[1, 0] <= 5.0
    assert abs(qd[1, 1]) < tol and abs(qd[1, 2]) < tol
    if strict_b:
        assert np.all(np.abs(qd[1, 3:6]) < tol)
