"""The reference's physical-validation scenes through the CUDA path, bit for bit against
the CPU oracle, with the reference's own assertions on the result.

Scenes (Z-up here; the reference's builder in these tests is Y-up):
  * static and dynamic friction: newton/tests/test_physics_validation.py:505-641
    (SolverXPBD(iterations=10, angular_damping=0), :1619-1622) -- body forces and an
    initial velocity through the contact path;
  * pendulum period: :83-158 (iterations 20, dt 3e-4) -- the revolute joint solve;
  * joint actuation: :321-409 -- joint forces on a revolute and a prismatic joint.
The oracle alone meets the same assertions in test_oracle_physics.py.
"""

import math

import numpy as np
import pytest
import torch

from newton_custom_contact_b200 import CollisionPipeline, ModelBuilder, SolverXPBD

pytestmark = pytest.mark.gpu


def _bits_equal(a, b):
    return np.array_equal(np.asarray(a, np.float32).view(np.uint32), np.asarray(b, np.float32).view(np.uint32))


def _run(orc, model, solver, dt, steps, body_f=None, joint_f=None, qd0=None):
    """CUDA and oracle loops side by side; body_f(i) gives the step's body forces.  Models
    without candidate pairs step without contacts (contacts=None)."""
    with_contacts = np.asarray(model.host("shape_contact_pairs")).size > 0
    pipe = CollisionPipeline(model)
    contacts = pipe.contacts() if with_contacts else None
    control = model.control()
    jf = np.zeros(model.joint_dof_count, np.float32) if joint_f is None else np.asarray(joint_f, np.float32)
    control.joint_f.copy_(torch.from_numpy(jf))
    s0, s1 = model.state(), model.state()
    q = model.host("body_q").copy()
    qd = model.host("body_qd").copy()
    if qd0 is not None:
        qd = np.asarray(qd0, np.float32).copy()
        s0.body_qd.copy_(torch.from_numpy(qd))
    zero = np.zeros((model.body_count, 6), np.float32)
    jt = control.joint_target_pos.cpu().numpy()
    jv = control.joint_target_vel.cpu().numpy()
    p = solver.params()
    for i in range(steps):
        f = zero if body_f is None else body_f(i)
        s0.clear_forces()
        s0.body_f.copy_(torch.from_numpy(f))
        if with_contacts:
            pipe.collide(s0, contacts)
        solver.step(s0, s1, control, contacts, dt)
        segs = orc.collide(model, pipe.layout, q) if with_contacts else None
        q, qd = orc.step(model, pipe.layout, p, q, qd, f, segs, dt, joint_target_pos=jt, joint_target_vel=jv,
                         joint_f=jf)[:2]
        s0, s1 = s1, s0
    torch.cuda.synchronize()
    gq, gqd = s0.body_q.cpu().numpy(), s0.body_qd.cpu().numpy()
    assert _bits_equal(gq, q) and _bits_equal(gqd, qd)
    return gq, gqd


def _boxes_on_ground(mu, ys):
    cfg = ModelBuilder.ShapeConfig(mu=mu, gap=0.1)
    b = ModelBuilder(up_axis="Z", gravity=-10.0)
    b.add_ground_plane(cfg=cfg)
    h = 0.25
    for y in ys:
        body = b.add_body(xform=[0.0, y, h + 0.001, 0.0, 0.0, 0.0, 1.0])
        b.add_shape_box(body, hx=h, hy=h, hz=h, cfg=cfg)
    return b.finalize(device="cuda"), h


def test_static_friction(cuda, orc):
    mu = 0.5
    model, h = _boxes_on_ground(mu, [0.0, 5.0])
    mass = 1000.0 * (2 * h) ** 3
    push = np.zeros((2, 6), np.float32)
    push[0, 0] = 0.3 * mu * mass * 10.0
    push[1, 0] = 2.0 * mu * mass * 10.0
    zero = np.zeros_like(push)
    solver = SolverXPBD(model, iterations=10, angular_damping=0.0)
    q, _ = _run(orc, model, solver, 1e-3, 200, body_f=lambda i: push if i > 20 else zero)
    assert abs(q[0, 0]) < 0.01 and q[0, 2] == pytest.approx(h, abs=0.01)
    assert q[1, 0] > 0.05 and q[1, 2] == pytest.approx(h, abs=0.01)


def test_dynamic_friction(cuda, orc):
    mu, v0, g = 0.4, 2.0, 10.0
    model, h = _boxes_on_ground(mu, [0.0])
    qd0 = model.host("body_qd").copy()
    qd0[0, 0] = v0
    solver = SolverXPBD(model, iterations=10, angular_damping=0.0)
    q, qd = _run(orc, model, solver, 1e-3, int(1.5 * v0 / (mu * g) / 1e-3), qd0=qd0)
    d_stop = v0 ** 2 / (2.0 * mu * g)
    assert q[0, 0] == pytest.approx(d_stop, abs=0.01 * d_stop)
    assert abs(qd[0, 0]) < 0.01 and q[0, 2] == pytest.approx(h, abs=0.01)


def test_pendulum_period(cuda, orc):
    g, L, theta0, dt = 10.0, 1.0, 0.05, 3e-4
    b = ModelBuilder(gravity=-g)
    s, c = math.sin(theta0), math.cos(theta0)
    link = b.add_link(xform=((-L * s, 0.0, -L * c), (0.0, math.sin(0.5 * theta0), 0.0, math.cos(0.5 * theta0))))
    b.add_shape_sphere(link, radius=0.01)
    ident = (0.0, 0.0, 0.0, 1.0)
    b.add_joint_revolute(-1, link, parent_xform=((0.0, 0.0, 0.0), ident), child_xform=((0.0, 0.0, L), ident),
                         axis=(0.0, 1.0, 0.0))
    model = b.finalize(device="cuda")
    m = float(model.host("body_mass")[0])
    period = 2.0 * math.pi * math.sqrt((float(model.host("body_inertia").reshape(-1, 3, 3)[0, 1, 1]) + m * L * L)
                                       / (m * g * L))
    solver = SolverXPBD(model, iterations=20, angular_damping=0.0)
    # a quarter period side by side with the oracle, bit for bit
    _run(orc, model, solver, dt, int(0.25 * period / dt))
    # then the reference's trajectory check on the CUDA path alone (no shape pairs: the
    # single link steps without contacts)
    assert np.asarray(model.host("shape_contact_pairs")).size == 0
    s0, s1 = model.state(), model.state()
    steps = int(3.5 * period / dt)
    angles = torch.empty(steps, device="cuda")
    for i in range(steps):
        s0.clear_forces()
        solver.step(s0, s1, None, None, dt)
        s0, s1 = s1, s0
        angles[i] = torch.atan2(-s0.body_q[0, 0], -s0.body_q[0, 2])
    a = angles.cpu().numpy()
    t = np.arange(1, steps + 1) * dt
    err = np.mean(np.abs(a - theta0 * np.cos(2.0 * math.pi / period * t))) / theta0
    assert err < 0.01, err


def test_joint_actuation(cuda, orc):
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
    model = b.finalize(device="cuda")
    i_zz = float(model.host("body_inertia").reshape(-1, 3, 3)[rev, 2, 2])
    m_pri = float(model.host("body_mass")[pri])
    qd_start = model.host("joint_qd_start")
    jf = np.zeros(model.joint_dof_count, np.float32)
    jf[qd_start[0]] = tau
    jf[qd_start[1]] = force
    solver = SolverXPBD(model, iterations=20, angular_damping=0.0)
    _, qd = _run(orc, model, solver, dt, steps, joint_f=jf)
    t = steps * dt
    assert qd[rev, 5] == pytest.approx(tau * t / i_zz, abs=max(tau / i_zz * dt, 1e-3))
    assert qd[pri, 0] == pytest.approx(force * t / m_pri, abs=max(force / m_pri * dt, 1e-3))


def test_kinematic_platform_drags_boxes(cuda, orc):
    """Kinematic bodies through the CUDA path, bit for bit against the oracle: a kinematic platform
    (effective inverse mass and inertia zero, solver.py:160-174) that the caller moves every substep
    at 0.5 m/s carries boxes resting on it through the contacts' kinematic friction term
    (kernels.py:2220-2225); the step passes the platform's own state through unchanged
    (copy_kinematic_body_state_kernel, kernels.py:18-31)."""
    cfg = ModelBuilder.ShapeConfig(mu=0.8, gap=0.05)
    b = ModelBuilder(up_axis="Z", gravity=-9.81)
    platform = b.add_body(xform=[0.0, 0.0, 0.1, 0.0, 0.0, 0.0, 1.0], is_kinematic=True)
    b.add_shape_box(platform, hx=1.0, hy=1.0, hz=0.1, cfg=cfg)
    h = 0.1
    for x in (-0.5, 0.0, 0.5):
        body = b.add_body(xform=[x, 0.0, 0.2 + h + 0.002, 0.0, 0.0, 0.0, 1.0])
        b.add_shape_box(body, hx=h, hy=h, hz=h, cfg=cfg)
    model = b.finalize(device="cuda")
    dt = 1.0 / 60.0 / 8
    speed = 0.5
    solver = SolverXPBD(model, iterations=8)
    pipe = CollisionPipeline(model)
    contacts = pipe.contacts()
    s0, s1 = model.state(), model.state()
    q = model.host("body_q").copy()
    qd = model.host("body_qd").copy()
    qd[platform, 0] = np.float32(speed)
    s0.body_qd.copy_(torch.from_numpy(qd))
    zero = np.zeros((model.body_count, 6), np.float32)
    p = solver.params()
    for i in range(240):
        # the caller drives the kinematic platform: its pose before substep i
        q[platform, 0] = np.float32(speed * dt * i)
        s0.body_q[platform, 0] = float(q[platform, 0])
        s0.clear_forces()
        pipe.collide(s0, contacts)
        solver.step(s0, s1, None, contacts, dt)
        segs = orc.collide(model, pipe.layout, q)
        q_in = q.copy()
        q, qd = orc.step(model, pipe.layout, p, q, qd, zero, segs, dt)[:2]
        # kinematic pass-through: the step leaves the platform as it got it
        assert np.array_equal(q[platform], q_in[platform])
        s0, s1 = s1, s0
        if i in (0, 15, 239):
            torch.cuda.synchronize()
            gq, gqd = s0.body_q.cpu().numpy(), s0.body_qd.cpu().numpy()
            assert _bits_equal(gq, q) and _bits_equal(gqd, qd), f"substep {i}"
    # after 0.5 s the boxes ride the platform: they move along +x at close to its speed and stay on it
    boxes = [i for i in range(model.body_count) if i != platform]
    vx = qd[boxes, 0]
    assert np.all(vx > 0.8 * speed) and np.all(vx < 1.2 * speed), vx
    assert np.all(np.abs(q[boxes, 2] - (0.2 + h)) < 0.01)
