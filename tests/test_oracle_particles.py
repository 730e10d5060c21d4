"""The particle oracle against answers it does not share with the CUDA kernels: closed-form free fall,
signed distances of known points, conservation laws, resting contact, and the builder's particle
arrays (newton/_src/sim/builder.py:7186-7320, 9818-9855)."""

import numpy as np
import pytest

from newton_custom_contact_b200 import ModelBuilder, particles, scenes
from oracle import oracle_particles as op

F = np.float32


def _model(build):
    b = ModelBuilder()
    build(b)
    return b.finalize(device="cpu")


def _step(m, q, qd, soft=None, dt=1.0 / 240.0, iterations=4, relaxation=0.9):
    return op.step(m._host, particles.params(m), q, qd, None, soft, dt, iterations, relaxation)


def test_free_fall_is_semi_implicit_euler():
    m = _model(lambda b: b.add_particle((0.0, 0.0, 1.0), (0.5, 0.0, 0.0), 1.0, radius=0.05))
    dt = 1.0 / 240.0
    q, qd = m.host("particle_q"), m.host("particle_qd")
    for _ in range(10):
        q, qd = _step(m, q, qd, dt=dt)
    # v_{k+1} = v_k + g dt, x_{k+1} = x_k + v_{k+1} dt (solver.py:40-46); apply_particle_deltas then
    # recomputes v = (x_new - x0) / dt, whose fp32 cancellation at |x| ~ 1 costs ~ulp(1) / dt per step
    n = 10
    tol_v = n * 2.0 * np.spacing(F(1.0)) / dt
    assert qd[0, 2] == pytest.approx(-9.81 * dt * n, abs=tol_v)
    assert q[0, 2] == pytest.approx(1.0 - 9.81 * dt * dt * n * (n + 1) / 2, abs=tol_v * dt * n)
    assert q[0, 0] == pytest.approx(0.5 * dt * n, abs=1e-6)


def test_zero_mass_particle_ignores_gravity_and_inactive_particle_is_frozen():
    def build(b):
        b.add_particle((0.0, 0.0, 1.0), (0.2, 0.0, 0.0), 0.0, radius=0.05)
        b.add_particle((1.0, 0.0, 1.0), (0.0, 0.0, -3.0), 1.0, radius=0.05, flags=0)

    m = _model(build)
    q, qd = _step(m, m.host("particle_q"), m.host("particle_qd"), dt=0.01)
    np.testing.assert_allclose(q[0], [0.002, 0.0, 1.0], rtol=1e-6)
    np.testing.assert_allclose(qd[0], [0.2, 0.0, 0.0], rtol=1e-6)
    np.testing.assert_array_equal(q[1], m.host("particle_q")[1])
    np.testing.assert_array_equal(qd[1], m.host("particle_qd")[1])


@pytest.mark.parametrize("geo,scale,point,dist,normal", [
    (op.GEO_SPHERE, (0.5, 0, 0), (0.0, 0.0, 2.0), 1.5, (0, 0, 1)),
    (op.GEO_SPHERE, (0.5, 0, 0), (0.3, 0.4, 0.0), 0.0, (0.6, 0.8, 0)),
    (op.GEO_BOX, (0.5, 0.25, 0.1), (1.5, 0.0, 0.0), 1.0, (1, 0, 0)),
    (op.GEO_BOX, (0.5, 0.25, 0.1), (0.0, 0.0, 0.05), -0.05, (0, 0, 1)),
    (op.GEO_BOX, (0.5, 0.25, 0.1), (0.8, 0.65, 0.1), 0.5, (0.6, 0.8, 0)),
    (op.GEO_CAPSULE, (0.1, 0.3, 0), (0.0, 0.0, 0.6), 0.2, (0, 0, 1)),
    (op.GEO_CAPSULE, (0.1, 0.3, 0), (0.0, -0.5, 0.0), 0.4, (0, -1, 0)),
    (op.GEO_PLANE, (0.0, 0.0, 0), (3.0, -2.0, 0.25), 0.25, (0, 0, 1)),
])
def test_signed_distance_known_points(geo, scale, point, dist, normal):
    d, n = op._sdf(geo, np.asarray([point], F), np.asarray(scale, F))
    assert float(d[0]) == pytest.approx(dist, abs=1e-6)
    np.testing.assert_allclose(n[0], normal, atol=1e-6)


def test_soft_contact_on_ground_and_box():
    def build(b):
        b.add_ground_plane()
        b.add_shape_box(-1, xform=(2.0, 0.0, 0.5, 0, 0, 0, 1), hx=0.5, hy=0.5, hz=0.5)
        b.add_particle((0.3, 0.2, 0.004), (0, 0, 0), 1.0, radius=0.01)  # touches the ground
        b.add_particle((2.0, 0.1, 1.005), (0, 0, 0), 1.0, radius=0.01)  # on the box top (and above the ground)
        b.add_particle((5.0, 0.0, 2.0), (0, 0, 0), 1.0, radius=0.01)    # touches nothing

    m = _model(build)
    count, cp, cs, bpos, bvel, cn = op.soft_collide(m._host, m.host("particle_q"), None, 0.01, 16)
    assert count == 2
    np.testing.assert_array_equal(cp, [0, 1])
    np.testing.assert_array_equal(cs, [0, 1])
    np.testing.assert_allclose(cn, [[0, 0, 1], [0, 0, 1]], atol=1e-6)
    np.testing.assert_allclose(bpos[0], [0.3, 0.2, 0.0], atol=1e-6)
    np.testing.assert_allclose(bpos[1], [2.0, 0.1, 1.0], atol=1e-6)  # box top; a static shape's body frame is the world
    # capacity: the first contacts are kept, the count reports all
    count1, cp1, *_ = op.soft_collide(m._host, m.host("particle_q"), None, 0.01, 1)
    assert count1 == 2 and cp1.tolist() == [0]


def test_particle_comes_to_rest_on_the_ground():
    r = 0.02

    def build(b):
        b.add_ground_plane()
        b.add_particle((0.0, 0.0, 0.3), (0.4, 0.0, 0.0), 0.05, radius=r)

    m = _model(build)
    q, qd = m.host("particle_q"), m.host("particle_qd")
    dt = 1.0 / 240.0
    for _ in range(240):
        soft = op.soft_collide(m._host, q, None, 0.01, 8)
        q, qd = _step(m, q, qd, soft=soft, dt=dt, iterations=4)
    assert abs(q[0, 2] - r) < 2e-3          # resting on the plane at its radius
    assert abs(qd[0, 2]) < 0.05
    assert abs(qd[0, 0]) < 0.4               # friction (mu 0.5 mean) slowed the slide


def test_spring_pair_conserves_momentum_and_restores_length():
    def build(b):
        b.add_particle((0.0, 0.0, 0.0), (0, 0, 0), 1.0, radius=0.01)
        b.add_particle((1.0, 0.0, 0.0), (0, 0, 0), 1.0, radius=0.01)
        b.add_spring(0, 1, 1.0e4, 1.0, 0.0)

    m = _model(build)
    m._host["gravity"] = np.zeros((1, 3), F)
    q = m.host("particle_q").copy()
    q[1, 0] = 1.2  # stretched by 0.2
    qd = m.host("particle_qd")
    for _ in range(60):
        q, qd = _step(m, q, qd, dt=1.0 / 240.0, iterations=8)
    # velocities are quantised to ~ulp(x) / dt by v = (x_new - x0) / dt (kernels.py:800): 3e-5 m/s here
    quantum = 4.0 * float(np.spacing(F(1.2))) * 240.0
    assert abs(float(q[0, 0] + q[1, 0]) - 1.2) < 60 * quantum / 240.0   # centre of mass fixed
    assert abs(float(qd[0, 0] + qd[1, 0])) < quantum                    # zero total momentum
    assert abs(float(q[1, 0] - q[0, 0]) - 1.0) < 0.05       # back near the rest length


def test_head_on_particle_collision_separates_and_conserves_momentum():
    def build(b):
        b.add_particle((0.0, 0.0, 0.0), (1.0, 0.0, 0.0), 1.0, radius=0.05)
        b.add_particle((0.12, 0.0, 0.0), (-1.0, 0.0, 0.0), 1.0, radius=0.05)

    m = _model(build)
    m._host["gravity"] = np.zeros((1, 3), F)
    q, qd = m.host("particle_q"), m.host("particle_qd")
    for _ in range(20):
        q, qd = _step(m, q, qd, dt=1.0 / 240.0, iterations=4)
    assert float(q[1, 0] - q[0, 0]) > 0.1 - 2e-3              # no interpenetration beyond 2 mm
    assert abs(float(qd[0, 0] + qd[1, 0])) < 1e-5            # momentum conserved


def test_builder_particle_arrays_and_add_builder():
    src = ModelBuilder()
    src.add_particle((0.0, 0.0, 0.0), (0, 0, 0), 2.0, radius=0.1)
    src.add_particle((0.3, 0.4, 0.0), (0, 0, 0), 0.0)
    src.add_spring(0, 1, 100.0, 1.0, 0.0)
    b = ModelBuilder()
    b.replicate(src, 2, spacing=(1.0, 0.0, 0.0))
    m = b.finalize(device="cpu")
    assert m.particle_count == 4 and m.spring_count == 2
    np.testing.assert_array_equal(m.host("spring_indices"), [0, 1, 2, 3])
    np.testing.assert_allclose(m.host("spring_rest_length"), [0.5, 0.5], rtol=1e-6)
    np.testing.assert_array_equal(m.host("particle_inv_mass"), np.asarray([0.5, 0.0, 0.5, 0.0], F))
    np.testing.assert_array_equal(m.host("particle_world"), [0, 0, 1, 1])
    np.testing.assert_allclose(m.host("particle_q")[2], [1.0, 0.0, 0.0])
    assert m.host("particle_radius")[1] == F(0.1)  # default_particle_radius
    np.testing.assert_array_equal(m.host("particle_spring_start"), [0, 1, 2, 3, 4])


def test_solver_rejects_particle_contacts_with_bodies():
    from newton_custom_contact_b200 import SolverXPBD

    def build(b):
        body = b.add_body(xform=(0, 0, 1, 0, 0, 0, 1))
        b.add_joint_free(body)
        b.add_shape_sphere(body, radius=0.1)
        b.add_particle((0.0, 0.0, 0.5), (0, 0, 0), 1.0, radius=0.02)

    with pytest.raises(NotImplementedError, match="body-attached"):
        SolverXPBD(_model(build))
    m, _ = scenes.scene_particles(device="cpu", cloth=3, loose=4, body_shapes=True)
    SolverXPBD(m)  # a body shape built with has_particle_collision=False is fine


def test_atan2_matches_float64_in_every_quadrant():
    rng = np.random.default_rng(0)
    y = rng.normal(size=20000).astype(F)
    x = rng.normal(size=20000).astype(F)
    y[:8] = [0, 1, -1, 0, 1, -1, 1e-30, -1e-30]
    x[:8] = [1, 0, 0, -1, -1, 1, -1, -1]
    got = op.atan2(y, x).astype(np.float64)
    ref = np.arctan2(y.astype(np.float64), x.astype(np.float64))
    # a few float32 ulps of the angle (|angle| <= pi)
    assert np.abs(got - ref).max() < 1e-6
    assert op.atan2(np.float32(0), np.float32(0)) == 0


def test_bending_hinge_rest_angle_and_relaxation():
    """Two triangles folded 90 degrees about the x axis: the builder's rest angle of the flat hinge is 0;
    the bending constraint (kernels.py:358-457) unfolds the hinge toward it."""

    def build(b):
        b.add_particle((0.0, 0.0, 0.0), (0, 0, 0), 1.0, radius=0.01)   # k
        b.add_particle((1.0, 0.0, 0.0), (0, 0, 0), 1.0, radius=0.01)   # l
        b.add_particle((0.5, -0.5, 0.0), (0, 0, 0), 1.0, radius=0.01)  # i
        b.add_particle((0.5, 0.5, 0.0), (0, 0, 0), 1.0, radius=0.01)   # j
        b.add_edge(2, 3, 0, 1, edge_ke=50.0, edge_kd=0.0)

    m = _model(build)
    assert m.host("edge_rest_angle")[0] == pytest.approx(0.0, abs=1e-7)
    np.testing.assert_array_equal(m.host("particle_edge_start"), [0, 1, 2, 3, 4])
    m._host["gravity"] = np.zeros((1, 3), F)
    q = m.host("particle_q").copy()
    q[3] = (0.5, 0.0, 0.5)  # fold j up by 90 degrees
    qd = m.host("particle_qd")

    def angle(q):
        n1 = np.cross(q[0] - q[2], q[1] - q[2])
        n2 = np.cross(q[1] - q[3], q[0] - q[3])
        e = (q[1] - q[0]) / np.linalg.norm(q[1] - q[0])
        n1, n2 = n1 / np.linalg.norm(n1), n2 / np.linalg.norm(n2)
        return float(np.arctan2(np.dot(np.cross(n1, n2), e), np.dot(n1, n2)))

    a0 = angle(q)
    assert abs(abs(a0) - np.pi / 2) < 1e-5
    for _ in range(40):
        q, qd = _step(m, q, qd, dt=1.0 / 240.0, iterations=8)
    assert abs(angle(q)) < 0.5 * abs(a0)
    assert abs(float(qd.sum(axis=0)[2])) < 1e-3  # internal constraint: no net momentum


def test_restitution_bounce_off_the_ground():
    """apply_particle_shape_restitution (kernels.py:34-112): a particle hitting the plane leaves it with
    the restitution coefficient times its approach speed."""
    r = 0.02

    def build(b):
        b.add_ground_plane()
        b.add_particle((0.0, 0.0, r - 0.0005), (0.0, 0.0, -2.0), 0.05, radius=r)  # touching at the start

    m = _model(build)
    m.soft_contact_restitution = 0.5
    m._host["gravity"] = np.zeros((1, 3), F)
    q, qd = m.host("particle_q"), m.host("particle_qd")
    dt = 1.0 / 240.0
    soft = op.soft_collide(m._host, q, None, 0.01, 8)
    q1, qd1 = op.step(m._host, particles.params(m), q, qd, None, soft, dt, 4, 0.9, restitution=True)
    assert qd1[0, 2] == pytest.approx(1.0, rel=1e-5)  # 0.5 x 2 m/s, upwards
    _, qd0 = op.step(m._host, particles.params(m), q, qd, None, soft, dt, 4, 0.9, restitution=False)
    assert qd0[0, 2] < 0.5  # without restitution it leaves at the projection speed only


def test_compressed_tetrahedron_recovers_its_volume():
    """solve_tetrahedra (kernels.py:459-628): a tet squashed to 60 % height regains volume; no net momentum."""

    def build(b):
        for p in ((0, 0, 0), (0.1, 0, 0), (0, 0.1, 0), (0, 0, 0.1)):
            b.add_particle(p, (0, 0, 0), 0.01, radius=0.005)
        assert b.add_tetrahedron(0, 1, 2, 3) == pytest.approx(0.1 ** 3 / 6)

    m = _model(build)
    assert m.tet_count == 1
    m._host["gravity"] = np.zeros((1, 3), F)
    q = m.host("particle_q").copy()
    q[3, 2] = 0.06
    qd = m.host("particle_qd")

    def vol(q):
        return float(np.linalg.det(np.stack([q[1] - q[0], q[2] - q[0], q[3] - q[0]], axis=1)) / 6)

    v0 = vol(q)
    for _ in range(30):
        q, qd = op.step(m._host, particles.params(m), q, qd, None, None, 1.0 / 240.0, 8, 0.9,
                        soft_body_relaxation=1e-6)
    assert vol(q) > v0 + 0.5 * (0.1 ** 3 / 6 - v0)
    assert np.abs(qd.sum(axis=0)).max() < 1e-3
