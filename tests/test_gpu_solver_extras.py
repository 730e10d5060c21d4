"""CUDA path vs the CPU oracle for the solver's optional parts, bit for bit:
restitution (apply_rigid_restitution, xpbd/kernels.py:2471-2620), per-contact
forces (accumulate_weighted_contact_impulse + convert_contact_impulse_to_force,
kernels.py:2301-2393, SolverXPBD.update_contacts, solver_xpbd.py:766-821) and
the articulated C3 scene (solve_body_joints with revolute drives and limits).
The oracle itself is checked against the reference's physical tests in
test_oracle_physics.py.
"""

import numpy as np
import pytest
import torch

from newton_custom_contact_b200 import CollisionPipeline, JointType, ModelBuilder, SolverXPBD, scenes

pytestmark = pytest.mark.gpu


def _bits_equal(a, b):
    return np.array_equal(np.asarray(a, np.float32).view(np.uint32), np.asarray(b, np.float32).view(np.uint32))


def _oracle_public_order(model, lay, segs):
    """Oracle slot index of every contact in public (world, key) order."""
    cs = 5 * lay.world_pair_start.astype(np.int64)
    return np.concatenate([np.arange(cs[w], cs[w] + int(segs.world_count[w])) for w in range(model.world_count)])


def _run(model, substeps, dt, iterations, orc, restitution=False, forces=False, joint_target_pos=None):
    """GPU and oracle loops side by side; per substep compares forces when requested."""
    if forces:
        model.request_contact_attributes("force")
    pipe = CollisionPipeline(model)
    solver = SolverXPBD(model, iterations=iterations, enable_restitution=restitution)
    control = model.control()
    if joint_target_pos is not None:
        control.joint_target_pos.copy_(torch.as_tensor(joint_target_pos, dtype=torch.float32))
    s0, s1 = model.state(), model.state()
    contacts = pipe.contacts()
    q = model.host("body_q").copy()
    qd = model.host("body_qd").copy()
    f = np.zeros((model.body_count, 6), np.float32)
    p = solver.params()
    jt = control.joint_target_pos.cpu().numpy() if model.joint_dof_count else None
    jv = control.joint_target_vel.cpu().numpy() if model.joint_dof_count else None
    jf = np.zeros(model.joint_dof_count, np.float32)
    checked = 0
    for _ in range(substeps):
        s0.clear_forces()
        pipe.collide(s0, contacts)
        solver.step(s0, s1, control, contacts, dt)
        segs = orc.collide(model, pipe.layout, q)
        out = orc.step(model, pipe.layout, p, q, qd, f, segs, dt, joint_target_pos=jt, joint_target_vel=jv,
                       joint_f=jf, want_impulse=forces)
        q, qd = out[0], out[1]
        if forces:
            solver.update_contacts(contacts)
            torch.cuda.synchronize()
            n = int(contacts.rigid_contact_count.item())
            got = contacts.force[:n].cpu().numpy()
            inv_dt = np.float32(1.0) / np.float32(dt)
            want = out[3][_oracle_public_order(model, pipe.layout, segs)] * inv_dt
            assert got.shape == want.shape
            assert _bits_equal(got, want), np.abs(got - want).max()
            assert not contacts.force[n:].any()
            checked += int(np.count_nonzero(np.abs(want).sum(axis=1)))
        s0, s1 = s1, s0
    torch.cuda.synchronize()
    return s0.body_q.cpu().numpy(), s0.body_qd.cpu().numpy(), q, qd, checked


def test_restitution_parity(cuda, orc):
    model, info = scenes.scene_c5(worlds=16, device="cuda", restitution=0.5)
    gq, gqd, q, qd, _ = _run(model, 16, 1.0 / 600.0, 8, orc, restitution=True)
    np.testing.assert_allclose(gq, q, rtol=1e-5, atol=1e-6)
    assert _bits_equal(gq, q) and _bits_equal(gqd, qd)


def test_restitution_changes_the_step(cuda, orc):
    """The restitution pass is live on this scene (not a no-op)."""
    model, _ = scenes.scene_c5(worlds=16, device="cuda", restitution=0.5)
    a = _run(model, 4, 1.0 / 600.0, 8, orc, restitution=True)
    model2, _ = scenes.scene_c5(worlds=16, device="cuda", restitution=0.5)
    b = _run(model2, 4, 1.0 / 600.0, 8, orc, restitution=False)
    assert not np.array_equal(a[1], b[1])


def test_contact_force_parity(cuda, orc):
    model, info = scenes.scene_c5(worlds=16, device="cuda")
    gq, gqd, q, qd, checked = _run(model, 8, 1.0 / 600.0, 8, orc, forces=True)
    assert checked > 0
    assert _bits_equal(gq, q) and _bits_equal(gqd, qd)


def test_contact_force_parity_c2_with_restitution(cuda, orc):
    model, info = scenes.scene_c2(seed=7, worlds=24, nmin=8, nmax=40, device="cuda")
    gq, gqd, q, qd, checked = _run(model, 4, info["dt"] / info["substeps"], info["iterations"], orc,
                                   restitution=True, forces=True)
    assert _bits_equal(gq, q) and _bits_equal(gqd, qd)


def test_forces_of_ingested_contacts(cuda, orc):
    """Custom contacts in reversed order: each contact's force lands on its own public row.  Each
    body sums its contacts' deltas in public order, so the reversed order moves the bodies and the
    forces by rounding only."""
    model, info = scenes.scene_c5(worlds=8, device="cuda")
    model.request_contact_attributes("force")
    pipe = CollisionPipeline(model)
    solver = SolverXPBD(model, iterations=8)
    s0 = model.state()
    c1 = pipe.contacts()
    pipe.collide(s0, c1)
    out_a = model.state()
    solver.step(s0, out_a, None, c1, 1.0 / 600.0)
    solver.update_contacts(c1)
    fa = c1.force.clone()
    c2 = pipe.contacts()
    n = int(c1.rigid_contact_count.item())
    idx = torch.arange(n - 1, -1, -1, device="cuda")
    for name in ("shape0", "shape1", "point0", "point1", "offset0", "offset1", "normal", "margin0", "margin1"):
        getattr(c2, f"rigid_contact_{name}")[:n] = getattr(c1, f"rigid_contact_{name}")[:n][idx]
    c2.rigid_contact_count.fill_(n)
    c2.mark_dense_modified()
    out_b = model.state()
    solver.step(s0, out_b, None, c2, 1.0 / 600.0)
    solver.update_contacts(c2)
    torch.cuda.synchronize()
    torch.testing.assert_close(out_b.body_q, out_a.body_q, rtol=1e-5, atol=1e-6)
    scale = float(fa[:n].abs().max())
    assert scale > 0
    torch.testing.assert_close(c2.force[:n], fa[:n][idx], rtol=1e-4, atol=1e-4 * scale)


def test_update_contacts_errors(cuda):
    b = ModelBuilder()
    b.add_ground_plane()
    body = b.add_body(xform=((0.0, 0.0, 0.25), (0.0, 0.0, 0.0, 1.0)))
    b.add_shape_sphere(body, radius=0.25)
    model = b.finalize(device="cuda")
    solver = SolverXPBD(model, iterations=2)
    s0, s1 = model.state(), model.state()
    contacts = model.contacts()
    model.collide(s0, contacts)
    solver.step(s0, s1, model.control(), contacts, 1.0 / 60.0)
    assert contacts.force is None
    with pytest.raises(ValueError):
        solver.update_contacts(contacts)
    model.request_contact_attributes("force")
    pipe = CollisionPipeline(model)
    c2 = pipe.contacts()
    fresh = SolverXPBD(model, iterations=2)
    with pytest.raises(ValueError):
        fresh.update_contacts(c2)  # no step yet
    pipe.collide(s0, c2)
    fresh.step(s0, s1, None, c2, 1.0 / 60.0)
    other = CollisionPipeline(model, rigid_contact_max=c2.rigid_contact_max + 7).contacts()
    with pytest.raises(ValueError):
        fresh.update_contacts(other)  # capacity mismatch


@pytest.mark.parametrize("substeps", [1, 8])
def test_step_parity_c3_arms(cuda, orc, substeps):
    """Revolute drives and limits (solve_body_joints).  The twist / swing angles
    use the library's own asin / acos on both sides (a device / host-libm
    last-ulp difference would be amplified by 1/dt into the velocities), so
    the trajectories agree bit for bit."""
    model, info = scenes.scene_c3(worlds=6, device="cuda")
    # drive targets A sin(phase) on the arms' revolute dofs (free joints of the boxes stay 0)
    rev = np.nonzero(model.host("joint_type") == int(JointType.REVOLUTE))[0]
    targets = np.zeros(model.joint_dof_count, np.float32)
    targets[model.host("joint_qd_start")[rev]] = 0.5 * np.sin(info["phases"]).reshape(-1)
    gq, gqd, q, qd, _ = _run(model, substeps, info["dt"] / info["substeps"], info["iterations"], orc,
                             joint_target_pos=targets)
    np.testing.assert_allclose(gq, q, rtol=1e-5, atol=1e-6)
    assert _bits_equal(gq, q) and _bits_equal(gqd, qd)
    # the arms are live: joint drives moved the links
    assert not np.allclose(gq[: 7], model.host("body_q")[: 7], atol=1e-7)


@pytest.mark.parametrize("mode,group", [("groups_compact", 32), ("groups", 64), ("batch", 64)])
def test_c3_arms_all_step_modes(cuda, orc, mode, group):
    """Joint worlds through the compact slab, 64-thread groups and the batch kernel."""
    model, info = scenes.scene_c3(worlds=4, device="cuda")
    pipe = CollisionPipeline(model)
    pipe.set_step_schedule(group, mode=mode)
    solver = SolverXPBD(model, iterations=info["iterations"])
    s0, s1 = model.state(), model.state()
    contacts = pipe.contacts()
    dt = info["dt"] / info["substeps"]
    q = model.host("body_q").copy()
    qd = model.host("body_qd").copy()
    f = np.zeros((model.body_count, 6), np.float32)
    zeros = np.zeros(model.joint_dof_count, np.float32)
    for _ in range(4):
        s0.clear_forces()
        pipe.collide(s0, contacts)
        solver.step(s0, s1, None, contacts, dt)
        segs = orc.collide(model, pipe.layout, q)
        q, qd, _ = orc.step(model, pipe.layout, solver.params(), q, qd, f, segs, dt, joint_target_pos=zeros,
                            joint_target_vel=zeros, joint_f=zeros)
        s0, s1 = s1, s0
    torch.cuda.synchronize()
    assert _bits_equal(s0.body_q.cpu().numpy(), q) and _bits_equal(s0.body_qd.cpu().numpy(), qd)


def test_body_parent_f_parity_c3(cuda, orc):
    """State.body_parent_f (joint reaction per child body) equals the oracle's, bit for bit,
    on the articulated scene; unrequested it stays None."""
    model, info = scenes.scene_c3(worlds=4, device="cuda")
    assert model.state().body_parent_f is None
    model.request_state_attributes("body_parent_f")
    pipe = CollisionPipeline(model)
    solver = SolverXPBD(model, iterations=info["iterations"])
    s0, s1 = model.state(), model.state()
    contacts = pipe.contacts()
    dt = info["dt"] / info["substeps"]
    q, qd = model.host("body_q").copy(), model.host("body_qd").copy()
    f = np.zeros((model.body_count, 6), np.float32)
    zeros = np.zeros(model.joint_dof_count, np.float32)
    for _ in range(4):
        s0.clear_forces()
        pipe.collide(s0, contacts)
        solver.step(s0, s1, None, contacts, dt)
        segs = orc.collide(model, pipe.layout, q)
        q, qd, _, pf = orc.step(model, pipe.layout, solver.params(), q, qd, f, segs, dt, joint_target_pos=zeros,
                                joint_target_vel=zeros, joint_f=zeros, want_parent_f=True)
        torch.cuda.synchronize()
        got = s1.body_parent_f.cpu().numpy()
        assert _bits_equal(got, pf)
        s0, s1 = s1, s0
    rev = model.host("joint_child")[model.host("joint_type") == int(JointType.REVOLUTE)]
    assert np.abs(pf[rev]).sum() > 0 and np.all(np.delete(pf, rev, axis=0) == 0.0)


def test_shapes_never_exceed_initial_z(cuda):
    """No shape dropped on the ground ever rises above max(2 m, its initial z) over 200
    frames at 100 fps with 10 substeps, 2 iterations, relaxation 0.8 and no angular
    damping (the reference's settings, test_shapes_no_bounce.py:186-226); the replicated
    worlds stay bit-identical to one another throughout."""
    worlds = 4
    model, z0 = scenes.scene_falling_shapes(worlds, device="cuda")
    pipe = CollisionPipeline(model)
    solver = SolverXPBD(model, iterations=2, rigid_contact_relaxation=0.8, angular_damping=0.0)
    s0, s1 = model.state(), model.state()
    contacts = pipe.contacts()
    limit = np.maximum(np.float32(2.0), z0)
    dt = 1.0 / 100.0 / 10
    in_contact = 0
    for frame in range(200):
        for _ in range(10):
            s0.clear_forces()
            pipe.collide(s0, contacts)
            solver.step(s0, s1, None, contacts, dt)
            s0, s1 = s1, s0
        q = s0.body_q.cpu().numpy()
        z = q[:, 2]
        assert np.all(z <= limit), f"frame {frame + 1}: max excess {float((z - limit).max()):.4f} m"
        in_contact = max(in_contact, int(contacts.rigid_contact_count.item()))
        per_world = q.reshape(worlds, -1, 7)
        assert all(_bits_equal(per_world[w], per_world[0]) for w in range(1, worlds)), frame
    assert np.all(np.isfinite(q))
    # the grid has landed: every body below its start, contacts live in every world
    assert in_contact >= worlds * 16 and np.all(z < z0)


def _shapes_on_plane_model():
    """newton/tests/test_rigid_contact.py:28-227 without its cylinder and mesh bodies."""
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
    return b.finalize(device="cuda"), np.asarray(expected)


def test_shapes_on_plane_parity(cuda, orc):
    """The reference's shapes-on-plane rest test (test_rigid_contact.py:28-227, XPBD with
    2 iterations) through the CUDA path: 120 frames of 30 substeps agree with the oracle
    bit for bit, and the bodies rest on the plane (|v|, |w| < 0.2, positions within 0.25,
    orientations within 0.1 of identity)."""
    model, expected = _shapes_on_plane_model()
    gq, gqd, q, qd, _ = _run(model, 120 * 30, 1.0 / 60.0 / 30, 2, orc)
    assert _bits_equal(gq, q) and _bits_equal(gqd, qd)
    assert np.abs(gqd[:, :3]).max() < 0.2 and np.abs(gqd[:, 3:]).max() < 0.2
    assert np.abs(gq[:, :3] - expected).max() < 0.25
    assert np.abs(gq[:, 3:] - np.array([0.0, 0.0, 0.0, 1.0])).max() < 0.1


def test_box_drop_parity(cuda, orc):
    """The reference's two-box drop (test_rigid_contact.py:766-831, XPBD with 2 iterations)
    through the CUDA path: 60 frames of 8 substeps agree with the oracle bit for bit; both
    boxes end near the origin, above the ground and nearly at rest."""
    from newton_custom_contact_b200.builder import quat_from_axis_angle

    h = 0.5
    b = ModelBuilder()
    b.add_ground_plane()
    body = b.add_body(xform=[0.0, 0.0, h * 1.2, 0.0, 0.0, 0.0, 1.0])
    b.add_shape_box(body, hx=h, hy=h, hz=h)
    body = b.add_body(xform=np.concatenate([[0.0, 0.0, h * 4.2], quat_from_axis_angle((1.0, 0.0, 0.0), 0.5)]))
    b.add_shape_box(body, hx=h, hy=h, hz=h)
    model = b.finalize(device="cuda")
    gq, gqd, q, qd, _ = _run(model, 60 * 8, 1.0 / 60.0 / 8, 2, orc)
    assert _bits_equal(gq, q) and _bits_equal(gqd, qd)
    assert np.all(np.abs(gq[:, :2]) < 1.0) and np.all(gq[:, 2] > 0.5 * h)
    assert np.all(np.linalg.norm(gqd[:, :3], axis=1) < 1.0)
