"""Frame-to-frame contact matching on the GPU.

The first group restates the scenarios and assertions of the reference's
newton/tests/test_contact_matching.py:58-660 (identity on a stable scene, new
and broken contacts, position / normal thresholds, the report, sticky
replay, option validation).  The last test compares match indices and sticky
geometry with the CPU oracle (oracle/oracle_match.cpp) along a drop
trajectory.
"""

import numpy as np
import pytest
import torch

from newton_custom_contact_b200 import CollisionPipeline, ModelBuilder, SolverXPBD, scenes

pytestmark = pytest.mark.gpu

ID = (0.0, 0.0, 0.0, 1.0)


def _simple_scene(xs=(-0.5, 0.0, 0.5), z=0.1, extra=None):
    b = ModelBuilder()
    b.add_ground_plane()
    for x in xs:
        body = b.add_body(xform=((x, 0.0, z), ID))
        b.add_shape_sphere(body, radius=0.1)
    shape = None
    if extra is not None:
        body = b.add_body(xform=(extra, ID))
        shape = b.add_shape_sphere(body, radius=0.1)
    model = b.finalize(device="cuda")
    return model, model.state(), shape


def _collide(pipe, state, contacts):
    contacts.clear()
    pipe.collide(state, contacts)
    torch.cuda.synchronize()
    return int(contacts.rigid_contact_count.item())


def _mi(contacts, n):
    return contacts.rigid_contact_match_index[:n].cpu().numpy()


def _shift(state, body, xyz=None, dx=None):
    q = state.body_q.clone()
    if xyz is not None:
        q[body, :3] = torch.tensor(xyz, dtype=torch.float32)
    if dx is not None:
        q[:, 0] += dx
    state.body_q.copy_(q)


def test_first_frame_all_not_found(cuda):
    model, state, _ = _simple_scene()
    pipe = CollisionPipeline(model, broad_phase="nxn", contact_matching="latest")
    c = pipe.contacts()
    n = _collide(pipe, state, c)
    assert n > 0 and np.all(_mi(c, n) == -1)


def test_stable_scene_identity_three_frames(cuda):
    model, state, _ = _simple_scene()
    pipe = CollisionPipeline(model, broad_phase="nxn", contact_matching="latest")
    c = pipe.contacts()
    n1 = _collide(pipe, state, c)
    for _ in range(3):
        n = _collide(pipe, state, c)
        assert n == n1
        np.testing.assert_array_equal(_mi(c, n), np.arange(n, dtype=np.int32))


def test_new_contact_detection(cuda):
    model, state, _ = _simple_scene(xs=(-0.5, 0.5), extra=(0.0, 0.0, 10.0))
    pipe = CollisionPipeline(model, broad_phase="nxn", contact_matching="latest")
    c = pipe.contacts()
    n1 = _collide(pipe, state, c)
    _shift(state, 2, xyz=(0.0, 0.0, 0.1))
    n2 = _collide(pipe, state, c)
    mi = _mi(c, n2)
    assert n2 > n1 and np.sum(mi == -1) > 0 and np.sum(mi >= 0) == n1
    assert len(np.unique(mi[mi >= 0])) == np.sum(mi >= 0)


def test_broken_position_threshold_and_report(cuda):
    model, state, _ = _simple_scene()
    pipe = CollisionPipeline(model, broad_phase="nxn", contact_matching="latest", contact_report=True)
    c = pipe.contacts()
    n1 = _collide(pipe, state, c)
    _shift(state, None, dx=0.2)
    n2 = _collide(pipe, state, c)
    assert np.all(_mi(c, n2) == -2)
    nb = int(c.rigid_contact_broken_count.item())
    assert nb == n1
    np.testing.assert_array_equal(np.sort(c.rigid_contact_broken_indices[:nb].cpu().numpy()), np.arange(n1))


def test_within_position_threshold_still_matches(cuda):
    model, state, _ = _simple_scene()
    pipe = CollisionPipeline(model, broad_phase="nxn", contact_matching="latest")
    c = pipe.contacts()
    _collide(pipe, state, c)
    _shift(state, None, dx=0.0002)
    n2 = _collide(pipe, state, c)
    assert np.all(_mi(c, n2) >= 0)


def test_broken_normal_threshold(cuda):
    b = ModelBuilder()
    ba = b.add_body(xform=((0.0, 0.0, 0.0), ID))
    b.add_shape_sphere(ba, radius=0.1)
    bb = b.add_body(xform=((0.19, 0.0, 0.0), ID))
    b.add_shape_sphere(bb, radius=0.1)
    model = b.finalize(device="cuda")
    state = model.state()
    pipe = CollisionPipeline(model, broad_phase="nxn", contact_matching="latest", contact_matching_pos_threshold=10.0,
                             contact_matching_normal_dot_threshold=0.5)
    c = pipe.contacts()
    assert _collide(pipe, state, c) > 0
    _shift(state, 1, xyz=(0.0, 0.19, 0.0))
    n2 = _collide(pipe, state, c)
    assert n2 > 0 and np.all(_mi(c, n2) == -2)


def test_contact_report_new_and_stable(cuda):
    model, state, _ = _simple_scene()
    pipe = CollisionPipeline(model, broad_phase="nxn", contact_matching="latest", contact_report=True)
    c = pipe.contacts()
    n1 = _collide(pipe, state, c)
    nn = int(c.rigid_contact_new_count.item())
    assert nn == n1
    np.testing.assert_array_equal(np.sort(c.rigid_contact_new_indices[:nn].cpu().numpy()),
                                  np.nonzero(_mi(c, n1) < 0)[0])
    _collide(pipe, state, c)
    assert int(c.rigid_contact_new_count.item()) == 0 and int(c.rigid_contact_broken_count.item()) == 0


def test_contact_report_broken_indices(cuda):
    model, state, _ = _simple_scene(xs=(-0.5, 0.5))
    pipe = CollisionPipeline(model, broad_phase="nxn", contact_matching="latest", contact_report=True)
    c = pipe.contacts()
    n1 = _collide(pipe, state, c)
    _shift(state, 1, xyz=(0.5, 0.0, 10.0))
    n2 = _collide(pipe, state, c)
    nb = int(c.rigid_contact_broken_count.item())
    assert n2 < n1 and nb > 0
    bi = c.rigid_contact_broken_indices[:nb].cpu().numpy()
    assert np.all((bi >= 0) & (bi < n1))


def test_options_and_allocation(cuda):
    model, state, _ = _simple_scene()
    p = CollisionPipeline(model, broad_phase="nxn", contact_matching="latest")
    assert p.deterministic and p.contact_matching == "latest"
    off = CollisionPipeline(model, broad_phase="nxn", deterministic=True)
    c = off.contacts()
    assert c.rigid_contact_match_index is None and c.rigid_contact_new_indices is None
    assert c.rigid_contact_broken_indices is None and off.contact_matching == "disabled"
    for bad in ("bogus", True):
        with pytest.raises(ValueError):
            CollisionPipeline(model, broad_phase="nxn", contact_matching=bad)
    with pytest.raises(ValueError):
        CollisionPipeline(model, broad_phase="nxn", contact_matching="disabled", contact_report=True)
    latest = CollisionPipeline(model, broad_phase="nxn", contact_matching="latest")
    latest.contacts()
    assert latest._prev_point0 is None
    sticky = CollisionPipeline(model, broad_phase="nxn", contact_matching="sticky")
    sticky.contacts()
    assert sticky._prev_point0 is not None


def test_dynamic_bodies_and_box_manifold_identity(cuda):
    b = ModelBuilder()
    ba = b.add_body(xform=((0.0, 0.0, 0.0), ID))
    b.add_shape_sphere(ba, radius=0.1)
    bb = b.add_body(xform=((0.19, 0.0, 0.0), ID))
    b.add_shape_sphere(bb, radius=0.1)
    b.add_ground_plane()
    box = b.add_body(xform=((2.0, 0.0, 0.15), ID))
    b.add_shape_box(box, hx=0.1, hy=0.1, hz=0.1)
    model = b.finalize(device="cuda")
    state = model.state()
    pipe = CollisionPipeline(model, broad_phase="nxn", contact_matching="latest")
    c = pipe.contacts()
    n1 = _collide(pipe, state, c)
    n2 = _collide(pipe, state, c)
    assert n1 == n2 and n1 > 2
    np.testing.assert_array_equal(_mi(c, n2), np.arange(n2, dtype=np.int32))


def test_sticky_replays_matched_rows(cuda):
    model, state, _ = _simple_scene()
    pipe = CollisionPipeline(model, broad_phase="nxn", contact_matching="sticky")
    c = pipe.contacts()
    n1 = _collide(pipe, state, c)
    snap = {f: getattr(c, f"rigid_contact_{f}")[:n1].clone() for f in ("point0", "point1", "offset0", "offset1",
                                                                        "normal")}
    _shift(state, None, dx=0.0001)
    fresh_pipe = CollisionPipeline(model, broad_phase="nxn")
    fresh = fresh_pipe.contacts()
    _collide(fresh_pipe, state, fresh)
    assert not torch.equal(fresh.rigid_contact_point0[:n1], snap["point0"])
    n2 = _collide(pipe, state, c)
    assert n2 == n1 and np.all(_mi(c, n2) >= 0)
    for f, v in snap.items():
        assert torch.equal(getattr(c, f"rigid_contact_{f}")[:n2], v), f
    # the solver records carry the replayed geometry too: a step sees the sticky contacts
    rec = c._seg["rec"][:n2].cpu().numpy()
    np.testing.assert_array_equal(rec[:, 0:3], snap["point0"].cpu().numpy())
    np.testing.assert_array_equal(rec[:, 8:11], snap["normal"].cpu().numpy())


def test_sticky_unmatched_rows_pass_through(cuda):
    model, state, new_shape = _simple_scene(xs=(-0.5, 0.5), extra=(0.0, 0.0, 10.0))
    pipe = CollisionPipeline(model, broad_phase="nxn", contact_matching="sticky")
    c = pipe.contacts()
    n1 = _collide(pipe, state, c)
    _shift(state, 2, xyz=(0.0, 0.0, 0.1))
    n2 = _collide(pipe, state, c)
    assert n2 > n1
    mi = _mi(c, n2)
    s0 = c.rigid_contact_shape0[:n2].cpu().numpy()
    s1 = c.rigid_contact_shape1[:n2].cpu().numpy()
    assert (((s0 == new_shape) | (s1 == new_shape)) & (mi < 0)).any()
    assert np.all(s0[mi >= 0] >= 0) and np.all(s1[mi >= 0] >= 0)


@pytest.mark.parametrize("mode", ["latest", "sticky"])
def test_matching_matches_oracle_along_trajectory(cuda, orc, mode):
    """Match indices, report and (sticky) replayed geometry equal the oracle's, bit for bit."""
    model, info = scenes.scene_c2(seed=9, worlds=24, nmin=8, nmax=30, device="cuda")
    pipe = CollisionPipeline(model, contact_matching=mode, contact_report=True,
                             contact_matching_pos_threshold=0.002)
    solver = SolverXPBD(model, iterations=info["iterations"])
    matcher = orc.Matcher(pos_threshold=0.002, sticky=(mode == "sticky"))
    s0, s1 = model.state(), model.state()
    c = pipe.contacts()
    dt = info["dt"] / info["substeps"]
    seen_matched = 0
    for step in range(40):
        s0.clear_forces()
        q = s0.body_q.cpu().numpy()
        pipe.collide(s0, c)
        torch.cuda.synchronize()
        n = int(c.rigid_contact_count.item())
        # oracle input: the freshly published (pre-replay) contacts are what the GPU matched;
        # rebuild them from a non-matching pipeline on the same poses
        ref_pipe = CollisionPipeline(model, deterministic=True) if step == 0 else ref_pipe
        rc = ref_pipe.contacts() if step == 0 else rc
        ref_pipe.collide(s0, rc)
        torch.cuda.synchronize()
        pub = {"count": n, "world_offset": rc._world_offset.cpu().numpy()}
        for f in ("sort_key", "point0", "point1", "offset0", "offset1", "normal", "shape0", "shape1"):
            pub[f] = getattr(rc, f"rigid_contact_{f}")[:n].cpu().numpy().copy()
        mi, new_idx, broken = matcher.step(model, pipe.layout, q, pub)
        np.testing.assert_array_equal(_mi(c, n), mi)
        nn = int(c.rigid_contact_new_count.item())
        nb = int(c.rigid_contact_broken_count.item())
        np.testing.assert_array_equal(np.sort(c.rigid_contact_new_indices[:nn].cpu().numpy()), new_idx)
        np.testing.assert_array_equal(np.sort(c.rigid_contact_broken_indices[:nb].cpu().numpy()), broken)
        for f in ("point0", "point1", "offset0", "offset1", "normal"):
            got = getattr(c, f"rigid_contact_{f}")[:n].cpu().numpy()
            assert np.array_equal(got.view(np.uint32), pub[f].view(np.uint32)), f
        seen_matched += int(np.sum(mi >= 0))
        solver.step(s0, s1, None, c, dt)
        s0, s1 = s1, s0
    assert seen_matched > 0
