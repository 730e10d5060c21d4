"""The vectorised scene assembler against the ModelBuilder path.

``scenes.assemble_free_bodies`` builds the free-body benchmark scenes as model
arrays directly; these tests build the same bodies with ``ModelBuilder`` (one
body + one shape each, a free joint to world, a shared ground plane) and
require identical model arrays and the same explicit contact-pair set
(builder.py:10855-10913; free joints to world do not filter the ground,
builder.py:1258-1263).
"""

import numpy as np
import pytest

from newton_custom_contact_b200 import GeoType, ModelBuilder, scenes


def _builder_scene(body_world, types, scales, poses, mu, worlds):
    b = ModelBuilder()
    plane_cfg = ModelBuilder.ShapeConfig()
    plane_cfg.mu = 0.5
    b.add_ground_plane(cfg=plane_cfg)
    for w in range(worlds):
        b.begin_world()
        for i in np.nonzero(body_world == w)[0]:
            cfg = ModelBuilder.ShapeConfig()
            cfg.mu = float(mu[i])
            body = b.add_body(xform=(tuple(poses[i, :3]), tuple(poses[i, 3:])))
            t = int(types[i])
            if t == int(GeoType.BOX):
                b.add_shape_box(body, hx=scales[i, 0], hy=scales[i, 1], hz=scales[i, 2], cfg=cfg)
            elif t == int(GeoType.SPHERE):
                b.add_shape_sphere(body, radius=scales[i, 0], cfg=cfg)
            else:
                b.add_shape_capsule(body, radius=scales[i, 0], half_height=scales[i, 1], cfg=cfg)
        b.end_world()
    return b.finalize(device="cpu")


def _random_bodies(seed=3, worlds=3, n=5):
    rng = np.random.default_rng(seed)
    bw = np.repeat(np.arange(worlds), n)
    types = rng.choice([int(GeoType.BOX), int(GeoType.SPHERE), int(GeoType.CAPSULE)], size=bw.size)
    scales = np.zeros((bw.size, 3))
    scales[:, 0] = rng.uniform(0.03, 0.2, bw.size)
    scales[:, 1] = rng.uniform(0.05, 0.2, bw.size)
    scales[:, 2] = rng.uniform(0.03, 0.2, bw.size)
    scales[types == int(GeoType.SPHERE), 1:] = 0.0
    scales[types == int(GeoType.CAPSULE), 2] = 0.0
    q = scenes.random_quats(rng, bw.size)
    poses = np.concatenate([rng.uniform(-0.5, 0.5, (bw.size, 3)) + [0, 0, 1.0], q], axis=1)
    mu = rng.uniform(0.3, 1.0, bw.size)
    return bw, types, scales, poses, mu, worlds


@pytest.mark.parametrize("seed", [3, 4])
def test_assembler_matches_builder(seed):
    bw, types, scales, poses, mu, W = _random_bodies(seed)
    a = scenes.assemble_free_bodies(bw, types, scales, poses, mu, W, plane_mu=0.5, device="cpu")
    b = _builder_scene(bw, types, scales, poses, mu, W)
    assert a.body_count == b.body_count and a.shape_count == b.shape_count and a.world_count == b.world_count
    for name in ("body_q", "body_inv_mass", "body_inertia", "body_world", "shape_body", "shape_type",
                 "shape_scale", "shape_material_mu", "shape_gap", "shape_world", "joint_type", "joint_parent",
                 "joint_child", "joint_qd_start"):
        np.testing.assert_allclose(a.host(name), b.host(name), rtol=1e-5, atol=1e-6, err_msg=name)
    np.testing.assert_allclose(a.host("body_inv_inertia"), b.host("body_inv_inertia"), rtol=1e-4, atol=1e-3)
    pa = {tuple(p) for p in a.host("shape_contact_pairs").tolist()}
    pb = {tuple(p) for p in b.host("shape_contact_pairs").tolist()}
    assert pa == pb
    # every body shape pairs with the ground plane (shape 0)
    assert all((0, s) in pb for s in range(1, b.shape_count))


def test_fixed_joint_to_world_filters_ground():
    b = ModelBuilder()
    b.add_ground_plane()
    body = b.add_link(xform=((0.0, 0.0, 1.0), (0.0, 0.0, 0.0, 1.0)))
    b.add_shape_sphere(body, radius=0.1)
    b.add_joint_fixed(-1, body)
    other = b.add_body(xform=((0.0, 0.0, 2.0), (0.0, 0.0, 0.0, 1.0)))
    b.add_shape_sphere(other, radius=0.1)
    pairs = {tuple(p) for p in b.find_shape_contact_pairs().tolist()}
    assert (0, 1) not in pairs and (0, 2) in pairs and (1, 2) in pairs


def test_desc_all_joints_free():
    """NbModelDesc.all_joints_free (which lets the step use its lean kernel) is 1 only when
    every joint is FREE: the free-body scenes, not the revolute arms."""
    bw, types, scales, poses, mu, W = _random_bodies(3)
    free = scenes.assemble_free_bodies(bw, types, scales, poses, mu, W, plane_mu=0.5, device="cpu")
    assert free.make_desc(free.host_arrays()).all_joints_free == 1
    arms, _ = scenes.scene_c3(worlds=2, device="cpu")
    assert arms.make_desc(arms.host_arrays()).all_joints_free == 0
    b = ModelBuilder()
    b.add_ground_plane()
    body = b.add_link(xform=((0.0, 0.0, 1.0), (0.0, 0.0, 0.0, 1.0)))
    b.add_shape_sphere(body, radius=0.1)
    b.add_joint_fixed(-1, body)
    fixed = b.finalize(device="cpu")
    assert fixed.make_desc(fixed.host_arrays()).all_joints_free == 0


def test_c1_batch_worlds_are_c1_scenes():
    """scene_c1_batch(seed, W): world w holds exactly scene_c1(seed + w)'s boxes and poses."""
    batch, info = scenes.scene_c1_batch(seed=100, worlds=5, device="cpu")
    assert batch.world_count == 5 and batch.body_count == 5 * 64
    hb = batch.host_arrays()
    for w in (0, 3):
        one, _ = scenes.scene_c1(seed=100 + w, device="cpu")
        h1 = one.host_arrays()
        sl = slice(64 * w, 64 * (w + 1))
        assert np.array_equal(hb["body_q"][sl], h1["body_q"])
        assert np.array_equal(hb["body_inv_mass"][sl], h1["body_inv_mass"])
        assert np.array_equal(hb["shape_scale"][1 + 64 * w:1 + 64 * (w + 1)], h1["shape_scale"][1:])
    assert info["substeps"] == 10 and info["iterations"] == 4
