"""Known-answer tests of the CPU oracle's narrow phase.

Expected values are the assertions of the reference's own tests:
newton/tests/test_collision_primitives.py (plane-sphere :429, sphere-sphere :505,
sphere-capsule :587, capsule-capsule :696, sphere-box :1136, plane-capsule :1251,
plane-box :1335, box-box :1529, box-box with margin :1613, capsule-box :1749,
box-box depths :1881) and
newton/tests/test_narrow_phase.py (sphere-box corner :591, box-box face :635,
edge :708, capsules :801-895, plane-capsule :1083, per-shape gap :1271) and
newton/tests/test_collision_pipeline.py (sphere-pair normal direction :590,
box-box quaternion perturbation :720).  Contacts here run the full pipeline path
(primitive routing, MPR/GJK, manifold, write_contact gap test) with gap 0 on
both shapes, i.e. the reference primitive with margin 0.
"""

import math

import numpy as np
import pytest

from newton_custom_contact_b200 import GeoType

P, S, C, B = int(GeoType.PLANE), int(GeoType.SPHERE), int(GeoType.CAPSULE), int(GeoType.BOX)
ID = [0.0, 0.0, 0.0, 1.0]


def xf(p, q=ID):
    return list(p) + list(q)


def run(orc, ta, pa, sa, tb, pb, sb, gap=0.0, qa=ID, qb=ID):
    return orc.collide_pair(ta, xf(pa, qa), sa, tb, xf(pb, qb), sb, gap_a=gap, gap_b=gap)


@pytest.mark.parametrize("z,n,dist", [(2.0, 0, None), (1.0, 4, 0.0), (0.9, 4, -0.1), (0.8, 4, -0.2),
                                      (0.7, 4, -0.3), (0.5, 4, -0.5)])
def test_plane_box(orc, z, n, dist):
    rows = run(orc, P, [0, 0, 0], [0, 0, 0], B, [0, 0, z], [1, 1, 1])
    assert rows.shape[0] == n
    for r in rows:
        # analytic: the box's bottom corners sit at depth z - 1 along the plane normal
        assert r[11] == pytest.approx(dist, abs=1e-5)
        assert r[6:9] == pytest.approx([0, 0, 1], abs=1e-6)


@pytest.mark.parametrize("z,dist", [(1.0, 0.0), (0.8, -0.2), (0.5, -0.5), (0.2, -0.8)])
def test_plane_sphere(orc, z, dist):
    rows = run(orc, P, [0, 0, 0], [0, 0, 0], S, [0, 0, z], [1, 0, 0])
    assert rows.shape[0] == 1
    assert rows[0, 11] == pytest.approx(dist, abs=1e-5)


def test_plane_sphere_separated_beyond_gap(orc):
    assert run(orc, P, [0, 0, 0], [0, 0, 0], S, [0, 0, 2.0], [1, 0, 0]).shape[0] == 0
    # within the summed gap the speculative contact is kept
    rows = run(orc, P, [0, 0, 0], [0, 0, 0], S, [0, 0, 1.5], [1, 0, 0], gap=0.3)
    assert rows.shape[0] == 1 and rows[0, 11] == pytest.approx(0.5, abs=1e-5)


@pytest.mark.parametrize("x2,r1,dist", [(2.0, 1.0, 0.0), (1.8, 1.0, -0.2), (1.5, 1.0, -0.5), (1.2, 1.0, -0.8),
                                        (1.5, 0.5, 0.0), (1.2, 0.5, -0.3)])
def test_sphere_sphere(orc, x2, r1, dist):
    rows = run(orc, S, [0, 0, 0], [r1, 0, 0], S, [x2, 0, 0], [1, 0, 0])
    assert rows.shape[0] == 1
    assert rows[0, 11] == pytest.approx(dist, abs=1e-5)
    assert rows[0, 6:9] == pytest.approx([1, 0, 0], abs=1e-6)


@pytest.mark.parametrize("p,r,dist", [([1.5, 0, 0], 0.5, 0.0), ([1.4, 0, 0], 0.5, -0.1), ([1.3, 0, 0], 0.5, -0.2),
                                      ([1.2, 0, 0], 0.5, -0.3), ([0, 0, 1.5], 0.5, 0.0), ([0, 0, 1.3], 0.5, -0.2),
                                      ([0, 0, 0.4], 0.3, -0.9)])
def test_sphere_box(orc, p, r, dist):
    rows = run(orc, S, p, [r, 0, 0], B, [0, 0, 0], [1, 1, 1])
    assert rows.shape[0] == 1
    # analytic: distance from the sphere's centre to the face minus the radius
    assert rows[0, 11] == pytest.approx(dist, abs=1e-5)


def test_box_box_separated_and_overlapping(orc):
    assert run(orc, B, [0, 0, 0], [1, 1, 1], B, [3.0, 0, 0], [1, 1, 1]).shape[0] == 0
    rows = run(orc, B, [0, 0, 0], [1, 1, 1], B, [1.5, 0, 0], [1, 1, 1])
    assert rows.shape[0] > 0
    for r in rows:
        assert np.linalg.norm(r[6:9]) == pytest.approx(1.0, abs=0.01)
        assert np.dot(r[6:9], [1, 0, 0]) > -0.1


def test_box_box_face_depth(orc):
    rows = run(orc, B, [0, 0, 0], [1, 1, 1], B, [1.8, 0, 0], [1, 1, 1])
    assert rows.shape[0] > 0
    xs = [r for r in rows if abs(r[6]) > 0.9]
    assert xs, "expected a contact with an x-axis normal"
    for r in xs:
        assert r[11] == pytest.approx(-0.2, abs=0.05)
        assert r[6] > 0


@pytest.mark.parametrize("z,dist", [(1.1, 0.1), (1.0, 0.0), (0.9, -0.1), (0.8, -0.2), (0.7, -0.3)])
def test_box_box_face_steps(orc, z, dist):
    rows = run(orc, B, [0, 0, 0], [0.5, 0.5, 0.5], B, [0, 0, z], [0.5, 0.5, 0.5], gap=0.1)
    assert rows.shape[0] >= 1
    deepest = rows[:, 11].min()
    assert deepest == pytest.approx(dist, abs=0.02)
    assert np.all(rows[:, 8] > 0.99)


def test_box_box_edge(orc):
    a = math.pi / 4
    rows = run(orc, B, [0, 0, 0], [0.5, 0.5, 0.5], B, [1.2, 0, 0], [0.5, 0.5, 0.5],
               qb=[0, 0, math.sin(a / 2), math.cos(a / 2)])
    assert rows.shape[0] > 0
    assert np.linalg.norm(rows[0, 6:9]) == pytest.approx(1.0, abs=1e-5)


def test_capsule_capsule_parallel_two_contacts(orc):
    # both along z, side by side: the parallel branch emits two contacts
    rows = run(orc, C, [0, 0, 0], [0.5, 1.0, 0], C, [0.9, 0, 0], [0.5, 1.0, 0])
    assert rows.shape[0] == 2
    assert np.allclose(rows[:, 11], -0.1, atol=1e-5)


def test_capsule_capsule_crossed_one_contact(orc):
    qx = [math.sin(math.pi / 4), 0, 0, math.cos(math.pi / 4)]
    rows = run(orc, C, [0, 0, 0], [0.5, 1.0, 0], C, [0.9, 0, 0], [0.5, 1.0, 0], qb=qx)
    assert rows.shape[0] == 1
    assert rows[0, 11] == pytest.approx(-0.1, abs=1e-5)


def test_plane_capsule_resting(orc):
    qx = [math.sin(math.pi / 4), 0, 0, math.cos(math.pi / 4)]  # axis along y, lying on the plane
    rows = run(orc, P, [0, 0, 0], [0, 0, 0], C, [0, 0, 0.5], [0.5, 1.0, 0], qb=qx)
    assert rows.shape[0] == 2
    assert np.allclose(rows[:, 11], 0.0, atol=1e-5)


def test_capsule_box_gjk(orc):
    # capsule lying on top of a box face: routed to MPR/GJK + manifold
    qx = [math.sin(math.pi / 4), 0, 0, math.cos(math.pi / 4)]
    rows = run(orc, C, [0, 0, 1.45], [0.5, 0.5, 0], B, [0, 0, 0], [1, 1, 1], qa=qx)
    assert rows.shape[0] >= 1
    assert rows[:, 11].min() == pytest.approx(-0.05, abs=0.01)


def test_sort_sub_keys(orc):
    # plane-box writes sub keys 0..3; manifold sub keys (0 << 3) | i
    rows = run(orc, P, [0, 0, 0], [0, 0, 0], B, [0, 0, 0.9], [1, 1, 1])
    assert sorted(rows[:, 12].astype(int).tolist()) == [0, 1, 2, 3]
    rows = run(orc, B, [0, 0, 0], [0.5, 0.5, 0.5], B, [0, 0, 0.95], [0.5, 0.5, 0.5], gap=0.1)
    subs = rows[:, 12].astype(int)
    assert np.all(np.diff(subs) > 0) and subs.max() <= 4


# ---- more of newton/tests/test_collision_primitives.py: sphere-capsule :587,
# capsule-capsule :696, plane-capsule :1251, box-box with margin :1613,
# capsule-box :1749 (the reference's distances are checked within its own
# tolerances; separated cases need a summed gap larger than the distance)

QY90 = [0.0, math.sin(math.pi / 4), 0.0, math.cos(math.pi / 4)]   # local z -> world x
QX90 = [math.sin(math.pi / 4), 0.0, 0.0, math.cos(math.pi / 4)]   # local z -> world -y


def _dist_to_capsule(p, c, axis, r, hh):
    p, c, axis = np.asarray(p, float), np.asarray(c, float), np.asarray(axis, float)
    t = np.clip(np.dot(p - c, axis), -hh, hh)
    return abs(np.linalg.norm(p - (c + t * axis)) - r)


@pytest.mark.parametrize("p,dist", [([0, 1.5, 0], 0.5), ([0, 1.0, 0], 0.0), ([0, 0.9, 0], -0.1), ([0, 0.8, 0], -0.2),
                                    ([0, 0, 2.5], 0.5), ([0, 0, 2.0], 0.0), ([0, 0, 1.9], -0.1), ([0, 0, 1.8], -0.2)])
def test_sphere_capsule(orc, p, dist):
    gap = 0.3 if dist > 0 else 0.0
    rows = run(orc, S, p, [0.5, 0, 0], C, [0, 0, 0], [0.5, 1.0, 0], gap=gap)
    assert rows.shape[0] == 1
    r = rows[0]
    assert r[11] == pytest.approx(dist, abs=0.01)
    n = r[6:9]
    assert np.dot(n, -np.asarray(p, float)) > 0.99 * np.linalg.norm(p)  # from the sphere into the capsule
    if dist < 0:
        on_sphere = r[0:3] + n * r[9]
        on_capsule = r[3:6] - n * r[10]
        assert abs(np.linalg.norm(on_sphere - np.asarray(p, float)) - 0.5) < 0.05
        assert _dist_to_capsule(on_capsule, [0, 0, 0], [0, 0, 1], 0.5, 1.0) < 0.05
    assert run(orc, S, p, [0.5, 0, 0], C, [0, 0, 0], [0.5, 1.0, 0]).shape[0] == (0 if dist > 0 else 1)


@pytest.mark.parametrize("y,dist", [(2.0, 1.0), (1.5, 0.5), (1.0, 0.0), (0.9, -0.1), (0.8, -0.2), (0.6, -0.4)])
def test_capsule_capsule_parallel(orc, y, dist):
    gap = 0.6 if dist > 0 else 0.0
    rows = run(orc, C, [0, 0, 0], [0.5, 1.0, 0], C, [0, y, 0], [0.5, 1.0, 0], gap=gap, qa=QY90, qb=QY90)
    assert rows.shape[0] >= 1
    assert np.allclose(rows[:, 11], dist, atol=0.01)
    assert np.all(rows[:, 7] > 0.99)  # normal along +y, from the first capsule into the second


def test_capsule_capsule_perpendicular_through_centre(orc):
    rows = run(orc, C, [0, 0, 0], [0.5, 1.0, 0], C, [0, 0, 0], [0.5, 1.0, 0], qa=QY90, qb=QX90)
    assert rows.shape[0] >= 1
    assert rows[0, 11] == pytest.approx(-1.0, abs=0.01)


@pytest.mark.parametrize("z,dist", [(2.0, 1.5), (1.5, 1.0), (1.0, 0.5), (0.5, 0.0), (0.4, -0.1), (0.3, -0.2),
                                    (0.2, -0.3)])
def test_plane_capsule_horizontal(orc, z, dist):
    gap = 0.8 if dist > 0 else 0.0
    rows = run(orc, P, [0, 0, 0], [0, 0, 0], C, [0, 0, z], [0.5, 1.0, 0], gap=gap, qb=QY90)
    assert rows.shape[0] == 2  # one contact per end of the horizontal capsule
    assert np.allclose(rows[:, 11], dist, atol=0.01)
    assert np.all(rows[:, 8] > 0.99)


@pytest.mark.parametrize("gap_sum,contacts", [(0.0, False), (0.3, True), (0.1, False)])
def test_box_box_margin(orc, gap_sum, contacts):
    # stacked boxes 0.2 apart: a contact only when the contact threshold exceeds the gap
    rows = run(orc, B, [0, 0, 0], [0.5, 0.5, 0.5], B, [0, 0, 1.2], [0.5, 0.5, 0.5], gap=0.5 * gap_sum)
    assert (rows.shape[0] > 0) == contacts
    if contacts:
        assert np.allclose(rows[:, 11], 0.2, atol=0.01)
        assert np.all(rows[:, 8] > 0.99)


@pytest.mark.parametrize("z,dist", [(3.0, 0.5), (2.5, 0.0), (2.4, -0.1), (2.3, -0.2), (2.2, -0.3)])
def test_capsule_box_upright(orc, z, dist):
    gap = 0.3 if dist > 0 else 0.0
    rows = run(orc, C, [0, 0, z], [0.5, 1.0, 0], B, [0, 0, 0], [1, 1, 1], gap=gap)
    assert rows.shape[0] >= 1
    assert rows[:, 11].min() == pytest.approx(dist, abs=0.05)
    assert np.all(rows[:, 8] < -0.99)  # from the capsule down into the box


# ---- newton/tests/test_narrow_phase.py: sphere-box corner :591, per-shape gap :1271

def _dist_to_box(p, half):
    q = np.abs(np.asarray(p, float)) - np.asarray(half, float)
    outside = np.linalg.norm(np.maximum(q, 0.0))
    return outside if outside > 0.0 else -q.max()  # inside: distance to the nearest face


def test_sphere_box_corner(orc):
    c = np.ones(3) / np.sqrt(3.0) * 1.5
    rows = run(orc, S, c, [0.5, 0, 0], B, [0, 0, 0], [1, 1, 1])
    assert rows.shape[0] == 1
    r = rows[0]
    n = r[6:9]
    assert np.linalg.norm(n) == pytest.approx(1.0, abs=0.01)
    # the centre (0.866, 0.866, 0.866) lies inside the box: pushed out through the nearest
    # face, depth -(1 - 0.866 + r)
    assert r[11] == pytest.approx(-(1.0 - c[0] + 0.5), abs=0.01)
    on_sphere = r[0:3] + n * r[9]
    on_box = r[3:6] - n * r[10]
    assert abs(np.linalg.norm(on_sphere - c) - 0.5) < 0.05
    assert abs(_dist_to_box(on_box, [1, 1, 1])) < 0.05


@pytest.mark.parametrize("z,gap_sphere,contact", [(0.25, 0.02, False), (0.15, 0.02, True), (0.23, 0.06, True)])
def test_per_shape_gap(orc, z, gap_sphere, contact):
    # plane gap 0.01; a sphere of radius 0.2 has a contact only within the summed gap
    rows = orc.collide_pair(P, xf([0, 0, 0]), [0, 0, 0], S, xf([0, 0, z]), [0.2, 0, 0], gap_a=0.01,
                            gap_b=gap_sphere)
    assert (rows.shape[0] == 1) == contact
    if contact:
        assert rows[0, 11] == pytest.approx(z - 0.2, abs=1e-5)


# ---- newton/tests/test_collision_pipeline.py:590-717 (contact normal direction for
# sphere pairs) and :720-771 (box-box under a 1e-14 quaternion perturbation), through
# the pipeline's oracle with a model of free bodies

def _model_contacts(orc, model):
    from newton_custom_contact_b200 import CollisionPipeline

    pipe = CollisionPipeline(model)
    segs = orc.collide(model, pipe.layout, model.host("body_q"))
    return orc.contacts_table(model, pipe.layout, segs)


def test_sphere_pair_normals_point_from_shape0_to_shape1(orc):
    from newton_custom_contact_b200 import ModelBuilder

    half_dists, ys, expect = [0.3, 0.5, 0.54, 0.75], [0.0, 3.0, 6.0, 9.0], [True, True, True, False]
    b = ModelBuilder(gravity=0.0)
    b.rigid_gap = 0.05
    centres = []
    for hd, y in zip(half_dists, ys):
        for x in (-hd, hd):
            centres.append((x, y, 0.0))
            b.add_shape_sphere(b.add_body(xform=[x, y, 0.0, 0.0, 0.0, 0.0, 1.0]), radius=0.5)
    model = b.finalize(device="cpu")
    tab = _model_contacts(orc, model)
    centres = np.asarray(centres)
    per_pair = {k: [r for r in tab if int(r[1]) // 2 == k] for k in range(4)}
    for k in range(4):
        assert (len(per_pair[k]) > 0) == expect[k]
        for r in per_pair[k]:
            s0, s1 = int(r[1]), int(r[2])
            n = r[10:13]
            assert np.linalg.norm(n) == pytest.approx(1.0, abs=1e-3)
            d = centres[s1] - centres[s0]
            assert np.dot(n, d / np.linalg.norm(d)) > 0.95
            mid = 0.5 * ((r[4:7] + centres[s0]) + (r[7:10] + centres[s1]))
            lo, hi = min(centres[s0, 0], centres[s1, 0]), max(centres[s0, 0], centres[s1, 0])
            assert lo - 1e-3 <= mid[0] <= hi + 1e-3


def test_box_box_quaternion_perturbation(orc):
    """Face-to-face cubes rotated 30 deg about x, the second with a 1e-14 quaternion
    perturbation: four face-corner contacts, body-frame points inside the cube, normals
    along x (the support deadband of support_function.py:39)."""
    from newton_custom_contact_b200 import ModelBuilder

    half = 0.495
    q_clean = [0.2588233343021173, 0.0, 0.0, 0.9659246769912934]
    q_noisy = [0.2588233343021173, -2.27e-14, 9.25e-15, 0.9659246769912934]
    y, z = 6.680443286895752, 4.4285125732421875
    b = ModelBuilder()
    b.add_shape_box(b.add_body(xform=[half, y, z] + q_clean), hx=half, hy=half, hz=half)
    b.add_shape_box(b.add_body(xform=[-half, y, z] + q_noisy), hx=half, hy=half, hz=half)
    model = b.finalize(device="cpu")
    tab = _model_contacts(orc, model)
    assert tab.shape[0] == 4
    for r in tab:
        assert np.all(np.abs(r[4:7]) <= half * 1.01)
        assert abs(r[10]) == pytest.approx(1.0, abs=0.01)
