"""Host-side logic of CollisionPipeline, checked on CPU against the reference's own tests.

* Contact capacity estimate: newton/tests/test_collision_pipeline.py:796-865
  (TestContactEstimator, the cases with primitive shapes only; the estimate
  follows newton/_src/sim/collide.py:278-376).
* Candidate-pair count per world: :866-979 (TestShapePairsMaxScaling: the
  pair set grows linearly with the world count, global shapes join every
  world's segment).
* Constructor errors: newton/_src/sim/collide.py:587-603.
* Shape collision filter pairs: :460-573 (an excluded pair makes no contacts; the
  explicit, NxN and SAP modes report the same pairs).
* Candidate pairs across worlds and collision groups: newton/tests/test_broad_phase.py:
  22-68, 271-428 (the builder's explicit list and the NxN list against the rule).
* Per-shape gaps in the broad and narrow phase: test_broad_phase.py:2024-2130.
"""

import numpy as np
import pytest

from newton_custom_contact_b200 import CollisionPipeline, GeoType, ModelBuilder
from newton_custom_contact_b200.collide import _estimate_rigid_contact_max


class _Shapes:
    """The fields the estimate reads: shape types and worlds, world count, pair count."""

    def __init__(self, shape_type, shape_world, world_count, pair_count):
        self._h = {"shape_type": np.asarray(shape_type, np.int32), "shape_world": np.asarray(shape_world, np.int32)}
        self.world_count = world_count
        self.shape_contact_pair_count = pair_count

    def host_arrays(self):
        return self._h


def test_estimate_world_aware_planes():
    # 4 worlds of 10 boxes and 10 planes: 40*20*5 // 2 = 2000 box contacts and
    # 4 * (10 * 10) plane pairs * 5 = 2000 plane contacts, not a cross-world square
    st = ([int(GeoType.BOX)] * 10 + [int(GeoType.PLANE)] * 10) * 4
    sw = np.repeat(np.arange(4), 20)
    assert _estimate_rigid_contact_max(_Shapes(st, sw, 4, 0)) == 4000


def test_estimate_pair_count_tighter_than_heuristic():
    # 40 boxes in 4 worlds: heuristic 2000, 300 known pairs * 5 = 1500
    st = [int(GeoType.BOX)] * 40
    sw = np.repeat(np.arange(4), 10)
    assert _estimate_rigid_contact_max(_Shapes(st, sw, 4, 300)) == 1500


def test_estimate_floor_and_no_shapes():
    assert _estimate_rigid_contact_max(_Shapes([], [], 1, 0)) == 1000
    assert _estimate_rigid_contact_max(_Shapes([int(GeoType.SPHERE)] * 3, [0, 0, 0], 1, 0)) == 1000


def _worlds_of_boxes(worlds, per_world, ground=False):
    rb = ModelBuilder()
    for _ in range(per_world):
        b = rb.add_body()
        rb.add_shape_box(body=b, hx=0.1, hy=0.1, hz=0.1)
    mb = ModelBuilder()
    if ground:
        mb.add_ground_plane()
    for _ in range(worlds):
        mb.add_world(rb)
    return mb.finalize(device="cpu")


@pytest.mark.parametrize("broad_phase", ["explicit", "nxn", "sap"])
def test_shape_pairs_scale_linearly_with_worlds(broad_phase):
    for worlds in (1, 2, 4, 64):
        model = _worlds_of_boxes(worlds, 5)
        pipe = CollisionPipeline(model, broad_phase=broad_phase)
        assert pipe.shape_pairs_max == worlds * (5 * 4 // 2)
    n = model.shape_count
    assert pipe.shape_pairs_max < n * (n - 1) // 2 / 10


@pytest.mark.parametrize("broad_phase", ["explicit", "nxn", "sap"])
def test_global_shape_joins_every_world(broad_phase):
    # each world: 3 boxes + the global ground plane -> 3 box pairs + 3 plane pairs
    model = _worlds_of_boxes(2, 3, ground=True)
    assert CollisionPipeline(model, broad_phase=broad_phase).shape_pairs_max == 2 * 6


def test_constructor_errors():
    model = _worlds_of_boxes(1, 2)
    with pytest.raises(ValueError):
        CollisionPipeline(model, broad_phase="octree")
    with pytest.raises(ValueError):
        CollisionPipeline(model, shape_pairs_max=0)
    with pytest.raises(ValueError):
        CollisionPipeline(model, max_triangle_pairs=0)
    with pytest.raises(ValueError):
        CollisionPipeline(model, contact_matching="always")
    with pytest.raises(ValueError):
        CollisionPipeline(model, contact_report=True)
    with pytest.raises(NotImplementedError):
        CollisionPipeline(model, sdf_hydroelastic_config=object())


# ---- newton/tests/test_collision_pipeline.py:460-573: excluded shape pairs make no
# contacts, and every broad-phase mode reports the same contacting pairs (the
# contacts come from the CPU oracle of the pipeline here)

def _overlapping_spheres(n, exclude):
    b = ModelBuilder(gravity=0.0)
    b.rigid_gap = 0.01
    shapes = []
    for _ in range(n):
        body = b.add_body(xform=[0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 1.0])
        shapes.append(b.add_shape_sphere(body=body, radius=0.5))
    a, c = shapes[exclude[0]], shapes[exclude[1]]
    b.shape_collision_filter_pairs.append((min(a, c), max(a, c)))  # appended, as the reference test does
    return b.finalize(device="cpu"), (min(a, c), max(a, c))


def _contact_pairs(orc, model, broad_phase):
    pipe = CollisionPipeline(model, broad_phase=broad_phase)
    segs = orc.collide(model, pipe.layout, model.host("body_q"))
    tab = orc.contacts_table(model, pipe.layout, segs)
    return {(min(int(r[1]), int(r[2])), max(int(r[1]), int(r[2]))) for r in tab}


@pytest.mark.parametrize("broad_phase", ["nxn", "sap", "explicit"])
def test_filtered_pair_makes_no_contacts(orc, broad_phase):
    model, _ = _overlapping_spheres(2, (0, 1))
    assert _contact_pairs(orc, model, broad_phase) == set()


def test_filter_consistent_across_broad_phases(orc):
    model, excluded = _overlapping_spheres(3, (0, 1))
    sets = {bp: _contact_pairs(orc, model, bp) for bp in ("explicit", "nxn", "sap")}
    for pairs in sets.values():
        assert excluded not in pairs
        assert len(pairs) == 2
    assert sets["explicit"] == sets["nxn"] == sets["sap"]


# ---- newton/tests/test_broad_phase.py:22-68 and :271-428: the candidate pairs across
# worlds and collision groups (positive groups collide with themselves and with
# negative groups, a negative group with everything but itself, group 0 with nothing;
# world -1 shapes with every world; shapes of one body, the static ones included,
# never pair: builder.py:5539-5542)

def _group_pair(a, b):
    if a == 0 or b == 0:
        return False
    return (a == b or b < 0) if a > 0 else a != b


def _world_group_pair(wa, wb, ga, gb):
    if wa != -1 and wb != -1 and wa != wb:
        return False
    return _group_pair(ga, gb)


@pytest.mark.parametrize("seed", [123, 7])
def test_pairs_follow_world_and_group_rules(seed):
    from newton_custom_contact_b200.collide import nxn_pairs

    rng = np.random.Generator(np.random.PCG64(seed))
    worlds, per_world, n_global = 4, 10, 5
    groups = rng.integers(1, 6, size=worlds * per_world + n_global)
    groups[rng.choice(groups.size, size=int(np.sqrt(groups.size)), replace=False)] = -1
    groups[rng.choice(groups.size, size=2, replace=False)] = 0
    b = ModelBuilder()
    meta = []  # (shape, world, group, body)
    k = 0
    for _ in range(n_global):  # static shapes outside any world
        g = int(groups[k])
        k += 1
        s = b.add_shape_box(-1, xform=list(rng.random(3) * 5.0) + [0.0, 0.0, 0.0, 1.0], hx=0.2, hy=0.2, hz=0.2,
                            cfg=ModelBuilder.ShapeConfig(collision_group=g))
        meta.append((s, -1, g, -1))
    for w in range(worlds):
        b.begin_world()
        for _ in range(per_world):
            g = int(groups[k])
            k += 1
            body = b.add_body(xform=list(rng.random(3) * 5.0) + [0.0, 0.0, 0.0, 1.0])
            s = b.add_shape_sphere(body, radius=0.2, cfg=ModelBuilder.ShapeConfig(collision_group=g))
            meta.append((s, w, g, body))
        b.end_world()
    want = set()
    for i in range(len(meta)):
        for j in range(i + 1, len(meta)):
            (sa, wa, ga, ba), (sb, wb, gb, bb) = meta[i], meta[j]
            if ba != bb and _world_group_pair(wa, wb, ga, gb):
                want.add((min(sa, sb), max(sa, sb)))
    model = b.finalize(device="cpu")
    explicit = {tuple(p) for p in model.host("shape_contact_pairs").tolist()}
    nxn = {tuple(p) for p in np.asarray(nxn_pairs(model)).reshape(-1, 2).tolist()}
    assert explicit == want
    assert nxn == want
    # the draw exercises every rule: global-world pairs, negative and zero groups
    assert any(-1 in (meta[a][1], meta[b][1]) for a, b in [(0, len(meta) - 1)])
    assert (groups < 0).any() and (groups == 0).any()


def test_per_shape_gap_through_the_pipeline(orc):
    """newton/tests/test_broad_phase.py:2024-2130: two spheres (r 0.2) hover 0.04 above the
    ground (gap 0.01); A with gap 0.02 (summed 0.03) gets no contact, B with gap 0.06
    (summed 0.07) does, with separation 0.04 -- the broad phase and the narrow phase
    of the pipeline both apply each shape's own gap."""
    b = ModelBuilder(gravity=0.0)
    b.add_ground_plane(cfg=ModelBuilder.ShapeConfig(gap=0.01))
    a = b.add_shape_sphere(b.add_body(xform=[0.0, 0.0, 0.24, 0.0, 0.0, 0.0, 1.0]), radius=0.2,
                           cfg=ModelBuilder.ShapeConfig(gap=0.02))
    c = b.add_shape_sphere(b.add_body(xform=[10.0, 0.0, 0.24, 0.0, 0.0, 0.0, 1.0]), radius=0.2,
                           cfg=ModelBuilder.ShapeConfig(gap=0.06))
    model = b.finalize(device="cpu")
    pipe = CollisionPipeline(model)
    segs = orc.collide(model, pipe.layout, model.host("body_q"))
    tab = orc.contacts_table(model, pipe.layout, segs)
    shapes = {int(r[1]) for r in tab} | {int(r[2]) for r in tab}
    assert c in shapes and a not in shapes
    row = [r for r in tab if c in (int(r[1]), int(r[2]))][0]
    n, p0, p1 = row[10:13], row[4:7], row[7:10]
    # ground point in world space (static: body frame = world) and sphere centre offset
    centre = np.array([10.0, 0.0, 0.24])
    sep = abs(float(np.dot(n, (p1 + centre if int(row[2]) == c else p1) - (p0 + centre if int(row[1]) == c else p0))))
    assert sep - (row[19] + row[20]) == pytest.approx(0.04, abs=1e-5)


def test_sap_pair_table_indexes_the_pair_list():
    """The sweep-and-prune pair table: for every listed pair both orientations of its slots give its
    index in the pair list, and every other slot pair gives -1."""
    from newton_custom_contact_b200 import scenes

    model, _ = scenes.scene_c2(seed=5, worlds=6, nmin=8, nmax=20, device="cpu")
    pipe = CollisionPipeline(model, broad_phase="sap")
    lay = pipe.layout
    table, start = lay.pair_table(model)
    nloc = np.diff(model._part["world_shape_start"].astype(np.int64))
    ns = nloc + model._part["global_shapes"].size
    assert start[-1] == int(np.sum(ns * ns))
    wps = lay.world_pair_start.astype(np.int64)
    for w in range(model.world_count):
        t = table[start[w]:start[w + 1]].reshape(ns[w], ns[w])
        expect = np.full((ns[w], ns[w]), -1, np.int32)
        for p in range(wps[w], wps[w + 1]):
            a, b = lay.pair_slots[p]
            expect[a, b] = expect[b, a] = p
        assert np.array_equal(t, expect)
    assert "pair_table" in pipe._layout_dev
