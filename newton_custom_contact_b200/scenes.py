"""Seeded synthetic scenes of the benchmark configurations.

No dataset is involved: every scene is generated from a seed.  Free-body
scenes are assembled directly as model arrays (vectorised; the Python
ModelBuilder would take minutes for 4096 worlds) with exactly the
ModelBuilder semantics: one shape per body at the body origin, density
1000 kg/m^3 inertia (newton/_src/geometry/inertia.py), a free joint per body
(builder.py:3649-3722), the shared ground plane as shape 0 in world -1 with
the infinite-plane bounding radius 1e6 (geometry/utils.py:98-102), gap 0.1
(builder.py:1165) and the builder's explicit pair list (builder.py:10855-10913).
``tests/test_scenes.py`` checks the assembler against the ModelBuilder path.

  C1  1 world, 64 boxes (half-extents U[0.05,0.15]^3) on a jittered 4x4x4
      grid over [-0.5,0.5]^2 x [0.2,2.0], uniform random orientation, mu 0.5.
  C2  4096 worlds of N ~ U{8..128} bodies; box / sphere / capsule uniform;
      poses in a 1 x 1 x 2 m column with bounding-sphere rejection, bounding
      sphere above the plane; mu per world U[0.3,1.0]; shared ground plane (mu 0.5).
  C3  4096 worlds: 7-link revolute capsule arm (r 0.04, length 0.3, 1 kg,
      limits +-2.5 rad, drive ke 500 kd 20, sinusoid targets) reaching into
      8..48 loose boxes (half-extent U[0.03,0.08]) on a table plane.
  C5  1024 worlds of 16-box stacks (half-extent 0.1, lateral jitter +-1 cm,
      mu U[0.4,0.8]), initial twists N(0, 0.1).
  falling shapes  the scene of newton/tests/test_shapes_no_bounce.py with the
      shapes this solver collides (spheres, boxes, capsules in turn), every
      world the same grid.
"""

from __future__ import annotations

import math

import numpy as np

from ._abi import BodyFlags, GeoType, JointType, ShapeFlags
from .builder import ModelBuilder, compute_inertia_shape, compute_shape_radius, quat_from_axis_angle
from .model import Model

_SHAPE_FLAGS = int(ShapeFlags.VISIBLE | ShapeFlags.COLLIDE_SHAPES | ShapeFlags.COLLIDE_PARTICLES)


def random_quats(rng: np.random.Generator, n: int) -> np.ndarray:
    q = rng.normal(size=(n, 4))
    q /= np.linalg.norm(q, axis=1, keepdims=True)
    return q


def _inertia_batch(types, scales, density=1000.0):
    """Vectorised compute_inertia_shape for solid boxes, spheres and capsules (inertia.py:42-245)."""
    n = types.shape[0]
    mass = np.zeros(n)
    diag = np.zeros((n, 3))
    s = np.asarray(scales, dtype=np.float64)
    bx = types == int(GeoType.BOX)
    m = density * (8.0 * s[bx, 0] * s[bx, 1] * s[bx, 2])
    mass[bx] = m
    diag[bx] = np.stack([1.0 / 3.0 * m * (s[bx, 1] ** 2 + s[bx, 2] ** 2), 1.0 / 3.0 * m * (s[bx, 0] ** 2 + s[bx, 2] ** 2),
                         1.0 / 3.0 * m * (s[bx, 0] ** 2 + s[bx, 1] ** 2)], axis=1)
    sp = types == int(GeoType.SPHERE)
    r = s[sp, 0]
    m = density * (4.0 / 3.0 * math.pi * r * r * r)
    mass[sp] = m
    ia = 2.0 / 5.0 * m * r * r
    diag[sp] = np.stack([ia, ia, ia], axis=1)
    cp = types == int(GeoType.CAPSULE)
    r, hh = s[cp, 0], s[cp, 1]
    h = 2.0 * hh
    ms = density * (4.0 / 3.0) * math.pi * r * r * r
    mc = density * math.pi * r * r * h
    mass[cp] = ms + mc
    ia = mc * (0.25 * r * r + (1.0 / 12.0) * h * h) + ms * (0.4 * r * r + 0.375 * r * h + 0.25 * h * h)
    ib = (mc * 0.5 + ms * 0.4) * r * r
    diag[cp] = np.stack([ia, ia, ib], axis=1)
    inertia = np.zeros((n, 3, 3))
    inertia[:, 0, 0], inertia[:, 1, 1], inertia[:, 2, 2] = diag[:, 0], diag[:, 1], diag[:, 2]
    return mass, inertia


def _radius_batch(types, scales):
    s = np.asarray(scales, dtype=np.float64)
    r = np.where(types == int(GeoType.SPHERE), s[:, 0], s[:, 0] + s[:, 1])
    return np.where(types == int(GeoType.BOX), np.linalg.norm(s, axis=1), r)


def assemble_free_bodies(body_world: np.ndarray, types: np.ndarray, scales: np.ndarray, poses: np.ndarray,
                         mu: np.ndarray, world_count: int, plane_mu: float = 0.5, qd: np.ndarray | None = None,
                         device=None, uses_worlds: bool = True, gravity=(0.0, 0.0, -9.81),
                         restitution: float = 0.0) -> Model:
    """Model of free bodies (one primitive shape each) + a global ground plane (shape 0)."""
    B = types.shape[0]
    f32 = np.float32
    order = np.argsort(body_world, kind="stable")
    if np.any(order != np.arange(B)):
        raise ValueError("bodies must be given sorted by world")
    mass, inertia = _inertia_batch(types, scales)
    inv_inertia = np.linalg.inv(inertia) if B else np.zeros((0, 3, 3))
    S = B + 1
    h = {}
    h["body_q"] = poses.astype(f32).reshape(B, 7)
    h["body_qd"] = (np.zeros((B, 6)) if qd is None else qd).astype(f32).reshape(B, 6)
    h["body_com"] = np.zeros((B, 3), f32)
    h["body_mass"] = mass.astype(f32)
    h["body_inv_mass"] = (1.0 / mass).astype(f32)
    h["body_inertia"] = inertia.astype(f32).reshape(B, 9)
    h["body_inv_inertia"] = inv_inertia.astype(f32).reshape(B, 9)
    h["body_flags"] = np.full(B, int(BodyFlags.DYNAMIC), np.int32)
    h["body_world"] = (body_world if uses_worlds else np.full(B, -1)).astype(np.int32)
    st = np.concatenate([[int(GeoType.PLANE)], types]).astype(np.int32)
    h["shape_body"] = np.concatenate([[-1], np.arange(B)]).astype(np.int32)
    h["shape_type"] = st
    xf = np.zeros((S, 7), f32)
    xf[:, 6] = 1.0
    h["shape_transform"] = xf
    sc = np.zeros((S, 3), f32)
    sc[1:] = scales
    h["shape_scale"] = sc
    h["shape_margin"] = np.zeros(S, f32)
    h["shape_gap"] = np.full(S, 0.1, f32)
    h["shape_collision_radius"] = np.concatenate([[1.0e6], _radius_batch(types, scales)]).astype(f32)
    h["shape_material_mu"] = np.concatenate([[plane_mu], mu]).astype(f32)
    h["shape_material_mu_torsional"] = np.full(S, 0.005, f32)
    h["shape_material_mu_rolling"] = np.full(S, 0.0001, f32)
    h["shape_material_restitution"] = np.full(S, restitution, f32)
    h["shape_world"] = np.concatenate([[-1], body_world if uses_worlds else np.full(B, -1)]).astype(np.int32)
    h["shape_flags"] = np.full(S, _SHAPE_FLAGS, np.int32)
    h["shape_collision_group"] = np.ones(S, np.int32)
    J = B
    h["joint_type"] = np.full(J, int(JointType.FREE), np.int32)
    h["joint_enabled"] = np.ones(J, np.int32)
    h["joint_parent"] = np.full(J, -1, np.int32)
    h["joint_child"] = np.arange(J, dtype=np.int32)
    h["joint_X_p"] = poses.astype(f32).reshape(J, 7)
    xc = np.zeros((J, 7), f32)
    xc[:, 6] = 1.0
    h["joint_X_c"] = xc
    h["joint_qd_start"] = (6 * np.arange(J)).astype(np.int32)
    h["joint_dof_dim"] = np.tile(np.array([[3, 3]], np.int32), (J, 1))
    h["joint_world"] = h["body_world"].copy()
    D = 6 * J
    h["joint_axis"] = np.tile(np.concatenate([np.eye(3), np.eye(3)]).astype(f32), (J, 1)).reshape(D, 3)
    h["joint_limit_lower"] = np.full(D, -1e6, f32)
    h["joint_limit_upper"] = np.full(D, 1e6, f32)
    h["joint_target_ke"] = np.zeros(D, f32)
    h["joint_target_kd"] = np.zeros(D, f32)
    h["joint_target_pos"] = np.zeros(D, f32)
    h["joint_target_vel"] = np.zeros(D, f32)
    W = max(1, world_count)
    h["gravity"] = np.tile(np.asarray(gravity, f32), (W, 1))
    # explicit pairs: plane with every body shape, all body pairs inside a world
    chunks = [np.stack([np.zeros(B, np.int64), np.arange(1, S)], axis=1)]
    bounds = np.searchsorted(body_world, np.arange(W + 1))
    for w in range(W):
        lo, hi = bounds[w], bounds[w + 1]
        n = hi - lo
        if n < 2:
            continue
        i, j = np.triu_indices(n, 1)
        chunks.append(np.stack([lo + 1 + i, lo + 1 + j], axis=1))
    h["shape_contact_pairs"] = np.concatenate(chunks).astype(np.int32)
    return Model._from_arrays(h, world_count=W, uses_worlds=uses_worlds, device=device)


def scene_c1(seed: int = 0, device=None):
    """64 boxes, 1 world.  Returns (model, info)."""
    rng = np.random.default_rng(seed)
    n = 64
    half = rng.uniform(0.05, 0.15, size=(n, 3))
    gx = np.linspace(-0.5, 0.5, 4)
    gz = np.linspace(0.2, 2.0, 4)
    cx, cy, cz = np.meshgrid(gx, gx, gz, indexing="ij")
    centers = np.stack([cx.ravel(), cy.ravel(), cz.ravel()], axis=1)
    centers += rng.uniform(-0.02, 0.02, size=centers.shape)
    quats = random_quats(rng, n)
    poses = np.concatenate([centers, quats], axis=1)
    types = np.full(n, int(GeoType.BOX))
    model = assemble_free_bodies(np.zeros(n, np.int64), types, half, poses, np.full(n, 0.5), 1, plane_mu=0.5,
                                 device=device, uses_worlds=False)
    return model, dict(dt=1.0 / 60.0, substeps=10, iterations=4, name="C1: 64 boxes, 1 world")


def scene_c1_batch(seed: int = 100, worlds: int = 1024, device=None):
    """C1 scenes side by side: world w is scene_c1(seed + w) (64 boxes, its own random half-extents,
    jittered grid and orientations), all on one global ground plane (mu 0.5).  The learned warm start's
    C1 training and evaluation sets.  Returns (model, info) with C1's dt / substeps / iterations."""
    n = 64
    half, poses = [], []
    gx = np.linspace(-0.5, 0.5, 4)
    gz = np.linspace(0.2, 2.0, 4)
    cx, cy, cz = np.meshgrid(gx, gx, gz, indexing="ij")
    grid = np.stack([cx.ravel(), cy.ravel(), cz.ravel()], axis=1)
    for w in range(worlds):
        # the same draws, in the same order, as scene_c1(seed + w)
        rng = np.random.default_rng(seed + w)
        h = rng.uniform(0.05, 0.15, size=(n, 3))
        centers = grid + rng.uniform(-0.02, 0.02, size=grid.shape)
        quats = random_quats(rng, n)
        half.append(h)
        poses.append(np.concatenate([centers, quats], axis=1))
    body_world = np.repeat(np.arange(worlds), n)
    types = np.full(worlds * n, int(GeoType.BOX))
    model = assemble_free_bodies(body_world, types, np.concatenate(half), np.concatenate(poses),
                                 np.full(worlds * n, 0.5), worlds, plane_mu=0.5, device=device)
    return model, dict(dt=1.0 / 60.0, substeps=10, iterations=4, name=f"C1 x {worlds} (seeds {seed}..)")


def _bounding_radius(t, s):
    if t == int(GeoType.BOX):
        return float(np.linalg.norm(s))
    if t == int(GeoType.SPHERE):
        return float(s[0])
    return float(s[0] + s[1])


def _c2_counts(rng, worlds, nmin, nmax):
    return rng.integers(nmin, nmax + 1, size=worlds)


def c2_world_body_counts(seed: int = 1, worlds: int = 4096, nmin: int = 8, nmax: int = 128) -> np.ndarray:
    """Bodies per world of scene_c2(seed, worlds, nmin, nmax) without building it (for sharding)."""
    return _c2_counts(np.random.default_rng(seed), worlds, nmin, nmax)


def scene_c2(seed: int = 1, worlds: int = 4096, nmin: int = 8, nmax: int = 128, device=None,
             keep_worlds: int | None = None, world_range: tuple[int, int] | None = None):
    """Uneven worlds of box / sphere / capsule bodies.  Returns (model, info).

    Body i of every world is placed in the same vectorised round: up to 64
    uniform draws in the 1 x 1 x 2 m column, accepting the first that keeps
    bounding spheres apart; otherwise it is raised above the world's bodies.
    ``keep_worlds`` keeps only the first worlds of the generated scene and
    ``world_range = (a, b)`` worlds a..b-1 (the same bodies and poses as in the
    full scene), e.g. for a CPU sample or one rank's shard.
    """
    rng = np.random.default_rng(seed)
    counts = _c2_counts(rng, worlds, nmin, nmax)
    kinds = np.array([int(GeoType.BOX), int(GeoType.SPHERE), int(GeoType.CAPSULE)])
    nmax_w = int(counts.max())
    types = kinds[rng.integers(0, 3, size=(worlds, nmax_w))]
    scales = np.zeros((worlds, nmax_w, 3))
    box = types == int(GeoType.BOX)
    sph = types == int(GeoType.SPHERE)
    cap = types == int(GeoType.CAPSULE)
    scales[box] = rng.uniform(0.03, 0.2, size=(int(box.sum()), 3))
    scales[sph, 0] = rng.uniform(0.03, 0.2, size=int(sph.sum()))
    scales[cap, 0] = rng.uniform(0.02, 0.08, size=int(cap.sum()))
    scales[cap, 1] = rng.uniform(0.05, 0.2, size=int(cap.sum()))
    rad = _radius_batch(types.reshape(-1), scales.reshape(-1, 3)).reshape(worlds, nmax_w)
    pos = np.zeros((worlds, nmax_w, 3))
    for i in range(nmax_w):
        active = counts > i
        placed = ~active
        cand = np.zeros((worlds, 3))
        for _ in range(64):
            todo = ~placed
            if not todo.any():
                break
            k = int(todo.sum())
            c = np.stack([rng.uniform(-0.5, 0.5, k), rng.uniform(-0.5, 0.5, k), rng.uniform(0.2, 2.0, k)], axis=1)
            # dropped bodies start above the plane: bounding sphere clear of z = 0
            c[:, 2] = np.maximum(c[:, 2], rad[todo, i] + 0.001)
            if i > 0:
                diff = pos[todo, :i] - c[:, None, :]
                d2 = np.einsum("wij,wij->wi", diff, diff)
                rs = rad[todo, :i] + rad[todo, i][:, None]
                ok = ~np.any(d2 < rs * rs, axis=1)
            else:
                ok = np.ones(k, bool)
            idx = np.nonzero(todo)[0]
            cand[idx[ok]] = c[ok]
            placed[idx[ok]] = True
        fail = ~placed
        if fail.any():
            idx = np.nonzero(fail)[0]
            cand[idx] = np.stack([rng.uniform(-0.5, 0.5, idx.size), rng.uniform(-0.5, 0.5, idx.size),
                                  pos[idx, :i, 2].max(axis=1) + 2.0 * rad[idx].max(axis=1)], axis=1)
        pos[active, i] = cand[active]
    quats = random_quats(rng, worlds * nmax_w).reshape(worlds, nmax_w, 4)
    mu_w = rng.uniform(0.3, 1.0, size=worlds)
    mask = np.arange(nmax_w)[None, :] < counts[:, None]
    lo, hi = 0, worlds
    if keep_worlds is not None:
        if not 0 < keep_worlds <= worlds:
            raise ValueError("keep_worlds must be in [1, worlds]")
        hi = keep_worlds
    if world_range is not None:
        lo, hi = int(world_range[0]), int(world_range[1])
        if not 0 <= lo < hi <= worlds:
            raise ValueError("world_range must satisfy 0 <= a < b <= worlds")
    wid = np.arange(worlds)
    mask &= ((wid >= lo) & (wid < hi))[:, None]
    worlds = hi - lo
    bw = np.broadcast_to((wid - lo)[:, None], mask.shape)[mask]
    poses = np.concatenate([pos, quats], axis=2)[mask]
    mu = np.broadcast_to(mu_w[:, None], mask.shape)[mask]
    model = assemble_free_bodies(bw, types[mask], scales[mask], poses, mu, worlds, plane_mu=0.5, device=device)
    return model, dict(dt=1.0 / 60.0, substeps=8, iterations=8, name=f"C2: {worlds} uneven worlds")


def scene_c5(seed: int = 5, worlds: int = 1024, height: int = 16, device=None, restitution: float = 0.0):
    """16-box stacks with random initial twists.  Returns (model, info)."""
    rng = np.random.default_rng(seed)
    h = 0.1
    n = worlds * height
    pos = np.zeros((n, 3))
    k = np.tile(np.arange(height), worlds)
    pos[:, 0:2] = rng.uniform(-0.01, 0.01, size=(n, 2))
    pos[:, 2] = h + 2.0 * h * k
    quats = np.tile(np.array([0.0, 0.0, 0.0, 1.0]), (n, 1))
    poses = np.concatenate([pos, quats], axis=1)
    mu_w = rng.uniform(0.4, 0.8, size=worlds)
    mu = np.repeat(mu_w, height)
    qd = rng.normal(0.0, 0.1, size=(n, 6))
    model = assemble_free_bodies(np.repeat(np.arange(worlds), height), np.full(n, int(GeoType.BOX)),
                                 np.full((n, 3), h), poses, mu, worlds, plane_mu=0.6, qd=qd, device=device,
                                 restitution=restitution)
    return model, dict(dt=1.0 / 600.0, substeps=64, iterations=8, name=f"C5: {worlds} x {height}-box stacks")


def scene_c3(seed: int = 3, worlds: int = 4096, device=None):
    """7-link revolute arms among loose boxes.  Returns (model, info) with info['control_fn']."""
    rng = np.random.default_rng(seed)
    b = ModelBuilder()
    table_cfg = ModelBuilder.ShapeConfig(mu=0.6)
    b.add_ground_plane(cfg=table_cfg)
    r, L, m_link = 0.04, 0.3, 1.0
    link_cfg = ModelBuilder.ShapeConfig(density=0.0, mu=0.6)
    box_cfg = ModelBuilder.ShapeConfig(mu=0.6)
    _, _, Ic = compute_inertia_shape(int(GeoType.CAPSULE), (r, 0.5 * L, 0.0), 1000.0)
    mc, _, _ = compute_inertia_shape(int(GeoType.CAPSULE), (r, 0.5 * L, 0.0), 1000.0)
    I_link = Ic * (m_link / mc)
    phases = []
    for w in range(worlds):
        b.begin_world()
        base = np.array([0.0, 0.0, 0.35])
        parent = -1
        qx = quat_from_axis_angle((0.0, 1.0, 0.0), 0.5 * math.pi)  # links along +x
        for k in range(7):
            center = base + np.array([L * (k + 0.5), 0.0, 0.0])
            body = b.add_link(xform=np.concatenate([center, qx]), mass=m_link, inertia=I_link, lock_inertia=True)
            b.add_shape_capsule(body, radius=r, half_height=0.5 * L, cfg=link_cfg)
            axis = (0.0, 1.0, 0.0) if k % 2 == 0 else (0.0, 0.0, 1.0)
            if parent == -1:
                pxf = np.concatenate([base, qx])
            else:
                pxf = np.array([0.0, 0.0, 0.5 * L, 0.0, 0.0, 0.0, 1.0])
            cxf = np.array([0.0, 0.0, -0.5 * L, 0.0, 0.0, 0.0, 1.0])
            b.add_joint_revolute(parent, body, parent_xform=pxf, child_xform=cxf, axis=axis, target_ke=500.0,
                                 target_kd=20.0, limit_lower=-2.5, limit_upper=2.5)
            parent = body
        nbox = int(rng.integers(8, 49))
        placed = []  # (centre, bounding radius) of the world's boxes
        for _ in range(nbox):
            he = rng.uniform(0.03, 0.08, size=3)
            quat = random_quats(rng, 1)[0]
            qx_, qy_, qz_, qw_ = quat
            # the rotated box's half extent along z: its lowest corner clears the table
            row_z = np.array([2.0 * (qx_ * qz_ - qw_ * qy_), 2.0 * (qy_ * qz_ + qw_ * qx_),
                              1.0 - 2.0 * (qx_ * qx_ + qy_ * qy_)])
            ext_z = float(np.abs(row_z) @ he)
            rb = float(np.linalg.norm(he))
            p = None
            for _try in range(64):
                c = np.array([rng.uniform(0.2, 2.0), rng.uniform(-0.6, 0.6), ext_z + rng.uniform(0.0, 0.3)])
                # bounding spheres clear of the other boxes and of the arm's capsules (straight at rest)
                t = np.clip((c[0] - base[0]) / (7 * L), 0.0, 1.0)
                arm_d = np.linalg.norm(c - (base + np.array([7 * L * t, 0.0, 0.0])))
                if arm_d >= rb + r and all(np.linalg.norm(c - pc) >= rb + rc for pc, rc in placed):
                    p = c
                    break
            if p is None:
                # no room: raised above the arm and the world's boxes
                top = max([base[2] + r] + [pc[2] + rc for pc, rc in placed])
                p = np.array([rng.uniform(0.2, 2.0), rng.uniform(-0.6, 0.6), top + rb + 0.01])
            placed.append((p, rb))
            body = b.add_body(xform=np.concatenate([p, quat]))
            b.add_shape_box(body, hx=he[0], hy=he[1], hz=he[2], cfg=box_cfg)
        b.end_world()
        phases.append(rng.uniform(0.0, 2.0 * math.pi, size=7))
    model = b.finalize(device=device)
    phases = np.asarray(phases)
    return model, dict(dt=1.0 / 120.0, substeps=4, iterations=8, phases=phases,
                       name=f"C3: {worlds} arm worlds")


def scene_falling_shapes(worlds: int = 1, device=None):
    """The falling-shapes scene of newton/tests/test_shapes_no_bounce.py:32-184 with the
    shapes this solver collides: a 4 x 4 x 8 grid (spacing 1.5 m, offset (-5, -5, 1),
    +-0.2 m jitter from default_rng(42)) of spheres (r 0.3), boxes (half 0.3) and capsules
    (r 0.2, half height 0.4) in turn, each a free body (add_body's own free joint), above a
    ground plane at z = -0.5 (the reference's 2-triangle ground mesh at that height).  Every
    world holds the same grid.  Returns (model, initial z of every body as float32)."""
    b = ModelBuilder()
    b.add_ground_plane(height=-0.5)
    z0 = []
    for _ in range(worlds):
        rng = np.random.default_rng(42)
        b.begin_world()
        k = 0
        for ix in range(4):
            for iy in range(4):
                for iz in range(8):
                    base = np.array([-5.0 + 1.5 * ix, -5.0 + 1.5 * iy, 1.0 + 1.5 * iz])
                    pos = base + np.array([(rng.random() - 0.5) * 0.4 for _ in range(3)])
                    z0.append(np.float32(pos[2]))
                    body = b.add_body(xform=np.concatenate([pos, [0.0, 0.0, 0.0, 1.0]]))
                    kind = k % 3
                    k += 1
                    if kind == 0:
                        b.add_shape_sphere(body, radius=0.3)
                    elif kind == 1:
                        b.add_shape_box(body, hx=0.3, hy=0.3, hz=0.3)
                    else:
                        b.add_shape_capsule(body, radius=0.2, half_height=0.4)
        b.end_world()
    return b.finalize(device=device), np.asarray(z0, np.float32)


def scene_particles(seed: int = 7, cloth: int = 12, loose: int = 200, radius: float = 0.02, device=None,
                    body_shapes: bool = False, loose_extent: float = 0.3, loose_height=(0.33, 0.7)):
    """Particles dropped onto static shapes: a square cloth of ``cloth`` x ``cloth`` particles joined by
    structural and shear springs and bent across each quad's diagonal (bending edges), and ``loose`` free particles of radius U[0.5, 1] x ``radius`` above it.

    Static colliders: the ground plane, a box, a sphere and a capsule under the drop (world -1).  With
    ``body_shapes`` a free box body is added whose shape does not collide with particles.  The scene
    exercises every particle kernel: soft contacts with all four shape types, particle-particle contacts
    (cloth layers and loose particles pile), springs, and one inactive and one kinematic (mass 0) particle.
    Returns (model, info) with dt 1/60 split into 4 substeps and 8 iterations.
    """
    rng = np.random.default_rng(seed)
    b = ModelBuilder()
    b.add_ground_plane()
    b.add_shape_box(-1, xform=(0.15, 0.0, 0.1, 0.0, 0.0, 0.0, 1.0), hx=0.12, hy=0.2, hz=0.1)
    b.add_shape_sphere(-1, xform=(-0.2, 0.1, 0.12, 0.0, 0.0, 0.0, 1.0), radius=0.12)
    q = quat_from_axis_angle((1.0, 0.0, 0.0), math.pi / 2)
    b.add_shape_capsule(-1, xform=(0.0, -0.25, 0.06, *q), radius=0.06, half_height=0.2)
    if body_shapes:
        cfg = ModelBuilder.ShapeConfig(has_particle_collision=False)
        body = b.add_body(xform=(0.6, 0.6, 0.3, 0.0, 0.0, 0.0, 1.0))
        b.add_joint_free(body)
        b.add_shape_box(body, hx=0.05, hy=0.05, hz=0.05, cfg=cfg)
    spacing = 2.2 * radius
    origin = np.array([-0.5 * (cloth - 1) * spacing, -0.5 * (cloth - 1) * spacing, 0.28])
    idx = {}
    for i in range(cloth):
        for j in range(cloth):
            p = origin + np.array([i * spacing, j * spacing, 0.0]) + rng.uniform(-1e-3, 1e-3, 3)
            idx[i, j] = b.add_particle(tuple(p), (0.0, 0.0, 0.0), 0.1, radius=radius)
    for i in range(cloth):
        for j in range(cloth):
            for di, dj in ((1, 0), (0, 1), (1, 1), (1, -1)):
                if (i + di, j + dj) in idx:
                    b.add_spring(idx[i, j], idx[i + di, j + dj], 1.0e3 if di * dj == 0 else 2.5e2, 0.5, 0.0)
    # bending hinges across every quad's diagonal, flat at rest (add_edge: triangles (i, k, l), (j, l, k))
    for i in range(cloth - 1):
        for j in range(cloth - 1):
            b.add_edge(idx[i + 1, j], idx[i, j + 1], idx[i, j], idx[i + 1, j + 1], edge_ke=20.0, edge_kd=0.0)
    for _ in range(loose):
        p = (rng.uniform(-loose_extent, loose_extent), rng.uniform(-loose_extent, loose_extent),
             rng.uniform(*loose_height))
        v = tuple(rng.normal(0.0, 0.3, 3) + np.array([0.0, 0.0, -1.5]))
        b.add_particle(p, v, float(rng.uniform(0.005, 0.02)), radius=float(radius * rng.uniform(0.5, 1.0)))
    # an inactive particle and a kinematic one (mass 0: no gravity, no corrections)
    b.add_particle((0.4, 0.4, 0.5), (0.0, 0.0, -1.0), 0.01, radius=radius, flags=0)
    b.add_particle((-0.4, 0.4, 0.02), (0.1, 0.0, 0.0), 0.0, radius=radius)
    model = b.finalize(device=device)
    model.particle_mu = 0.4
    model.particle_cohesion = 0.002
    model.soft_contact_mu = 0.6
    return model, {"dt": 1.0 / 60.0, "substeps": 4, "iterations": 8}
