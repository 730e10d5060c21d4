"""ModelBuilder for the rigid-contact path.

Host-side scene construction with the reference's semantics and defaults
(newton/_src/sim/builder.py): ShapeConfig defaults (:231-305), rigid_gap 0.1
(:1165), add_body = add_link + add_joint_free + add_articulation (:3649-3722),
add_shape mass/inertia accumulation and same-body collision filtering
(:5449-5611, :8534-8566), ground plane (:5611-5700), worlds (:2815-2910,
:2116-2153) and the explicit contact-pair list (:10855-10913).
Supported geometry: plane, sphere, capsule, box.
"""

from __future__ import annotations

import copy
import dataclasses
import math
from typing import Sequence

import numpy as np

from ._abi import BodyFlags, GeoType, JointType, ShapeFlags


def _cross(a, b):
    # the component formulas of np.cross for 3-vectors, without its axis handling
    return np.array([a[1] * b[2] - a[2] * b[1], a[2] * b[0] - a[0] * b[2], a[0] * b[1] - a[1] * b[0]])


def _quat_rotate(q, v):
    q = np.asarray(q, dtype=np.float64)
    v = np.asarray(v, dtype=np.float64)
    u = q[:3]
    w = q[3]
    return v * (2.0 * w * w - 1.0) + u * (2.0 * np.dot(u, v)) + _cross(u, v) * (2.0 * w)


def _quat_to_matrix(q):
    return np.stack([_quat_rotate(q, e) for e in np.eye(3)], axis=1)


def _quat_mul(a, b):
    ax, ay, az, aw = a
    bx, by, bz, bw = b
    return np.array(
        [
            aw * bx + bw * ax + ay * bz - by * az,
            aw * by + bw * ay + az * bx - bz * ax,
            aw * bz + bw * az + ax * by - bx * ay,
            aw * bw - ax * bx - ay * by - az * bz,
        ]
    )


def _transform_point(xf, p):
    xf = np.asarray(xf, dtype=np.float64)
    return _quat_rotate(xf[3:7], p) + xf[:3]


def _quat_between_vectors(a, b):
    """Shortest-arc rotation taking unit vector a to unit vector b."""
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    c = np.cross(a, b)
    d = float(np.dot(a, b))
    if d < -1.0 + 1e-9:
        axis = np.cross(a, [1.0, 0.0, 0.0])
        if np.linalg.norm(axis) < 1e-6:
            axis = np.cross(a, [0.0, 1.0, 0.0])
        axis /= np.linalg.norm(axis)
        return np.array([axis[0], axis[1], axis[2], 0.0])
    q = np.array([c[0], c[1], c[2], 1.0 + d])
    return q / np.linalg.norm(q)


def quat_from_axis_angle(axis, angle):
    axis = np.asarray(axis, dtype=np.float64)
    axis = axis / np.linalg.norm(axis)
    s = math.sin(0.5 * angle)
    return np.array([axis[0] * s, axis[1] * s, axis[2] * s, math.cos(0.5 * angle)])


def _as_xform(xform) -> np.ndarray:
    if xform is None:
        return np.array([0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 1.0])
    if isinstance(xform, tuple) and len(xform) == 2:
        p, q = xform
        return np.array([*p, *q], dtype=np.float64)
    a = np.asarray(xform, dtype=np.float64).reshape(-1)
    if a.shape[0] != 7:
        raise ValueError(f"transform must have 7 components (p, q), got {a.shape[0]}")
    return a


def transform_inertia(mass, inertia, offset, quat):
    """Rotate + parallel-axis shift (newton/_src/geometry/inertia.py:454-489)."""
    r = _quat_to_matrix(quat)
    offset = np.asarray(offset, dtype=np.float64)
    return r @ inertia @ r.T + mass * (np.dot(offset, offset) * np.eye(3) - np.outer(offset, offset))


def compute_inertia_shape(geo_type, scale, density, is_solid=True, thickness=0.001):
    """Mass, COM and COM inertia of a primitive (newton/_src/geometry/inertia.py:42-245, 492-560)."""
    if density == 0.0 or geo_type == GeoType.PLANE:
        return 0.0, np.zeros(3), np.zeros((3, 3))

    def sphere(r):
        m = density * (4.0 / 3.0 * math.pi * r * r * r)
        ia = 2.0 / 5.0 * m * r * r
        return m, np.diag([ia, ia, ia])

    def box(hx, hy, hz):
        m = density * (8.0 * hx * hy * hz)
        return m, np.diag(
            [1.0 / 3.0 * m * (hy * hy + hz * hz), 1.0 / 3.0 * m * (hx * hx + hz * hz), 1.0 / 3.0 * m * (hx * hx + hy * hy)]
        )

    def capsule(r, hh):
        h = 2.0 * hh
        ms = density * (4.0 / 3.0) * math.pi * r * r * r
        mc = density * math.pi * r * r * h
        m = ms + mc
        ia = mc * (0.25 * r * r + (1.0 / 12.0) * h * h) + ms * (0.4 * r * r + 0.375 * r * h + 0.25 * h * h)
        ib = (mc * 0.5 + ms * 0.4) * r * r
        return m, np.diag([ia, ia, ib])

    if geo_type == GeoType.SPHERE:
        fn, args, hargs = sphere, (scale[0],), (scale[0] - thickness,)
    elif geo_type == GeoType.BOX:
        fn, args, hargs = box, tuple(scale[:3]), tuple(s - thickness for s in scale[:3])
    elif geo_type == GeoType.CAPSULE:
        fn, args, hargs = capsule, (scale[0], scale[1]), (scale[0] - thickness, scale[1] - thickness)
    else:
        raise NotImplementedError(f"inertia of {GeoType(geo_type).name} is not supported")
    m, inertia = fn(*args)
    if not is_solid:
        mh, ih = fn(*hargs)
        m, inertia = m - mh, inertia - ih
    return m, np.zeros(3), inertia


def compute_shape_radius(geo_type, scale) -> float:
    """Bounding radius for broad phase (newton/_src/geometry/utils.py:73-113)."""
    if geo_type == GeoType.SPHERE:
        return float(scale[0])
    if geo_type == GeoType.BOX:
        return float(np.linalg.norm(scale))
    if geo_type == GeoType.CAPSULE:
        return float(scale[0] + scale[1])
    if geo_type == GeoType.PLANE:
        if scale[0] > 0.0 and scale[1] > 0.0:
            return float(np.linalg.norm(scale) * 0.5)
        return 1.0e6
    raise NotImplementedError(f"{GeoType(geo_type).name} shapes are not supported")


class ModelBuilder:
    """Scene builder for the rigid-contact XPBD path (subset of newton.ModelBuilder)."""

    @dataclasses.dataclass
    class ShapeConfig:
        """Shape properties (newton/_src/sim/builder.py:231-305 defaults)."""

        density: float = 1000.0
        ke: float = 2.5e3
        kd: float = 100.0
        kf: float = 1000.0
        ka: float = 0.0
        mu: float = 1.0
        restitution: float = 0.0
        mu_torsional: float = 0.005
        mu_rolling: float = 0.0001
        margin: float = 0.0
        gap: float | None = None
        is_solid: bool = True
        collision_group: int = 1
        collision_filter_parent: bool = True
        has_shape_collision: bool = True
        has_particle_collision: bool = True
        is_visible: bool = True
        is_site: bool = False

        @property
        def flags(self) -> int:
            f = 0
            if self.is_visible:
                f |= ShapeFlags.VISIBLE
            if self.has_shape_collision:
                f |= ShapeFlags.COLLIDE_SHAPES
            if self.has_particle_collision:
                f |= ShapeFlags.COLLIDE_PARTICLES
            if self.is_site:
                f |= ShapeFlags.SITE
            return int(f)

        def copy(self):
            return copy.copy(self)

    def __init__(self, up_axis: str = "Z", gravity: float = -9.81):
        if str(up_axis).upper() not in ("Z", "2"):
            raise NotImplementedError("only up_axis='Z' is supported")
        self.up_vector = (0.0, 0.0, 1.0)
        self.gravity = gravity
        self.rigid_gap = 0.1
        self.default_shape_cfg = ModelBuilder.ShapeConfig()
        self.world_count = 0
        self._current_world = -1
        self.world_gravity: list[tuple[float, float, float]] = []
        # bodies
        self.body_q: list[np.ndarray] = []
        self.body_qd: list[np.ndarray] = []
        self.body_com: list[np.ndarray] = []
        self.body_mass: list[float] = []
        self.body_inv_mass: list[float] = []
        self.body_inertia: list[np.ndarray] = []
        self.body_inv_inertia: list[np.ndarray] = []
        self.body_flags: list[int] = []
        self.body_world: list[int] = []
        self.body_label: list[str] = []
        self.body_lock_inertia: list[bool] = []
        self.body_shapes: dict[int, list[int]] = {-1: []}
        # shapes
        self.shape_body: list[int] = []
        self.shape_type: list[int] = []
        self.shape_transform: list[np.ndarray] = []
        self.shape_scale: list[tuple] = []
        self.shape_margin: list[float] = []
        self.shape_gap: list[float] = []
        self.shape_radius: list[float] = []
        self.shape_mu: list[float] = []
        self.shape_mu_torsional: list[float] = []
        self.shape_mu_rolling: list[float] = []
        self.shape_restitution: list[float] = []
        self.shape_flags: list[int] = []
        self.shape_collision_group: list[int] = []
        self.shape_world: list[int] = []
        self.shape_label: list[str] = []
        # a list, as in the reference builder (builder.py:966), so that callers may append;
        # the pair list canonicalises and de-duplicates it
        self.shape_collision_filter_pairs: list[tuple[int, int]] = []
        # joints
        self.joint_type: list[int] = []
        self.joint_enabled: list[bool] = []
        self.joint_parent: list[int] = []
        self.joint_child: list[int] = []
        self.joint_X_p: list[np.ndarray] = []
        self.joint_X_c: list[np.ndarray] = []
        self.joint_qd_start: list[int] = []
        self.joint_q_start: list[int] = []
        self.joint_dof_dim: list[tuple[int, int]] = []
        self.joint_world: list[int] = []
        self.joint_collision_filter_parent: list[bool] = []
        self.joint_parents: dict[int, list[tuple[int, int]]] = {}
        self.joint_children: dict[int, list[tuple[int, int]]] = {}
        self.joint_axis: list[np.ndarray] = []
        self.joint_limit_lower: list[float] = []
        self.joint_limit_upper: list[float] = []
        self.joint_target_ke: list[float] = []
        self.joint_target_kd: list[float] = []
        self.joint_target_pos: list[float] = []
        self.joint_target_vel: list[float] = []
        self.joint_q: list[float] = []
        self.articulation_start: list[int] = []
        self.num_rigid_contacts_per_world: int | None = None
        # particles and springs (builder.py:816, 899; add_particle / add_spring at 7186-7320)
        self.default_particle_radius = 0.1
        self.particle_max_velocity: float = 1e5
        self.particle_q: list[tuple] = []
        self.particle_qd: list[tuple] = []
        self.particle_mass: list[float] = []
        self.particle_radius: list[float] = []
        self.particle_flags: list[int] = []
        self.particle_world: list[int] = []
        self.spring_indices: list[int] = []
        self.spring_rest_length: list[float] = []
        self.spring_stiffness: list[float] = []
        self.spring_damping: list[float] = []
        self.spring_control: list[float] = []
        # bending edges (builder.py:840-843, 999-1006; add_edge at 7589-7650)
        self.default_edge_ke = 100.0
        self.default_edge_kd = 0.0
        self.edge_indices: list[tuple[int, int, int, int]] = []
        self.edge_rest_angle: list[float] = []
        self.edge_rest_length: list[float] = []
        self.edge_bending_properties: list[tuple[float, float]] = []
        # tetrahedra (builder.py:7522-7587)
        self.tet_indices: list[tuple[int, int, int, int]] = []
        self.tet_poses: list[list] = []
        self.tet_activations: list[float] = []
        self.tet_materials: list[tuple[float, float, float]] = []
        self._requested_contact_attributes: set[str] = set()
        self._requested_state_attributes: set[str] = set()

    # ------------------------------------------------------------------ counts
    @property
    def body_count(self) -> int:
        return len(self.body_q)

    @property
    def shape_count(self) -> int:
        return len(self.shape_type)

    @property
    def joint_count(self) -> int:
        return len(self.joint_type)

    @property
    def joint_dof_count(self) -> int:
        return len(self.joint_axis)

    @property
    def particle_count(self) -> int:
        return len(self.particle_q)

    @property
    def spring_count(self) -> int:
        return len(self.spring_rest_length)

    @property
    def tet_count(self) -> int:
        return len(self.tet_indices)

    @property
    def edge_count(self) -> int:
        return len(self.edge_rest_angle)

    @property
    def current_world(self) -> int:
        return self._current_world

    # ------------------------------------------------------------------ worlds
    def begin_world(self, label: str | None = None, attributes=None, gravity=None):
        if self._current_world != -1:
            raise RuntimeError(
                f"Cannot begin a new world: already in world context (current_world={self._current_world}). "
                "Call end_world() first to close the current world context."
            )
        self._current_world = self.world_count
        self.world_count += 1
        if gravity is not None:
            self.world_gravity.append(tuple(float(g) for g in gravity))
        else:
            u = self.up_vector
            self.world_gravity.append((u[0] * self.gravity, u[1] * self.gravity, u[2] * self.gravity))

    def end_world(self):
        if self._current_world == -1:
            raise RuntimeError("Cannot end world: not currently in a world context (current_world is already -1).")
        self._current_world = -1

    def add_world(self, builder: "ModelBuilder", xform=None, label: str | None = None):
        """Copy every entity of ``builder`` into a new world, offset by ``xform``."""
        self.begin_world(label=label)
        self.add_builder(builder, xform=xform)
        self.end_world()

    def replicate(self, builder: "ModelBuilder", world_count: int, spacing=(0.0, 0.0, 0.0)):
        for i in range(world_count):
            off = np.asarray(spacing, dtype=np.float64) * i
            self.add_world(builder, xform=np.array([off[0], off[1], off[2], 0.0, 0.0, 0.0, 1.0]))

    def add_builder(self, builder: "ModelBuilder", xform=None):
        xf = _as_xform(xform)
        p_off = self.particle_count
        for i in range(builder.particle_count):
            self.particle_q.append(tuple(_transform_point(xf, np.asarray(builder.particle_q[i], dtype=np.float64))))
            v = _quat_rotate(xf[3:], np.asarray(builder.particle_qd[i], dtype=np.float64))
            self.particle_qd.append(tuple(v))
            self.particle_mass.append(builder.particle_mass[i])
            self.particle_radius.append(builder.particle_radius[i])
            self.particle_flags.append(builder.particle_flags[i])
            self.particle_world.append(self._current_world)
        self.spring_indices.extend(int(i) + p_off for i in builder.spring_indices)
        self.spring_rest_length.extend(builder.spring_rest_length)
        self.spring_stiffness.extend(builder.spring_stiffness)
        self.spring_damping.extend(builder.spring_damping)
        self.spring_control.extend(builder.spring_control)
        for e in builder.edge_indices:
            self.edge_indices.append(tuple(int(v) + p_off if v != -1 else -1 for v in e))
        self.edge_rest_angle.extend(builder.edge_rest_angle)
        self.edge_rest_length.extend(builder.edge_rest_length)
        self.edge_bending_properties.extend(builder.edge_bending_properties)
        self.tet_indices.extend(tuple(int(v) + p_off for v in t) for t in builder.tet_indices)
        self.tet_poses.extend(builder.tet_poses)
        self.tet_activations.extend(builder.tet_activations)
        self.tet_materials.extend(builder.tet_materials)
        b_off = self.body_count
        s_off = self.shape_count
        j_off = self.joint_count
        d_off = self.joint_dof_count
        for i in range(builder.body_count):
            q = builder.body_q[i]
            p = _transform_point(xf, q[:3])
            r = _quat_mul(xf[3:], q[3:])
            self._append_body(
                np.concatenate([p, r]),
                builder.body_com[i],
                builder.body_mass[i],
                builder.body_inertia[i],
                builder.body_flags[i],
                builder.body_label[i],
                builder.body_lock_inertia[i],
                inv_mass=builder.body_inv_mass[i],
                inv_inertia=builder.body_inv_inertia[i],
                qd=builder.body_qd[i],
            )
        for s in range(builder.shape_count):
            b = builder.shape_body[s]
            nb = b + b_off if b >= 0 else -1
            sxf = builder.shape_transform[s]
            if b < 0:
                p = _transform_point(xf, sxf[:3])
                sxf = np.concatenate([p, _quat_mul(xf[3:], sxf[3:])])
            self.shape_body.append(nb)
            self.body_shapes.setdefault(nb, []).append(self.shape_count)
            self.shape_type.append(builder.shape_type[s])
            self.shape_transform.append(np.array(sxf))
            self.shape_scale.append(builder.shape_scale[s])
            self.shape_margin.append(builder.shape_margin[s])
            self.shape_gap.append(builder.shape_gap[s])
            self.shape_radius.append(builder.shape_radius[s])
            self.shape_mu.append(builder.shape_mu[s])
            self.shape_mu_torsional.append(builder.shape_mu_torsional[s])
            self.shape_mu_rolling.append(builder.shape_mu_rolling[s])
            self.shape_restitution.append(builder.shape_restitution[s])
            self.shape_flags.append(builder.shape_flags[s])
            self.shape_collision_group.append(builder.shape_collision_group[s])
            self.shape_world.append(self._current_world)
            self.shape_label.append(builder.shape_label[s])
        for a, b in builder.shape_collision_filter_pairs:
            self.shape_collision_filter_pairs.append((a + s_off, b + s_off))
        for j in range(builder.joint_count):
            p = builder.joint_parent[j]
            c = builder.joint_child[j]
            xp = builder.joint_X_p[j]
            if p < 0:
                pp = _transform_point(xf, xp[:3])
                xp = np.concatenate([pp, _quat_mul(xf[3:], xp[3:])])
            self.joint_type.append(builder.joint_type[j])
            self.joint_enabled.append(builder.joint_enabled[j])
            self.joint_parent.append(p + b_off if p >= 0 else -1)
            self.joint_child.append(c + b_off)
            self.joint_X_p.append(np.array(xp))
            self.joint_X_c.append(np.array(builder.joint_X_c[j]))
            self.joint_qd_start.append(builder.joint_qd_start[j] + d_off)
            self.joint_q_start.append(builder.joint_q_start[j])
            self.joint_dof_dim.append(builder.joint_dof_dim[j])
            self.joint_world.append(self._current_world)
            self.joint_collision_filter_parent.append(builder.joint_collision_filter_parent[j])
        for d in range(builder.joint_dof_count):
            self.joint_axis.append(np.array(builder.joint_axis[d]))
            self.joint_limit_lower.append(builder.joint_limit_lower[d])
            self.joint_limit_upper.append(builder.joint_limit_upper[d])
            self.joint_target_ke.append(builder.joint_target_ke[d])
            self.joint_target_kd.append(builder.joint_target_kd[d])
            self.joint_target_pos.append(builder.joint_target_pos[d])
            self.joint_target_vel.append(builder.joint_target_vel[d])

    # ------------------------------------------------------------------ bodies
    def _append_body(self, q, com, mass, inertia, flags, label, lock, inv_mass=None, inv_inertia=None, qd=None):
        self.body_q.append(np.asarray(q, dtype=np.float64))
        self.body_qd.append(np.zeros(6) if qd is None else np.asarray(qd, dtype=np.float64))
        self.body_com.append(np.asarray(com, dtype=np.float64))
        self.body_mass.append(float(mass))
        self.body_inertia.append(np.asarray(inertia, dtype=np.float64))
        if inv_mass is None:
            inv_mass = 1.0 / mass if mass > 0.0 else 0.0
        if inv_inertia is None:
            inv_inertia = np.linalg.inv(inertia) if np.any(inertia) else np.asarray(inertia, dtype=np.float64)
        self.body_inv_mass.append(float(inv_mass))
        self.body_inv_inertia.append(np.asarray(inv_inertia, dtype=np.float64))
        self.body_flags.append(int(flags))
        self.body_world.append(self._current_world)
        self.body_label.append(label)
        self.body_lock_inertia.append(bool(lock))
        self.body_shapes.setdefault(len(self.body_q) - 1, [])
        return len(self.body_q) - 1

    def add_link(self, xform=None, com=None, inertia=None, mass: float = 0.0, label=None, lock_inertia=False,
                 is_kinematic: bool = False, armature=None):
        xf = _as_xform(xform)
        inertia = np.zeros((3, 3)) if inertia is None else np.asarray(inertia, dtype=np.float64).reshape(3, 3)
        com = np.zeros(3) if com is None else np.asarray(com, dtype=np.float64)
        flags = BodyFlags.KINEMATIC if is_kinematic else BodyFlags.DYNAMIC
        return self._append_body(xf, com, mass, inertia, flags, label or f"body_{self.body_count}", lock_inertia)

    def add_body(self, xform=None, armature=None, com=None, inertia=None, mass: float = 0.0, label=None,
                 lock_inertia=False, is_kinematic=False):
        """Free-floating body: add_link + add_joint_free (builder.py:3649-3722)."""
        b = self.add_link(xform=xform, com=com, inertia=inertia, mass=mass, label=label,
                          lock_inertia=lock_inertia, is_kinematic=is_kinematic)
        self.add_joint_free(child=b)
        self.articulation_start.append(self.joint_count - 1)
        return b

    # ------------------------------------------------------------------ joints
    @staticmethod
    def _default_filter_parent(joint_type, parent: int) -> bool:
        """builder.py:1258-1263: False for non-fixed joints to world, True otherwise."""
        if parent == -1:
            return int(joint_type) == int(JointType.FIXED)
        return True

    def _add_joint(self, jtype, parent, child, parent_xform, child_xform, lin_axes, ang_axes,
                   collision_filter_parent=None, enabled=True):
        if collision_filter_parent is None:
            collision_filter_parent = self._default_filter_parent(jtype, parent)
        j = self.joint_count
        self.joint_type.append(int(jtype))
        self.joint_enabled.append(bool(enabled))
        self.joint_parent.append(int(parent))
        self.joint_child.append(int(child))
        self.joint_X_p.append(_as_xform(parent_xform))
        self.joint_X_c.append(_as_xform(child_xform))
        self.joint_qd_start.append(self.joint_dof_count)
        self.joint_q_start.append(len(self.joint_q))
        self.joint_dof_dim.append((len(lin_axes), len(ang_axes)))
        self.joint_world.append(self._current_world)
        self.joint_collision_filter_parent.append(bool(collision_filter_parent))
        for ax in list(lin_axes) + list(ang_axes):
            self.joint_axis.append(np.asarray(ax["axis"], dtype=np.float64))
            self.joint_limit_lower.append(float(ax.get("limit_lower", -1e6)))
            self.joint_limit_upper.append(float(ax.get("limit_upper", 1e6)))
            self.joint_target_ke.append(float(ax.get("target_ke", 0.0)))
            self.joint_target_kd.append(float(ax.get("target_kd", 0.0)))
            self.joint_target_pos.append(float(ax.get("target_pos", 0.0)))
            self.joint_target_vel.append(float(ax.get("target_vel", 0.0)))
        self.joint_parents.setdefault(child, []).append((parent, j))
        self.joint_children.setdefault(parent, []).append((child, j))
        if collision_filter_parent:
            # builder.py:3878-3885 (parent -1: the static shapes)
            for cs in self.body_shapes.get(child, []):
                if not self.shape_flags[cs] & ShapeFlags.COLLIDE_SHAPES:
                    continue
                for ps in self.body_shapes.get(parent, []):
                    if not self.shape_flags[ps] & ShapeFlags.COLLIDE_SHAPES:
                        continue
                    self.add_shape_collision_filter_pair(ps, cs)
        return j

    def add_joint_free(self, child: int, parent_xform=None, child_xform=None, parent: int = -1, label=None):
        if parent_xform is None and parent == -1:
            parent_xform = self.body_q[child]
        axes = [{"axis": e, "limit_lower": -1e6, "limit_upper": 1e6} for e in np.eye(3)]
        return self._add_joint(JointType.FREE, parent, child, parent_xform, child_xform, axes, axes)

    def add_joint_revolute(self, parent: int, child: int, parent_xform=None, child_xform=None, axis=(1.0, 0.0, 0.0),
                           target_pos: float = 0.0, target_vel: float = 0.0, target_ke: float = 0.0,
                           target_kd: float = 0.0, limit_lower: float = -1e6, limit_upper: float = 1e6,
                           collision_filter_parent: bool | None = None, enabled: bool = True, label=None):
        ax = {"axis": axis, "limit_lower": limit_lower, "limit_upper": limit_upper, "target_ke": target_ke,
              "target_kd": target_kd, "target_pos": target_pos, "target_vel": target_vel}
        return self._add_joint(JointType.REVOLUTE, parent, child, parent_xform, child_xform, [], [ax],
                               collision_filter_parent, enabled)

    def add_joint_prismatic(self, parent: int, child: int, parent_xform=None, child_xform=None,
                            axis=(1.0, 0.0, 0.0), target_pos=0.0, target_vel=0.0, target_ke=0.0, target_kd=0.0,
                            limit_lower=-1e6, limit_upper=1e6, collision_filter_parent=None, enabled=True,
                            label=None):
        ax = {"axis": axis, "limit_lower": limit_lower, "limit_upper": limit_upper, "target_ke": target_ke,
              "target_kd": target_kd, "target_pos": target_pos, "target_vel": target_vel}
        return self._add_joint(JointType.PRISMATIC, parent, child, parent_xform, child_xform, [ax], [],
                               collision_filter_parent, enabled)

    def add_joint_fixed(self, parent: int, child: int, parent_xform=None, child_xform=None,
                        collision_filter_parent=None, enabled=True, label=None):
        return self._add_joint(JointType.FIXED, parent, child, parent_xform, child_xform, [], [],
                               collision_filter_parent, enabled)

    def add_joint_ball(self, parent: int, child: int, parent_xform=None, child_xform=None,
                       collision_filter_parent=None, enabled=True, label=None):
        axes = [{"axis": e} for e in np.eye(3)]
        return self._add_joint(JointType.BALL, parent, child, parent_xform, child_xform, [], axes,
                               collision_filter_parent, enabled)

    def add_articulation(self, joints: Sequence[int], label=None):
        self.articulation_start.append(int(joints[0]) if len(joints) else self.joint_count)

    # ------------------------------------------------------------------ shapes
    def add_shape_collision_filter_pair(self, shape_a: int, shape_b: int) -> None:
        a, b = (shape_a, shape_b) if shape_a < shape_b else (shape_b, shape_a)
        self.shape_collision_filter_pairs.append((a, b))

    def add_shape(self, *, body: int, type: int, xform=None, cfg=None, scale=None, is_static: bool = False,
                  label=None) -> int:
        if int(type) not in [int(g) for g in (GeoType.PLANE, GeoType.SPHERE, GeoType.CAPSULE, GeoType.BOX)]:
            raise NotImplementedError(f"shape type {GeoType(type).name} is not supported by this build")
        xf = _as_xform(xform)
        if cfg is None:
            cfg = self.default_shape_cfg
        if scale is None:
            scale = (1.0, 1.0, 1.0)
        shape = self.shape_count
        self.shape_body.append(int(body))
        if cfg.has_shape_collision:
            for other in self.body_shapes.get(body, []):
                self.add_shape_collision_filter_pair(other, shape)
        self.body_shapes.setdefault(body, []).append(shape)
        self.shape_label.append(label or f"shape_{shape}")
        self.shape_transform.append(xf)
        self.shape_flags.append(cfg.flags)
        self.shape_type.append(int(type))
        self.shape_scale.append((float(scale[0]), float(scale[1]), float(scale[2])))
        self.shape_margin.append(float(cfg.margin))
        self.shape_gap.append(float(cfg.gap if cfg.gap is not None else self.rigid_gap))
        self.shape_radius.append(compute_shape_radius(int(type), scale))
        self.shape_mu.append(float(cfg.mu))
        self.shape_mu_torsional.append(float(cfg.mu_torsional))
        self.shape_mu_rolling.append(float(cfg.mu_rolling))
        self.shape_restitution.append(float(cfg.restitution))
        self.shape_collision_group.append(int(cfg.collision_group))
        self.shape_world.append(self._current_world)
        if cfg.has_shape_collision and cfg.collision_filter_parent:
            for parent_body, j in self.joint_parents.get(body, ()):
                if not self.joint_collision_filter_parent[j]:
                    continue
                for ps in self.body_shapes.get(parent_body, []):
                    self.add_shape_collision_filter_pair(ps, shape)
            for child_body, j in self.joint_children.get(body, ()):
                if not self.joint_collision_filter_parent[j]:
                    continue
                for cs in self.body_shapes.get(child_body, []):
                    self.add_shape_collision_filter_pair(shape, cs)
        if not is_static and cfg.density > 0.0 and body >= 0 and not self.body_lock_inertia[body]:
            m, c, inertia = compute_inertia_shape(int(type), scale, cfg.density, cfg.is_solid, cfg.margin)
            com_body = _transform_point(xf, c)
            self._update_body_mass(body, m, inertia, com_body, xf[3:])
        return shape

    def _update_body_mass(self, i, m, inertia, p, q):
        """builder.py:8534-8566."""
        new_mass = self.body_mass[i] + m
        if new_mass == 0.0:
            return
        new_com = (self.body_com[i] * self.body_mass[i] + p * m) / new_mass
        com_offset = new_com - self.body_com[i]
        shape_offset = new_com - p
        new_inertia = transform_inertia(self.body_mass[i], self.body_inertia[i], com_offset,
                                        np.array([0.0, 0.0, 0.0, 1.0])) + transform_inertia(m, inertia,
                                                                                            shape_offset, q)
        self.body_mass[i] = new_mass
        self.body_inertia[i] = new_inertia
        self.body_com[i] = new_com
        self.body_inv_mass[i] = 1.0 / new_mass if new_mass > 0.0 else 0.0
        self.body_inv_inertia[i] = np.linalg.inv(new_inertia) if np.any(new_inertia) else new_inertia

    def add_shape_box(self, body: int, xform=None, hx: float = 0.5, hy: float = 0.5, hz: float = 0.5, cfg=None,
                      label=None) -> int:
        return self.add_shape(body=body, type=GeoType.BOX, xform=xform, cfg=cfg, scale=(hx, hy, hz), label=label)

    def add_shape_sphere(self, body: int, xform=None, radius: float = 1.0, cfg=None, label=None) -> int:
        return self.add_shape(body=body, type=GeoType.SPHERE, xform=xform, cfg=cfg, scale=(radius, 0.0, 0.0),
                              label=label)

    def add_shape_capsule(self, body: int, xform=None, radius: float = 1.0, half_height: float = 0.5, cfg=None,
                          label=None) -> int:
        return self.add_shape(body=body, type=GeoType.CAPSULE, xform=xform, cfg=cfg,
                              scale=(radius, half_height, 0.0), label=label)

    def add_shape_plane(self, plane=(0.0, 0.0, 1.0, 0.0), xform=None, width: float = 10.0, length: float = 10.0,
                        body: int = -1, cfg=None, label=None) -> int:
        if xform is None:
            normal = np.array(plane[:3], dtype=np.float64)
            norm = np.linalg.norm(normal)
            normal /= norm
            d = plane[3] / norm
            pos = -d * normal
            rot = _quat_between_vectors([0.0, 0.0, 1.0], normal)
            xform = np.concatenate([pos, rot])
        return self.add_shape(body=body, type=GeoType.PLANE, xform=xform, cfg=cfg, scale=(width, length, 0.0),
                              is_static=True, label=label)

    def add_ground_plane(self, height: float = 0.0, cfg=None, label=None) -> int:
        return self.add_shape_plane(plane=(*self.up_vector, -height), width=0.0, length=0.0, cfg=cfg,
                                    label=label or "ground_plane")

    # ------------------------------------------------------------------ particles
    def add_particle(self, pos, vel, mass: float, radius: float | None = None, flags: int = 1,
                     custom_attributes=None) -> int:
        """Add one particle (builder.py:7186-7230); mass 0 makes it kinematic."""
        if custom_attributes:
            raise NotImplementedError("custom attributes are not supported")
        self.particle_q.append(tuple(float(x) for x in pos))
        self.particle_qd.append(tuple(float(x) for x in vel))
        self.particle_mass.append(float(mass))
        self.particle_radius.append(float(self.default_particle_radius if radius is None else radius))
        self.particle_flags.append(int(flags))
        self.particle_world.append(self._current_world)
        return self.particle_count - 1

    def add_particles(self, pos, vel, mass, radius=None, flags=None, custom_attributes=None) -> None:
        """Add a group of particles (builder.py:7232-7276)."""
        n = len(pos)
        radius = [self.default_particle_radius] * n if radius is None else radius
        flags = [1] * n if flags is None else flags
        for i in range(n):
            self.add_particle(pos[i], vel[i], mass[i], radius[i], flags[i], custom_attributes)

    def add_spring(self, i: int, j: int, ke: float, kd: float, control: float, custom_attributes=None) -> None:
        """Spring between particles i and j; its rest length is their current distance (builder.py:7278-7320)."""
        if custom_attributes:
            raise NotImplementedError("custom attributes are not supported")
        self.spring_indices.extend((int(i), int(j)))
        self.spring_stiffness.append(float(ke))
        self.spring_damping.append(float(kd))
        self.spring_control.append(float(control))
        p = np.asarray(self.particle_q[i], dtype=np.float32)
        q = np.asarray(self.particle_q[j], dtype=np.float32)
        delta = np.subtract(p, q)
        self.spring_rest_length.append(float(np.sqrt(np.dot(delta, delta))))

    def add_edge(self, i: int, j: int, k: int, l: int, rest: float | None = None, edge_ke: float | None = None,
                 edge_kd: float | None = None, custom_attributes=None) -> int:
        """Bending edge k-l between the triangles (i, k, l) and (j, l, k) (builder.py:7589-7650); the rest
        angle defaults to the current dihedral angle."""
        if custom_attributes:
            raise NotImplementedError("custom attributes are not supported")
        edge_ke = self.default_edge_ke if edge_ke is None else edge_ke
        edge_kd = self.default_edge_kd if edge_kd is None else edge_kd
        x3 = np.asarray(self.particle_q[k], dtype=np.float32)
        x4 = np.asarray(self.particle_q[l], dtype=np.float32)
        if rest is None:
            rest = 0.0
            if i != -1 and j != -1:
                x1 = np.asarray(self.particle_q[i], dtype=np.float32)
                x2 = np.asarray(self.particle_q[j], dtype=np.float32)
                unit = lambda a: a / np.linalg.norm(a)  # noqa: E731
                n1 = unit(np.cross(x3 - x1, x4 - x1))
                n2 = unit(np.cross(x4 - x2, x3 - x2))
                e = unit(x4 - x3)
                cos_theta = np.clip(np.dot(n1, n2), -1.0, 1.0)
                sin_theta = np.dot(np.cross(n1, n2), e)
                rest = math.atan2(sin_theta, cos_theta)
        self.edge_indices.append((int(i), int(j), int(k), int(l)))
        self.edge_rest_angle.append(float(rest))
        self.edge_rest_length.append(float(np.linalg.norm(x4 - x3)))
        self.edge_bending_properties.append((float(edge_ke), float(edge_kd)))
        return len(self.edge_indices) - 1

    def add_tetrahedron(self, i: int, j: int, k: int, l: int, k_mu: float = 1.0e3, k_lambda: float = 1.0e3,
                        k_damp: float = 0.0, custom_attributes=None) -> float:
        """Tetrahedral element (builder.py:7522-7587): its inverse rest matrix from the particles' current
        positions; returns the rest volume (an inverted element is reported and not added)."""
        if custom_attributes:
            raise NotImplementedError("custom attributes are not supported")
        p, q, r, s = (np.array(self.particle_q[x]) for x in (i, j, k, l))
        Dm = np.array((q - p, r - p, s - p)).T
        volume = np.linalg.det(Dm) / 6.0
        if volume <= 0.0:
            print("inverted tetrahedral element")
        else:
            self.tet_indices.append((int(i), int(j), int(k), int(l)))
            self.tet_poses.append(np.linalg.inv(Dm).tolist())
            self.tet_activations.append(0.0)
            self.tet_materials.append((float(k_mu), float(k_lambda), float(k_damp)))
        return volume

    def request_state_attributes(self, *attributes: str) -> None:
        bad = sorted(set(attributes) - {"body_parent_f"})
        if bad:
            raise ValueError(f"Unknown state attribute(s): {', '.join(bad)}. Allowed: body_parent_f.")
        self._requested_state_attributes.update(attributes)

    def request_contact_attributes(self, *attributes: str) -> None:
        allowed = {"force"}
        bad = sorted(set(attributes) - allowed)
        if bad:
            raise ValueError(f"Unknown extended contact attribute(s): {', '.join(bad)}. Allowed: force.")
        self._requested_contact_attributes.update(attributes)

    # ------------------------------------------------------------------ pairs
    @staticmethod
    def _test_group_pair(a: int, b: int) -> bool:
        if a == 0 or b == 0:
            return False
        if a > 0:
            return a == b or b < 0
        return a != b

    def _test_world_and_group_pair(self, wa, wb, ga, gb) -> bool:
        if wa != -1 and wb != -1 and wa != wb:
            return False
        return self._test_group_pair(ga, gb)

    def find_shape_contact_pairs(self) -> np.ndarray:
        """Explicit pair list (builder.py:10855-10913): canonical (min, max) pairs."""
        flags = np.asarray(self.shape_flags, dtype=np.int64)
        colliding = [i for i in range(self.shape_count) if flags[i] & ShapeFlags.COLLIDE_SHAPES]
        order = sorted(colliding, key=lambda i: self.shape_world[i])
        pairs = []
        filters = {(min(a, b), max(a, b)) for a, b in self.shape_collision_filter_pairs}
        for i1 in range(len(order)):
            s1 = order[i1]
            w1 = self.shape_world[s1]
            g1 = self.shape_collision_group[s1]
            for i2 in range(i1 + 1, len(order)):
                s2 = order[i2]
                w2 = self.shape_world[s2]
                if w1 != -1 and w2 != -1 and w1 != w2:
                    break
                if not self._test_world_and_group_pair(w1, w2, g1, self.shape_collision_group[s2]):
                    continue
                a, b = (s2, s1) if s1 > s2 else (s1, s2)
                if (a, b) not in filters:
                    pairs.append((a, b))
        return np.asarray(pairs, dtype=np.int32).reshape(-1, 2)

    # ------------------------------------------------------------------ finalize
    def finalize(self, device=None, requires_grad: bool = False):
        from .model import Model

        return Model._from_builder(self, device=device, requires_grad=requires_grad)
