"""Model / State / Control containers (newton/_src/sim/{model,state,control}.py).

Arrays are torch tensors on the model's device, in the reference's layouts
(transform = 7 floats, spatial_vector = 6 floats, mat33 = 9 floats).  The
model also carries the per-world partition the B200 kernels work on: the
bodies, shapes and joints of a world are contiguous index ranges, and shapes
of world -1 (static, e.g. the ground plane) are shared by every world.
"""

from __future__ import annotations

import numpy as np
import torch

from ._abi import BodyFlags, JointType, NbModelDesc, ptr


def _dev(device) -> torch.device:
    if device is None:
        device = "cuda" if torch.cuda.is_available() else "cpu"
    d = torch.device(device)
    if d.type == "cuda" and d.index is None and torch.cuda.is_available():
        d = torch.device("cuda", torch.cuda.current_device())
    return d


class State:
    """Time-varying body state (newton/_src/sim/state.py)."""

    def __init__(self):
        self.body_q: torch.Tensor | None = None
        self.body_qd: torch.Tensor | None = None
        self.body_f: torch.Tensor | None = None
        self.particle_q: torch.Tensor | None = None
        self.particle_qd: torch.Tensor | None = None
        self.particle_f: torch.Tensor | None = None
        self.body_parent_f: torch.Tensor | None = None
        self.requires_grad = False

    def clear_forces(self) -> None:
        """Zero body_f and particle_f (state.py:156): body_f by a memset on the current stream through the
        library when it is a CUDA tensor."""
        if self.particle_f is not None:
            self.particle_f.zero_()
        if self.body_f is None:
            return
        if self.body_f.is_cuda and self.body_f.is_contiguous() and self.body_f.dtype == torch.float32:
            from . import _lib

            lib = _lib.load()
            _lib.check("nb_clear_forces", lib.nb_clear_forces(self.body_f.data_ptr(), int(self.body_f.shape[0]),
                                                               _lib.stream_handle(self.body_f.device)))
        else:
            self.body_f.zero_()

    def assign(self, other: "State") -> None:
        """Copy the arrays of ``other`` into this state (state.py:169)."""
        for name in ("body_q", "body_qd", "body_f", "particle_q", "particle_qd", "particle_f"):
            a, b = getattr(self, name), getattr(other, name)
            if a is not None and b is not None:
                a.copy_(b)

    @property
    def body_count(self) -> int:
        return 0 if self.body_q is None else int(self.body_q.shape[0])


class Control:
    """Control inputs (newton/_src/sim/control.py)."""

    def __init__(self):
        self.joint_target_pos: torch.Tensor | None = None
        self.joint_target_vel: torch.Tensor | None = None
        self.joint_f: torch.Tensor | None = None

    def clear(self) -> None:
        if self.joint_f is not None:
            self.joint_f.zero_()


class Model:
    """Static scene description (subset of newton.Model used by collide + SolverXPBD)."""

    def __init__(self, device=None):
        self.device = _dev(device)
        self.requires_grad = False
        self.body_count = 0
        self.shape_count = 0
        self.joint_count = 0
        self.joint_dof_count = 0
        self.world_count = 1
        self.rigid_contact_max = 0
        self.particle_count = 0
        self.spring_count = 0
        self.edge_count = 0
        self.tet_count = 0
        self.particle_max_radius = 0.0
        self._collision_pipeline = None
        self._requested_contact_attributes: set[str] = set()
        self._requested_state_attributes: set[str] = set()
        self._host: dict[str, np.ndarray] = {}

    # ------------------------------------------------------------ construction
    @classmethod
    def _from_builder(cls, b, device=None, requires_grad=False) -> "Model":
        m = cls(device)
        m.requires_grad = requires_grad
        B, S, J, D = b.body_count, b.shape_count, b.joint_count, b.joint_dof_count
        m.body_count, m.shape_count, m.joint_count, m.joint_dof_count = B, S, J, D
        f32 = np.float32
        h = {}
        h["body_q"] = np.asarray(b.body_q, dtype=f32).reshape(B, 7)
        h["body_qd"] = np.asarray(b.body_qd, dtype=f32).reshape(B, 6)
        h["body_com"] = np.asarray(b.body_com, dtype=f32).reshape(B, 3)
        h["body_mass"] = np.asarray(b.body_mass, dtype=f32).reshape(B)
        h["body_inv_mass"] = np.asarray(b.body_inv_mass, dtype=f32).reshape(B)
        h["body_inertia"] = np.asarray(b.body_inertia, dtype=f32).reshape(B, 9)
        h["body_inv_inertia"] = np.asarray(b.body_inv_inertia, dtype=f32).reshape(B, 9)
        h["body_flags"] = np.asarray(b.body_flags, dtype=np.int32).reshape(B)
        h["body_world"] = np.asarray(b.body_world, dtype=np.int32).reshape(B)
        h["shape_body"] = np.asarray(b.shape_body, dtype=np.int32).reshape(S)
        h["shape_type"] = np.asarray(b.shape_type, dtype=np.int32).reshape(S)
        h["shape_transform"] = np.asarray(b.shape_transform, dtype=f32).reshape(S, 7)
        h["shape_scale"] = np.asarray(b.shape_scale, dtype=f32).reshape(S, 3)
        h["shape_margin"] = np.asarray(b.shape_margin, dtype=f32).reshape(S)
        h["shape_gap"] = np.asarray(b.shape_gap, dtype=f32).reshape(S)
        h["shape_collision_radius"] = np.asarray(b.shape_radius, dtype=f32).reshape(S)
        h["shape_material_mu"] = np.asarray(b.shape_mu, dtype=f32).reshape(S)
        h["shape_material_mu_torsional"] = np.asarray(b.shape_mu_torsional, dtype=f32).reshape(S)
        h["shape_material_mu_rolling"] = np.asarray(b.shape_mu_rolling, dtype=f32).reshape(S)
        h["shape_material_restitution"] = np.asarray(b.shape_restitution, dtype=f32).reshape(S)
        h["shape_world"] = np.asarray(b.shape_world, dtype=np.int32).reshape(S)
        h["shape_flags"] = np.asarray(b.shape_flags, dtype=np.int32).reshape(S)
        h["shape_collision_group"] = np.asarray(b.shape_collision_group, dtype=np.int32).reshape(S)
        h["joint_type"] = np.asarray(b.joint_type, dtype=np.int32).reshape(J)
        h["joint_enabled"] = np.asarray(b.joint_enabled, dtype=np.int32).reshape(J)
        h["joint_parent"] = np.asarray(b.joint_parent, dtype=np.int32).reshape(J)
        h["joint_child"] = np.asarray(b.joint_child, dtype=np.int32).reshape(J)
        h["joint_X_p"] = np.asarray(b.joint_X_p, dtype=f32).reshape(J, 7)
        h["joint_X_c"] = np.asarray(b.joint_X_c, dtype=f32).reshape(J, 7)
        h["joint_qd_start"] = np.asarray(b.joint_qd_start, dtype=np.int32).reshape(J)
        h["joint_dof_dim"] = np.asarray(b.joint_dof_dim, dtype=np.int32).reshape(J, 2)
        h["joint_world"] = np.asarray(b.joint_world, dtype=np.int32).reshape(J)
        h["joint_axis"] = np.asarray(b.joint_axis, dtype=f32).reshape(D, 3)
        h["joint_limit_lower"] = np.asarray(b.joint_limit_lower, dtype=f32).reshape(D)
        h["joint_limit_upper"] = np.asarray(b.joint_limit_upper, dtype=f32).reshape(D)
        h["joint_target_ke"] = np.asarray(b.joint_target_ke, dtype=f32).reshape(D)
        h["joint_target_kd"] = np.asarray(b.joint_target_kd, dtype=f32).reshape(D)
        h["joint_target_pos"] = np.asarray(b.joint_target_pos, dtype=f32).reshape(D)
        h["joint_target_vel"] = np.asarray(b.joint_target_vel, dtype=f32).reshape(D)
        W = max(1, b.world_count)
        grav = list(b.world_gravity)
        u = b.up_vector
        default_g = (u[0] * b.gravity, u[1] * b.gravity, u[2] * b.gravity)
        while len(grav) < W:
            grav.append(default_g)
        h["gravity"] = np.asarray(grav, dtype=f32).reshape(W, 3)
        h["shape_contact_pairs"] = b.find_shape_contact_pairs()
        m._init_from_host(h, world_count=W, uses_worlds=b.world_count > 0,
                          filter_pairs={(min(x, y), max(x, y)) for x, y in b.shape_collision_filter_pairs},
                          requested=set(b._requested_contact_attributes))
        m._requested_state_attributes = set(b._requested_state_attributes)
        if b.particle_count:
            from . import particles

            particles.attach(m, b)
        return m

    @classmethod
    def _from_arrays(cls, h: dict, world_count: int, uses_worlds: bool = True, filter_pairs=None, device=None,
                     requires_grad=False) -> "Model":
        """Model from ready host arrays (same keys and layouts as a finalized builder)."""
        m = cls(device)
        m.requires_grad = requires_grad
        m.body_count = int(h["body_q"].shape[0])
        m.shape_count = int(h["shape_type"].shape[0])
        m.joint_count = int(h["joint_type"].shape[0])
        m.joint_dof_count = int(h["joint_axis"].shape[0])
        m._init_from_host(h, world_count=world_count, uses_worlds=uses_worlds,
                          filter_pairs=set(filter_pairs or ()), requested=set())
        return m

    def _init_from_host(self, h, world_count, uses_worlds, filter_pairs, requested):
        self.world_count = int(world_count)
        self.shape_collision_filter_pairs = filter_pairs
        self.shape_contact_pair_count = int(h["shape_contact_pairs"].shape[0])
        self.up_vector = (0.0, 0.0, 1.0)
        self._requested_contact_attributes = requested
        self._uses_worlds = uses_worlds
        self._host = h
        self._build_partition()
        dev = self.device
        for k, v in h.items():
            if k == "shape_contact_pairs":
                continue
            setattr(self, k, torch.from_numpy(np.ascontiguousarray(v)).to(dev))
        self.shape_contact_pairs = torch.from_numpy(np.ascontiguousarray(h["shape_contact_pairs"]))
        self._part_dev = {k: torch.from_numpy(np.ascontiguousarray(v)).to(dev) for k, v in self._part.items()}
        self._part_dev["body_pack"] = torch.zeros((max(self.body_count, 1), 24), dtype=torch.float32, device=dev)
        self.update_body_pack()

    def update_body_pack(self) -> None:
        """Refresh the packed per-body mass properties the step reads (``NbModelDesc.body_pack``): com,
        effective inverse mass, inertia, effective inverse inertia -- zero inverse mass and inertia for
        kinematic bodies, as the solver's ``_update_effective_inv_mass_inertia``
        (newton/_src/solvers/solver.py:160-174), which the reference runs at solver construction and
        in ``notify_model_changed``.  Updated in place, so descriptors keep their pointer."""
        B = self.body_count
        if B == 0:
            return
        kin = (self.body_flags.to(torch.int32) & int(BodyFlags.KINEMATIC)) != 0
        zero = torch.zeros((), dtype=torch.float32, device=self.device)
        inv_m = torch.where(kin, zero, self.body_inv_mass.reshape(B))
        inv_I = torch.where(kin[:, None], zero, self.body_inv_inertia.reshape(B, 9))
        pack = torch.cat([self.body_com.reshape(B, 3), inv_m[:, None], self.body_inertia.reshape(B, 9), inv_I,
                          torch.zeros((B, 2), dtype=torch.float32, device=self.device)], dim=1)
        self._part_dev["body_pack"].copy_(pack)

    def _build_partition(self) -> None:
        """World ranges + per-world candidate pair layout for the per-world kernels."""
        h = self._host
        W = self.world_count
        if self._uses_worlds:
            bw = h["body_world"]
            sw = h["shape_world"]
            jw = h["joint_world"]
        else:  # every entity in world -1: one world, static shapes included
            bw = np.zeros(self.body_count, np.int32)
            sw = np.zeros(self.shape_count, np.int32)
            jw = np.zeros(self.joint_count, np.int32)
        if np.any(bw < 0):
            raise ValueError("bodies in world -1 are not supported when worlds are used; add them inside a world")
        for name, arr, n in (("body", bw, self.body_count), ("joint", jw, self.joint_count)):
            if n and np.any(np.diff(arr) < 0):
                raise ValueError(f"{name}s of each world must be contiguous and in world order")
        local = sw[sw >= 0]
        if local.size and np.any(np.diff(local) < 0):
            raise ValueError("shapes of each world must be contiguous and in world order")
        glob = np.nonzero(sw < 0)[0].astype(np.int32)
        if np.any(h["shape_body"][glob] >= 0):
            raise ValueError("shapes in world -1 must be static (body -1)")
        # world-local shapes must form one block [l0, l1) ordered by world;
        # global shapes sit before or after it
        lidx = np.nonzero(sw >= 0)[0]
        if lidx.size and lidx[-1] - lidx[0] + 1 != lidx.size:
            raise ValueError("global (world -1) shapes must be added before or after all world shapes")

        def starts(arr, n_items, base=0):
            cnt = np.bincount(arr[arr >= 0], minlength=W)[:W] if n_items else np.zeros(W, np.int64)
            st = np.zeros(W + 1, np.int64)
            st[1:] = np.cumsum(cnt)
            return st + base

        if self.joint_count:
            for name in ("joint_child", "joint_parent"):
                jb = h[name]
                ok = (jb < 0) | (bw[np.clip(jb, 0, max(self.body_count - 1, 0))] == jw)
                if name == "joint_child":
                    ok &= jb >= 0
                if not np.all(ok):
                    raise ValueError(f"{name} of a joint is not a body of the joint's world")
        body_start = starts(bw, self.body_count)
        joint_start = starts(jw, self.joint_count)
        shape_start = starts(sw, lidx.size, int(lidx[0]) if lidx.size else 0)
        self._part = {
            "world_body_start": body_start.astype(np.int32),
            "world_joint_start": joint_start.astype(np.int32),
            "world_shape_start": shape_start.astype(np.int32),
            "global_shapes": glob,
        }
        cnts = np.diff(shape_start)
        self._world_of_shape = sw
        self._world_of_body = bw
        self.max_world_bodies = int(np.max(np.diff(body_start))) if W else 0
        self.max_world_joints = int(np.max(np.diff(joint_start))) if W else 0
        self.max_world_shapes = int(cnts.max() if cnts.size else 0) + int(glob.size)

    # ------------------------------------------------------------ factories
    def request_state_attributes(self, *attributes: str) -> None:
        """Optional State arrays (model.py request_state_attributes); "body_parent_f" only."""
        bad = sorted(set(attributes) - {"body_parent_f"})
        if bad:
            raise ValueError(f"Unknown state attribute(s): {', '.join(bad)}. Allowed: body_parent_f.")
        self._requested_state_attributes.update(attributes)

    def state(self, requires_grad: bool | None = None) -> State:
        s = State()
        s.body_q = self.body_q.clone()
        s.body_qd = self.body_qd.clone()
        s.body_f = torch.zeros((self.body_count, 6), dtype=torch.float32, device=self.device)
        if self.particle_count:
            s.particle_q = self.particle_q.clone()
            s.particle_qd = self.particle_qd.clone()
            s.particle_f = torch.zeros((self.particle_count, 3), dtype=torch.float32, device=self.device)
        if "body_parent_f" in self._requested_state_attributes:
            s.body_parent_f = torch.zeros((self.body_count, 6), dtype=torch.float32, device=self.device)
        s.requires_grad = bool(requires_grad) if requires_grad is not None else self.requires_grad
        return s

    def control(self, clone_variables: bool = True) -> Control:
        c = Control()
        if clone_variables:
            c.joint_target_pos = self.joint_target_pos.clone()
            c.joint_target_vel = self.joint_target_vel.clone()
        else:
            c.joint_target_pos = self.joint_target_pos
            c.joint_target_vel = self.joint_target_vel
        c.joint_f = torch.zeros(self.joint_dof_count, dtype=torch.float32, device=self.device)
        return c

    def request_contact_attributes(self, *attributes: str) -> None:
        bad = sorted(set(attributes) - {"force"})
        if bad:
            raise ValueError(f"Unknown extended contact attribute(s): {', '.join(bad)}. Allowed: force.")
        self._requested_contact_attributes.update(attributes)

    def get_requested_contact_attributes(self) -> set[str]:
        return set(self._requested_contact_attributes)

    def _default_pipeline(self):
        from .collide import CollisionPipeline

        if self._collision_pipeline is None:
            self._collision_pipeline = CollisionPipeline(self, broad_phase="explicit")
        return self._collision_pipeline

    def contacts(self, collision_pipeline=None):
        """Allocate a Contacts buffer for the default (or given) pipeline (model.py:970-994)."""
        pipe = collision_pipeline if collision_pipeline is not None else self._default_pipeline()
        return pipe.contacts()

    def collide(self, state: State, contacts=None, *, collision_pipeline=None):
        """Run collision detection (model.py:996-1022); returns the Contacts."""
        pipe = collision_pipeline if collision_pipeline is not None else self._default_pipeline()
        if contacts is None:
            contacts = pipe.contacts()
        pipe.collide(state, contacts)
        return contacts

    # ------------------------------------------------------------ descriptors
    def host(self, name: str) -> np.ndarray:
        return self._host[name]

    def make_desc(self, arrays: dict, pair_info: dict | None = None) -> NbModelDesc:
        """Fill an NbModelDesc from ``arrays`` (numpy or torch, same keys as the model)."""
        d = NbModelDesc()
        d.body_count = self.body_count
        d.shape_count = self.shape_count
        d.joint_count = self.joint_count
        d.joint_dof_count = self.joint_dof_count
        d.world_count = self.world_count
        d.global_shape_count = int(self._part["global_shapes"].size)
        d.max_world_bodies = self.max_world_bodies
        d.max_world_shapes = self.max_world_shapes
        d.max_world_joints = self.max_world_joints
        jt = np.asarray(self._host["joint_type"])
        d.all_joints_free = int(bool(np.all(jt == int(JointType.FREE))))
        names = {
            "body_com": "body_com", "body_mass": "body_mass", "body_inv_mass": "body_inv_mass",
            "body_inertia": "body_inertia", "body_inv_inertia": "body_inv_inertia", "body_flags": "body_flags",
            "body_world": "body_world", "gravity": "gravity", "shape_body": "shape_body",
            "shape_type": "shape_type", "shape_transform": "shape_transform", "shape_scale": "shape_scale",
            "shape_margin": "shape_margin", "shape_gap": "shape_gap", "shape_radius": "shape_collision_radius",
            "shape_mu": "shape_material_mu", "shape_mu_torsional": "shape_material_mu_torsional",
            "shape_mu_rolling": "shape_material_mu_rolling", "shape_restitution": "shape_material_restitution",
            "joint_type": "joint_type", "joint_enabled": "joint_enabled", "joint_parent": "joint_parent",
            "joint_child": "joint_child", "joint_X_p": "joint_X_p", "joint_X_c": "joint_X_c",
            "joint_qd_start": "joint_qd_start", "joint_dof_dim": "joint_dof_dim", "joint_axis": "joint_axis",
            "joint_limit_lower": "joint_limit_lower", "joint_limit_upper": "joint_limit_upper",
            "joint_target_ke": "joint_target_ke", "joint_target_kd": "joint_target_kd",
            "world_body_start": "world_body_start", "world_joint_start": "world_joint_start",
            "world_shape_start": "world_shape_start", "global_shapes": "global_shapes",
        }
        for field, key in names.items():
            setattr(d, field, ptr(arrays[key]))
        if pair_info is not None:
            d.pair_count = int(pair_info["pair_count"])
            d.max_world_pairs = int(pair_info["max_world_pairs"])
            d.contact_capacity = int(pair_info["contact_capacity"])
            d.world_pair_start = ptr(arrays["world_pair_start"])
            d.pair_shapes = ptr(arrays["pair_shapes"])
            d.world_order = ptr(arrays["world_order"])
        sched = arrays.get("schedule")
        if sched is not None:
            d.batch_count = int(sched.batch_count)
            d.worlds_per_group = 1
            d.group_threads = int(sched.group_threads)
            d.cta_threads = int(sched.cta_threads)
            d.smem_floats_per_batch = int(sched.arena_words)
            d.step_mode = int(sched.step_mode)
            d.batch_world = ptr(arrays["batch_world"])
            d.batch_slab = ptr(arrays["batch_slab"])
        if "body_pack" in arrays:
            d.body_pack = ptr(arrays["body_pack"])
        return d

    def host_arrays(self) -> dict:
        a = dict(self._host)
        a.update(self._part)
        return a

    def device_arrays(self) -> dict:
        a = {k: getattr(self, k) for k in self._host if k != "shape_contact_pairs"}
        a.update(self._part_dev)
        return a
