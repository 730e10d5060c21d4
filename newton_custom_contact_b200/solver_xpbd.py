"""SolverXPBD (newton/_src/solvers/xpbd/solver_xpbd.py) for rigid bodies on B200.

``step(state_in, state_out, control, contacts, dt)`` is one launch of the fused
per-world substep kernel (integrate, ``iterations`` x contact + joint
projection, delta application) from libnewton_b200.so.  Differences from the
reference that a caller can observe:
  * ``state_in`` is left unchanged (the reference ping-pongs through it,
    solver_xpbd.py:203-257);
  * per-body constraint deltas are summed in float in contact (joint) order --
    the reference's sums run sequentially -- so results are bit-reproducible
    where the reference's atomic order is unspecified;
  * particles (particles.py: integration, springs, particle-particle and
    particle-static-shape contacts) run before the bodies in every substep;
    particle contacts with body-attached shapes, particle restitution,
    triangles, bending edges and tetrahedra raise ``NotImplementedError``;
  * an optional learned warm start (``solver.warm_start``, warmstart.py) has
    no counterpart in the reference; it is off by default.
"""

from __future__ import annotations

import ctypes as C

import torch

from . import _lib
from ._abi import NbContactSeg, NbStepIO, NbXpbdParams, ptr
from .contacts import Contacts


class SolverNotifyFlags:
    JOINT_PROPERTIES = 1 << 0
    JOINT_DOF_PROPERTIES = 1 << 1
    BODY_PROPERTIES = 1 << 2
    BODY_INERTIAL_PROPERTIES = 1 << 3
    SHAPE_PROPERTIES = 1 << 4
    MODEL_PROPERTIES = 1 << 5


class SolverXPBD:
    """Rigid-body XPBD substep (Macklin et al. 2016, Müller et al. 2020)."""

    def __init__(self, model, iterations: int = 2, soft_body_relaxation: float = 0.9,
                 soft_contact_relaxation: float = 0.9, joint_linear_relaxation: float = 0.7,
                 joint_angular_relaxation: float = 0.4, joint_linear_compliance: float = 0.0,
                 joint_angular_compliance: float = 0.0, rigid_contact_relaxation: float = 0.8,
                 rigid_contact_con_weighting: bool = True, angular_damping: float = 0.0,
                 enable_restitution: bool = False):
        if iterations < 0:
            raise ValueError("iterations must be non-negative")
        self.model = model
        # the effective mass properties, as SolverBase._init_kinematic_state (solver.py:196-215)
        model.update_body_pack()
        self.iterations = int(iterations)
        self.soft_body_relaxation = soft_body_relaxation
        self.soft_contact_relaxation = soft_contact_relaxation
        self.joint_linear_relaxation = joint_linear_relaxation
        self.joint_angular_relaxation = joint_angular_relaxation
        self.joint_linear_compliance = joint_linear_compliance
        self.joint_angular_compliance = joint_angular_compliance
        self.rigid_contact_relaxation = rigid_contact_relaxation
        self.rigid_contact_con_weighting = rigid_contact_con_weighting
        self.angular_damping = angular_damping
        self.enable_restitution = enable_restitution
        self.compute_body_velocity_from_position_delta = False
        self._desc_cache = {}
        self._empty_seg = None
        self._last_dt = None
        self._contact_impulse = None
        self._contact_impulse_capacity = 0
        self._joint_impulse = None
        # optional learned warm start (warmstart.WarmStart); None = the plain solver
        self.warm_start = None
        self._particles = None
        if getattr(model, "particle_count", 0):
            from .particles import ParticleSolver

            self._particles = ParticleSolver(model, self)

    @property
    def device(self):
        return self.model.device

    def notify_model_changed(self, flags: int) -> None:
        """Model arrays are read at every step, except the effective (kinematic-aware) mass properties,
        which are refreshed here as in the reference (solver.py:160-174); cached descriptors are
        dropped."""
        self.model.update_body_pack()
        self._desc_cache.clear()

    def params(self) -> NbXpbdParams:
        p = NbXpbdParams()
        p.iterations = self.iterations
        p.rigid_contact_con_weighting = 1 if self.rigid_contact_con_weighting else 0
        p.enable_restitution = 1 if self.enable_restitution else 0
        p.joint_linear_relaxation = self.joint_linear_relaxation
        p.joint_angular_relaxation = self.joint_angular_relaxation
        p.joint_linear_compliance = self.joint_linear_compliance
        p.joint_angular_compliance = self.joint_angular_compliance
        p.rigid_contact_relaxation = self.rigid_contact_relaxation
        p.angular_damping = self.angular_damping
        return p

    def _desc_for(self, contacts: Contacts | None):
        pipe = contacts._layout if contacts is not None and contacts._layout is not None else None
        if pipe is None:
            pipe = self.model._default_pipeline()
        return pipe, pipe.desc()

    @staticmethod
    def _check_state(name, t, shape):
        if t is None or t.dtype != torch.float32 or not t.is_contiguous() or tuple(t.shape) != shape:
            raise TypeError(f"{name} must be a contiguous float32 tensor of shape {shape}")

    def step(self, state_in, state_out, control, contacts: Contacts | None, dt: float) -> None:
        model = self.model
        _lib.require_cuda(model.device)
        if self._particles is not None:
            # particles touch static shapes only, so their substep is independent of the bodies'
            self._particles.step(state_in, state_out, contacts, dt)
        if model.body_count == 0:
            return
        # control=None: the model's default targets and no joint forces (the reference builds
        # model.control(), whose joint_f is zero; a null joint_f skips the same work without a fill)
        joint_f = None if control is None else control.joint_f
        if control is None:
            control = model
        B = model.body_count
        self._check_state("state_in.body_q", state_in.body_q, (B, 7))
        self._check_state("state_in.body_qd", state_in.body_qd, (B, 6))
        self._check_state("state_in.body_f", state_in.body_f, (B, 6))
        self._check_state("state_out.body_q", state_out.body_q, (B, 7))
        self._check_state("state_out.body_qd", state_out.body_qd, (B, 6))
        lib = _lib.load()
        stream = _lib.stream_handle(model.device)
        pipe, desc = self._desc_for(contacts)
        if contacts is not None:
            if contacts._seg is None or contacts._layout is None:
                pipe.attach_segments(contacts)
            if not contacts._seg_valid:
                pub = pipe.public_struct(contacts)
                seg = pipe.seg_struct(contacts)
                _lib.check("nb_ingest_contacts", lib.nb_ingest_contacts(C.byref(desc), C.byref(pub), C.byref(seg),
                                                                        C.c_void_p(stream)))
                contacts._seg_valid = True
            seg = pipe.seg_struct(contacts)
        else:
            if self._empty_seg is None:
                self._empty_seg = {"work_counter": torch.zeros(8, dtype=torch.int32, device=model.device),
                                   "status": torch.zeros(1, dtype=torch.int32, device=model.device)}
            seg = NbContactSeg()
            seg.work_counter = ptr(self._empty_seg["work_counter"])
            seg.world_count = None
            seg.status = ptr(self._empty_seg["status"])
        io = NbStepIO()
        io.body_q_in = ptr(state_in.body_q)
        io.body_qd_in = ptr(state_in.body_qd)
        io.body_f_in = ptr(state_in.body_f)
        io.body_q_out = ptr(state_out.body_q)
        io.body_qd_out = ptr(state_out.body_qd)
        io.joint_target_pos = ptr(control.joint_target_pos)
        io.joint_target_vel = ptr(control.joint_target_vel)
        io.joint_f = ptr(joint_f)
        if state_out.body_parent_f is not None:
            # incoming joint wrench per body (solver_xpbd.py:294-297, 636-655)
            self._check_state("state_out.body_parent_f", state_out.body_parent_f, (B, 6))
            io.body_parent_f = ptr(state_out.body_parent_f)
            if model.joint_count > 0:
                if self._joint_impulse is None or self._joint_impulse.device != model.device:
                    self._joint_impulse = torch.zeros((model.joint_count, 6), dtype=torch.float32,
                                                      device=model.device)
                io.joint_impulse = ptr(self._joint_impulse)
        impulse = None
        if contacts is not None and contacts.force is not None:
            # solver-owned accumulated impulse (solver_xpbd.py:286-291), zeroed every step
            cap = contacts.rigid_contact_max
            impulse = self._contact_impulse
            if impulse is None or impulse.shape[0] != cap or impulse.device != model.device:
                impulse = torch.zeros((max(cap, 1), 6), dtype=torch.float32, device=model.device)
            else:
                impulse.zero_()
            io.contact_impulse = ptr(impulse)
            io.impulse_scratch = ptr(contacts._seg["impulse_scratch"])
            io.contact_impulse_capacity = cap
        params = self.params()
        ws = self.warm_start if contacts is not None else None
        if ws is not None:
            ws.before_step(model, pipe, desc, state_in, contacts, dt, io)
            if ws.enabled() and ws.iterations is not None:
                params.iterations = int(ws.iterations)
        grid = pipe.grid()
        _lib.check("nb_xpbd_step", lib.nb_xpbd_step(C.byref(desc), C.byref(params), C.byref(io), C.byref(seg),
                                                    float(dt), grid, C.c_void_p(stream)))
        if ws is not None:
            ws.after_step(contacts)
        self._contact_impulse = impulse
        self._contact_impulse_capacity = contacts.rigid_contact_max if contacts is not None else 0
        self._last_dt = dt

    def step_substeps(self, state_in, state_out, contacts: Contacts, dt: float, substeps: int) -> None:
        """`substeps` x (collide, step) in one library call (``nb_xpbd_substeps``; no counterpart in the
        reference, whose examples loop ``model.collide`` + ``solver.step`` on the host): the pipeline that
        made `contacts` collides at every substep, ``state_in.body_f`` is applied at every substep,
        ``state_out`` receives the final state and ``state_in`` is overwritten (ping-pong buffer).
        The plain solve only: no contact forces, ``body_parent_f`` or warm start."""
        model = self.model
        _lib.require_cuda(model.device)
        if substeps < 0:
            raise ValueError("substeps must be non-negative")
        if model.body_count == 0 or substeps == 0:
            return
        if contacts.force is not None or state_out.body_parent_f is not None or self.warm_start is not None:
            raise ValueError("step_substeps runs the plain solve only (no contact forces, body_parent_f or warm "
                             "start)")
        B = model.body_count
        for name, t, shape in (("state_in.body_q", state_in.body_q, (B, 7)), ("state_in.body_qd", state_in.body_qd, (B, 6)),
                               ("state_in.body_f", state_in.body_f, (B, 6)), ("state_out.body_q", state_out.body_q, (B, 7)),
                               ("state_out.body_qd", state_out.body_qd, (B, 6))):
            self._check_state(name, t, shape)
        pipe = contacts._layout
        if pipe is None:
            raise ValueError("contacts must come from a CollisionPipeline (pipeline.contacts())")
        if getattr(pipe, "contact_matching", "disabled") != "disabled":
            raise ValueError("step_substeps does not run contact matching; call collide and step per substep")
        if contacts._seg is None:
            pipe.attach_segments(contacts)
        if contacts._world_offset.numel() != model.world_count + 1:
            contacts._world_offset = torch.zeros(model.world_count + 1, dtype=torch.int64, device=model.device)
        lib = _lib.load()
        desc = pipe.desc()
        io = NbStepIO()
        io.body_q_in, io.body_qd_in, io.body_f_in = ptr(state_in.body_q), ptr(state_in.body_qd), ptr(state_in.body_f)
        io.body_q_out, io.body_qd_out = ptr(state_out.body_q), ptr(state_out.body_qd)
        # the model's default targets, no joint forces (a default Control's joint_f is zero)
        io.joint_target_pos = ptr(model.joint_target_pos)
        io.joint_target_vel = ptr(model.joint_target_vel)
        params = self.params()
        _lib.check("nb_xpbd_substeps", lib.nb_xpbd_substeps(
            C.byref(desc), C.byref(params), C.byref(io), C.byref(pipe.seg_struct(contacts)),
            C.byref(pipe.public_struct(contacts)), float(dt), int(substeps), pipe.grid(),
            C.c_void_p(_lib.stream_handle(model.device))))
        contacts._seg_valid = True
        self._last_dt = dt

    def update_contacts(self, contacts: Contacts, state=None) -> None:
        """Populate ``contacts.force`` (force [N], torque [N m] per contact) from the impulses the last
        ``step`` accumulated (solver_xpbd.py:766-821); same errors as the reference."""
        if contacts.force is None:
            raise ValueError("contacts.force is not allocated. Call model.request_contact_attributes('force') "
                             "before creating the Contacts object.")
        if self._contact_impulse is None:
            raise ValueError("No contact impulse data available. Call step() before update_contacts().")
        if contacts.rigid_contact_max != self._contact_impulse_capacity:
            raise ValueError(
                f"Contacts capacity mismatch: update_contacts() received rigid_contact_max="
                f"{contacts.rigid_contact_max}, but step() used {self._contact_impulse_capacity}. "
                f"Pass the same Contacts instance to both step() and update_contacts().")
        lib = _lib.load()
        stream = _lib.stream_handle(self.model.device)
        _lib.check("nb_contact_forces", lib.nb_contact_forces(
            C.c_void_p(ptr(self._contact_impulse)), C.c_void_p(ptr(contacts.rigid_contact_count)),
            int(contacts.rigid_contact_max), float(self._last_dt), C.c_void_p(ptr(contacts.force)),
            C.c_void_p(stream)))
