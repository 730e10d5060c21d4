"""Particles: model arrays, soft contacts and the XPBD particle substep.

The particle branch of the reference's pipeline, on the library's kernels
(``nb_soft_collide`` and ``nb_particle_step``):

  * ``Model`` particle / spring arrays (newton/_src/sim/model.py; finalized
    from ``ModelBuilder.add_particle`` / ``add_spring``, builder.py:9818-9855);
  * soft contacts of particles with shapes, filled by
    ``CollisionPipeline.collide`` (collide.py:1194-1230);
  * the particle part of ``SolverXPBD.step`` (solver_xpbd.py:303-320,
    377-505, 657-660): integration, particle-shape contacts,
    particle-particle contacts, springs, position corrections.

Particles collide with each other and with STATIC shapes: the solver raises
for a model where a particle-colliding shape is attached to a body (the
two-way particle-body coupling is not built).  Bending edges, tetrahedra
and particle restitution are built.
"""

from __future__ import annotations

import ctypes as C

import numpy as np
import torch

from . import _lib
from ._abi import NbParticleDesc, NbParticleIO, NbSoftContacts, ShapeFlags, ptr


def attach(model, b) -> None:
    """Copy the builder's particles and springs into ``model`` (host arrays + device tensors)."""
    P, S = b.particle_count, b.spring_count
    model.particle_count = P
    model.spring_count = S
    model.particle_max_velocity = float(b.particle_max_velocity)
    model.particle_mu = 0.5
    model.particle_cohesion = 0.0
    model.particle_adhesion = 0.0
    model.soft_contact_mu = 0.5
    model.soft_contact_restitution = 0.0
    f32 = np.float32
    h = {}
    h["particle_q"] = np.asarray(b.particle_q, dtype=f32).reshape(P, 3)
    h["particle_qd"] = np.asarray(b.particle_qd, dtype=f32).reshape(P, 3)
    ms = np.asarray(b.particle_mass, dtype=f32).reshape(P)
    h["particle_mass"] = ms
    h["particle_inv_mass"] = np.divide(f32(1.0), ms, out=np.zeros_like(ms), where=ms != 0.0)
    h["particle_radius"] = np.asarray(b.particle_radius, dtype=f32).reshape(P)
    h["particle_flags"] = np.asarray(b.particle_flags, dtype=np.int32).reshape(P)
    h["particle_world"] = np.asarray(b.particle_world, dtype=np.int32).reshape(P)
    h["spring_indices"] = np.asarray(b.spring_indices, dtype=np.int32).reshape(S * 2)
    h["spring_rest_length"] = np.asarray(b.spring_rest_length, dtype=f32).reshape(S)
    h["spring_stiffness"] = np.asarray(b.spring_stiffness, dtype=f32).reshape(S)
    h["spring_damping"] = np.asarray(b.spring_damping, dtype=f32).reshape(S)
    h["spring_control"] = np.asarray(b.spring_control, dtype=f32).reshape(S)
    # springs of each particle, ascending spring index (the order the corrections are summed in)
    ends = h["spring_indices"].reshape(S, 2)
    owner = np.concatenate([ends[:, 0], ends[:, 1]]).astype(np.int64)
    spring = np.concatenate([np.arange(S), np.arange(S)]).astype(np.int64)
    order = np.lexsort((spring, owner))
    h["particle_spring_list"] = spring[order].astype(np.int32)
    start = np.zeros(P + 1, dtype=np.int32)
    np.cumsum(np.bincount(owner, minlength=P), out=start[1:])
    h["particle_spring_start"] = start
    E = b.edge_count
    model.edge_count = E
    h["edge_indices"] = np.asarray(b.edge_indices, dtype=np.int32).reshape(E, 4)
    h["edge_rest_angle"] = np.asarray(b.edge_rest_angle, dtype=f32).reshape(E)
    h["edge_rest_length"] = np.asarray(b.edge_rest_length, dtype=f32).reshape(E)
    h["edge_bending_properties"] = np.asarray(b.edge_bending_properties, dtype=f32).reshape(E, 2)
    # bending edges of each particle, ascending edge index (an edge with a -1 vertex does nothing)
    ev = h["edge_indices"]
    live = np.nonzero((ev >= 0).all(axis=1))[0]
    owner = ev[live].reshape(-1).astype(np.int64)
    edge = np.repeat(live, 4).astype(np.int64)
    pairs = np.unique(np.stack([owner, edge], axis=1), axis=0) if owner.size else np.zeros((0, 2), np.int64)
    h["particle_edge_list"] = pairs[:, 1].astype(np.int32)
    estart = np.zeros(P + 1, dtype=np.int32)
    np.cumsum(np.bincount(pairs[:, 0], minlength=P), out=estart[1:])
    h["particle_edge_start"] = estart
    T = b.tet_count
    model.tet_count = T
    h["tet_indices"] = np.asarray(b.tet_indices, dtype=np.int32).reshape(T, 4)
    h["tet_poses"] = np.asarray(b.tet_poses, dtype=f32).reshape(T, 9)
    h["tet_activations"] = np.asarray(b.tet_activations, dtype=f32).reshape(T)
    h["tet_materials"] = np.asarray(b.tet_materials, dtype=f32).reshape(T, 3)
    tv = h["tet_indices"]
    tpairs = (np.unique(np.stack([tv.reshape(-1).astype(np.int64), np.repeat(np.arange(T), 4)], axis=1), axis=0)
              if T else np.zeros((0, 2), np.int64))
    h["particle_tet_list"] = tpairs[:, 1].astype(np.int32)
    tstart = np.zeros(P + 1, dtype=np.int32)
    np.cumsum(np.bincount(tpairs[:, 0], minlength=P), out=tstart[1:])
    h["particle_tet_start"] = tstart
    model.particle_max_radius = float(h["particle_radius"].max()) if P else 0.0
    model._host.update(h)
    dev = model.device
    for k, v in h.items():
        setattr(model, k, torch.from_numpy(np.ascontiguousarray(v)).to(dev))


def params(model) -> dict:
    """The model's particle scalars (the oracle reads the same dict)."""
    return {k: float(getattr(model, k)) for k in ("particle_max_velocity", "particle_max_radius", "particle_mu",
                                                  "particle_cohesion", "particle_adhesion", "soft_contact_mu",
                                                  "soft_contact_restitution")}


def desc(model) -> NbParticleDesc:
    d = NbParticleDesc()
    d.particle_count = model.particle_count
    d.spring_count = model.spring_count
    d.shape_count = model.shape_count
    d.world_count = int(model.gravity.shape[0])
    for k, v in params(model).items():
        setattr(d, k, v)
    for k in ("particle_inv_mass", "particle_radius", "particle_flags", "particle_world", "gravity",
              "spring_indices", "spring_rest_length", "spring_stiffness", "spring_damping", "particle_spring_start",
              "particle_spring_list", "shape_body", "shape_type", "shape_transform", "shape_scale", "shape_world",
              "shape_flags"):
        setattr(d, k, ptr(getattr(model, k)))
    d.shape_mu = ptr(model.shape_material_mu)
    d.tet_count = model.tet_count
    for k in ("tet_indices", "tet_poses", "particle_tet_start", "particle_tet_list"):
        setattr(d, k, ptr(getattr(model, k)))
    d.edge_count = model.edge_count
    for k in ("edge_indices", "edge_rest_angle", "edge_bending_properties", "particle_edge_start",
              "particle_edge_list"):
        setattr(d, k, ptr(getattr(model, k)))
    return d


def soft_scratch_len(P: int) -> int:
    return P + 2 + (P + 1023) // 1024


def soft_struct(contacts, P: int) -> NbSoftContacts:
    sc = NbSoftContacts()
    sc.count = ptr(contacts.soft_contact_count)
    sc.particle = ptr(contacts.soft_contact_particle)
    sc.shape = ptr(contacts.soft_contact_shape)
    sc.body_pos = ptr(contacts.soft_contact_body_pos)
    sc.body_vel = ptr(contacts.soft_contact_body_vel)
    sc.normal = ptr(contacts.soft_contact_normal)
    sc.max = contacts.soft_contact_max
    sc.margin = float(contacts._soft_margin)
    n = soft_scratch_len(P)
    if contacts._soft_particle_start is None or contacts._soft_particle_start.numel() < n:
        contacts._soft_particle_start = torch.zeros(n, dtype=torch.int32, device=contacts.device)
    sc.particle_start = ptr(contacts._soft_particle_start)
    return sc


def soft_collide(model, state, contacts, margin: float) -> None:
    """Soft contacts of the state's particles with the model's shapes (collide.py:1194-1230)."""
    if state.particle_q is None:
        raise ValueError("state.particle_q is missing: create the state with model.state()")
    lib = _lib.load()
    contacts._soft_margin = float(margin)
    sc = soft_struct(contacts, model.particle_count)
    d = desc(model)
    bq = state.body_q if model.body_count else None
    _lib.check("nb_soft_collide", lib.nb_soft_collide(C.byref(d), C.c_void_p(ptr(state.particle_q)),
                                                      C.c_void_p(ptr(bq)), C.byref(sc),
                                                      C.c_void_p(_lib.stream_handle(model.device))))
    contacts._soft_valid = True


class ParticleSolver:
    """The particle half of SolverXPBD.step, with its work buffers."""

    def __init__(self, model, solver):
        flags = model.host("shape_flags")
        body = model.host("shape_body")
        coupled = np.nonzero(((flags & int(ShapeFlags.COLLIDE_PARTICLES)) != 0) & (body >= 0))[0]
        if coupled.size:
            raise NotImplementedError(
                f"particle contacts with body-attached shapes (e.g. shape {int(coupled[0])}) are not supported: "
                "this build couples particles to static shapes only; build those shapes with "
                "has_particle_collision=False")
        self.model = model
        self.solver = solver
        P = model.particle_count
        dev = model.device
        self.grid_size = 1 << max(6, int(2 * P - 1).bit_length())
        self.delta = torch.zeros((P, 3), dtype=torch.float32, device=dev)
        self.grid_head = torch.full((2 * self.grid_size,), -1, dtype=torch.int32, device=dev)
        self.grid_next = torch.full((max(P, 1),), -1, dtype=torch.int32, device=dev)
        self.status_word = torch.zeros(1, dtype=torch.int32, device=dev)

    def step(self, state_in, state_out, contacts, dt: float) -> None:
        model = self.model
        P = model.particle_count
        for name, st in (("state_in", state_in), ("state_out", state_out)):
            for k in ("particle_q", "particle_qd"):
                t = getattr(st, k)
                if t is None or t.dtype != torch.float32 or not t.is_contiguous() or tuple(t.shape) != (P, 3):
                    raise TypeError(f"{name}.{k} must be a contiguous float32 tensor of shape ({P}, 3)")
        io = NbParticleIO()
        io.particle_q = ptr(state_in.particle_q)
        io.particle_qd = ptr(state_in.particle_qd)
        io.particle_f = ptr(state_in.particle_f)
        io.particle_q_out = ptr(state_out.particle_q)
        io.particle_qd_out = ptr(state_out.particle_qd)
        io.delta = ptr(self.delta)
        io.grid_head = ptr(self.grid_head)
        io.grid_next = ptr(self.grid_next)
        io.grid_size = self.grid_size
        io.enable_restitution = int(bool(self.solver.enable_restitution))
        io.status = ptr(self.status_word)
        sc = None
        if contacts is not None and contacts.soft_contact_max > 0 and getattr(contacts, "_soft_valid", False):
            sc = soft_struct(contacts, P)
        d = desc(model)
        d.soft_body_relaxation = float(self.solver.soft_body_relaxation)
        lib = _lib.load()
        _lib.check("nb_particle_step", lib.nb_particle_step(
            C.byref(d), C.byref(io), C.byref(sc) if sc is not None else None, float(dt),
            int(self.solver.iterations), float(self.solver.soft_contact_relaxation),
            C.c_void_p(_lib.stream_handle(model.device))))

    def status(self) -> int:
        """Sticky NB_STATUS_* bits of the particle step (synchronises)."""
        return int(self.status_word.item())
