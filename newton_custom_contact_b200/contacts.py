"""Contacts container (newton/_src/sim/contacts.py:43-358).

Holds the reference's dense rigid-contact arrays (what users read and what a
custom contact writer fills) plus the solver-format per-world segments the
B200 kernels work on.  ``CollisionPipeline.collide`` fills both; contacts
written by hand into the dense arrays are moved into the segments by the
solver (``nb_ingest_contacts``) when ``contacts.mark_dense_modified()`` was
called or the buffer was never filled by a pipeline.
"""

from __future__ import annotations

import torch


class Contacts:
    EXTENDED_ATTRIBUTES: frozenset[str] = frozenset(("force",))

    @classmethod
    def validate_extended_attributes(cls, attributes) -> None:
        if not attributes:
            return
        invalid = sorted(set(attributes).difference(cls.EXTENDED_ATTRIBUTES))
        if invalid:
            allowed = ", ".join(sorted(cls.EXTENDED_ATTRIBUTES))
            raise ValueError(f"Unknown extended contact attribute(s): {', '.join(invalid)}. Allowed: {allowed}.")

    def __init__(self, rigid_contact_max: int, soft_contact_max: int = 0, requires_grad: bool = False, device=None,
                 per_contact_shape_properties: bool = False, clear_buffers: bool = False,
                 requested_attributes: set[str] | None = None, contact_matching: bool = False,
                 contact_report: bool = False, world_count: int | None = None, deterministic: bool = True):
        if contact_report and not contact_matching:
            raise ValueError("contact_report=True requires contact_matching=True")
        if rigid_contact_max < 0:
            raise ValueError("rigid_contact_max must be non-negative")
        self.validate_extended_attributes(requested_attributes)
        from .model import _dev

        dev = _dev(device)
        self.device = dev
        self.requires_grad = requires_grad
        self.per_contact_shape_properties = per_contact_shape_properties
        self.clear_buffers = clear_buffers
        n = int(rigid_contact_max)
        i32 = dict(dtype=torch.int32, device=dev)
        f32 = dict(dtype=torch.float32, device=dev)
        self.contact_counters = torch.zeros(2, **i32)
        self.rigid_contact_count = self.contact_counters[0:1]
        self.contact_generation = torch.zeros(1, **i32)
        self.rigid_contact_point_id = torch.zeros(n, **i32)
        self.rigid_contact_shape0 = torch.full((n,), -1, **i32)
        self.rigid_contact_shape1 = torch.full((n,), -1, **i32)
        self.rigid_contact_point0 = torch.zeros((n, 3), **f32)
        self.rigid_contact_point1 = torch.zeros((n, 3), **f32)
        self.rigid_contact_offset0 = torch.zeros((n, 3), **f32)
        self.rigid_contact_offset1 = torch.zeros((n, 3), **f32)
        self.rigid_contact_normal = torch.zeros((n, 3), **f32)
        self.rigid_contact_margin0 = torch.zeros(n, **f32)
        self.rigid_contact_margin1 = torch.zeros(n, **f32)
        self.rigid_contact_tids = torch.full((n,), -1, **i32)
        self.rigid_contact_force = torch.zeros((n, 3), **f32)
        self.rigid_contact_stiffness = torch.zeros(0, **f32)
        self.rigid_contact_damping = torch.zeros(0, **f32)
        self.rigid_contact_friction = torch.zeros(0, **f32)
        self.rigid_contact_sort_key = torch.zeros(n if deterministic else 0, dtype=torch.int64, device=dev)
        self.contact_matching = bool(contact_matching)
        self.contact_report = bool(contact_report)
        self.rigid_contact_match_index = torch.full((n,), -1, **i32) if contact_matching else None
        if contact_report:
            self.rigid_contact_new_indices = torch.zeros(n, **i32)
            self.rigid_contact_new_count = torch.zeros(1, **i32)
            self.rigid_contact_broken_indices = torch.zeros(n, **i32)
            self.rigid_contact_broken_count = torch.zeros(1, **i32)
        else:
            self.rigid_contact_new_indices = None
            self.rigid_contact_new_count = None
            self.rigid_contact_broken_indices = None
            self.rigid_contact_broken_count = None
        self.force = torch.zeros((n, 6), **f32) if requested_attributes and "force" in requested_attributes else None
        self.soft_contact_max = int(soft_contact_max)
        self.soft_contact_count = self.contact_counters[1:2]
        ns = self.soft_contact_max
        self.soft_contact_particle = torch.zeros(ns, **i32)
        self.soft_contact_shape = torch.zeros(ns, **i32)
        self.soft_contact_body_pos = torch.zeros((ns, 3), **f32)
        self.soft_contact_body_vel = torch.zeros((ns, 3), **f32)
        self.soft_contact_normal = torch.zeros((ns, 3), **f32)
        # per-particle first contact, written with the soft contacts (allocated by the first collide)
        self._soft_particle_start: torch.Tensor | None = None
        self._soft_margin = 0.0
        self._soft_valid = False
        self.rigid_contact_max = n
        # solver-format segments; attached by CollisionPipeline.contacts()
        self._seg: dict[str, torch.Tensor] | None = None
        self._layout = None
        self._seg_valid = False
        self._world_offset = torch.zeros((world_count or 1) + 1, dtype=torch.int64, device=dev)

    def clear(self, bump_generation: bool = True) -> None:
        self.contact_counters.zero_()
        self._soft_valid = False
        if bump_generation:
            self.contact_generation.add_(1)
        if self.clear_buffers:
            self.rigid_contact_shape0.fill_(-1)
            self.rigid_contact_shape1.fill_(-1)
            for t in (self.rigid_contact_point0, self.rigid_contact_point1, self.rigid_contact_offset0,
                      self.rigid_contact_offset1, self.rigid_contact_normal, self.rigid_contact_margin0,
                      self.rigid_contact_margin1):
                t.zero_()
        self._seg_valid = False

    def mark_dense_modified(self) -> None:
        """Declare that the dense arrays were written by the caller (custom contact writer)."""
        self._seg_valid = False

    @property
    def device_count(self) -> int:
        return int(self.rigid_contact_count.item())
