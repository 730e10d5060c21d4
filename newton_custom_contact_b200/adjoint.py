"""Differentiable XPBD substeps: the hand-written adjoint behind torch.autograd.

The reference differentiates a rollout by recording ``collide`` +
``SolverXPBD.step`` on a ``wp.Tape`` (state arrays created with
``model.state(requires_grad=True)``, newton/_src/solvers/xpbd/solver_xpbd.py)
and calling ``tape.backward``.  Here ``simulate(...)`` runs the rollout with
the library's forward kernels and returns torch tensors whose gradients
(``loss.backward()``) come from ``nb_xpbd_step_adjoint``, one reverse
substep at a time:

* the forward pass keeps the body state every ``checkpoint_every`` substeps
  (16 by default) and nothing else, so memory is bounded by the checkpoint
  count plus one segment;
* the backward pass re-simulates each segment from its checkpoint (collide
  included, so every substep sees the contacts the forward pass saw), then
  runs the adjoint kernel over the segment's substeps in reverse.

What is differentiated: free rigid bodies with contacts; gradients with
respect to the initial ``body_q``, ``body_qd``, a constant ``body_f``
(applied at every substep) and, optionally, the shapes' friction
coefficients ``shape_mu`` (a contact's coefficient is the mean of its two
shapes', newton/_src/solvers/xpbd/kernels.py:2160-2178; a per-world friction
is a differentiable map from world to shape coefficients that the caller
builds in torch).  Within a substep the contact set and the
contacts' body-frame points, offsets, normals and margins are held fixed,
as are which contacts are active, the contact counts of the weighting and
the friction-cone / velocity-threshold branches.  Not differentiated
(raise): enabled non-free joints, restitution, contact matching, the
learned warm start.
"""

from __future__ import annotations

import ctypes as C

import torch

from . import _lib
from ._abi import NbAdjointIO, ptr


class SubstepAdjoint:
    """Scratch buffers and the call of ``nb_xpbd_step_adjoint`` for one solver."""

    def __init__(self, solver):
        self.solver = solver
        self.model = solver.model
        self._bufs = None

    def _alloc(self, active_capacity: int = 0):
        m, K = self.model, self.solver.iterations
        B = max(m.body_count, 1)
        key = (B, K, active_capacity)
        if self._bufs is None or self._bufs["key"] != key:
            dev = m.device
            f = dict(dtype=torch.float32, device=dev)
            self._bufs = {
                "key": key,
                "tape_state": torch.empty((K + 1) * B * 13, **f),
                "tape_delta": torch.empty(max(K, 1) * B * 6, **f),
                "tape_weight": torch.empty(max(K, 1) * B, **f),
                "grad_acc": torch.empty(B * 13, dtype=torch.float64, device=dev),
                "delta_acc": torch.empty(B * 6, dtype=torch.float32, device=dev),
                "count_acc": torch.empty(B, dtype=torch.int32, device=dev),
                # active contacts per iteration: (record, world), at most every published contact
                "active": torch.empty(max(K, 1) * max(active_capacity, 1) * 2, dtype=torch.int32, device=dev),
                "active_count": torch.zeros(max(K, 1), dtype=torch.int32, device=dev),
                "active_capacity": active_capacity,
                "status": torch.zeros(1, dtype=torch.int32, device=dev) if self._bufs is None else self._bufs["status"],
            }
        return self._bufs

    def __call__(self, contacts, body_q, body_qd, body_f, grad_q_out, grad_qd_out, dt: float,
                 forward_out: tuple | None = None, grad_shape_mu: torch.Tensor | None = None):
        """Cotangents (grad_body_q, grad_body_qd, grad_body_f) of one substep's inputs given those of its
        outputs; `contacts` as the step used them (after collide).  With `forward_out = (q, qd)` the
        recomputed forward state is written there; with `grad_shape_mu` (float64 [shape_count]) the
        cotangent of the shapes' friction coefficients is added to it."""
        solver, m = self.solver, self.model
        _lib.require_cuda(m.device)
        B = m.body_count
        for name, t, shape in (("body_q", body_q, (B, 7)), ("body_qd", body_qd, (B, 6)), ("body_f", body_f, (B, 6)),
                               ("grad_q_out", grad_q_out, (B, 7)), ("grad_qd_out", grad_qd_out, (B, 6))):
            solver._check_state(name, t, shape)
        gq, gqd, gf = torch.empty_like(body_q), torch.empty_like(body_qd), torch.empty_like(body_f)
        io = self._io(contacts, body_q, body_qd, body_f)
        io.grad_q_out, io.grad_qd_out = ptr(grad_q_out), ptr(grad_qd_out)
        io.grad_q_in, io.grad_qd_in, io.grad_f_in = ptr(gq), ptr(gqd), ptr(gf)
        if forward_out is not None:
            io.body_q_out, io.body_qd_out = ptr(forward_out[0]), ptr(forward_out[1])
        if grad_shape_mu is not None:
            if (grad_shape_mu.dtype != torch.float64 or not grad_shape_mu.is_contiguous()
                    or grad_shape_mu.numel() != m.shape_count or grad_shape_mu.device != body_q.device):
                raise TypeError("grad_shape_mu must be a contiguous float64 tensor of shape_count entries on the "
                                "model device")
            io.grad_shape_mu = ptr(grad_shape_mu)
        self._launch(contacts, io, dt)
        return gq, gqd, gf

    def branch_buffers(self, contacts):
        """Zeroed (contact, body) branch arrays of one substep for ``forward(..., branches=...)``: one byte
        per contact record and iteration, one per body and iteration."""
        m, K = self.model, max(self.solver.iterations, 1)
        pipe, desc = self.solver._desc_for(contacts)
        ncap = int(desc.contact_capacity) if contacts is not None else 0
        dev = m.device
        return (torch.zeros(K * max(ncap, 1), dtype=torch.uint8, device=dev),
                torch.zeros(K * max(m.body_count, 1), dtype=torch.uint8, device=dev))

    def forward(self, contacts, body_q, body_qd, body_f, dt: float, q_out, qd_out, branches=None,
                replay: bool = False) -> None:
        """The adjoint's forward pass alone: one substep from (body_q, body_qd) into (q_out, qd_out), equal
        to ``solver.step`` on the same contacts.  With `branches` (from ``branch_buffers``) it records the
        substep's branch decisions there, or, with `replay`, takes them from there: a finite difference
        whose two sides replay the nominal substep's branches stays on the piece whose derivative the
        adjoint computes."""
        m = self.model
        _lib.require_cuda(m.device)
        B = m.body_count
        for name, t, shape in (("body_q", body_q, (B, 7)), ("body_qd", body_qd, (B, 6)), ("body_f", body_f, (B, 6)),
                               ("q_out", q_out, (B, 7)), ("qd_out", qd_out, (B, 6))):
            self.solver._check_state(name, t, shape)
        if replay and branches is None:
            raise ValueError("replay needs the recorded branches")
        io = self._io(contacts, body_q, body_qd, body_f)
        io.body_q_out, io.body_qd_out = ptr(q_out), ptr(qd_out)
        io.forward_only = 1
        if branches is not None:
            bc, bb = branches
            want = self.branch_buffers(contacts)
            for t, w in ((bc, want[0]), (bb, want[1])):
                if t.dtype != torch.uint8 or not t.is_contiguous() or t.numel() != w.numel() or t.device != w.device:
                    raise TypeError("branches must be the uint8 arrays branch_buffers() returns")
            io.branch_contact, io.branch_body = ptr(bc), ptr(bb)
            io.branch_mode = 2 if replay else 1
        self._launch(contacts, io, dt)

    def _io(self, contacts, body_q, body_qd, body_f) -> NbAdjointIO:
        if self.solver.enable_restitution:
            raise NotImplementedError("the adjoint does not differentiate restitution")
        b = self._alloc(contacts.rigid_contact_max if contacts is not None else 0)
        io = NbAdjointIO()
        io.body_q_in, io.body_qd_in, io.body_f_in = ptr(body_q), ptr(body_qd), ptr(body_f)
        for k in ("tape_state", "tape_delta", "tape_weight", "grad_acc", "delta_acc", "count_acc", "active",
                  "active_count", "status"):
            setattr(io, k, ptr(b[k]))
        io.active_capacity = b["active_capacity"]
        return io

    def _launch(self, contacts, io, dt: float) -> None:
        solver, m = self.solver, self.model
        pipe, desc = solver._desc_for(contacts)
        if contacts is not None:
            if contacts._seg is None or not contacts._seg_valid:
                raise ValueError("run collide (or a step) on these contacts before the adjoint")
            seg = pipe.seg_struct(contacts)
        else:
            from ._abi import NbContactSeg

            seg = NbContactSeg()
        params = solver.params()
        lib = _lib.load()
        _lib.check("nb_xpbd_step_adjoint", lib.nb_xpbd_step_adjoint(
            C.byref(desc), C.byref(params), C.byref(io), C.byref(seg), float(dt),
            C.c_void_p(_lib.stream_handle(m.device))))

    def status(self) -> int:
        return 0 if self._bufs is None else int(self._bufs["status"].item())


class Rollout:
    """Collide + step for `substeps` substeps from given initial tensors (the differentiable unit)."""

    def __init__(self, pipeline, solver, dt: float, checkpoint_every: int = 16):
        if checkpoint_every < 1:
            raise ValueError("checkpoint_every must be >= 1")
        if getattr(pipeline, "contact_matching", "disabled") != "disabled":
            raise NotImplementedError("differentiable rollouts need contact_matching='disabled'")
        if getattr(solver, "warm_start", None) is not None:
            raise NotImplementedError("the learned warm start is not differentiated")
        self.pipe, self.solver, self.dt = pipeline, solver, float(dt)
        self.checkpoint_every = int(checkpoint_every)
        m = solver.model
        self.model = m
        self.a, self.b = m.state(), m.state()
        self.contacts = pipeline.contacts()
        self.adjoint = SubstepAdjoint(solver)

    def _substep(self, q, qd, f):
        """One collide + step from (q, qd) with force f; returns the new (q, qd) (copies)."""
        a, b = self.a, self.b
        a.body_q.copy_(q)
        a.body_qd.copy_(qd)
        a.body_f.copy_(f)
        self.pipe.collide(a, self.contacts)
        self.solver.step(a, b, None, self.contacts, self.dt)
        return b.body_q.clone(), b.body_qd.clone()

    def forward(self, q, qd, f, substeps: int):
        checkpoints = [(q.clone(), qd.clone())]
        for i in range(substeps):
            q, qd = self._substep(q, qd, f)
            if (i + 1) % self.checkpoint_every == 0 and i + 1 < substeps:
                checkpoints.append((q.clone(), qd.clone()))
        return q, qd, checkpoints

    def backward(self, checkpoints, f, substeps: int, gq, gqd, want_mu: bool = False):
        gf_total = torch.zeros_like(f)
        gmu = torch.zeros(self.model.shape_count, dtype=torch.float64, device=f.device) if want_mu else None
        self.adjoint._alloc(self.contacts.rigid_contact_max)["status"].zero_()
        n_seg = len(checkpoints)
        for s in range(n_seg - 1, -1, -1):
            start = s * self.checkpoint_every
            n = min(self.checkpoint_every, substeps - start)
            states = [checkpoints[s]]
            for _ in range(n - 1):
                states.append(self._substep(states[-1][0], states[-1][1], f))
            for j in range(n - 1, -1, -1):
                q, qd = states[j]
                a = self.a
                a.body_q.copy_(q)
                a.body_qd.copy_(qd)
                a.body_f.copy_(f)
                self.pipe.collide(a, self.contacts)
                gq, gqd, gf = self.adjoint(self.contacts, a.body_q, a.body_qd, a.body_f, gq.contiguous(),
                                           gqd.contiguous(), self.dt, grad_shape_mu=gmu)
                gf_total += gf
        st = self.adjoint.status()
        if st:
            raise RuntimeError(f"adjoint status bits 0x{st:x} (a world with an enabled non-free joint, or "
                               "active-contact overflow)")
        return gq, gqd, gf_total, gmu


class _RolloutFn(torch.autograd.Function):
    @staticmethod
    def forward(ctx, body_q, body_qd, body_f, shape_mu, rollout, substeps):
        if shape_mu is not None:
            # the rollout runs with these coefficients: they become the model's
            rollout.model.shape_material_mu.copy_(shape_mu.detach().to(torch.float32))
        q, qd, checkpoints = rollout.forward(body_q.detach().contiguous(), body_qd.detach().contiguous(),
                                             body_f.detach().contiguous(), substeps)
        ctx.rollout, ctx.substeps, ctx.checkpoints = rollout, substeps, checkpoints
        ctx.body_f = body_f.detach().contiguous()
        ctx.want_mu = shape_mu is not None and shape_mu.requires_grad
        ctx.mu_dtype = shape_mu.dtype if shape_mu is not None else None
        return q, qd

    @staticmethod
    def backward(ctx, gq, gqd):
        gq = torch.zeros_like(ctx.checkpoints[0][0]) if gq is None else gq
        gqd = torch.zeros_like(ctx.checkpoints[0][1]) if gqd is None else gqd
        g_q, g_qd, g_f, g_mu = ctx.rollout.backward(ctx.checkpoints, ctx.body_f, ctx.substeps, gq.float(), gqd.float(),
                                                    want_mu=ctx.want_mu)
        if g_mu is not None:
            g_mu = g_mu.to(ctx.mu_dtype)
        return g_q, g_qd, g_f, g_mu, None, None


def simulate(pipeline, solver, body_q: torch.Tensor, body_qd: torch.Tensor, body_f: torch.Tensor | None = None,
             substeps: int = 1, dt: float = 1.0 / 480.0, checkpoint_every: int = 16,
             rollout: Rollout | None = None, shape_mu: torch.Tensor | None = None):
    """`substeps` substeps of collide + ``solver.step`` from (body_q, body_qd) with the constant body
    force `body_f`; returns (body_q, body_qd) after the last substep, differentiable with respect to
    the three inputs.  With `shape_mu` ([shape_count]), the rollout uses those friction coefficients
    (they are copied into ``model.shape_material_mu``) and the result is differentiable with respect
    to them too."""
    m = solver.model
    if body_f is None:
        body_f = torch.zeros((m.body_count, 6), dtype=torch.float32, device=body_q.device)
    if shape_mu is not None and shape_mu.shape != (m.shape_count,):
        raise ValueError(f"shape_mu must have shape ({m.shape_count},)")
    if rollout is None:
        rollout = Rollout(pipeline, solver, dt, checkpoint_every)
    return _RolloutFn.apply(body_q, body_qd, body_f, shape_mu, rollout, int(substeps))
