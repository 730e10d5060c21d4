"""Run metrics reported next to the throughput: max penetration and max joint violation.

Both are evaluated on the device with torch (they are reporting, not part of
the substep) from the current body poses:

* penetration of a contact: -d with d = n . (X_b p1 - X_a p0) - (margin0 +
  margin1), the separation solve_body_contact_positions tests
  (newton/_src/solvers/xpbd/kernels.py:2100-2130); max over contacts of
  max(-d, 0);
* joint violation: distance between the parent and child joint anchors
  (X_wp = X_p(parent) * X_pj, X_wc = X_c * X_cj) for joints whose linear
  motion is fully constrained (revolute, ball, fixed), and its part
  perpendicular to the axis for prismatic joints.
"""

from __future__ import annotations

import torch

from ._abi import JointType


def _qrot(q, v):
    """Rotate v by unit quaternions q (xyzw), batched."""
    u = q[..., :3]
    w = q[..., 3:4]
    t = 2.0 * torch.cross(u, v, dim=-1)
    return v + w * t + torch.cross(u, t, dim=-1)


def _tf_point(x, p):
    return _qrot(x[..., 3:7], p) + x[..., :3]


def _tf_mul(a, b):
    qa, qb = a[..., 3:7], b[..., 3:7]
    xyz = qa[..., 3:4] * qb[..., :3] + qb[..., 3:4] * qa[..., :3] + torch.cross(qa[..., :3], qb[..., :3], dim=-1)
    w = qa[..., 3:4] * qb[..., 3:4] - (qa[..., :3] * qb[..., :3]).sum(-1, keepdim=True)
    return torch.cat([_tf_point(a, b[..., :3]), xyz, w], dim=-1)


def max_penetration(model, contacts, body_q) -> float:
    """Largest penetration [m] among the live contacts at poses `body_q`."""
    pen = contact_penetrations(model, contacts, body_q)
    return float(pen.max().item()) if pen.numel() else 0.0


def penetration_stats(model, contacts, body_q) -> dict:
    """max, 99th percentile and mean penetration [m] over the live contacts, and their sum."""
    pen = contact_penetrations(model, contacts, body_q)
    if pen.numel() == 0:
        return {"max": 0.0, "p99": 0.0, "mean": 0.0, "sum": 0.0}
    return {"max": float(pen.max()), "p99": float(torch.quantile(pen.float()[:2**24], 0.99)),
            "mean": float(pen.mean()), "sum": float(pen.sum())}


def contact_penetrations(model, contacts, body_q) -> torch.Tensor:
    """max(-d, 0) [m] per live contact at poses `body_q` (float64)."""
    n = min(int(contacts.rigid_contact_count.item()), contacts.rigid_contact_max)
    if n == 0:
        return torch.zeros(0, dtype=torch.float64, device=body_q.device)
    dev = body_q.device
    q = body_q.to(torch.float64)
    shape_body = model.shape_body.to(dev).long()
    ident = torch.tensor([0, 0, 0, 0, 0, 0, 1], dtype=torch.float64, device=dev)

    def pose(shapes):
        s = shapes.long()
        b = torch.where(s >= 0, shape_body[s.clamp(min=0)], torch.full_like(s, -1))
        return torch.where((b >= 0)[:, None], q[b.clamp(min=0)], ident.expand(s.numel(), 7))

    xa = pose(contacts.rigid_contact_shape0[:n])
    xb = pose(contacts.rigid_contact_shape1[:n])
    pa = _tf_point(xa, contacts.rigid_contact_point0[:n].to(torch.float64))
    pb = _tf_point(xb, contacts.rigid_contact_point1[:n].to(torch.float64))
    nrm = contacts.rigid_contact_normal[:n].to(torch.float64)
    thick = (contacts.rigid_contact_margin0[:n] + contacts.rigid_contact_margin1[:n]).to(torch.float64)
    d = (nrm * (pb - pa)).sum(-1) - thick
    return torch.clamp(-d, min=0.0)


def max_joint_violation(model, body_q) -> float:
    """Largest joint anchor error [m] over enabled revolute / ball / fixed / prismatic joints."""
    if model.joint_count == 0:
        return 0.0
    dev = body_q.device
    jt = model.joint_type.to(dev).long()
    en = model.joint_enabled.to(dev).bool()
    kinds = torch.tensor([int(JointType.REVOLUTE), int(JointType.BALL), int(JointType.FIXED),
                          int(JointType.PRISMATIC)], device=dev)
    sel = en & torch.isin(jt, kinds)
    if not bool(sel.any()):
        return 0.0
    idx = torch.nonzero(sel).flatten()
    q = body_q.to(torch.float64)
    par = model.joint_parent.to(dev).long()[idx]
    chi = model.joint_child.to(dev).long()[idx]
    xp = model.joint_X_p.to(dev).to(torch.float64)[idx]
    xc = model.joint_X_c.to(dev).to(torch.float64)[idx]
    ident = torch.tensor([0, 0, 0, 0, 0, 0, 1], dtype=torch.float64, device=dev).expand(idx.numel(), 7)
    wp = torch.where((par >= 0)[:, None], _tf_mul(q[par.clamp(min=0)], xp), xp)
    wc = _tf_mul(q[chi], xc)
    err = wc[:, :3] - wp[:, :3]
    prism = jt[idx] == int(JointType.PRISMATIC)
    if bool(prism.any()):
        qs = model.joint_qd_start.to(dev).long()[idx]
        axis = model.joint_axis.to(dev).to(torch.float64)[qs.clamp(max=model.joint_axis.shape[0] - 1)]
        axw = _qrot(wp[:, 3:7], axis)
        along = (err * axw).sum(-1, keepdim=True) * axw
        err = torch.where(prism[:, None], err - along, err)
    del ident
    return float(err.norm(dim=-1).max().item())
