"""TEST INFRASTRUCTURE ONLY -- CPU oracle of the XPBD particle path.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg may use it.

A numpy float32 restatement of the reference's particle kernels, vectorised
over particles, contacts and springs (a different structure from the CUDA
kernels, which run one thread per particle):

  create_soft_contacts       newton/_src/geometry/kernels.py:1000-1140
  sdf_* and their gradients  newton/_src/geometry/kernels.py:165-330, 568-590
  integrate_particles        newton/_src/solvers/solver.py:11-47
  solve_particle_shape_contacts   newton/_src/solvers/xpbd/kernels.py:114-222
  solve_particle_particle_contacts newton/_src/solvers/xpbd/kernels.py:225-289
  solve_springs              newton/_src/solvers/xpbd/kernels.py:292-356
  bending_constraint         newton/_src/solvers/xpbd/kernels.py:358-457
  solve_tetrahedra           newton/_src/solvers/xpbd/kernels.py:459-628
  apply_particle_deltas      newton/_src/solvers/xpbd/kernels.py:776-807
  apply_particle_shape_restitution newton/_src/solvers/xpbd/kernels.py:34-112 (static shapes)
  iteration order            newton/_src/solvers/xpbd/solver_xpbd.py:303-320, 377-505

Every float operation is a float32 numpy operation in the order the
reference writes it (numpy never fuses a*b+c, sqrt and division are
correctly rounded).  Where the reference scatters with atomic adds, whose
order varies from run to run, the oracle fixes one order per particle: its
soft contacts in list order, then its particle neighbours in ascending index
(all j within the contact distance, found by brute force), then its springs in
ascending index, then its bending edges in ascending index.  The dihedral
angle's atan2 is the library's: asin (the C oracle's ``orc_asin``) of the
smaller coordinate over the radius, shifted into its quadrant.
"""

from __future__ import annotations

import numpy as np

F = np.float32
ACTIVE = 1
COLLIDE_PARTICLES = 1 << 2
GEO_PLANE, GEO_SPHERE, GEO_CAPSULE, GEO_BOX = 1, 3, 4, 7


def _dot(a, b):
    return a[..., 0] * b[..., 0] + a[..., 1] * b[..., 1] + a[..., 2] * b[..., 2]


def _length(a):
    return np.sqrt(_dot(a, a))


def _normalize(a):
    n = _length(a)
    safe = np.where(n > 0, n, F(1))
    return np.where((n > 0)[..., None], a / safe[..., None], F(0))


def _cross(a, b):
    return np.stack([a[..., 1] * b[..., 2] - a[..., 2] * b[..., 1], a[..., 2] * b[..., 0] - a[..., 0] * b[..., 2],
                     a[..., 0] * b[..., 1] - a[..., 1] * b[..., 0]], axis=-1)


def _max(a, b):  # wp.max: a > b ? a : b
    return np.where(a > b, a, b)


def _min(a, b):
    return np.where(a < b, a, b)


def _qrot(q, v, sign=1):
    """wp.quat_rotate (sign=1) / quat_rotate_inv (sign=-1) for quaternions (x, y, z, w)."""
    qx, qy, qz, qw = q[..., 0], q[..., 1], q[..., 2], q[..., 3]
    vx, vy, vz = v[..., 0], v[..., 1], v[..., 2]
    c = F(2) * qw * qw - F(1)
    d = F(2) * (qx * vx + qy * vy + qz * vz)
    tx = (qy * vz - qz * vy) * qw * F(2)
    ty = (qz * vx - qx * vz) * qw * F(2)
    tz = (qx * vy - qy * vx) * qw * F(2)
    if sign > 0:
        return np.stack([vx * c + qx * d + tx, vy * c + qy * d + ty, vz * c + qz * d + tz], axis=-1)
    return np.stack([vx * c + qx * d - tx, vy * c + qy * d - ty, vz * c + qz * d - tz], axis=-1)


def _qmul(a, b):
    ax, ay, az, aw = a[..., 0], a[..., 1], a[..., 2], a[..., 3]
    bx, by, bz, bw = b[..., 0], b[..., 1], b[..., 2], b[..., 3]
    return np.stack([aw * bx + bw * ax + ay * bz - by * az, aw * by + bw * ay + az * bx - bz * ax,
                     aw * bz + bw * az + ax * by - bx * ay, aw * bw - ax * bx - ay * by - az * bz], axis=-1)


def _tf_point(p, q, v):
    return _qrot(q, v) + p


def _sdf(geo, x, scale):
    """Signed distance and gradient of one shape type for an array of local points."""
    P = x.shape[0]
    with np.errstate(divide="ignore", invalid="ignore"):
        if geo == GEO_SPHERE:
            l = _length(x)
            d = l - scale[0]
            n = np.where((l > F(1e-8))[:, None], x / np.where(l > 0, l, F(1))[:, None], np.array([0, 0, 1], F))
            return d, n
        if geo == GEO_BOX:
            hx, hy, hz = scale
            qx, qy, qz = np.abs(x[:, 0]) - hx, np.abs(x[:, 1]) - hy, np.abs(x[:, 2]) - hz
            e = np.stack([_max(qx, F(0)), _max(qy, F(0)), _max(qz, F(0))], axis=-1)
            d = _length(e) + _min(_max(qx, _max(qy, qz)), F(0))
            cl = np.stack([_min(_max(x[:, 0], -hx), hx), _min(_max(x[:, 1], -hy), hy),
                           _min(_max(x[:, 2], -hz), hz)], axis=-1)
            ext = _normalize(x - cl)
            sgn = np.where(x < 0, F(-1), F(1))
            z = np.zeros(P, F)
            nx = np.stack([sgn[:, 0], z, z], -1)
            ny = np.stack([z, sgn[:, 1], z], -1)
            nz = np.stack([z, z, sgn[:, 2]], -1)
            outside = (qx > 0) | (qy > 0) | (qz > 0)
            use_x = ((qx > qy) & (qx > qz)) | ((qy == 0) & (qz == 0))
            use_y = ((qy > qx) & (qy > qz)) | ((qx == 0) & (qz == 0))
            inner = np.where(use_x[:, None], nx, np.where(use_y[:, None], ny, nz))
            return d, np.where(outside[:, None], ext, inner)
        if geo == GEO_CAPSULE:
            r, hh = scale[0], scale[1]
            top, bot = x[:, 2] > hh, x[:, 2] < -hh
            vz = np.where(top, x[:, 2] - hh, np.where(bot, x[:, 2] + hh, F(0)))
            v = np.stack([x[:, 0], x[:, 1], vz], -1)
            l = _length(v)
            d = l - r
            fb = np.where(bot[:, None], np.array([0, 0, -1], F), np.array([0, 0, 1], F))
            n = np.where((l > F(1e-8))[:, None], v / np.where(l > 0, l, F(1))[:, None], fb)
            return d, n
        if geo == GEO_PLANE:
            w, ln = scale[0] * F(0.5), scale[1] * F(0.5)
            if w > 0 and ln > 0:
                d = _max(_max(np.abs(x[:, 0]) - w, np.abs(x[:, 1]) - ln), np.abs(x[:, 2]))
            else:
                d = x[:, 2].copy()
            return d, np.tile(np.array([0, 0, 1], F), (P, 1))
    return np.full(P, F(1e6)), np.zeros((P, 3), F)


def soft_collide(h: dict, particle_q, body_q, margin: float, soft_contact_max: int):
    """Soft contacts in (particle, shape) order.  ``h`` holds the model's host arrays (particle_*, shape_*).

    Returns (count, particle, shape, body_pos, body_vel, normal) with the first soft_contact_max stored.
    """
    x = np.asarray(particle_q, F).reshape(-1, 3)
    P, S = x.shape[0], h["shape_type"].shape[0]
    radius = h["particle_radius"].astype(F)
    act = (h["particle_flags"] & ACTIVE) != 0
    pw = h["particle_world"]
    margin = F(margin)
    hit = np.zeros((P, S), bool)
    out = {k: np.zeros((P, S, 3), F) for k in ("body_pos", "body_vel", "normal")}
    ident = np.array([0, 0, 0, 0, 0, 0, 1], F)
    for s in range(S):
        if not (h["shape_flags"][s] & COLLIDE_PARTICLES):
            continue
        sw = h["shape_world"][s]
        ok = act & ~((pw != -1) & (sw != -1) & (pw != sw))
        b = h["shape_body"][s]
        X_wb = np.asarray(body_q, F).reshape(-1, 7)[b] if b >= 0 else ident
        X_bs = h["shape_transform"][s].astype(F)
        ws_p = _tf_point(X_wb[:3], X_wb[3:], X_bs[:3])
        ws_q = _qmul(X_wb[3:], X_bs[3:])
        qi = ws_q * np.array([-1, -1, -1, 1], F)
        sw_p = -_qrot(qi, ws_p)
        xl = _tf_point(sw_p, qi, x)
        d, n = _sdf(int(h["shape_type"][s]), xl, h["shape_scale"][s].astype(F))
        hit[:, s] = ok & (d < margin + radius)
        out["body_pos"][:, s] = _tf_point(X_bs[:3], X_bs[3:], xl - n * d[:, None])
        out["body_vel"][:, s] = _qrot(X_bs[3:], np.zeros((P, 3), F))
        out["normal"][:, s] = _qrot(ws_q, n)
    pi, si = np.nonzero(hit)
    count = int(pi.shape[0])
    keep = min(count, int(soft_contact_max))
    return (count, pi[:keep].astype(np.int32), si[:keep].astype(np.int32),
            out["body_pos"][pi, si][:keep], out["body_vel"][pi, si][:keep], out["normal"][pi, si][:keep])


def _asin(u):
    import oracle

    f = oracle.load().orc_asin
    return np.asarray([f(float(x)) for x in np.asarray(u, F).reshape(-1)], F).reshape(np.shape(u))


def atan2(y, x):
    """Elementwise float32 atan2 as the particle kernels compute it (see the module docstring)."""
    y, x = np.asarray(y, F), np.asarray(x, F)
    with np.errstate(divide="ignore", invalid="ignore"):
        r = np.sqrt(x * x + y * y)
        safe = np.where(r == 0, F(1), r)
        lo = np.abs(y) <= np.abs(x)
        a_lo = _asin(np.where(lo, y / safe, F(0)))
        a_lo = np.where(x > 0, a_lo, np.where(y < 0, F(-3.1415927410125732) - a_lo, F(3.1415927410125732) - a_lo))
        a_hi = F(1.5707963705062866) - _asin(np.where(lo, F(0), x / safe))
        a_hi = np.where(y < 0, -a_hi, a_hi)
    return np.where(r == 0, F(0), np.where(lo, a_lo, a_hi)).astype(F)


def _bending(h, x, v, w, dt):
    """Per-edge corrections of bending_constraint: (owner particle, correction) in edge order, roles i, j, k, l."""
    ev = h["edge_indices"].reshape(-1, 4)
    if ev.shape[0] == 0:
        return [], []
    live = (ev >= 0).all(axis=1)
    idx = np.where(ev >= 0, ev, 0)
    x1, x2, x3, x4 = (x[idx[:, r]] for r in range(4))
    n1 = _cross(x3 - x1, x4 - x1)
    n2 = _cross(x4 - x2, x3 - x2)
    e = x4 - x3
    n1l, n2l, el = _length(n1), _length(n2), _length(e)
    ok = live & ~((n1l < F(1e-6)) | (n2l < F(1e-6)) | (el < F(1e-6)))
    with np.errstate(divide="ignore", invalid="ignore"):
        n1h, n2h, eh = n1 / n1l[:, None], n2 / n2l[:, None], e / el[:, None]
        theta = atan2(_dot(_cross(n1h, n2h), eh), _dot(n1h, n2h))
        c = theta - h["edge_rest_angle"].astype(F)
        g = [-n1h * el[:, None], -n2h * el[:, None],
             -n1h * _dot(x1 - x4, eh)[:, None] - n2h * _dot(x2 - x4, eh)[:, None],
             -n1h * _dot(x3 - x1, eh)[:, None] - n2h * _dot(x3 - x2, eh)[:, None]]
        ws = [w[idx[:, r]] for r in range(4)]
        den = ws[0] * _dot(g[0], g[0]) + ws[1] * _dot(g[1], g[1]) + ws[2] * _dot(g[2], g[2]) + ws[3] * _dot(g[3], g[3])
        bp = h["edge_bending_properties"].reshape(-1, 2).astype(F)
        ke, kd = bp[:, 0], bp[:, 1]
        ok &= ~((den <= 0) | (ke <= 0) | (kd < 0))
        alpha = F(1) / (ke * dt * dt)
        gamma = kd / (ke * dt)
        gdv = dt * (_dot(g[0], v[idx[:, 0]]) + _dot(g[1], v[idx[:, 1]]) + _dot(g[2], v[idx[:, 2]]) +
                    _dot(g[3], v[idx[:, 3]]))
        dl = F(-1) * (c + alpha * F(0) + gamma * gdv) / ((F(1) + gamma) * den + alpha)
    owners, contribs = [], []
    for e_i in np.nonzero(ok)[0]:
        for r in range(4):
            owners.append(int(idx[e_i, r]))
            contribs.append(g[r][e_i] * (ws[r][e_i] * dl[e_i]))
    return owners, contribs


def _det3(m):
    return (m[..., 0, 0] * (m[..., 1, 1] * m[..., 2, 2] - m[..., 1, 2] * m[..., 2, 1]) -
            m[..., 0, 1] * (m[..., 1, 0] * m[..., 2, 2] - m[..., 1, 2] * m[..., 2, 0]) +
            m[..., 0, 2] * (m[..., 1, 0] * m[..., 2, 1] - m[..., 1, 1] * m[..., 2, 0]))


def _matmul3(a, b):
    """Row-by-column products summed k = 0, 1, 2 in order (no BLAS, whose summation order is its own)."""
    out = np.empty(np.broadcast_shapes(a.shape, b.shape), F)
    for i in range(3):
        for j in range(3):
            out[..., i, j] = a[..., i, 0] * b[..., 0, j] + a[..., i, 1] * b[..., 1, j] + a[..., i, 2] * b[..., 2, j]
    return out


def _tets(h, x, w, dt, relax):
    """Corrections of solve_tetrahedra: (owner, correction) in tet order, stretch then volume term, roles."""
    tv = h["tet_indices"].reshape(-1, 4)
    if tv.shape[0] == 0:
        return [], []
    X = [x[tv[:, r]] for r in range(4)]
    ws = [w[tv[:, r]] for r in range(4)]
    Ds = np.stack([X[1] - X[0], X[2] - X[0], X[3] - X[0]], axis=-1)  # columns
    Dm = h["tet_poses"].reshape(-1, 3, 3).astype(F)
    inv_QT = np.swapaxes(Dm, -1, -2)
    inv_rest_volume = _det3(Dm) * F(6)
    Fm = _matmul3(Ds, Dm)
    f1, f2, f3 = Fm[..., :, 0], Fm[..., :, 1], Fm[..., :, 2]
    tr = _dot(f1, f1) + _dot(f2, f2) + _dot(f3, f3)
    terms = [(tr - F(3), Fm * F(2)),
             (_det3(Fm) - F(1), np.stack([_cross(f2, f3), _cross(f3, f1), _cross(f1, f2)], axis=-1))]
    alpha = F(relax) / dt / dt
    alpha = np.where(inv_rest_volume > 0, alpha * inv_rest_volume, alpha)
    per_term = []
    for C, dC in terms:
        dP = _matmul3(dC, inv_QT)
        g1, g2, g3 = dP[..., :, 0], dP[..., :, 1], dP[..., :, 2]
        g0 = -g1 - g2 - g3
        g = [g0, g1, g2, g3]
        wsum = _dot(g0, g0) * ws[0] + _dot(g1, g1) * ws[1] + _dot(g2, g2) * ws[2] + _dot(g3, g3) * ws[3]
        ok = (C != 0) & (wsum > 0)
        with np.errstate(divide="ignore", invalid="ignore"):
            dl = -C / (wsum + alpha)
        per_term.append((ok, g, dl))
    owners, contribs = [], []
    for t in range(tv.shape[0]):
        for ok, g, dl in per_term:
            if not ok[t]:
                continue
            for r in range(4):
                owners.append(int(tv[t, r]))
                contribs.append(g[r][t] * (ws[r][t] * dl[t]))
    return owners, contribs


def _spring_csr(h):
    P = h["particle_radius"].shape[0]
    idx = h["spring_indices"].reshape(-1, 2)
    lists = [[] for _ in range(P)]
    for s, (a, b) in enumerate(idx):
        lists[a].append(s)
        lists[b].append(s)
    return [sorted(x) for x in lists]


def _accumulate(delta, owner, contrib):
    """delta[owner[k]] += contrib[k] for k in list order, sequentially per owner."""
    if owner.size == 0:
        return
    order = np.argsort(owner, kind="stable")
    owner, contrib = owner[order], contrib[order]
    first = np.r_[0, np.nonzero(np.diff(owner))[0] + 1]
    rank = np.arange(owner.size) - np.repeat(first, np.diff(np.r_[first, owner.size]))
    for lvl in range(int(rank.max()) + 1):
        m = rank == lvl
        delta[owner[m]] = delta[owner[m]] + contrib[m]


def step(h: dict, params: dict, q, qd, f, soft, dt: float, iterations: int, relaxation: float,
         restitution: bool = False, soft_body_relaxation: float = 0.9):
    """One particle substep; returns (q_out, qd_out).  ``soft`` is soft_collide's tuple or None."""
    dt, relax = F(dt), F(relaxation)
    x0 = np.asarray(q, F).reshape(-1, 3)
    v0 = np.asarray(qd, F).reshape(-1, 3)
    P = x0.shape[0]
    f0 = np.zeros_like(x0) if f is None else np.asarray(f, F).reshape(-1, 3)
    w = h["particle_inv_mass"].astype(F)
    radius = h["particle_radius"].astype(F)
    act = (h["particle_flags"] & ACTIVE) != 0
    vmax = F(params["particle_max_velocity"])
    grav = h["gravity"].astype(F).reshape(-1, 3)[np.maximum(h["particle_world"], 0)]
    gate = np.where(-w < 0, F(1), F(0))
    v1 = v0 + (f0 * w[:, None] + grav * gate[:, None]) * dt
    mag = _length(v1)
    with np.errstate(divide="ignore", invalid="ignore"):
        v1 = np.where((mag > vmax)[:, None], v1 * (vmax / mag)[:, None], v1)
    x1 = x0 + v1 * dt
    x = np.where(act[:, None], x1, x0)
    v = np.where(act[:, None], v1, v0)

    max_r = F(params["particle_max_radius"])
    coh = F(params["particle_cohesion"])
    pp_on = max_r > 0 and P > 1
    springs = h["spring_indices"].reshape(-1, 2)
    csr = _spring_csr(h) if springs.shape[0] else None
    shape_mu = h["shape_material_mu"].astype(F)
    for _ in range(iterations):
        delta = np.zeros((P, 3), F)
        with np.errstate(divide="ignore", invalid="ignore"):
            # particle-shape contacts (static shapes)
            if soft is not None and soft[0] > 0:
                cnt, cp, cs, bpos, bvel, cn = soft
                ok = act[cp] & (h["shape_body"][cs] < 0)
                bx = bpos + np.zeros(3, F)  # identity body transform
                r = bx - np.zeros(3, F)
                c = _dot(cn, x[cp] - bx) - radius[cp]
                ok &= ~(c > F(params["particle_adhesion"]))
                mu = F(0.5) * (F(params["soft_contact_mu"]) + shape_mu[cs])
                bv = (np.zeros(3, F) + _cross(np.zeros_like(r), r)) + bvel
                vr = v[cp] - bv
                dn = cn * c[:, None]
                vt = vr - cn * _dot(cn, vr)[:, None]
                denom = w[cp] + F(0)
                ok &= denom != 0
                lf = _max(mu * c, -_length(vt) * dt)
                df = _normalize(vt) * lf[:, None]
                dtot = (df - dn) / denom[:, None] * relax
                _accumulate(delta, cp[ok], w[cp][ok][:, None] * dtot[ok])
            # particle-particle contacts, neighbours in ascending index
            if pp_on:
                nvec = x[:, None, :] - x[None, :, :]
                d = _length(nvec)
                err = d - radius[:, None] - radius[None, :]
                denom = w[:, None] + w[None, :]
                acc = (act[:, None] & act[None, :] & ~np.eye(P, dtype=bool) & (err <= coh) & (denom > 0))
                n = nvec / d[..., None]
                vrel = v[:, None, :] - v[None, :, :]
                dn = n * err[..., None]
                vt = vrel - n * _dot(n, vrel)[..., None]
                lf = _max(F(params["particle_mu"]) * err, -_length(vt) * dt)
                df = _normalize(vt) * lf[..., None]
                contrib = np.where(acc[..., None], (df - dn) / denom[..., None], F(0))
                dpp = np.zeros((P, 3), F)
                for j in range(P):  # sequential over j: dpp += contribution of j where accepted
                    m = acc[:, j]
                    dpp[m] = dpp[m] + contrib[m, j]
                delta = np.where(act[:, None], delta + dpp * w[:, None] * relax, delta)
            # springs, ascending spring index per particle
            if csr is not None:
                a, b = springs[:, 0], springs[:, 1]
                xij = x[a] - x[b]
                vij = v[a] - v[b]
                l = _length(xij)
                n = xij / l[:, None]
                c = l - h["spring_rest_length"].astype(F)
                wi, wj = w[a], w[b]
                den = wi + wj
                ke, kd = h["spring_stiffness"].astype(F), h["spring_damping"].astype(F)
                ok = (l != 0) & ~((den <= 0) | (ke <= 0) | (kd < 0))
                alpha = F(1) / (ke * dt * dt)
                gamma = kd / (ke * dt)
                gcv = dt * _dot(n, vij)
                dl = F(-1) * (c + alpha * F(0) + gamma * gcv) / ((F(1) + gamma) * den + alpha)
                dxi = n * (wi * dl)[:, None]
                dxj = (F(-1) * n) * (wj * dl)[:, None]
                owners, contribs = [], []
                for p in range(P):
                    for s in csr[p]:
                        if not ok[s]:
                            continue
                        if a[s] == p:
                            owners.append(p)
                            contribs.append(dxi[s])
                        if b[s] == p:
                            owners.append(p)
                            contribs.append(dxj[s])
                if owners:
                    _accumulate(delta, np.asarray(owners), np.asarray(contribs, F))
            # bending edges, ascending edge index per particle
            owners, contribs = _bending(h, x, v, w, dt)
            if owners:
                _accumulate(delta, np.asarray(owners), np.asarray(contribs, F))
            # tetrahedra, ascending per particle
            if "tet_indices" in h:
                owners, contribs = _tets(h, x, w, dt, soft_body_relaxation)
                if owners:
                    _accumulate(delta, np.asarray(owners), np.asarray(contribs, F))
        # apply_particle_deltas
        xn = x + delta
        vn = (xn - x0) / dt
        mag = _length(vn)
        with np.errstate(divide="ignore", invalid="ignore"):
            vn = np.where((mag > vmax)[:, None], vn * (vmax / mag)[:, None], vn)
        x = np.where(act[:, None], xn, x)
        v = np.where(act[:, None], vn, v)
    if restitution and soft is not None and soft[0] > 0:
        # velocity change of every soft contact, tested at the substep's start position and computed from
        # the velocity after the iterations, added per particle in list order
        cnt, cp, cs, bpos, bvel, cn = soft
        ok = act[cp] & (h["shape_body"][cs] < 0)
        c = _dot(cn, x0[cp] - (bpos + np.zeros(3, F))) - radius[cp]
        ok &= ~(c > F(params["particle_adhesion"]))
        rvo = _dot(cn, v0[cp] - bvel)
        rvn = _dot(cn, v[cp] - bvel)
        ok &= rvo < 0
        dv = cn * (-rvn + _max(-F(params["soft_contact_restitution"]) * rvo, F(0)))[:, None]
        _accumulate(v, cp[ok], dv[ok])
    return x, v
