"""TEST INFRASTRUCTURE ONLY: ctypes bindings of the CPU oracle (liboracle.so).

The oracle restates the reference's collide + SolverXPBD rigid path in
sequential C++ (oracle_collide.cpp, oracle_xpbd.cpp).  Only tests/,
__graft_entry__.smoke() and bench.py's CPU-baseline leg may import it; the
product package never does.
"""

from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "liboracle.so")

ACC_FIXED = 0
ACC_FLOAT = 1

_lib = None


def build() -> str:
    subprocess.run(["make", "-s", "-C", HERE], check=True)
    return LIB


def load() -> C.CDLL:
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            build()
        lib = C.CDLL(LIB)
        lib.orc_collide.restype = C.c_int
        lib.orc_collide.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p]
        lib.orc_step.restype = C.c_int
        lib.orc_step.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_float, C.c_int,
                                 C.POINTER(C.c_uint32)]
        lib.orc_contact_midpoints.restype = C.c_int
        lib.orc_contact_midpoints.argtypes = [C.c_void_p, C.c_void_p, C.c_int] + [C.c_void_p] * 5
        lib.orc_match_contacts.restype = C.c_int
        lib.orc_match_contacts.argtypes = ([C.c_int, C.c_int] + [C.c_void_p] * 4 + [C.c_int] + [C.c_void_p] * 4 +
                                           [C.c_float, C.c_float, C.c_void_p, C.c_void_p])
        lib.orc_asin.restype = C.c_float
        lib.orc_asin.argtypes = [C.c_float]
        lib.orc_acos.restype = C.c_float
        lib.orc_acos.argtypes = [C.c_float]
        lib.orc_shape_aabbs.restype = C.c_int
        lib.orc_shape_aabbs.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
        lib.orc_collide_pair.restype = C.c_int
        lib.orc_collide_pair.argtypes = [C.c_int, C.c_void_p, C.c_void_p, C.c_float, C.c_float,
                                         C.c_int, C.c_void_p, C.c_void_p, C.c_float, C.c_float,
                                         C.c_void_p, C.c_int]
        _lib = lib
    return _lib


def _f32(a):
    return np.ascontiguousarray(np.asarray(a, dtype=np.float32))


def collide_pair(type_a, xf_a, scale_a, type_b, xf_b, scale_b, margin_a=0.0, margin_b=0.0, gap_a=0.1, gap_b=0.1):
    """Narrow phase of one pair of static shapes in world space.

    Returns an array [n, 16]: point0(3) point1(3) normal(3) margin0 margin1 d sub shape0 shape1 0,
    where d = n.(p1 - p0) - (margin0 + margin1) is the signed separation.
    """
    lib = load()
    out = np.zeros((8, 16), np.float32)
    xa, sa, xb, sb = _f32(xf_a), _f32(scale_a), _f32(xf_b), _f32(scale_b)
    n = lib.orc_collide_pair(int(type_a), xa.ctypes.data, sa.ctypes.data, margin_a, gap_a,
                             int(type_b), xb.ctypes.data, sb.ctypes.data, margin_b, gap_b,
                             out.ctypes.data, 8)
    return out[:n].copy()


class OrcSeg(C.Structure):
    _fields_ = [("rec0", C.c_void_p), ("rec1", C.c_void_p), ("rec2", C.c_void_p), ("rec3", C.c_void_p),
                ("rec4", C.c_void_p), ("world_count", C.c_void_p)]


class HostSegments:
    """Host-side solver-format contact segments for one pipeline layout."""

    def __init__(self, capacity: int, world_count: int):
        cap = max(1, capacity)
        self.rec = [np.zeros((cap, 4), np.float32) for _ in range(5)]
        self.world_count = np.zeros(world_count, np.int32)
        self.status = np.zeros(1, np.uint32)
        self.work = np.zeros(4, np.int32)

    def struct(self):
        s = OrcSeg()
        for k in range(5):
            setattr(s, f"rec{k}", self.rec[k].ctypes.data)
        s.world_count = self.world_count.ctypes.data
        return s


def model_desc(model, layout):
    """NbModelDesc over host numpy arrays of `model` and a PairLayout."""
    arrays = model.host_arrays()
    hd = layout.host_dict()
    arrays.update(hd)
    keep = [arrays, hd]
    desc = model.make_desc(arrays, layout.info())
    desc._keep = keep
    return desc


def collide(model, layout, body_q: np.ndarray) -> HostSegments:
    lib = load()
    segs = HostSegments(layout.contact_capacity, model.world_count)
    desc = model_desc(model, layout)
    bq = _f32(body_q)
    st = segs.struct()
    rc = lib.orc_collide(C.addressof(desc), bq.ctypes.data, C.addressof(st))
    if rc != 0:
        raise RuntimeError(f"orc_collide failed ({rc})")
    return segs


def step(model, layout, params, body_q, body_qd, body_f, segs: HostSegments | None, dt: float,
         joint_target_pos=None, joint_target_vel=None, joint_f=None, acc_mode: int = ACC_FLOAT,
         want_impulse: bool = False, want_parent_f: bool = False):
    """One SolverXPBD.step on the CPU (per-body deltas summed in float in contact / joint order, like the
    CUDA kernels, unless ``acc_mode`` is ACC_FIXED).  Returns (body_q_out, body_qd_out, status), then the
    accumulated weighted contact impulse [slot, 6] (indexed like ``segs``) when ``want_impulse``,
    then body_parent_f [B, 6] when ``want_parent_f``."""
    from newton_custom_contact_b200._abi import NbStepIO

    lib = load()
    desc = model_desc(model, layout)
    q_in, qd_in, f_in = _f32(body_q), _f32(body_qd), _f32(body_f)
    q_out = np.zeros_like(q_in)
    qd_out = np.zeros_like(qd_in)
    io = NbStepIO()
    io.body_q_in = q_in.ctypes.data
    io.body_qd_in = qd_in.ctypes.data
    io.body_f_in = f_in.ctypes.data
    io.body_q_out = q_out.ctypes.data
    io.body_qd_out = qd_out.ctypes.data
    keep = []
    for name, arr in (("joint_target_pos", joint_target_pos), ("joint_target_vel", joint_target_vel),
                      ("joint_f", joint_f)):
        if arr is not None and np.asarray(arr).size:
            a = _f32(arr)
            keep.append(a)
            setattr(io, name, a.ctypes.data)
    parent_f = None
    if want_parent_f:
        parent_f = np.full((q_in.shape[0], 6), np.nan, np.float32)
        io.body_parent_f = parent_f.ctypes.data
    imp = None
    if want_impulse:
        imp = np.zeros((segs.rec[0].shape[0] if segs is not None else 1, 6), np.float32)
        io.contact_impulse = imp.ctypes.data
    status = C.c_uint32(0)
    st = segs.struct() if segs is not None else None
    rc = lib.orc_step(C.addressof(desc), C.addressof(params), C.addressof(io),
                      C.addressof(st) if st is not None else None, float(dt), int(acc_mode), C.byref(status))
    if rc != 0:
        raise RuntimeError(f"orc_step failed ({rc})")
    out = [q_out, qd_out, int(status.value)]
    if want_impulse:
        out.append(imp)
    if want_parent_f:
        out.append(parent_f)
    return tuple(out)


def contacts_table(model, layout, segs: HostSegments) -> np.ndarray:
    """All live contacts as rows (world, shape0, shape1, sub, p0(3), p1(3), n(3), o0(3), o1(3), m0, m1)."""
    rows = []
    cs = 5 * layout.world_pair_start.astype(np.int64)
    for w in range(model.world_count):
        n = int(segs.world_count[w])
        for k in range(cs[w], cs[w] + n):
            r0, r1, r2, r3, r4 = (segs.rec[i][k] for i in range(5))
            s0 = int(r2[3:4].view(np.int32)[0])
            s1 = int(r3[3:4].view(np.int32)[0])
            tag = int(r4[3:4].view(np.int32)[0])
            rows.append([w, s0, s1, (tag >> 24) & 0xFF, *r0[:3], *r1[:3], *r2[:3], *r3[:3], *r4[:3], r0[3], r1[3]])
    return np.asarray(rows, dtype=np.float64).reshape(-1, 21)


class Matcher:
    """Frame-to-frame contact matching on the CPU (oracle_match.cpp + bookkeeping).

    ``step(model, body_q, pub)`` takes one frame's published contacts (dict of
    numpy arrays in public order: count, world_offset, sort_key, point0/1,
    offset0/1, normal, shape0/1), returns (match_index, new_indices,
    broken_indices) and, in sticky mode, replays matched rows into ``pub`` in
    place (ContactMatcher.match / replay_matched / build_report /
    save_sorted_state, contact_match.py:720-990).
    """

    def __init__(self, pos_threshold=0.0005, normal_dot_threshold=0.995, sticky=False):
        self.pos_thr_sq = np.float32(pos_threshold) * np.float32(pos_threshold)
        self.ndot = np.float32(normal_dot_threshold)
        self.sticky = sticky
        self.prev = None

    def step(self, model, layout, body_q, pub):
        lib = load()
        desc = model_desc(model, layout)
        n = int(pub["count"])
        W = model.world_count
        f32 = lambda a: np.ascontiguousarray(np.asarray(a, np.float32))  # noqa: E731
        i64 = lambda a: np.ascontiguousarray(np.asarray(a, np.int64))  # noqa: E731
        i32 = lambda a: np.ascontiguousarray(np.asarray(a, np.int32))  # noqa: E731
        bq = f32(body_q)
        p0, p1, s0, s1 = f32(pub["point0"][:n]), f32(pub["point1"][:n]), i32(pub["shape0"][:n]), i32(pub["shape1"][:n])
        mid = np.zeros((max(n, 1), 3), np.float32)
        lib.orc_contact_midpoints(C.addressof(desc), bq.ctypes.data, n, p0.ctypes.data, p1.ctypes.data,
                                  s0.ctypes.data, s1.ctypes.data, mid.ctypes.data)
        keys, wo, nrm = i64(pub["sort_key"][:n]), i64(pub["world_offset"]), f32(pub["normal"][:n])
        match = np.full(max(n, 1), -1, np.int32)
        prev = self.prev
        n_old = 0 if prev is None else prev["count"]
        matched = np.zeros(max(n_old, 1), np.uint8)
        if prev is not None:
            lib.orc_match_contacts(W, n, wo.ctypes.data, keys.ctypes.data, mid.ctypes.data, nrm.ctypes.data, n_old,
                                   prev["world_offset"].ctypes.data, prev["keys"].ctypes.data,
                                   prev["mid"].ctypes.data, prev["normal"].ctypes.data, self.pos_thr_sq, self.ndot,
                                   match.ctypes.data, matched.ctypes.data)
        match = match[:n]
        if self.sticky and prev is not None:
            for i in np.nonzero(match >= 0)[0]:
                k = match[i]
                for f in ("point0", "point1", "offset0", "offset1", "normal"):
                    pub[f][i] = prev[f][k]
            p0 = f32(pub["point0"][:n])
            p1 = f32(pub["point1"][:n])
            nrm = f32(pub["normal"][:n])
            lib.orc_contact_midpoints(C.addressof(desc), bq.ctypes.data, n, p0.ctypes.data, p1.ctypes.data,
                                      s0.ctypes.data, s1.ctypes.data, mid.ctypes.data)
        new_idx = np.nonzero(match < 0)[0].astype(np.int32)
        broken = np.nonzero(matched[:n_old] == 0)[0].astype(np.int32) if n_old else np.zeros(0, np.int32)
        self.prev = {"count": n, "world_offset": wo.copy(), "keys": keys.copy(), "mid": mid[:max(n, 1)].copy(),
                     "normal": f32(pub["normal"][:max(n, 1)]).copy()}
        if self.sticky:
            for f in ("point0", "point1", "offset0", "offset1"):
                self.prev[f] = f32(pub[f][:n]).copy()
            self.prev["normal"] = f32(pub["normal"][:n]).copy() if n else self.prev["normal"]
        return match, new_idx, broken
