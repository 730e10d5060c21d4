"""CollisionPipeline (newton/_src/sim/collide.py:483-1230) on the B200 kernels.

``collide(state, contacts)`` launches two kernels of libnewton_b200.so:
``nb_collide`` (per-world AABBs, broad phase, narrow phase and key-ordered
compaction into solver-format segments) and ``nb_publish_contacts`` (the
reference's dense Contacts arrays, ordered by (world, key)).  Both run on the
current torch stream without host synchronisation, so a substep loop of
collide + SolverXPBD.step can be captured in a CUDA graph.
"""

from __future__ import annotations

import ctypes as C
from typing import Literal

import numpy as np
import torch

from . import _lib
from ._abi import GeoType, NbContactSeg, NbContactsPublic, NbMatchState, ShapeFlags, ptr
from .contacts import Contacts

BROAD_PHASE_MODES = ("nxn", "sap", "explicit")

_PRIMITIVE_CPP = 5
_MAX_NEIGHBORS_PER_SHAPE = 20


def _estimate_rigid_contact_max(model) -> int:
    """Capacity estimate of newton/_src/sim/collide.py:278-376 (primitive shapes only)."""
    h = model.host_arrays()
    st = h["shape_type"]
    if st.size == 0:
        return 1000
    plane = st == int(GeoType.PLANE)
    non_plane = ~plane
    n_np = int(non_plane.sum())
    non_plane_contacts = (n_np * _MAX_NEIGHBORS_PER_SHAPE * _PRIMITIVE_CPP) // 2
    avg_cpp = _PRIMITIVE_CPP if n_np > 0 else 0
    plane_contacts = 0
    if plane.any() and n_np > 0:
        sw = h["shape_world"]
        W = model.world_count
        gmask = sw == -1
        lmask = ~gmask
        gp = int(np.count_nonzero(gmask & plane))
        gnp = int(np.count_nonzero(gmask & non_plane))
        lp = np.bincount(sw[lmask & plane], minlength=W)[:W]
        lnp = np.bincount(sw[lmask & non_plane], minlength=W)[:W]
        cnt = int(np.sum((lp + gp) * (lnp + gnp)))
        if W > 1:
            cnt -= (W - 1) * gp * gnp
        plane_contacts = cnt * avg_cpp
    total = non_plane_contacts + plane_contacts
    if model.shape_contact_pair_count > 0:
        total = min(total, int(model.shape_contact_pair_count) * max(avg_cpp, _PRIMITIVE_CPP))
    return max(1000, total)


def _max_contacts(ta: int, tb: int) -> int:
    """Upper bound of contacts one pair can emit (narrow_phase.py:153-776)."""
    P, S, C_, B = int(GeoType.PLANE), int(GeoType.SPHERE), int(GeoType.CAPSULE), int(GeoType.BOX)
    table = {(P, S): 1, (S, S): 1, (S, C_): 1, (S, B): 1, (P, C_): 2, (C_, C_): 2}
    return table.get((ta, tb), 5)


def nxn_pairs(model) -> np.ndarray:
    """The NxN candidate set (broad_phase_nxn.py:129-214 + broad_phase_common.py:132-180).

    Pairs of colliding shapes that pass the world / collision-group test and are
    not filtered; identical to the builder's explicit list by construction.
    """
    h = model.host_arrays()
    flags = h["shape_flags"]
    sw = model._world_of_shape
    grp = h["shape_collision_group"].astype(np.int64)
    filters = model.shape_collision_filter_pairs
    col = (flags & int(ShapeFlags.COLLIDE_SHAPES)) != 0
    glob = np.nonzero(col & (sw < 0))[0]
    chunks = []
    wss = model._part["world_shape_start"]
    for w in range(model.world_count):
        loc = np.arange(wss[w], wss[w + 1])
        loc = loc[col[loc]]
        ids = np.sort(np.concatenate([loc, glob]))
        if ids.size < 2:
            continue
        i, j = np.triu_indices(ids.size, 1)
        a, b = ids[i], ids[j]
        both_global = (sw[a] < 0) & (sw[b] < 0)
        ga, gb = grp[a], grp[b]
        ok = (ga != 0) & (gb != 0) & np.where(ga > 0, (ga == gb) | (gb < 0), ga != gb) & ~both_global
        chunks.append(np.stack([a[ok], b[ok]], axis=1))
    pairs = np.concatenate(chunks) if chunks else np.zeros((0, 2), np.int64)
    if filters and pairs.size:
        keep = np.array([(int(x), int(y)) not in filters for x, y in pairs], dtype=bool)
        pairs = pairs[keep]
    return pairs.astype(np.int32).reshape(-1, 2)


class PairLayout:
    """Per-world candidate pairs sorted by contact key and contact slot ranges."""

    def __init__(self, model, pairs: np.ndarray):
        h = model.host_arrays()
        W = model.world_count
        types = h["shape_type"]
        sws = model._world_of_shape
        wss = model._part["world_shape_start"].astype(np.int64)
        glob = model._part["global_shapes"].astype(np.int64)
        pairs = np.asarray(pairs, dtype=np.int64).reshape(-1, 2)
        a, b = pairs[:, 0], pairs[:, 1]
        wa, wb = sws[a], sws[b]
        keep = (wa >= 0) | (wb >= 0)
        a, b, wa, wb = a[keep], b[keep], wa[keep], wb[keep]
        if np.any((wa >= 0) & (wb >= 0) & (wa != wb)):
            raise ValueError("candidate pair spans two worlds")
        w = np.where(wa >= 0, wa, wb).astype(np.int64)
        swap = types[a] > types[b]
        sa = np.where(swap, b, a)
        sb = np.where(swap, a, b)
        if model.shape_count < (1 << 21):
            order = np.argsort((w << 42) | (sa << 21) | sb, kind="stable")
        else:
            order = np.lexsort((sb, sa, w))
        sa, sb, w = sa[order], sb[order], w[order]
        nloc = np.diff(wss)
        gslot = np.full(model.shape_count, -1, np.int64)
        gslot[glob] = np.arange(glob.size)

        def local(s):
            ws = sws[s]
            out = s - wss[w]
            g = ws < 0
            out[g] = nloc[w[g]] + gslot[s[g]]
            return out

        la, lb = local(sa), local(sb)
        P = sa.size
        # every slot must address the world's shapes or the global shapes (the
        # kernels index shared memory with it)
        lim = nloc[w] + glob.size
        if P and (la.min() < 0 or lb.min() < 0 or np.any(la >= lim) or np.any(lb >= lim)):
            raise AssertionError("pair layout produced an out-of-range shape slot")
        if P and np.any(np.diff(w) < 0):
            raise AssertionError("pair layout is not grouped by world")
        cnt = np.bincount(w, minlength=W)[:W] if P else np.zeros(W, np.int64)
        pstart = np.zeros(W + 1, np.int64)
        pstart[1:] = np.cumsum(cnt)
        nb = np.diff(model._part["world_body_start"].astype(np.int64))
        cost = cnt + 4 * nb
        self.world_order = np.argsort(-cost, kind="stable").astype(np.int32)
        self.world_pair_start = pstart.astype(np.int32)
        if P and max(la.max(), lb.max()) >= (1 << 16):
            raise ValueError("a world has more than 65535 shapes")
        # packed (slot_a | slot_b << 16), padded so the kernel can read 4 pairs per 16-byte load
        packed = np.zeros(P + 4, np.uint32)
        packed[:P] = (la.astype(np.uint32) & 0xFFFF) | (lb.astype(np.uint32) << 16)
        self.pair_shapes = packed
        self.pair_slots = np.stack([la, lb], axis=1).astype(np.int32).reshape(-1, 2)
        self.pair_global = np.stack([sa, sb], axis=1).astype(np.int32).reshape(-1, 2)
        self.pair_count = int(P)
        self.max_world_pairs = int(cnt.max()) if W else 0
        self.contact_capacity = 5 * int(P)
        self.world_count = W

    def host_dict(self) -> dict:
        return {
            "world_pair_start": self.world_pair_start,
            "pair_shapes": self.pair_shapes,
            "world_order": self.world_order,
        }

    def pair_table(self, model) -> tuple:
        """Per world a dense ns x ns table (ns = the world's shape slots: its own shapes, then the global
        ones) of pair indices, -1 where the slots form no listed pair, both orientations filled; and the
        tables' int64 start offsets [W + 1].  The sweep and prune broad phase looks its overlaps up here."""
        W = self.world_count
        nloc = np.diff(model._part["world_shape_start"].astype(np.int64))
        ns = nloc + model._part["global_shapes"].size
        start = np.zeros(W + 1, np.int64)
        start[1:] = np.cumsum(ns * ns)
        table = np.full(int(start[-1]), -1, np.int32)
        P = self.pair_count
        if P:
            w = np.repeat(np.arange(W), np.diff(self.world_pair_start.astype(np.int64)))
            la = self.pair_slots[:, 0].astype(np.int64)
            lb = self.pair_slots[:, 1].astype(np.int64)
            idx = np.arange(P, dtype=np.int32)
            table[start[w] + la * ns[w] + lb] = idx
            table[start[w] + lb * ns[w] + la] = idx
        return table, start

    def info(self) -> dict:
        return {"pair_count": self.pair_count, "max_world_pairs": self.max_world_pairs,
                "contact_capacity": self.contact_capacity}


class CollisionPipeline:
    """Broad phase + primitive/MPR-GJK narrow phase + deterministic compaction on B200."""

    def __init__(self, model, *, reduce_contacts: bool = True, rigid_contact_max: int | None = None,
                 max_triangle_pairs: int = 1000000, shape_pairs_filtered=None, soft_contact_max: int | None = None,
                 soft_contact_margin: float = 0.01, requires_grad: bool | None = None,
                 broad_phase: Literal["nxn", "sap", "explicit"] | None = None, narrow_phase=None,
                 sdf_hydroelastic_config=None, shape_pairs_max: int | None = None, deterministic: bool = False,
                 contact_matching: str = "disabled", contact_matching_pos_threshold: float = 0.0005,
                 contact_matching_normal_dot_threshold: float = 0.995, contact_report: bool = False,
                 verify_buffers: bool = True):
        if not isinstance(contact_matching, str) or contact_matching not in ("disabled", "latest", "sticky"):
            raise ValueError(
                f"contact_matching must be one of 'disabled', 'latest', 'sticky', got {contact_matching!r}")
        if contact_matching_pos_threshold < 0.0:
            raise ValueError(f"contact_matching_pos_threshold must be non-negative, got {contact_matching_pos_threshold}")
        if not -1.0 <= contact_matching_normal_dot_threshold <= 1.0:
            raise ValueError("contact_matching_normal_dot_threshold must be in [-1, 1], got "
                             f"{contact_matching_normal_dot_threshold}")
        if contact_report and contact_matching == "disabled":
            raise ValueError('contact_report=True requires contact_matching != "disabled"')
        if contact_matching != "disabled":
            deterministic = True  # matching works on the sorted keys (collide.py:605-607)
        if max_triangle_pairs <= 0:
            raise ValueError("max_triangle_pairs must be > 0")
        if narrow_phase is not None or sdf_hydroelastic_config is not None:
            raise NotImplementedError("custom narrow phases / hydroelastic contacts are not supported")
        if shape_pairs_max is not None and shape_pairs_max <= 0:
            raise ValueError(f"shape_pairs_max must be a positive integer or None, got {shape_pairs_max}")
        mode = "explicit" if broad_phase is None else str(broad_phase).lower()
        if mode not in BROAD_PHASE_MODES:
            raise ValueError(f"Unsupported broad phase mode: {broad_phase!r}")
        self.model = model
        self.device = model.device
        self.broad_phase_mode = mode
        self.deterministic = deterministic
        self.contact_matching = contact_matching
        self.contact_report = bool(contact_report)
        self.contact_matching_pos_threshold = float(contact_matching_pos_threshold)
        self.contact_matching_normal_dot_threshold = float(contact_matching_normal_dot_threshold)
        self._match = None  # previous-frame state, allocated with the first contacts buffer
        self.requires_grad = model.requires_grad if requires_grad is None else requires_grad
        self.soft_contact_margin = soft_contact_margin
        if rigid_contact_max is None:
            mrc = int(getattr(model, "rigid_contact_max", 0) or 0)
            rigid_contact_max = mrc if mrc > 0 else _estimate_rigid_contact_max(model)
        self._rigid_contact_max = int(rigid_contact_max)
        model.rigid_contact_max = self._rigid_contact_max
        # the reference's default capacity: every (particle, shape) pair (collide.py:814-815)
        self._soft_contact_max = (int(soft_contact_max) if soft_contact_max is not None
                                  else model.shape_count * getattr(model, "particle_count", 0))
        if mode == "explicit":
            if shape_pairs_filtered is None:
                shape_pairs_filtered = model.host("shape_contact_pairs")
            if shape_pairs_filtered is None:
                raise ValueError("shape_pairs_filtered must be provided for broad_phase=EXPLICIT "
                                 "(or set model.shape_contact_pairs)")
            pairs = shape_pairs_filtered
            if isinstance(pairs, torch.Tensor):
                pairs = pairs.detach().cpu().numpy()
        else:
            # NxN and SAP find the same AABB-overlapping pairs among the pairs the world, group and filter
            # rules allow (the NxN list): NxN tests every listed pair, SAP sorts the world's boxes along x
            # and sweeps, keeping the overlaps that are in the list.
            pairs = nxn_pairs(model)
        self.shape_pairs_max = int(np.asarray(pairs).reshape(-1, 2).shape[0])
        self.layout = PairLayout(model, pairs)
        hd = self.layout.host_dict()
        self._layout_host = hd
        self._layout_dev = {k: torch.from_numpy(np.ascontiguousarray(v)).to(self.device) for k, v in hd.items()}
        if mode == "sap":
            table, start = self.layout.pair_table(model)
            self._layout_dev["pair_table"] = torch.from_numpy(table).to(self.device)
            self._layout_dev["world_table_start"] = torch.from_numpy(start).to(self.device)
        self._desc = None
        self._grid = None
        self._schedule = None

    @property
    def rigid_contact_max(self) -> int:
        return self._rigid_contact_max

    @property
    def soft_contact_max(self) -> int:
        return self._soft_contact_max

    # ------------------------------------------------------------ buffers
    def contacts(self) -> Contacts:
        c = Contacts(self._rigid_contact_max, self._soft_contact_max, requires_grad=self.requires_grad,
                     device=self.device, requested_attributes=self.model.get_requested_contact_attributes(),
                     world_count=self.model.world_count, deterministic=self.deterministic,
                     contact_matching=self.contact_matching != "disabled", contact_report=self.contact_report)
        self.attach_segments(c)
        if self.contact_matching != "disabled" and self._match is None:
            self._alloc_match(c.rigid_contact_max)
        return c

    # ------------------------------------------------------------ contact matching
    def _alloc_match(self, cap: int) -> None:
        dev = self.device
        sticky = self.contact_matching == "sticky"
        n = max(cap, 1)
        f3 = lambda: torch.zeros((n, 3), dtype=torch.float32, device=dev)  # noqa: E731
        m = {
            # [previous count, match_index rows written by the last call]
            "prev_count": torch.zeros(2, dtype=torch.int32, device=dev),
            "prev_world_offset": torch.zeros(self.model.world_count + 1, dtype=torch.int64, device=dev),
            "prev_keys": torch.zeros(n, dtype=torch.int64, device=dev),
            "prev_mid": f3(),
            "prev_normal": f3(),
            "prev_claim": torch.zeros(n, dtype=torch.int64, device=dev),
            "prev_was_matched": torch.zeros(n, dtype=torch.int32, device=dev) if self.contact_report else None,
        }
        for k in ("prev_point0", "prev_point1", "prev_offset0", "prev_offset1", "prev_normal_sticky"):
            m[k] = f3() if sticky else None
        m["capacity"] = cap
        self._match = m

    @property
    def _prev_point0(self):
        return None if self._match is None else self._match["prev_point0"]

    def reset_contact_matching(self) -> None:
        """Forget the previous frame (after teleporting / resetting bodies): the next
        collide reports every contact as new (ContactMatcher.reset)."""
        if self._match is not None:
            self._match["prev_count"][:1].zero_()

    def _match_struct(self, c: Contacts) -> NbMatchState:
        m = self._match
        if m["capacity"] != c.rigid_contact_max:
            raise ValueError("contacts buffer capacity differs from the one contact matching was set up for")
        st = NbMatchState()
        st.capacity = int(c.rigid_contact_max)
        st.sticky = 1 if self.contact_matching == "sticky" else 0
        st.pos_threshold_sq = self.contact_matching_pos_threshold ** 2
        st.normal_dot_threshold = self.contact_matching_normal_dot_threshold
        for k in ("prev_count", "prev_world_offset", "prev_keys", "prev_mid", "prev_normal", "prev_claim",
                  "prev_was_matched", "prev_point0", "prev_point1", "prev_offset0", "prev_offset1",
                  "prev_normal_sticky"):
            setattr(st, k, ptr(m[k]))
        st.match_index = ptr(c.rigid_contact_match_index)
        st.new_indices = ptr(c.rigid_contact_new_indices)
        st.new_count = ptr(c.rigid_contact_new_count)
        st.broken_indices = ptr(c.rigid_contact_broken_indices)
        st.broken_count = ptr(c.rigid_contact_broken_count)
        return st

    def attach_segments(self, c: Contacts) -> None:
        P = max(1, self.layout.pair_count)
        W = self.model.world_count
        dev = self.device
        i32 = dict(dtype=torch.int32, device=dev)
        # solver records: the contacts the public arrays hold, at most 5 per candidate pair
        R = max(1, min(P * 5, int(c.rigid_contact_max)))
        seg = {
            "slots": torch.zeros((P * 5, 20), dtype=torch.float32, device=dev),
            "rec": torch.zeros((R, 20), dtype=torch.float32, device=dev),
            "world_base": torch.zeros(W, dtype=torch.int64, device=dev),
            "cand": torch.zeros(P, **i32),
            "cand_count": torch.zeros(W, **i32),
            "counts": torch.zeros(P, dtype=torch.uint8, device=dev),
            "queue": torch.zeros((2 * P, 2), **i32),
            "world_count": torch.zeros(W, **i32),
            "geom": torch.zeros((max(1, self.model.shape_count), 20), dtype=torch.float32, device=dev),
            "work_counter": torch.zeros(8, **i32),
            "status": torch.zeros(1, **i32),
        }
        if c.force is not None:
            # per-contact impulses: public index of every solver record + the step's scratch
            seg["rec_index"] = torch.full((R,), -1, **i32)
            seg["impulse_scratch"] = torch.zeros((R, 6), dtype=torch.float32, device=dev)
        c._seg = seg
        c._layout = self
        c._seg_valid = False

    def set_step_schedule(self, group_threads: int | None = None, mode: str | None = None) -> None:
        """Choose how the step kernel maps worlds to thread groups (see schedule.py):
        ``mode`` "groups", "groups_compact" or "batch", with ``group_threads``; default: the
        smallest independent group whose arena share holds the largest world, else batches."""
        from .schedule import build_schedule

        sched = build_schedule(self.model, group_threads, mode)
        self._schedule = sched
        self._layout_dev["batch_world"] = torch.from_numpy(sched.batch_world.reshape(-1)).to(self.device)
        self._layout_dev["batch_slab"] = torch.from_numpy(sched.batch_slab.reshape(-1)).to(self.device)
        self._desc = None

    def desc(self):
        if self._desc is None:
            if getattr(self, "_schedule", None) is None:
                self.set_step_schedule()
            arrays = self.model.device_arrays()
            arrays.update(self._layout_dev)
            arrays["schedule"] = self._schedule
            self._desc = self.model.make_desc(arrays, self.layout.info())
            # broad_phase="sap": sweep and prune per world over the NxN candidate list
            self._desc.broad_phase = 1 if self.broad_phase_mode == "sap" else 0
            if "pair_table" in self._layout_dev:
                self._desc.pair_table = ptr(self._layout_dev["pair_table"])
                self._desc.world_table_start = ptr(self._layout_dev["world_table_start"])
        return self._desc

    def grid(self) -> int:
        if self._grid is None:
            self._grid = int(_lib.load().nb_default_grid())
        return self._grid

    @staticmethod
    def seg_struct(c: Contacts) -> NbContactSeg:
        s = c._seg
        st = NbContactSeg()
        for k in ("slots", "rec", "world_base", "cand", "cand_count", "counts", "queue", "world_count", "geom",
                  "work_counter", "status"):
            setattr(st, k, ptr(s[k]))
        st.rec_index = ptr(s["rec_index"]) if "rec_index" in s else None
        return st

    @staticmethod
    def public_struct(c: Contacts) -> NbContactsPublic:
        p = NbContactsPublic()
        p.capacity = c.rigid_contact_max
        p.count = ptr(c.rigid_contact_count)
        p.shape0 = ptr(c.rigid_contact_shape0)
        p.shape1 = ptr(c.rigid_contact_shape1)
        p.point0 = ptr(c.rigid_contact_point0)
        p.point1 = ptr(c.rigid_contact_point1)
        p.offset0 = ptr(c.rigid_contact_offset0)
        p.offset1 = ptr(c.rigid_contact_offset1)
        p.normal = ptr(c.rigid_contact_normal)
        p.margin0 = ptr(c.rigid_contact_margin0)
        p.margin1 = ptr(c.rigid_contact_margin1)
        p.sort_key = ptr(c.rigid_contact_sort_key) if c.rigid_contact_sort_key.numel() else None
        p.world_offset = ptr(c._world_offset)
        p.generation = ptr(c.contact_generation)
        return p

    # ------------------------------------------------------------ collide
    def collide(self, state, contacts: Contacts, *, soft_contact_margin: float | None = None) -> None:
        _lib.require_cuda(self.device)
        if self.model.body_count == 0:
            # no rigid contacts without bodies
            contacts.rigid_contact_count.zero_()
            contacts._seg_valid = False
        else:
            self._collide_rigid(state, contacts)
        if getattr(self.model, "particle_count", 0) and self.model.shape_count and contacts.soft_contact_max > 0:
            from . import particles

            margin = self.soft_contact_margin if soft_contact_margin is None else soft_contact_margin
            particles.soft_collide(self.model, state, contacts, margin)

    def _collide_rigid(self, state, contacts: Contacts) -> None:
        if contacts._seg is None or contacts._layout is not self:
            self.attach_segments(contacts)
        if contacts._world_offset.numel() != self.model.world_count + 1:
            contacts._world_offset = torch.zeros(self.model.world_count + 1, dtype=torch.int64, device=self.device)
        lib = _lib.load()
        grid = 0  # narrow-phase grid: library default
        desc = self.desc()
        seg = self.seg_struct(contacts)
        stream = _lib.stream_handle(self.device)
        bq = state.body_q
        if bq.dtype != torch.float32 or not bq.is_contiguous() or bq.device.type != "cuda":
            raise TypeError("state.body_q must be a contiguous float32 tensor on the model device")
        _lib.check("nb_collide", lib.nb_collide(C.byref(desc), C.c_void_p(ptr(bq)), C.byref(seg), grid,
                                                C.c_void_p(stream)))
        pub = self.public_struct(contacts)
        _lib.check("nb_publish_contacts", lib.nb_publish_contacts(C.byref(desc), C.byref(seg), C.byref(pub),
                                                                  C.c_void_p(stream)))
        if self.contact_matching != "disabled":
            if contacts.rigid_contact_match_index is None:
                raise ValueError("CollisionPipeline has contact_matching enabled but the Contacts buffer was "
                                 "created without contact_matching. Use pipeline.contacts() to create a "
                                 "compatible buffer.")
            if self.contact_report and contacts.rigid_contact_new_indices is None:
                raise ValueError("CollisionPipeline has contact_report enabled but the Contacts buffer was "
                                 "created without contact_report=True. Use pipeline.contacts() to create a "
                                 "compatible buffer.")
            if self._match is None:
                self._alloc_match(contacts.rigid_contact_max)
            st = self._match_struct(contacts)
            _lib.check("nb_match_contacts", lib.nb_match_contacts(C.byref(desc), C.c_void_p(ptr(bq)), C.byref(pub),
                                                                  C.byref(seg), C.byref(st), C.c_void_p(stream)))
        contacts._seg_valid = True

    def status(self, contacts: Contacts) -> int:
        """Device status bits (NB_STATUS_*) accumulated in this contacts buffer (synchronises)."""
        return int(contacts._seg["status"].item())
