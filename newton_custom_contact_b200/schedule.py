"""Work schedule and autotuner for the XPBD step kernel.

Two ways to map worlds to the GPU:

* group modes (``"groups"``, ``"groups_compact"``): the CTA's threads form
  independent groups of G = 32, 64 or 128 threads; every group owns G / 256 of
  its CTA's shared-memory arena and pulls whole worlds, largest first, from a
  device counter -- no CTA-wide barrier between worlds.  ``"groups"`` stages
  the full body slab (43 words per body), ``"groups_compact"`` only the
  mutable part (21 words per body; mass properties are read from the model).
  A G = 32 share holds 62 / 128 bodies, a G = 64 share 125 / 256.
* batch mode: one world per thread group of G threads (G = 32: a warp per
  world ... G = 256: a CTA per world); a CTA holds 256 / G groups that share
  one arena.  Worlds are packed, largest first, into batches that fit one
  arena; CTAs pull batches from a device counter.  Used for worlds too large
  for a warp's share.

``autotune`` times the candidate schedules on the caller's own scene and
keeps the fastest; results are cached per world-size histogram.
"""

from __future__ import annotations

import dataclasses

import numpy as np

CTA_THREADS = 256
WARPS_PER_CTA = CTA_THREADS // 32
SLAB_WORDS_PER_BODY = 6 + 13 + 4 + 9 + 9 + 1 + 1  # must match slab_words_per_body<false>() in nb_xpbd.cu
SLAB_WORDS_COMPACT = 6 + 13 + 1 + 1  # slab_words_per_body<true>()
STEP_MODES = {"batch": 0, "groups": 1, "groups_compact": 2}
GROUP_MODE_SIZES = (32, 64, 128)
# The step kernel's static shared memory (the groups' ordered-accumulation batches) is 21.8 KB for
# 32-thread groups and up to 28.9 KB for 64-thread groups; with the dynamic arena below, two CTAs
# still fit one SM's 228 KB.
ARENA_WORDS_TWO_CTAS = 21 * 1024  # 84 KB: two CTAs per SM
ARENA_WORDS_MAX = 48 * 1024       # 192 KB: the opt-in per-CTA maximum less the kernel's static shared memory
GROUP_SIZES = (32, 64, 128, 256)


@dataclasses.dataclass
class StepSchedule:
    group_threads: int
    cta_threads: int
    arena_words: int
    batch_count: int
    batch_world: np.ndarray   # [batch_count, groups] int32, -1 = empty group
    batch_slab: np.ndarray    # [batch_count, groups] int32 word offsets
    mode: str = "batch"

    @property
    def step_mode(self) -> int:
        return STEP_MODES[self.mode]

    @property
    def groups(self) -> int:
        return self.cta_threads // self.group_threads


def _sm_count() -> int:
    try:
        import torch

        if torch.cuda.is_available():
            return int(torch.cuda.get_device_properties(torch.cuda.current_device()).multi_processor_count)
    except Exception:
        pass
    return 148


def default_group_threads(world_count: int, sms: int | None = None) -> int:
    """Smallest group size that still fills every SM with two CTAs of worlds."""
    sms = sms or _sm_count()
    for g in GROUP_SIZES:
        groups_in_flight = sms * 2 * (CTA_THREADS // g)
        if world_count >= groups_in_flight or g == GROUP_SIZES[-1]:
            return g
    return GROUP_SIZES[-1]


def group_share_words(group_threads: int, arena_words: int = ARENA_WORDS_TWO_CTAS) -> int:
    """Arena words one group owns in the group modes (8-byte aligned)."""
    return (arena_words // (CTA_THREADS // group_threads)) & ~1


def default_mode(max_world_bodies: int) -> tuple:
    """(mode, group_threads): the smallest group whose share holds the largest world, with the full
    slab if it fits, else the compact one; else batches.  (Measured on the 4096-world drop: one
    warp per world with the compact slab beats 64-thread groups with the full slab.)"""
    for g in GROUP_MODE_SIZES:
        for words, mode in ((SLAB_WORDS_PER_BODY, "groups"), (SLAB_WORDS_COMPACT, "groups_compact")):
            if words * max_world_bodies <= group_share_words(g):
                return mode, g
    return "batch", None


def build_schedule(model, group_threads: int | None = None, mode: str | None = None) -> StepSchedule:
    part = model._part
    nb = np.diff(part["world_body_start"].astype(np.int64))
    W = nb.size
    maxb = int(nb.max()) if W else 1
    if mode is None:
        if group_threads is not None:
            mode = "batch"
        else:
            mode, group_threads = default_mode(maxb)
    if mode not in STEP_MODES:
        raise ValueError(f"mode must be one of {tuple(STEP_MODES)}")
    if mode != "batch":
        g = group_threads or 32
        if g not in GROUP_MODE_SIZES:
            raise ValueError(f"group modes take group_threads in {GROUP_MODE_SIZES}")
        words = SLAB_WORDS_PER_BODY if mode == "groups" else SLAB_WORDS_COMPACT
        if words * maxb > group_share_words(g):
            raise ValueError(f"mode {mode!r}: a world with {maxb} bodies does not fit a {g}-thread group's share")
        groups = CTA_THREADS // g
        return StepSchedule(group_threads=g, cta_threads=CTA_THREADS, arena_words=ARENA_WORDS_TWO_CTAS,
                            batch_count=0, batch_world=np.full((1, groups), -1, np.int32),
                            batch_slab=np.zeros((1, groups), np.int32), mode=mode)
    g = group_threads or default_group_threads(W)
    if g not in GROUP_SIZES:
        raise ValueError(f"group_threads must be one of {GROUP_SIZES}")
    groups = CTA_THREADS // g
    slab = SLAB_WORDS_PER_BODY * np.maximum(nb, 1)
    slab = slab + (slab & 1)  # keep every slab 8-byte aligned (int64 accumulators first)
    big = int(slab.max()) if W else 2
    arena = ARENA_WORDS_TWO_CTAS if big <= ARENA_WORDS_TWO_CTAS else big
    if arena > ARENA_WORDS_MAX:
        raise ValueError(f"a world with {int(nb.max())} bodies does not fit in one CTA's shared memory")
    order = np.argsort(-nb, kind="stable")
    batches_w, batches_o = [], []
    cur_w, cur_o, used = [], [], 0
    for w in order:
        s = int(slab[w])
        if len(cur_w) == groups or used + s > arena:
            batches_w.append(cur_w)
            batches_o.append(cur_o)
            cur_w, cur_o, used = [], [], 0
        cur_w.append(int(w))
        cur_o.append(used)
        used += s
    if cur_w:
        batches_w.append(cur_w)
        batches_o.append(cur_o)
    nbatch = len(batches_w)
    bw = np.full((max(nbatch, 1), groups), -1, np.int32)
    bo = np.zeros((max(nbatch, 1), groups), np.int32)
    for i, (ws, os_) in enumerate(zip(batches_w, batches_o)):
        bw[i, : len(ws)] = ws
        bo[i, : len(os_)] = os_
    return StepSchedule(group_threads=g, cta_threads=CTA_THREADS, arena_words=int(arena), batch_count=nbatch,
                        batch_world=bw, batch_slab=bo, mode="batch")


def histogram_key(model, bins=(16, 32, 64, 128, 256, 512)) -> tuple:
    nb = np.diff(model._part["world_body_start"].astype(np.int64))
    h = np.histogram(nb, bins=(0,) + tuple(bins) + (1 << 30,))[0]
    # coarse: log2 bucket of each count so near-identical scenes share an entry
    return tuple(int(np.ceil(np.log2(x + 1))) for x in h)


_CACHE: dict = {}


def candidate_schedules(model) -> list:
    """(mode, group_threads) pairs that can run this model's largest world."""
    nb = np.diff(model._part["world_body_start"].astype(np.int64))
    maxb = int(nb.max()) if nb.size else 1
    out = []
    for words, mode in ((SLAB_WORDS_PER_BODY, "groups"), (SLAB_WORDS_COMPACT, "groups_compact")):
        out += [(mode, g) for g in GROUP_MODE_SIZES if words * maxb <= group_share_words(g)]
    out += [("batch", g) for g in GROUP_SIZES]
    return out


def autotune(pipeline, solver, state_in, state_out, contacts, dt: float, candidates=None, reps: int = 3):
    """Time the step for every candidate schedule on this scene; keep the fastest.

    The state is restored after every trial, so tuning does not advance the
    simulation.  Returns {(mode, group_threads): ms}.
    """
    import torch

    key = histogram_key(pipeline.model)
    if key in _CACHE:
        mode, g = _CACHE[key]
        pipeline.set_step_schedule(g, mode=mode)
        return {}
    if candidates is None:
        candidates = candidate_schedules(pipeline.model)
    q0, qd0 = state_in.body_q.clone(), state_in.body_qd.clone()
    pipeline.collide(state_in, contacts)
    times = {}
    for mode, g in candidates:
        pipeline.set_step_schedule(g, mode=mode)
        solver.step(state_in, state_out, None, contacts, dt)  # warm-up / attribute setup
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        for _ in range(reps):
            solver.step(state_in, state_out, None, contacts, dt)
        b.record()
        torch.cuda.synchronize()
        times[(mode, g)] = a.elapsed_time(b) / reps
    best = min(times, key=times.get)
    _CACHE[key] = best
    pipeline.set_step_schedule(best[1], mode=best[0])
    state_in.body_q.copy_(q0)
    state_in.body_qd.copy_(qd0)
    return times
