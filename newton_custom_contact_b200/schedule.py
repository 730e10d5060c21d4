"""Work schedule and autotuner for the XPBD step kernel.

The step kernel runs one world per thread group of G threads (G = 32: a warp
per world ... G = 256: a CTA per world).  A CTA holds 256 / G groups that
share one shared-memory arena; each world gets a slab of
``SLAB_WORDS_PER_BODY * bodies`` 4-byte words for its body state, mass
properties and fixed-point delta accumulators.  ``build_schedule`` packs
worlds, largest first, into batches that fit one arena, so CTAs pulling
batches from the device counter get similar-size worlds (little idle time at
the batch barrier) and the biggest worlds start first.

``autotune`` times the candidate group sizes on the caller's own scene and
keeps the fastest; results are cached per world-size histogram.
"""

from __future__ import annotations

import dataclasses

import numpy as np

CTA_THREADS = 256
SLAB_WORDS_PER_BODY = 12 + 13 + 4 + 9 + 9 + 1 + 1  # must match slab_words_per_body() in nb_xpbd.cu
ARENA_WORDS_TWO_CTAS = 27 * 1024  # ~108 KB: two CTAs per SM
ARENA_WORDS_MAX = 55 * 1024       # ~220 KB: the opt-in per-CTA maximum less the kernel's static shared memory
GROUP_SIZES = (32, 64, 128, 256)


@dataclasses.dataclass
class StepSchedule:
    group_threads: int
    cta_threads: int
    arena_words: int
    batch_count: int
    batch_world: np.ndarray   # [batch_count, groups] int32, -1 = empty group
    batch_slab: np.ndarray    # [batch_count, groups] int32 word offsets

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


def build_schedule(model, group_threads: int | None = None) -> StepSchedule:
    part = model._part
    nb = np.diff(part["world_body_start"].astype(np.int64))
    W = nb.size
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
                        batch_world=bw, batch_slab=bo)


def histogram_key(model, bins=(16, 32, 64, 128, 256, 512)) -> tuple:
    nb = np.diff(model._part["world_body_start"].astype(np.int64))
    h = np.histogram(nb, bins=(0,) + tuple(bins) + (1 << 30,))[0]
    # coarse: log2 bucket of each count so near-identical scenes share an entry
    return tuple(int(np.ceil(np.log2(x + 1))) for x in h)


_CACHE: dict = {}


def autotune(pipeline, solver, state_in, state_out, contacts, dt: float, candidates=GROUP_SIZES, reps: int = 3):
    """Time one collide + step per candidate group size on this scene; keep the fastest.

    The state is restored after every trial, so tuning does not advance the
    simulation.  Returns {group_threads: ms}.
    """
    import torch

    key = histogram_key(pipeline.model)
    if key in _CACHE:
        pipeline.set_step_schedule(_CACHE[key])
        return {}
    q0, qd0 = state_in.body_q.clone(), state_in.body_qd.clone()
    pipeline.collide(state_in, contacts)
    times = {}
    for g in candidates:
        pipeline.set_step_schedule(g)
        solver.step(state_in, state_out, None, contacts, dt)  # warm-up / attribute setup
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        for _ in range(reps):
            solver.step(state_in, state_out, None, contacts, dt)
        b.record()
        torch.cuda.synchronize()
        times[g] = a.elapsed_time(b) / reps
    best = min(times, key=times.get)
    _CACHE[key] = best
    pipeline.set_step_schedule(best)
    state_in.body_q.copy_(q0)
    state_in.body_qd.copy_(qd0)
    return times
