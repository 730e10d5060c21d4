"""Benchmark: world-substeps/s of the rigid-contact XPBD step (collide + SolverXPBD.step).

Workload: 4096 uneven worlds of box / sphere / capsule bodies (N ~ U{8..128}),
dt = 1/60 s, 8 substeps, 8 iterations, FP32, seeded synthetic scene.  One
frame = 8 x (State.clear_forces, CollisionPipeline.collide, SolverXPBD.step),
captured once as a CUDA graph and replayed.

One benchmark step = one pass over the drop's frames 6..35 (30 frames = 240
substeps: bodies falling, landing and piling up).  Before every step the state
is reset to frame 6 and L2 is flushed, outside the timed events, so every step
times the same frames whatever --steps is.  Later frames are avoided because
the reference integrator's explicit gyroscopic term (integrate_rigid_body,
newton/_src/solvers/solver.py:80-86) lets a thin capsule spinning about its
axis diverge: with seed 1 the first world leaves the finite range at frame 42,
in the CUDA path and the CPU oracle alike.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Under torchrun (N > 1) every rank simulates its own 4096-world scene (weak
scaling, no data-path collective); rank 0 prints one JSON line.
"""

from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

METRIC = "world-substeps/s @4096 worlds, plain vs NN warm-start at equal max penetration"
UNIT = "world-substeps/s"
WORKLOAD = "C2: 4096 uneven worlds (8..128 box/sphere/capsule bodies), dt 1/60, 8 substeps x 8 iterations"
WINDOW_START = 6    # frames simulated before the timed window
WINDOW_FRAMES = 30  # one timed step = frames WINDOW_START .. WINDOW_START + 29
FRAMES = f"{WINDOW_START}..{WINDOW_START + WINDOW_FRAMES - 1}"
CPU_SAMPLE_WORLDS = 256


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--worlds", type=int, default=4096)
    ap.add_argument("--seed", type=int, default=1)
    ap.add_argument("--cpu-sample-seconds", type=float, default=12.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-warm-start", action="store_true", help="skip the learned-warm-start arm")
    ap.add_argument("--warm-start-iterations", type=int, default=2)
    ap.add_argument("--no-articulated", action="store_true", help="skip the articulated (C3) batch")
    ap.add_argument("--no-particles", action="store_true", help="skip the particle drop")
    ap.add_argument("--particles-only", action="store_true",
                    help="run only the particle drop and print its line (a diagnostic run, not the benchmark line)")
    ap.add_argument("--warm-start-sweep", default="", metavar="K1,K2,...",
                    help="also time the plain and the warm-started forms at these iteration counts")
    ap.add_argument("--step-schedule", default=None, metavar="MODE/G",
                    help="fix the step schedule (e.g. groups_compact/32) instead of autotuning it; a run "
                         "under a profiler serialises launches, so its autotuner may pick another schedule")
    ap.add_argument("--broad-phase", default="explicit", choices=["explicit", "nxn", "sap"],
                    help="CollisionPipeline broad phase of the main workload (the reference's default: explicit)")
    ap.add_argument("--build", default="product", choices=["product", "exact"],
                    help="library build: product (FMA contraction in the solver) or exact (the parity build)")
    ap.add_argument("--scaling", default="weak", choices=["weak", "strong"],
                    help="weak: every rank simulates its own --worlds scene; strong: the ranks split one scene")
    return ap.parse_args()


# ---------------------------------------------------------------- clocks
class ClockSampler:
    """nvidia-smi samples of SM clock and throttle reasons during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.rows = []
        self._stop = threading.Event()
        self._t = None

    def _run(self):
        while not self._stop.is_set():
            try:
                out = subprocess.run(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.FIELDS}",
                                      "--format=csv,noheader,nounits"], capture_output=True, text=True, timeout=5)
                if out.returncode == 0 and out.stdout.strip():
                    self.rows.append([x.strip() for x in out.stdout.strip().split(",")])
            except Exception:
                pass
            self._stop.wait(0.2)

    def __enter__(self):
        self._t = threading.Thread(target=self._run, daemon=True)
        self._t.start()
        return self

    def __exit__(self, *exc):
        self._stop.set()
        if self._t:
            self._t.join(timeout=10)

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if r[2].replace(".", "").isdigit()]
        reasons = set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in self.rows:
            for n, v in zip(names, r[5:9]):
                if "Active" in v and "Not" not in v:
                    reasons.add(n)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(self.rows)}


# ---------------------------------------------------------------- CPU baseline (oracle port)
def _oracle_sample(seed: int, worlds_total: int):
    """The first CPU_SAMPLE_WORLDS worlds of the C2 scene on the host, advanced to the window start."""
    import oracle
    from newton_custom_contact_b200 import SolverXPBD, scenes
    from newton_custom_contact_b200.collide import PairLayout

    oracle.build()
    sample_worlds = min(CPU_SAMPLE_WORLDS, worlds_total)
    model, info = scenes.scene_c2(seed=seed, worlds=worlds_total, device="cpu", keep_worlds=sample_worlds)
    lay = PairLayout(model, model.host("shape_contact_pairs"))
    p = SolverXPBD(model, iterations=info["iterations"]).params()
    dt = info["dt"] / info["substeps"]
    f = np.zeros((model.body_count, 6), np.float32)

    def frame(q, qd):
        for _ in range(info["substeps"]):
            segs = oracle.collide(model, lay, q)
            q, qd, _ = oracle.step(model, lay, p, q, qd, f, segs, dt)
        return q, qd

    q, qd = model.host("body_q").copy(), model.host("body_qd").copy()
    for _ in range(WINDOW_START):
        q, qd = frame(q, qd)
    return sample_worlds, info["substeps"], frame, q, qd


def cpu_baseline(seed: int, seconds: float, worlds_total: int):
    """Oracle (sequential C++ restatement, OpenMP over worlds) on a bounded sample of the C2 workload:
    the first CPU_SAMPLE_WORLDS worlds of the same scene over the same frames 6..35, whole windows
    (the state reset to frame 6 before each) until about `seconds` of CPU time were measured."""
    sample_worlds, substeps, frame, q0, qd0 = _oracle_sample(seed, worlds_total)
    windows = 0
    el = 0.0
    while el < seconds or windows == 0:
        q, qd = q0.copy(), qd0.copy()
        t0 = time.perf_counter()
        for _ in range(WINDOW_FRAMES):
            q, qd = frame(q, qd)
        el += time.perf_counter() - t0
        windows += 1
    n_sub = windows * WINDOW_FRAMES * substeps
    cores = int(os.environ.get("OMP_NUM_THREADS", os.cpu_count() or 1))
    value = sample_worlds * n_sub / el
    return {"value": value, "unit": UNIT, "cores": cores, "kind": "port",
            "sample": f"first {sample_worlds} of the {worlds_total} C2 worlds, {windows} passes over frames "
                      f"{FRAMES} ({n_sub} substeps of collide + step), {el:.1f} s measured, OpenMP over worlds; "
                      f"a per-world rate, compared with the GPU's 4096-world rate"}


# ---------------------------------------------------------------- reference arm
def run_reference(args, rank):
    """The reference's CPU path for this workload: warp-lang (the reference's runtime) is not installed
    on this image, so the CPU restatement of the reference kernels (oracle/) stands in for it, on all
    host cores.  One step = one pass over the window's 30 frames for the first CPU_SAMPLE_WORLDS worlds
    of the same scene (the state is reset to the window start before each step, outside the timing);
    --warmup untimed steps, then --steps timed ones."""
    if rank != 0:
        return
    sample_worlds, substeps, frame, q0, qd0 = _oracle_sample(args.seed, args.worlds)

    def window():
        q, qd = q0.copy(), qd0.copy()
        t0 = time.perf_counter()
        for _ in range(WINDOW_FRAMES):
            q, qd = frame(q, qd)
        return time.perf_counter() - t0

    for _ in range(args.warmup):
        window()
    times = [window() for _ in range(args.steps)]
    el = float(sum(times))
    units = sample_worlds * substeps * WINDOW_FRAMES * args.steps
    value = units / el
    cores = int(os.environ.get("OMP_NUM_THREADS", os.cpu_count() or 1))
    sample = (f"first {sample_worlds} of the {args.worlds} C2 worlds, frames {FRAMES} per step "
              f"({substeps * WINDOW_FRAMES} substeps of collide + step), {args.steps} timed steps after "
              f"{args.warmup} warm-up steps, {el:.1f} s measured; a per-world rate")
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * el / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded)",
            "config": {"workload": WORKLOAD, "worlds": sample_worlds, "frames": FRAMES,
                       "step": f"{WINDOW_FRAMES} frames x {substeps} substeps of {sample_worlds} worlds"},
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "port", "sample": sample},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "note": "warp-lang (the reference's runtime) is not installed on this image and cannot be installed "
                    "(no network), so the reference arm times the CPU restatement of the reference kernels "
                    "(oracle/) on the host cores; ms_per_step is the measured time of one step of the "
                    f"{sample_worlds}-world sample, and value is a per-world rate comparable with the GPU arm's"}
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------- ours
def algorithmic_bytes(model, layout, n_contacts: float):
    """Bytes one collide and one step launch must move (per substep, all worlds)."""
    B = model.body_count
    S = model.shape_count
    P = layout.pair_count
    # step: per body read q, qd, f (76 B) and static com, inverse mass, inertia,
    # inverse inertia, flags, world (96 B), write q, qd (52 B); each contact
    # record read once (80 B)
    step = B * (76 + 96 + 52) + n_contacts * 80
    # collide: shape transform/scale/type/body (44 B), body pose (28 B), packed pair (4 B), contact slot written (80 B)
    collide = S * 44 + B * 28 + P * 4 + n_contacts * 80
    # publish: slot read (80 B), solver record (80 B) and public row + sort key (84 B) written
    publish = n_contacts * (80 + 80 + 84)
    return {"step": step, "collide": collide, "publish": publish}


def _window_penetration(graph, stream, model, contacts, state, frames):
    """Replay `graph` (one frame) `frames` times from the current state; per frame the penetration
    statistics of the frame's last contacts at the frame's final poses."""
    import torch

    from newton_custom_contact_b200.metrics import penetration_stats

    out = []
    for _ in range(frames):
        with torch.cuda.stream(stream):
            graph.replay()
        torch.cuda.synchronize()
        out.append(penetration_stats(model, contacts, state.body_q))
    return out


def _pen_summary(stats):
    return {k: float(np.nanmean([p[k] for p in stats]) * 1e3) for k in ("max", "p99", "mean")} | {
        "worst": float(np.nanmax([p["max"] for p in stats]) * 1e3)}


def _state_snapshot(tensors):
    """Copies of the device tensors that carry state from one frame to the next; `restore()` puts them
    back (on the current stream)."""
    saved = [(t, t.clone()) for t in tensors]

    def restore():
        for t, v in saved:
            t.copy_(v)

    return restore


def time_windows(graph, stream, restore, flush, steps, warmup):
    """Per step: restore the window start and flush L2 (untimed), then replay `graph` (one frame) for the
    window's WINDOW_FRAMES frames between CUDA events on `stream`.  Returns the total ms of the timed steps."""
    import torch

    starts = [torch.cuda.Event(enable_timing=True) for _ in range(steps)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(steps)]
    with torch.cuda.stream(stream):
        for _ in range(warmup):
            restore()
            for _ in range(WINDOW_FRAMES):
                graph.replay()
        for k in range(steps):
            restore()
            flush.fill_(float(k))
            starts[k].record(stream)
            for _ in range(WINDOW_FRAMES):
                graph.replay()
            ends[k].record(stream)
    torch.cuda.synchronize()
    return sum(starts[k].elapsed_time(ends[k]) for k in range(steps))


def warm_start_arm(model, dt, substeps, sched, stream, flush, steps, warmup, iterations):
    """The learned-warm-start form on the same scene and frames: contact matching ("latest", for the
    previous-lambda feature) + warm start + `iterations` plain iterations per substep.  Timed like the
    plain form: each step replays frames 6..35 from the same frame-6 state, matching history and
    previous-substep lambdas (all restored before the step, untimed), L2 flushed; penetration statistics
    along one pass of the same window."""
    import torch

    from newton_custom_contact_b200 import CollisionPipeline, SolverXPBD
    from newton_custom_contact_b200.warmstart import WarmStart, WarmStartNet

    net = WarmStartNet.load(os.path.join(ROOT, "newton_custom_contact_b200", "data", "warmstart_c2.npz"),
                            device=model.device)
    pipe = CollisionPipeline(model, contact_matching="latest")
    pipe.set_step_schedule(sched.group_threads, sched.mode)
    solver = SolverXPBD(model, iterations=iterations)
    ws = WarmStart(net, iterations=iterations)
    solver.warm_start = ws
    a, b = model.state(), model.state()
    c = pipe.contacts()

    def frame():
        x, y = a, b
        for _ in range(substeps):
            x.clear_forces()
            pipe.collide(x, c)
            solver.step(x, y, None, c, dt)
            x, y = y, x

    # buffers allocated on the default stream above are used on `stream` below
    stream.wait_stream(torch.cuda.current_stream(stream.device))
    with torch.cuda.stream(stream):
        for _ in range(WINDOW_START):
            frame()
    torch.cuda.synchronize()
    carried = [a.body_q, a.body_qd]
    carried += [t for t in pipe._match.values() if isinstance(t, torch.Tensor)]
    carried += [t for t in ws._bufs.values() if isinstance(t, torch.Tensor)]
    restore = _state_snapshot(carried)
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g, stream=stream):
        frame()
    torch.cuda.synchronize()
    with torch.cuda.stream(stream):
        restore()
    fb0 = ws.fallback_count
    pen = _window_penetration(g, stream, model, c, a, WINDOW_FRAMES)
    fb1 = ws.fallback_count
    ms = time_windows(g, stream, restore, flush, steps, warmup)
    del g
    units = model.world_count * substeps * WINDOW_FRAMES * steps
    return {"iterations": iterations, "value": units / (ms / 1e3), "ms_per_step": ms / steps,
            "frames": FRAMES, "penetration_mm": _pen_summary(pen),
            "fallback_world_fraction": (fb1 - fb0) / float(model.world_count * substeps * WINDOW_FRAMES),
            "contact_matching": "latest", "network": "newton_custom_contact_b200/data/warmstart_c2.npz"}


ARM_AMPLITUDE = 0.5               # rad, joint target amplitude of the articulated batch
ARM_FREQUENCY = 0.5               # Hz


def articulated_arm(dev, stream, flush, steps, warmup):
    """The articulated batch (4096 worlds of a 7-link revolute arm among 8..48 loose boxes on a table
    plane; dt 1/120 s, 4 substeps x 8 iterations): joint targets A sin(2 pi f t + phase) with a random
    phase per joint, written into Control.joint_target_pos before every frame (inside the timed
    region).  Timed like the main workload: each step is frames 6..35 from the same frame-6 state."""
    import torch

    from newton_custom_contact_b200 import CollisionPipeline, JointType, SolverXPBD, scenes
    from newton_custom_contact_b200.metrics import max_joint_violation, max_penetration
    from newton_custom_contact_b200.schedule import autotune

    t0 = time.perf_counter()
    model, info = scenes.scene_c3(worlds=4096, device=dev)
    build_s = time.perf_counter() - t0
    substeps, iters = info["substeps"], info["iterations"]
    dt = info["dt"] / substeps
    pipe = CollisionPipeline(model)
    solver = SolverXPBD(model, iterations=iters)
    s0, s1 = model.state(), model.state()
    contacts = pipe.contacts()
    control = model.control()
    # joint target table: frame f sets the targets of time f * frame_dt
    jt = model.host("joint_type")
    rev = np.nonzero(jt == int(JointType.REVOLUTE))[0]
    dof = model.host("joint_qd_start")[rev]
    phases = np.asarray(info["phases"], np.float64).reshape(-1)
    n_frames = WINDOW_START + WINDOW_FRAMES
    table = np.zeros((n_frames, model.joint_dof_count), np.float32)
    for f in range(n_frames):
        table[f, dof] = ARM_AMPLITUDE * np.sin(2.0 * np.pi * ARM_FREQUENCY * f * info["dt"] + phases)
    table_d = torch.from_numpy(table).to(dev)

    def frame():
        a, b = s0, s1
        for _ in range(substeps):
            a.clear_forces()
            pipe.collide(a, contacts)
            solver.step(a, b, control, contacts, dt)
            a, b = b, a

    # buffers allocated on the default stream above are used on `stream` below
    stream.wait_stream(torch.cuda.current_stream(stream.device))
    with torch.cuda.stream(stream):
        for f in range(WINDOW_START):
            control.joint_target_pos.copy_(table_d[f])
            frame()
    torch.cuda.synchronize()
    snap = (s0.body_q.clone(), s0.body_qd.clone())
    with torch.cuda.stream(stream):
        s0.clear_forces()
        tune_ms = autotune(pipe, solver, s0, s1, contacts, dt, reps=3)
    torch.cuda.synchronize()
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g, stream=stream):
        frame()
    torch.cuda.synchronize()

    def window():
        for f in range(WINDOW_START, n_frames):
            control.joint_target_pos.copy_(table_d[f])
            g.replay()

    starts = [torch.cuda.Event(enable_timing=True) for _ in range(steps)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(steps)]
    with torch.cuda.stream(stream):
        for k in range(warmup + steps):
            s0.body_q.copy_(snap[0])
            s0.body_qd.copy_(snap[1])
            flush.fill_(float(k))
            if k >= warmup:
                starts[k - warmup].record(stream)
            window()
            if k >= warmup:
                ends[k - warmup].record(stream)
    torch.cuda.synchronize()
    ms = sum(starts[k].elapsed_time(ends[k]) for k in range(steps))
    with torch.cuda.stream(stream):
        pipe.collide(s0, contacts)
    torch.cuda.synchronize()
    pen, jv = max_penetration(model, contacts, s0.body_q), max_joint_violation(model, s0.body_q)
    finite = bool(torch.isfinite(s0.body_q).all().item())
    del g
    units = model.world_count * substeps * WINDOW_FRAMES * steps
    sched = pipe._schedule
    return {"workload": "C3: 4096 worlds of a 7-link revolute arm (capsules r 0.04 m, 0.3 m, 1 kg, limits "
                        "+-2.5 rad, drive ke 500 kd 20) among 8..48 boxes on a table plane; dt 1/120, 4 substeps "
                        "x 8 iterations",
            "value": units / (ms / 1e3), "unit": UNIT, "ms_per_step": ms / steps, "frames": FRAMES,
            "bodies": model.body_count, "joints": model.joint_count,
            "joint_targets": f"{ARM_AMPLITUDE} rad x sin(2 pi {ARM_FREQUENCY} Hz t + phase), set every frame",
            "max_joint_violation_m": jv, "max_penetration_m": pen, "final_state_finite": finite,
            "step_schedule": {"mode": sched.mode, "group_threads": sched.group_threads,
                              "autotune_ms": {f"{m}/{g_}": round(v, 4) for (m, g_), v in tune_ms.items()}},
            "scene_build_s": round(build_s, 1)}


def particles_arm(dev, stream, flush, steps, warmup):
    """The particle path: a 100 x 100 spring cloth (10,000 particles, 39,402 springs, 9,801 bending edges) and 100,000 loose
    particles dropped onto a ground plane, a box, a sphere and a capsule; dt 1/240 s, 8 iterations.  One
    step is 60 substeps (collide + solver step each, CUDA-graph captured) from the same start state,
    taken after 40 untimed substeps, when the cloth and the loose particles are landing."""
    import torch

    from newton_custom_contact_b200 import CollisionPipeline, SolverXPBD, scenes

    n_sub, pre = 60, 40
    t0 = time.perf_counter()
    model, info = scenes.scene_particles(seed=2, cloth=100, loose=100_000, radius=0.01, device=dev,
                                         loose_extent=1.0, loose_height=(0.33, 1.2))
    build_s = time.perf_counter() - t0
    dt = 1.0 / 240.0
    pipe = CollisionPipeline(model)
    solver = SolverXPBD(model, iterations=8)
    s0, s1 = model.state(), model.state()
    contacts = pipe.contacts()

    def substeps(n):
        a, b = s0, s1
        for _ in range(n // 2 * 2):
            pipe.collide(a, contacts)
            solver.step(a, b, None, contacts, dt)
            a, b = b, a

    stream.wait_stream(torch.cuda.current_stream(stream.device))
    with torch.cuda.stream(stream):
        substeps(pre)
    torch.cuda.synchronize()
    snap = (s0.particle_q.clone(), s0.particle_qd.clone())
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g, stream=stream):
        substeps(n_sub)
    torch.cuda.synchronize()
    starts = [torch.cuda.Event(enable_timing=True) for _ in range(steps)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(steps)]
    contacts_seen = []
    with torch.cuda.stream(stream):
        for k in range(warmup + steps):
            s0.particle_q.copy_(snap[0])
            s0.particle_qd.copy_(snap[1])
            flush.fill_(float(k))
            if k >= warmup:
                starts[k - warmup].record(stream)
            g.replay()
            if k >= warmup:
                ends[k - warmup].record(stream)
                contacts_seen.append(contacts.soft_contact_count.clone())
    torch.cuda.synchronize()
    ms = sum(starts[k].elapsed_time(ends[k]) for k in range(steps))
    q = s0.particle_q
    r = model.particle_radius
    act = (model.particle_flags & 1) != 0
    del g
    P = model.particle_count
    return {"workload": "particles: 100x100 spring + bending cloth + 100,000 loose particles (r 5..10 mm) dropped on a "
                        "plane, box, sphere and capsule; dt 1/240, 8 iterations, substeps 41..100 of the drop",
            "value": P * n_sub * steps / (ms / 1e3), "unit": "particle-substeps/s",
            "ms_per_substep": ms / steps / n_sub, "particles": P, "springs": model.spring_count,
            "soft_contacts_at_step_end": int(torch.stack(contacts_seen).float().mean().item()),
            "min_height_above_radius_m": float((q[act, 2] - r[act]).min().item()),
            "final_state_finite": bool(torch.isfinite(q).all().item()),
            # soft contacts 3 kernels, integrate 1, then constraints (+ bending) + apply per iteration
            "status": solver._particles.status(),
            "gpu_launches_per_substep": 3 + 1 + (3 if model.edge_count else 2) * 8, "bending_edges": model.edge_count,
            "scene_build_s": round(build_s, 1)}


def plain_arm(model, dt, substeps, sched, stream, flush, steps, warmup, iterations):
    """The plain form with `iterations` iterations on the same scene and frames (for the warm-start
    sweep): timed like the main workload, penetration statistics along one pass of the window."""
    import torch

    from newton_custom_contact_b200 import CollisionPipeline, SolverXPBD

    pipe = CollisionPipeline(model)
    pipe.set_step_schedule(sched.group_threads, sched.mode)
    solver = SolverXPBD(model, iterations=iterations)
    a, b = model.state(), model.state()
    c = pipe.contacts()

    def frame():
        x, y = a, b
        for _ in range(substeps):
            x.clear_forces()
            pipe.collide(x, c)
            solver.step(x, y, None, c, dt)
            x, y = y, x

    # buffers allocated on the default stream above are used on `stream` below
    stream.wait_stream(torch.cuda.current_stream(stream.device))
    with torch.cuda.stream(stream):
        for _ in range(WINDOW_START):
            frame()
    torch.cuda.synchronize()
    restore = _state_snapshot([a.body_q, a.body_qd])
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g, stream=stream):
        frame()
    torch.cuda.synchronize()
    with torch.cuda.stream(stream):
        restore()
    pen = _window_penetration(g, stream, model, c, a, WINDOW_FRAMES)
    ms = time_windows(g, stream, restore, flush, steps, warmup)
    del g
    units = model.world_count * substeps * WINDOW_FRAMES * steps
    return {"iterations": iterations, "value": units / (ms / 1e3), "ms_per_step": ms / steps,
            "penetration_mm": _pen_summary(pen)}


def warm_start_sweep(model, dt, substeps, sched, stream, flush, steps, warmup, iterations):
    """Plain and warm-started forms at each of `iterations` on the same frames: throughput and
    penetration, and for each warm-started form the plain form it matches or beats on the mean of the
    per-frame largest penetration, with the throughput ratio."""
    plain = [plain_arm(model, dt, substeps, sched, stream, flush, steps, warmup, k) for k in iterations]
    warm = [warm_start_arm(model, dt, substeps, sched, stream, flush, steps, warmup, k) for k in iterations]
    ref8 = next((p for p in plain if p["iterations"] == 8), plain[-1])
    best = None
    for w in warm:
        if w["penetration_mm"]["max"] <= ref8["penetration_mm"]["max"]:
            r = w["value"] / ref8["value"]
            if best is None or r > best["throughput_vs_plain"]:
                best = {"warm_iterations": w["iterations"], "throughput_vs_plain": r,
                        "plain_iterations": ref8["iterations"]}
    return {"plain": plain, "warm_start": warm, "best_at_equal_max_penetration": best,
            "penetration_metric": "mean over frames 6..35 of each frame's largest penetration [mm]"}


def run_ours(args, rank, world_size, local_rank):
    import torch

    from newton_custom_contact_b200 import CollisionPipeline, SolverXPBD, _lib, scenes

    _lib.use_build(args.build)
    dev = torch.device("cuda", local_rank)
    torch.cuda.set_device(dev)
    if args.particles_only:
        stream = torch.cuda.Stream(dev)
        flush = torch.empty(int(256 * 2**20) // 4, dtype=torch.float32, device=dev)
        if rank == 0:
            print(json.dumps({"particles": particles_arm(dev, stream, flush, args.steps, args.warmup)}), flush=True)
        return
    dist = None
    if world_size > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    from newton_custom_contact_b200.distributed import max_over_ranks, shard_range

    if args.scaling == "strong" and world_size > 1:
        lo, hi = shard_range(rank, world_size, scenes.c2_world_body_counts(args.seed, args.worlds))
        model, info = scenes.scene_c2(seed=args.seed, worlds=args.worlds, device=dev, world_range=(lo, hi))
    else:
        model, info = scenes.scene_c2(seed=args.seed + 1000 * rank, worlds=args.worlds, device=dev)
    substeps, iters = info["substeps"], info["iterations"]
    dt = info["dt"] / substeps
    pipe = CollisionPipeline(model, broad_phase=args.broad_phase)
    solver = SolverXPBD(model, iterations=iters)
    s0, s1 = model.state(), model.state()
    contacts = pipe.contacts()
    stream = torch.cuda.Stream(dev)
    # the scene's and the contacts' buffers were allocated (and zero-filled) on the default stream
    stream.wait_stream(torch.cuda.current_stream(dev))

    def frame():
        a, b = s0, s1
        for _ in range(substeps):
            a.clear_forces()
            pipe.collide(a, contacts)
            solver.step(a, b, None, contacts, dt)
            a, b = b, a

    # eager frames up to the window start (also load the library, set kernel attributes)
    with torch.cuda.stream(stream):
        for _ in range(WINDOW_START):
            frame()
    torch.cuda.synchronize()
    snap_q, snap_qd = s0.body_q.clone(), s0.body_qd.clone()
    # step schedule: autotuned on this scene (keyed on its world-size histogram); the
    # trials restore the state, so the trajectory does not move
    from newton_custom_contact_b200.schedule import autotune

    if args.step_schedule:
        mode, g_threads = args.step_schedule.split("/")
        pipe.set_step_schedule(int(g_threads), mode)
        tune_ms = {}
    else:
        with torch.cuda.stream(stream):
            s0.clear_forces()
            tune_ms = autotune(pipe, solver, s0, s1, contacts, dt, reps=3)
    torch.cuda.synchronize()
    sched = pipe._schedule

    def restore():
        s0.body_q.copy_(snap_q)
        s0.body_qd.copy_(snap_qd)

    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g, stream=stream):
        frame()
    torch.cuda.synchronize()
    flush = torch.empty(int(256 * 2**20) // 4, dtype=torch.float32, device=dev)
    with torch.cuda.stream(stream):
        restore()
        for _ in range(WINDOW_FRAMES):
            g.replay()
    torch.cuda.synchronize()
    # per-stage timing pass (same kernels, same frame window) for the roofline: each substep's stages
    # (clear_forces + nb_collide, nb_publish_contacts, the step) are captured as three small CUDA
    # graphs per state parity and replayed between events, so the host, which only launches graphs,
    # stays ahead of the device and no launch gap falls inside a pair of events
    import ctypes as C

    from newton_custom_contact_b200 import _lib

    lib = _lib.load()
    n_sub = WINDOW_FRAMES * substeps
    stage_graphs = []
    contacts._seg_valid = True
    for a, b in ((s0, s1), (s1, s0)):
        gc, gp, gs = torch.cuda.CUDAGraph(), torch.cuda.CUDAGraph(), torch.cuda.CUDAGraph()
        desc, seg, pub = pipe.desc(), pipe.seg_struct(contacts), pipe.public_struct(contacts)
        with torch.cuda.graph(gc, stream=stream):
            a.clear_forces()
            _lib.check("nb_collide", lib.nb_collide(C.byref(desc), C.c_void_p(a.body_q.data_ptr()), C.byref(seg), 0,
                                                    C.c_void_p(_lib.stream_handle(dev))))
        with torch.cuda.graph(gp, stream=stream):
            _lib.check("nb_publish_contacts", lib.nb_publish_contacts(C.byref(desc), C.byref(seg), C.byref(pub),
                                                                      C.c_void_p(_lib.stream_handle(dev))))
        with torch.cuda.graph(gs, stream=stream):
            solver.step(a, b, None, contacts, dt)
        stage_graphs.append((gc, gp, gs))
    evs = [[torch.cuda.Event(enable_timing=True) for _ in range(4)] for _ in range(n_sub)]
    n_contacts_acc = torch.zeros((), dtype=torch.float64, device=dev)
    with torch.cuda.stream(stream):
        restore()
        for i in range(n_sub):
            gc, gp, gs = stage_graphs[i % 2]
            ev = evs[i]
            ev[0].record(stream)
            gc.replay()
            ev[1].record(stream)
            gp.replay()
            ev[2].record(stream)
            gs.replay()
            ev[3].record(stream)
            n_contacts_acc += contacts._seg["world_count"].sum()
    torch.cuda.synchronize()
    del stage_graphs
    t_col = sum(e[0].elapsed_time(e[1]) for e in evs)
    t_pub = sum(e[1].elapsed_time(e[2]) for e in evs)
    t_step = sum(e[2].elapsed_time(e[3]) for e in evs)
    n_contacts = float(n_contacts_acc.item()) / n_sub
    # timed region: K steps, each the WINDOW_FRAMES frames from the window start (state restored and L2
    # flushed before every step, outside the events)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    with ClockSampler(local_rank) as clk:
        ms = time_windows(g, stream, restore, flush, args.steps, args.warmup)
    # run metrics at the end of the last timed window (max over ranks)
    from newton_custom_contact_b200.metrics import max_joint_violation, max_penetration

    with torch.cuda.stream(stream):
        pipe.collide(s0, contacts)
    torch.cuda.synchronize()
    pen, jv = max_penetration(model, contacts, s0.body_q), max_joint_violation(model, s0.body_q)
    ms = max_over_ranks(ms, device=dev)
    pen, jv = max_over_ranks([pen, jv], device=dev)
    if dist:
        dist.barrier()
    frames_timed = WINDOW_FRAMES * args.steps
    units = args.worlds * substeps * frames_timed * (world_size if args.scaling == "weak" else 1)
    value = units / (ms / 1e3)
    # e2e through the public API with host buffers: every step uploads its input state (body_q /
    # body_qd at the window start) from pinned host memory, runs the window's frames (collide + step
    # x 8 each) and downloads the resulting state.  One step = the same window of frames from the
    # same start state.
    host_q0, host_qd0 = snap_q.cpu(), snap_qd.cpu()
    hq = torch.empty(s0.body_q.shape, dtype=torch.float32).pin_memory()
    hqd = torch.empty(s0.body_qd.shape, dtype=torch.float32).pin_memory()
    e_s = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    e_e = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    for k in range(args.steps):
        torch.cuda.synchronize()
        hq.copy_(host_q0)
        hqd.copy_(host_qd0)
        with torch.cuda.stream(stream):
            flush.fill_(float(k))
            e_s[k].record(stream)
            s0.body_q.copy_(hq, non_blocking=True)
            s0.body_qd.copy_(hqd, non_blocking=True)
            for _ in range(WINDOW_FRAMES):
                g.replay()
            hq.copy_(s0.body_q, non_blocking=True)
            hqd.copy_(s0.body_qd, non_blocking=True)
            e_e[k].record(stream)
    torch.cuda.synchronize()
    e2e_ms = max_over_ranks(sum(e_s[k].elapsed_time(e_e[k]) for k in range(args.steps)), device=dev)
    e2e_value = units / (e2e_ms / 1e3)
    state_bytes = int(hq.numel() * 4 + hqd.numel() * 4)
    status = pipe.status(contacts)
    q = s0.body_q
    finite = bool(torch.isfinite(q).all().item())
    warm = None
    if not args.no_warm_start and world_size == 1:
        # the plain form's penetration along one pass of the same window, then the warm-start form
        with torch.cuda.stream(stream):
            restore()
        plain_pen = _pen_summary(_window_penetration(g, stream, model, contacts, s0, WINDOW_FRAMES))
        warm = warm_start_arm(model, dt, substeps, sched, stream, flush, args.steps, args.warmup,
                              args.warm_start_iterations)
        warm["plain_penetration_mm"] = plain_pen
        warm["vs_plain"] = warm["value"] / value
    sweep = None
    if args.warm_start_sweep and world_size == 1:
        its = [int(x) for x in args.warm_start_sweep.split(",")]
        sweep = warm_start_sweep(model, dt, substeps, sched, stream, flush, args.steps, args.warmup, its)
    arm = None
    if not args.no_articulated and world_size == 1:
        arm = articulated_arm(dev, stream, flush, args.steps, args.warmup)
    parts = None
    if not args.no_particles and world_size == 1:
        parts = particles_arm(dev, stream, flush, args.steps, args.warmup)
    del g
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return
    # roofline of the dominant kernel: the XPBD step (the largest single kernel of the launch list; the
    # collide stage is five kernels), with the stages' figures beside it
    algo = algorithmic_bytes(model, pipe.layout, n_contacts)
    per = {"collide": t_col / n_sub, "publish": t_pub / n_sub, "step": t_step / n_sub}
    dom = "step"
    peaks_path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    peak, peak_src = 6650.0, "fallback"
    if os.path.exists(peaks_path):
        peak = float(json.load(open(peaks_path))["hbm_gbs"])
        peak_src = "measured"
    tj = {}
    tpath = os.path.join(ROOT, "profiles", "traffic_per_world_substep.json")
    if os.path.exists(tpath):
        tj = json.load(open(tpath))
    # ncu DRAM bytes per world-substep (a 1024-world capture) scaled to this launch's worlds
    traffic = {k: float(tj[k]) * args.worlds if k in tj else None for k in per}
    stages = {k: {"ms": per[k], "achieved": algo[k] / (per[k] / 1e3) / 1e9,
                  "frac": algo[k] / (per[k] / 1e3) / 1e9 / peak, "algorithmic_bytes": algo[k],
                  "traffic": traffic[k]} for k in per}
    achieved = stages[dom]["achieved"]
    cpu = None
    if not args.no_cpu_baseline and world_size == 1:
        cpu = cpu_baseline(args.seed, args.cpu_sample_seconds, args.worlds)
    # own kernels per substep: broad phase, analytic narrow phase, MPR/GJK
    # prefilter, MPR/GJK, manifolds, world scan, publish, and the XPBD step
    launches_per_frame = substeps * 8
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world_size, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": args.scaling,
        "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded scene generator)",
        "config": {"workload": WORKLOAD, "worlds_per_gpu": model.world_count, "bodies_per_gpu": model.body_count,
                   "substeps": substeps, "iterations": iters, "form": "plain XPBD", "build": args.build,
                   "broad_phase": args.broad_phase,
                   "l2": "256 MiB buffer written before every timed step; the frame's working set (pair "
                         "lists, contact slots and records, body state) is larger than L2",
                   "cuda_graph": True,
                   "frames": f"{FRAMES} of the drop in every step (state reset to frame {WINDOW_START} before it)",
                   "step": f"{WINDOW_FRAMES} frames x {substeps} substeps",
                   "step_schedule": {"mode": sched.mode, "group_threads": sched.group_threads,
                                     "autotune_ms": {f"{m}/{g}": round(v, 4) for (m, g), v in tune_ms.items()}},
                   "mean_contacts_per_substep": int(n_contacts)},
        "roofline": {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "peak_source": peak_src, "traffic": traffic[dom],
                     "algorithmic_bytes_per_launch": algo[dom], "stages": stages},
        "kernel_ms_per_substep": per,
        "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": state_bytes,
                "d2h_bytes_per_step": state_bytes,
                "note": "every step uploads its input body_q / body_qd from pinned host memory and "
                        "downloads the resulting state (the window's 30 frames run in between)"},
        "gpu_launches": launches_per_frame * WINDOW_FRAMES * args.steps,
        "clocks": clk.summary(),
        "status_bits": status, "final_state_finite": finite,
        "max_penetration_m": pen, "max_joint_violation_m": jv,
    }
    if cpu is not None:
        line["cpu_baseline"] = cpu
    if warm is not None:
        line["warm_start"] = warm
    if arm is not None:
        line["articulated"] = arm
    if parts is not None:
        line["particles"] = parts
    if sweep is not None:
        line["warm_start_sweep"] = sweep
    print(json.dumps(line), flush=True)


def main():
    args = parse()
    rank = int(os.environ.get("RANK", "0"))
    world_size = int(os.environ.get("WORLD_SIZE", "1"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference(args, rank)
        return
    run_ours(args, rank, world_size, local_rank)


if __name__ == "__main__":
    main()
