"""Benchmark: world-substeps/s of the rigid-contact XPBD step (collide + SolverXPBD.step).

Workload: 4096 uneven worlds of box / sphere / capsule bodies (N ~ U{8..128}),
dt = 1/60 s, 8 substeps, 8 iterations, FP32, seeded synthetic scene.  One
benchmark step = one frame = 8 x (State.clear_forces, CollisionPipeline.collide,
SolverXPBD.step), captured once as a CUDA graph and replayed.

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


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=40)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--worlds", type=int, default=4096)
    ap.add_argument("--seed", type=int, default=1)
    ap.add_argument("--cpu-sample-seconds", type=float, default=12.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
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
def cpu_baseline(seed: int, seconds: float, worlds_total: int):
    """Oracle (sequential C++ restatement, OpenMP over worlds) on a bounded sample of the C2 workload."""
    import oracle
    from newton_custom_contact_b200 import SolverXPBD, scenes
    from newton_custom_contact_b200.collide import PairLayout

    oracle.build()
    sample_worlds = 256
    model, info = scenes.scene_c2(seed=seed, worlds=sample_worlds, device="cpu")
    lay = PairLayout(model, model.host("shape_contact_pairs"))
    p = SolverXPBD(model, iterations=info["iterations"]).params()
    dt = info["dt"] / info["substeps"]
    q, qd = model.host("body_q").copy(), model.host("body_qd").copy()
    f = np.zeros((model.body_count, 6), np.float32)
    substeps = 0
    t0 = time.perf_counter()
    while True:
        for _ in range(info["substeps"]):
            segs = oracle.collide(model, lay, q)
            q, qd, _ = oracle.step(model, lay, p, q, qd, f, segs, dt)
            substeps += 1
        el = time.perf_counter() - t0
        if el >= seconds:
            break
    cores = int(os.environ.get("OMP_NUM_THREADS", os.cpu_count() or 1))
    value = sample_worlds * substeps / el
    return {"value": value, "unit": UNIT, "cores": cores, "kind": "port",
            "sample": f"{sample_worlds} worlds of the same C2 generator, {substeps} substeps (collide + step), "
                      f"{el:.1f} s, OpenMP over worlds"}


# ---------------------------------------------------------------- reference arm
def run_reference(args, rank):
    if rank != 0:
        return
    res = cpu_baseline(args.seed, max(2.0, args.cpu_sample_seconds / 2), args.worlds)
    line = {"impl": "reference", "metric": METRIC, "value": res["value"], "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * args.worlds * 8 / res["value"],
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded)", "config": {"workload": WORKLOAD, "worlds": args.worlds},
            "cpu_baseline": res,
            "e2e": {"value": res["value"], "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "note": "warp-lang (the reference's runtime) is not installable here; the reference arm times the "
                    "CPU restatement of the reference kernels (oracle/) on the host cores"}
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------- ours
def algorithmic_bytes(model, layout, n_contacts: float):
    """Bytes one collide and one step launch must move (per substep, all worlds)."""
    B = model.body_count
    S = model.shape_count
    P = layout.pair_count
    step = B * (7 * 4 + 6 * 4 + 6 * 4 + 4 + 12 + 36 + 36 + 4 + 4) + B * (7 * 4 + 6 * 4) + n_contacts * 80
    collide = S * 44 + B * 28 + P * 8 + n_contacts * 80
    publish = n_contacts * (80 + 76)
    return {"step": step, "collide": collide, "publish": publish}


def run_ours(args, rank, world_size, local_rank):
    import torch

    from newton_custom_contact_b200 import CollisionPipeline, SolverXPBD, scenes

    dev = torch.device("cuda", local_rank)
    torch.cuda.set_device(dev)
    dist = None
    if world_size > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    model, info = scenes.scene_c2(seed=args.seed + 1000 * rank, worlds=args.worlds, device=dev)
    substeps, iters = info["substeps"], info["iterations"]
    dt = info["dt"] / substeps
    pipe = CollisionPipeline(model)
    solver = SolverXPBD(model, iterations=iters)
    s0, s1 = model.state(), model.state()
    contacts = pipe.contacts()
    stream = torch.cuda.Stream(dev)

    def frame():
        a, b = s0, s1
        for _ in range(substeps):
            a.clear_forces()
            pipe.collide(a, contacts)
            solver.step(a, b, None, contacts, dt)
            a, b = b, a

    # eager warm-up (also loads the library, sets kernel attributes)
    with torch.cuda.stream(stream):
        frame()
    torch.cuda.synchronize()
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g, stream=stream):
        frame()
    torch.cuda.synchronize()
    flush = torch.empty(int(256 * 2**20) // 4, dtype=torch.float32, device=dev)
    for _ in range(args.warmup):
        g.replay()
    torch.cuda.synchronize()
    # per-kernel timing pass (eager, same kernels) for the roofline
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(4)]
    t_col = t_pub = t_step = 0.0
    with torch.cuda.stream(stream):
        a, b = s0, s1
        import ctypes as C

        from newton_custom_contact_b200 import _lib
        lib = _lib.load()
        for _ in range(substeps):
            a.clear_forces()
            desc = pipe.desc()
            seg = pipe.seg_struct(contacts)
            h = _lib.stream_handle(dev)
            ev[0].record(stream)
            _lib.check("nb_collide", lib.nb_collide(C.byref(desc), C.c_void_p(a.body_q.data_ptr()), C.byref(seg),
                                                    0, C.c_void_p(h)))
            ev[1].record(stream)
            pub = pipe.public_struct(contacts)
            _lib.check("nb_publish_contacts", lib.nb_publish_contacts(C.byref(desc), C.byref(seg), C.byref(pub),
                                                                      C.c_void_p(h)))
            ev[2].record(stream)
            contacts._seg_valid = True
            solver.step(a, b, None, contacts, dt)
            ev[3].record(stream)
            stream.synchronize()
            t_col += ev[0].elapsed_time(ev[1])
            t_pub += ev[1].elapsed_time(ev[2])
            t_step += ev[2].elapsed_time(ev[3])
            a, b = b, a
    torch.cuda.synchronize()
    n_contacts = float(contacts._seg["world_count"].sum().item())
    n_candidates = float(contacts._seg["cand_count"].sum().item())
    # timed region: K graph replays, L2 flushed between them (outside the events)
    starts = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    with ClockSampler(local_rank) as clk:
        with torch.cuda.stream(stream):
            for k in range(args.steps):
                flush.fill_(float(k))
                starts[k].record(stream)
                g.replay()
                ends[k].record(stream)
        torch.cuda.synchronize()
    ms = sum(starts[k].elapsed_time(ends[k]) for k in range(args.steps))
    if dist:
        t = torch.tensor([ms], device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
        dist.barrier()
    units = args.worlds * substeps * args.steps * world_size
    value = units / (ms / 1e3)
    # e2e through the public API with host buffers
    # the host owns the state between steps: each step uploads body_q / body_qd
    # from pinned memory and downloads the new ones (the trajectory continues)
    hq = torch.empty(s0.body_q.shape, dtype=torch.float32).pin_memory()
    hqd = torch.empty(s0.body_qd.shape, dtype=torch.float32).pin_memory()
    hq.copy_(s0.body_q.cpu())
    hqd.copy_(s0.body_qd.cpu())
    e_s = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    e_e = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    with torch.cuda.stream(stream):
        for k in range(args.steps):
            flush.fill_(float(k))
            e_s[k].record(stream)
            s0.body_q.copy_(hq, non_blocking=True)
            s0.body_qd.copy_(hqd, non_blocking=True)
            g.replay()
            hq.copy_(s0.body_q, non_blocking=True)
            hqd.copy_(s0.body_qd, non_blocking=True)
            e_e[k].record(stream)
    torch.cuda.synchronize()
    e2e_ms = sum(e_s[k].elapsed_time(e_e[k]) for k in range(args.steps))
    if dist:
        t = torch.tensor([e2e_ms], device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_ms = float(t.item())
    e2e_value = units / (e2e_ms / 1e3)
    status = pipe.status(contacts)
    q = s0.body_q
    finite = bool(torch.isfinite(q).all().item())
    del g
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return
    # roofline of the dominant kernel
    algo = algorithmic_bytes(model, pipe.layout, n_contacts)
    per = {"collide": t_col / substeps, "publish": t_pub / substeps, "step": t_step / substeps}
    dom = max(per, key=per.get)
    peaks_path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    peak, peak_src = 6650.0, "fallback"
    if os.path.exists(peaks_path):
        peak = float(json.load(open(peaks_path))["hbm_gbs"])
        peak_src = "measured"
    achieved = algo[dom] / (per[dom] / 1e3) / 1e9
    traffic = None
    tpath = os.path.join(ROOT, "profiles", "traffic_per_world_substep.json")
    if os.path.exists(tpath):
        tj = json.load(open(tpath))
        if dom in tj:
            traffic = float(tj[dom]) * args.worlds
    cpu = None
    if not args.no_cpu_baseline and world_size == 1:
        cpu = cpu_baseline(args.seed, args.cpu_sample_seconds, args.worlds)
    launches_per_frame = substeps * 4  # collide, world scan, publish, step
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world_size, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded scene generator)",
        "config": {"workload": WORKLOAD, "worlds_per_gpu": args.worlds, "bodies_per_gpu": model.body_count,
                   "substeps": substeps, "iterations": iters, "form": "plain XPBD",
                   "l2": "256 MiB buffer written between timed steps", "cuda_graph": True,
                   "contacts_last_substep": int(n_contacts)},
        "roofline": {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "peak_source": peak_src, "traffic": traffic,
                     "algorithmic_bytes_per_launch": algo[dom]},
        "kernel_ms_per_substep": per,
        "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": int(hq.numel() * 4 + hqd.numel() * 4),
                "d2h_bytes_per_step": int(hq.numel() * 4 + hqd.numel() * 4)},
        "gpu_launches": launches_per_frame * args.steps,
        "clocks": clk.summary(),
        "status_bits": status, "final_state_finite": finite,
    }
    if cpu is not None:
        line["cpu_baseline"] = cpu
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
