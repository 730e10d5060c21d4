"""Train the learned warm start on the uneven-worlds scene and evaluate its gain.

    python -m newton_custom_contact_b200.train_warmstart [--scene c2|c5]

Samples are (features, lambda) pairs of the plain solver with the teacher's
iteration count: first along plain rollouts, then (DAgger rounds) at the
states the warm-started solver itself visits, so that the network sees the
states it will be used on.  The previous-lambda feature always comes from the
rollout that is being followed.  Training runs the library's own kernels
(nb_ws_grads, nb_ws_adam); evaluation compares, substep by substep over the
same window, the largest penetration and the substep time of the plain solver
at the teacher's and at the student's iteration count with the warm-started
student.
"""

from __future__ import annotations

import argparse
import json
import os
import time

import numpy as np
import torch

from . import CollisionPipeline, SolverXPBD, scenes
from .metrics import penetration_stats
from .warmstart import WarmStart, WarmStartNet, corrections

DT = 1.0 / 480.0
SCENE = "c2"  # "c2": uneven worlds of boxes / spheres / capsules; "c5": 16-box stacks (dt 1/600);
              # "c1": C1's 64-box worlds, one seed per world (dt 1/600)


def set_scene(kind: str) -> None:
    """Scene family the training / evaluation helpers build (and its substep)."""
    global SCENE, DT
    if kind not in ("c1", "c2", "c5"):
        raise ValueError("scene must be 'c1', 'c2' or 'c5'")
    SCENE = kind
    DT = 1.0 / 480.0 if kind == "c2" else 1.0 / 600.0


def make_scene(seed: int, worlds: int, device):
    if SCENE == "c5":
        m, _ = scenes.scene_c5(seed=seed, worlds=worlds, device=device)
    elif SCENE == "c1":
        # C1 seeds: training from 100 on, evaluation from 100000 on (unseen)
        m, _ = scenes.scene_c1_batch(seed=seed, worlds=worlds, device=device)
    else:
        m, _ = scenes.scene_c2(seed=seed, worlds=worlds, device=device)
    pipe = CollisionPipeline(m, contact_matching="latest")
    return m, pipe


def rollout(m, pipe, iterations: int, substeps: int, policy: WarmStart | None = None,
            teacher_iterations: int | None = None, recorder: WarmStart | None = None, warmup: int = 0,
            measure: bool = True):
    """Advance the scene `warmup + substeps` substeps with `iterations` (and `policy`, if given).
    With a recorder, each recorded substep also runs the teacher (plain, teacher_iterations) from the
    same state into a scratch state and records its samples, with the previous-lambda feature of the
    rollout.  Returns per-substep (max penetration after the step, step ms) when `measure`."""
    solver = SolverXPBD(m, iterations=iterations)
    teacher = SolverXPBD(m, iterations=teacher_iterations or iterations)
    a, b, scratch = m.state(), m.state(), m.state()
    c = pipe.contacts()
    pipe.reset_contact_matching()
    pens, times = [], []
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    for i in range(warmup + substeps):
        a.clear_forces()
        pipe.collide(a, c)
        live = i >= warmup
        if live and recorder is not None:
            if policy is not None and policy._bufs is not None:
                recorder._alloc(m, c)
                recorder._bufs["prev"] = policy._bufs["prev"]  # the followed rollout's lambdas
            recorder.update_prev = policy is None
            teacher.warm_start = recorder
            teacher.step(a, scratch, None, c, DT)
            teacher.warm_start = None
        solver.warm_start = policy
        if measure and live:
            ev0.record()
        solver.step(a, b, None, c, DT)
        if measure and live:
            ev1.record()
            torch.cuda.synchronize()
            times.append(ev0.elapsed_time(ev1))
            pens.append(penetration_stats(m, c, b.body_q))
        a, b = b, a
    return pens, np.array(times)


def collect(m, pipe, teacher_iterations: int, substeps: int, warmup: int, fraction: float,
            policy: WarmStart | None = None, student_iterations: int = 2, seed: int = 0):
    rec = WarmStart(None, iterations=None, record=True, record_fraction=fraction, seed=seed)
    rollout(m, pipe, student_iterations if policy is not None else teacher_iterations, substeps, policy=policy,
            teacher_iterations=teacher_iterations, recorder=rec, warmup=warmup, measure=False)
    return rec.samples()


def r2_scores(net: WarmStartNet, x: torch.Tensor, t: torch.Tensor) -> list[float]:
    """Coefficient of determination per output (normal, tangent 1, tangent 2) of nb_ws_infer's predicted
    corrections c = lambda * w against the samples' (features x, lambdas t)."""
    out = torch.empty_like(t)
    status = torch.zeros(1, dtype=torch.int32, device=x.device)
    net.infer(x, torch.tensor([x.shape[0]], dtype=torch.int32, device=x.device), out, status)
    c, ct = corrections(x, out), corrections(x, t)
    res = ((c - ct) ** 2).sum(0)
    tot = ((ct - ct.mean(0)) ** 2).sum(0).clamp_min(1e-30)
    return [float(v) for v in (1.0 - res / tot)]


def train(device="cuda", worlds: int = 1024, seed: int = 2, teacher_iterations: int = 8,
          student_iterations: int = 2, substeps: int = 240, warmup: int = 48, fraction: float = 0.1,
          dagger_rounds: int = 1, epochs: int = 20, batch: int = 2048, log=print) -> tuple[WarmStartNet, dict]:
    dev = torch.device(device)
    m, pipe = make_scene(seed, worlds, dev)
    x, t = collect(m, pipe, teacher_iterations, substeps, warmup, fraction, seed=seed)
    log(f"plain rollout: {x.shape[0]} samples")
    net = WarmStartNet(device=dev, seed=seed)
    net.fit(x, t, epochs=epochs, batch=batch, log=log)
    info = {"samples": [int(x.shape[0])], "fallbacks": []}
    for r in range(dagger_rounds):
        pol = WarmStart(net, iterations=student_iterations)
        xr, tr = collect(m, pipe, teacher_iterations, substeps, warmup, fraction, policy=pol,
                         student_iterations=student_iterations, seed=seed + r + 1)
        log(f"DAgger round {r}: {xr.shape[0]} samples, fallbacks {pol.fallback_count}")
        info["samples"].append(int(xr.shape[0]))
        info["fallbacks"].append(pol.fallback_count)
        x, t = torch.cat([x, xr]), torch.cat([t, tr])
        net = WarmStartNet(device=dev, seed=seed)
        net.fit(x, t, epochs=epochs, batch=batch, log=log)
    info["train_r2"] = r2_scores(net, x[:200000], t[:200000])
    return net, info


def timed_frames(m, pipe, iterations: int, policy: WarmStart | None, warmup: int, frames: int,
                 substeps_per_frame: int = 8) -> float:
    """Median ms per substep (collide + step, warm start included) over `frames` replays of a CUDA graph
    of one frame, after `warmup` eager substeps."""
    solver = SolverXPBD(m, iterations=iterations)
    solver.warm_start = policy
    s0, s1 = m.state(), m.state()
    c = pipe.contacts()
    pipe.reset_contact_matching()
    stream = torch.cuda.Stream()
    # the contacts' buffers were allocated (and zero-filled) on the default stream
    stream.wait_stream(torch.cuda.current_stream())

    def frame():
        a, b = s0, s1
        for _ in range(substeps_per_frame):
            a.clear_forces()
            pipe.collide(a, c)
            solver.step(a, b, None, c, DT)
            a, b = b, a

    with torch.cuda.stream(stream):
        for _ in range(max(warmup // substeps_per_frame, 1)):
            frame()
    torch.cuda.synchronize()
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g, stream=stream):
        frame()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(frames)]
    with torch.cuda.stream(stream):
        for e0, e1 in ev:
            e0.record(stream)
            g.replay()
            e1.record(stream)
    torch.cuda.synchronize()
    ms = sorted(e0.elapsed_time(e1) for e0, e1 in ev)
    del g
    return ms[len(ms) // 2] / substeps_per_frame


def evaluate(net: WarmStartNet, device="cuda", worlds: int = 1024, seed: int = 1, teacher_iterations: int = 8,
             student_iterations=(2, 4), gains=((1.0, 1.0), (1.0, 0.0), (0.8, 0.5)), substeps: int = 240,
             warmup: int = 48) -> dict:
    """Penetration after each substep over the window (largest over all contacts, 99th percentile, mean
    and sum over the live contacts; each averaged over the substeps) and the substep time, for the plain
    solver (teacher and student iteration counts) and the warm-started student(s)."""
    dev = torch.device(device)
    m, pipe = make_scene(seed, worlds, dev)
    cfgs = [("plain", teacher_iterations, None)] + [("plain", k, None) for k in student_iterations]
    cfgs += [("warm", k, gn) for k in student_iterations for gn in gains]
    out = {}
    for kind, iters, gain in cfgs:
        pol = WarmStart(net, iterations=iters, gain=gain) if kind == "warm" else None
        pens, _ = rollout(m, pipe, iters, substeps, policy=pol, warmup=warmup)
        fb = pol.fallback_count if pol is not None else 0
        tpol = WarmStart(net, iterations=iters, gain=gain) if kind == "warm" else None
        ms = timed_frames(m, pipe, iters, tpol, warmup, frames=substeps // 8)
        name = f"{kind}_{iters}" + (f"_g{gain[0]}_{gain[1]}" if gain is not None else "")
        row = {"iterations": iters, "gain": gain, "substep_ms": ms,
               "fallback_rate": fb / float(worlds * (warmup + substeps))}
        for k in ("max", "p99", "mean", "sum"):
            v = np.array([p[k] for p in pens])
            row[f"{k}_pen_mm"] = float(np.nanmean(v) * 1e3)
        row["worst_pen_mm"] = float(np.nanmax([p["max"] for p in pens]) * 1e3)
        out[name] = row
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--scene", default="c2", choices=["c1", "c2", "c5"])
    ap.add_argument("--out", default=None, help="network file (default: data/warmstart_<scene>.npz)")
    ap.add_argument("--train-seed", type=int, default=None)
    ap.add_argument("--eval-seed", type=int, default=None)
    ap.add_argument("--worlds", type=int, default=1024)
    ap.add_argument("--substeps", type=int, default=240)
    ap.add_argument("--dagger", type=int, default=1)
    ap.add_argument("--epochs", type=int, default=20)
    ap.add_argument("--fraction", type=float, default=0.1)
    ap.add_argument("--student-iterations", type=int, default=2)
    ap.add_argument("--report", default=None)
    ap.add_argument("--eval-only", action="store_true", help="evaluate the network saved at --out")
    a = ap.parse_args()
    set_scene(a.scene)
    if a.out is None:
        a.out = os.path.join(os.path.dirname(__file__), "data", f"warmstart_{a.scene}.npz")
    # training and evaluation scenes differ (unseen seed at evaluation)
    train_seed = a.train_seed if a.train_seed is not None else {"c1": 100, "c2": 2, "c5": 6}[a.scene]
    eval_seed = a.eval_seed if a.eval_seed is not None else {"c1": 100000, "c2": 1, "c5": 5}[a.scene]
    t0 = time.time()
    if a.eval_only:
        net = WarmStartNet.load(a.out)
        res = {}
    else:
        net, info = train(worlds=a.worlds, seed=train_seed, substeps=a.substeps, dagger_rounds=a.dagger,
                          epochs=a.epochs, student_iterations=a.student_iterations, fraction=a.fraction)
        os.makedirs(os.path.dirname(a.out), exist_ok=True)
        net.save(a.out)
        res = {"train": info, "train_s": time.time() - t0}
    res["scene"] = a.scene
    res["eval"] = evaluate(net, worlds=a.worlds, seed=eval_seed, student_iterations=(a.student_iterations, 4))
    print(json.dumps(res, indent=1))
    if a.report:
        with open(a.report, "w") as f:
            json.dump(res, f, indent=1)


if __name__ == "__main__":
    main()
