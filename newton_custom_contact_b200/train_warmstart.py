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
from .metrics import contact_penetrations, penetration_stats
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


def _world_residuals(m, c, body_q, world_of_contact):
    """Largest penetration [m] of each world's contacts at poses `body_q` (0 for a world without any)."""
    pen = contact_penetrations(m, c, body_q)
    out = torch.zeros(m.world_count, dtype=torch.float64, device=body_q.device)
    if pen.numel():
        out.scatter_reduce_(0, world_of_contact[:pen.numel()], pen, reduce="amax")
    return out


def judge_check(net: WarmStartNet, device="cuda", worlds: int = 1024, seed: int = 1, iterations: int = 2,
                substeps: int = 120, warmup: int = 48) -> dict:
    """How often the warm start's fallback proxy (a world falls back when the prediction raises its largest
    penetration before the iterations) disagrees with the north-star rule (a world falls back when its
    residual after the iterations -- here its largest penetration at the end of the substep -- is worse
    than the plain solver's).  Every measured substep runs, from the same state and contacts, the plain
    solver (A), the warm start keeping every prediction (B) and the warm start with the proxy (C), and
    follows C.  A world falls back under the proxy when C equals A bit for bit (a rejected prediction
    reproduces the plain step exactly) and under the rule when B's residual exceeds A's; worlds whose
    prediction changes nothing (B equals A) are not counted."""
    dev = torch.device(device)
    m, pipe = make_scene(seed, worlds, dev)
    plain = SolverXPBD(m, iterations=iterations)
    solver = SolverXPBD(m, iterations=iterations)
    ws = WarmStart(net, iterations=iterations)
    a, A, B, Cs = m.state(), m.state(), m.state(), m.state()
    c = pipe.contacts()
    pipe.reset_contact_matching()
    bw = m.body_world.to(dev).long()
    stats = {"worlds_judged": 0, "agree": 0, "proxy_keeps_rule_rejects": 0, "proxy_rejects_rule_keeps": 0,
             "residual_mm": {"plain": 0.0, "proxy": 0.0, "rule": 0.0}}
    n_meas = 0
    for i in range(warmup + substeps):
        a.clear_forces()
        pipe.collide(a, c)
        live = i >= warmup
        if live:
            plain.step(a, A, None, c, DT)
            prev = ws._bufs["prev"].clone() if ws._bufs is not None else None
            ws.judge = "none"
            solver.warm_start = ws
            solver.step(a, B, None, c, DT)
            if prev is not None:
                ws._bufs["prev"].copy_(prev)
            ws.judge = "proxy"
        solver.warm_start = ws
        solver.step(a, Cs, None, c, DT)
        if live:
            wo = c._world_offset
            woc = torch.repeat_interleave(torch.arange(m.world_count, device=dev), (wo[1:] - wo[:-1]).clamp(min=0))
            r_a = _world_residuals(m, c, A.body_q, woc)
            r_b = _world_residuals(m, c, B.body_q, woc)
            r_c = _world_residuals(m, c, Cs.body_q, woc)

            def world_all(eq):
                out = torch.ones(m.world_count, dtype=torch.int32, device=dev)
                return out.scatter_reduce(0, bw, eq.to(torch.int32), reduce="amin") == 1

            same_ab = world_all((A.body_q == B.body_q).all(1) & (A.body_qd == B.body_qd).all(1))
            same_ac = world_all((A.body_q == Cs.body_q).all(1) & (A.body_qd == Cs.body_qd).all(1))
            judged = ~same_ab
            proxy_fb = same_ac & judged
            rule_fb = (r_b > r_a) & judged
            stats["worlds_judged"] += int(judged.sum())
            stats["agree"] += int((judged & (proxy_fb == rule_fb)).sum())
            stats["proxy_keeps_rule_rejects"] += int((judged & ~proxy_fb & rule_fb).sum())
            stats["proxy_rejects_rule_keeps"] += int((judged & proxy_fb & ~rule_fb).sum())
            r_rule = torch.where(rule_fb, r_a, r_b)
            for k, r in (("plain", r_a), ("proxy", r_c), ("rule", r_rule)):
                stats["residual_mm"][k] += float(r.max()) * 1e3
            n_meas += 1
        a, Cs = Cs, a
    for k in stats["residual_mm"]:
        stats["residual_mm"][k] /= max(n_meas, 1)
    stats["agree_fraction"] = stats["agree"] / max(stats["worlds_judged"], 1)
    stats["iterations"] = iterations
    stats["substeps"] = substeps
    return stats


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
    ap.add_argument("--judge-check", action="store_true",
                    help="also measure how often the fallback proxy disagrees with the residual rule")
    ap.add_argument("--profile-arm", default=None, metavar="plain|warm",
                    help="only run one arm (--student-iterations iterations, warm: the network at --out) for "
                         "--profile-substeps substeps after 64 warm-up substeps, for a profiler's launch list")
    ap.add_argument("--profile-substeps", type=int, default=16)
    a = ap.parse_args()
    set_scene(a.scene)
    if a.profile_arm is not None:
        if a.out is None:
            a.out = os.path.join(os.path.dirname(__file__), "data", f"warmstart_{a.scene}.npz")
        m, pipe = make_scene(a.eval_seed if a.eval_seed is not None else 1, a.worlds, torch.device("cuda"))
        pol = WarmStart(WarmStartNet.load(a.out), iterations=a.student_iterations) if a.profile_arm == "warm" else None
        rollout(m, pipe, a.student_iterations, a.profile_substeps, policy=pol, warmup=64, measure=False)
        torch.cuda.synchronize()
        return
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
    if a.judge_check:
        res["judge"] = judge_check(net, worlds=a.worlds, seed=eval_seed, iterations=a.student_iterations)
    print(json.dumps(res, indent=1))
    if a.report:
        with open(a.report, "w") as f:
            json.dump(res, f, indent=1)


if __name__ == "__main__":
    main()
