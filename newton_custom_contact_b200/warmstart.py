"""Learned warm start of the XPBD contact solve (no counterpart in the reference).

A small network predicts, for every contact of a substep, the impulse the
plain solver would end up applying to it -- the weighted, accumulated
per-contact impulse that ``SolverXPBD.update_contacts`` reports
(newton/_src/solvers/xpbd/kernels.py:2301-2393), expressed in the contact
frame (normal, two tangents).  The step applies the predictions to the
bodies before its (fewer) plain iterations, which then correct whatever the
network got wrong; a world whose largest penetration the warm start makes
worse falls back to no warm start (the solver restores its state).

Network: BF16 MLP 24 -> 128 -> 128 -> 3 with SiLU and FP32 accumulation,
predicting the ratio y of the contact's velocity correction c = lambda * w
(w: generalised inverse mass) to a physical prior -- the previous substep's
correction of the matched contact, else the velocity that removes the depth
expected after the integration; lambda_n >= 0 and the tangential part is
kept inside the friction cone --
evaluated by the tensor-core kernel ``nb_ws_infer`` (tcgen05); trained by the
library's own forward / backward / Adam kernels (``nb_ws_grads``,
``nb_ws_adam``) on (features, lambda) samples collected from plain-solver
rollouts (train_warmstart.py).  Features (``nb_ws_features``): a matched
flag, ratios to the prior of the depth estimate, of the previous correction
(normal, tangents), of the relative velocity, depth, gravity and thickness;
normal, inverse-mass shares, friction, contacts per body, log2 prior,
direction to the other body, which side is static.
"""

from __future__ import annotations

import ctypes as C

import numpy as np
import torch

from . import _lib
from ._abi import NB_WS_KEEP_ALL, NbWsNet, NbWsTrain, ptr

N_IN, N_HID, N_OUT = 24, 128, 3
N_FEAT = 27  # network inputs + generalised inverse masses (normal, tangents) + prior
COL_WN, COL_WT, COL_PRIOR, COL_MU = 24, 25, 26, 17


def corrections(features: torch.Tensor, lam: torch.Tensor) -> torch.Tensor:
    """Velocity corrections c = lambda * w (w: the contact's generalised inverse mass along the normal /
    the tangents)."""
    w = features[:, [COL_WN, COL_WT, COL_WT]]
    return (lam * w).contiguous()


def ratio_targets(features: torch.Tensor, lam: torch.Tensor) -> tuple[torch.Tensor, torch.Tensor]:
    """(network inputs, targets y = c / prior) of the rows that have a prior; y_n in [0, 10], y_t in
    [-10, 10]."""
    keep = features[:, COL_PRIOR] > 0
    f, c = features[keep], corrections(features[keep], lam[keep])
    y = c / f[:, COL_PRIOR:COL_PRIOR + 1]
    y = torch.stack([y[:, 0].clamp(0.0, 10.0), y[:, 1].clamp(-10.0, 10.0), y[:, 2].clamp(-10.0, 10.0)], 1)
    return f[:, :N_IN].contiguous(), y.contiguous()


def moments(x: torch.Tensor, group=None) -> tuple[torch.Tensor, torch.Tensor]:
    """Per-column mean and standard deviation (unbiased) of x [R, C]; with a process group, of the
    rows of every rank (sums all-reduced in float64)."""
    s = torch.stack([torch.full((x.shape[1],), float(x.shape[0]), dtype=torch.float64, device=x.device),
                     x.double().sum(0), (x.double() ** 2).sum(0)])
    if group is not None:
        import torch.distributed as dist

        dist.all_reduce(s, op=dist.ReduceOp.SUM, group=group)
    n, sx, sxx = s[0], s[1], s[2]
    mean = sx / n
    var = (sxx - n * mean * mean) / (n - 1).clamp_min(1.0)
    return mean.float(), var.clamp_min(0.0).sqrt().float()


def allreduce_mean(grads: dict, group) -> None:
    """Average gradient tensors over the ranks of `group`, in place (one flat all-reduce)."""
    import torch.distributed as dist

    keys = sorted(grads)
    flat = torch.cat([grads[k].reshape(-1) for k in keys])
    dist.all_reduce(flat, op=dist.ReduceOp.SUM, group=group)
    flat /= dist.get_world_size(group)
    o = 0
    for k in keys:
        n = grads[k].numel()
        grads[k].copy_(flat[o:o + n].view_as(grads[k]))
        o += n


def _bf16_bits(t: torch.Tensor) -> torch.Tensor:
    return t.to(torch.bfloat16).view(torch.int16).contiguous()


class WarmStartNet:
    """FP32 master weights + normalisation, and their packed BF16 copy for inference."""

    def __init__(self, device="cuda", seed: int = 0):
        dev = torch.device(device)
        g = torch.Generator().manual_seed(seed)

        def init(o, i):
            return (torch.randn(o, i, generator=g) * (1.0 / np.sqrt(i))).to(dev)

        self.params = {
            "w1": init(N_HID, N_IN), "b1": torch.zeros(N_HID, device=dev),
            "w2": init(N_HID, N_HID), "b2": torch.zeros(N_HID, device=dev),
            "w3": init(N_OUT, N_HID) * 0.1, "b3": torch.zeros(N_OUT, device=dev),
        }
        self.in_mean = torch.zeros(N_IN, device=dev)
        self.in_inv_std = torch.ones(N_IN, device=dev)
        self.out_scale = torch.ones(N_OUT, device=dev)
        self.device = dev
        self._packed = None

    # ------------------------------------------------------------ inference layout
    def packed(self) -> dict:
        if self._packed is None:
            p = self.params
            w1 = torch.zeros(N_HID, 32, device=self.device)
            w1[:, :N_IN] = p["w1"]
            w3 = torch.zeros(16, N_HID, device=self.device)
            w3[:N_OUT] = p["w3"]
            b3 = torch.zeros(16, device=self.device)
            b3[:N_OUT] = p["b3"]
            self._packed = {"w1": _bf16_bits(w1), "b1": p["b1"].contiguous(), "w2": _bf16_bits(p["w2"]),
                            "b2": p["b2"].contiguous(), "w3": _bf16_bits(w3), "b3": b3,
                            "in_mean": self.in_mean.contiguous(), "in_inv_std": self.in_inv_std.contiguous(),
                            "out_scale": self.out_scale.contiguous()}
        return self._packed

    def struct(self, gain=1.0) -> NbWsNet:
        """Inference arguments; `gain` (scalar or (normal, tangent)) scales the predictions."""
        pk = self.packed()
        g = (float(gain), float(gain)) if np.isscalar(gain) else (float(gain[0]), float(gain[1]))
        if g != (1.0, 1.0):
            key = ("out_scale", g)
            if key not in pk:
                pk[key] = (pk["out_scale"] * torch.tensor([g[0], g[1], g[1]], device=self.device)).contiguous()
            osc = pk[key]
        else:
            osc = pk["out_scale"]
        s = NbWsNet()
        for k in ("w1", "b1", "w2", "b2", "w3", "b3", "in_mean", "in_inv_std"):
            setattr(s, k, ptr(pk[k]))
        s.out_scale = ptr(osc)
        s._keep = pk
        return s

    def infer(self, features: torch.Tensor, count: torch.Tensor, out: torch.Tensor, status: torch.Tensor,
              gain=1.0) -> None:
        """gain x lambda[i] for i < min(count, len(features)) on the tensor cores (nb_ws_infer);
        features [cap, 27] as written by nb_ws_features."""
        if features.shape[1] != N_FEAT:
            raise ValueError(f"features must have {N_FEAT} columns")
        lib = _lib.load()
        net = self.struct(gain)
        _lib.check("nb_ws_infer", lib.nb_ws_infer(C.byref(net), C.c_void_p(ptr(features)), C.c_void_p(ptr(count)),
                                                  int(features.shape[0]), C.c_void_p(ptr(out)),
                                                  C.c_void_p(ptr(status)), C.c_void_p(_lib.stream_handle(self.device))))

    # ------------------------------------------------------------ training
    def set_normalisation(self, x: torch.Tensor, t: torch.Tensor, group=None) -> None:
        """Input mean / inverse std and output scale of the samples (over every rank's shard with a
        process group)."""
        (xm, xs), (_, ts) = moments(x, group), moments(t, group)
        self.in_mean = xm.contiguous()
        self.in_inv_std = 1.0 / torch.maximum(xs, 1e-4 + 1e-3 * xm.abs())
        self.out_scale = ts.clamp_min(1e-8).contiguous()
        self._packed = None

    def grads(self, x: torch.Tensor, t: torch.Tensor) -> tuple[dict, float]:
        """Gradients of the mean squared error of the normalised outputs on (network inputs x [R, 24],
        targets t [R, 3]), and the loss."""
        lib = _lib.load()
        R = int(x.shape[0])
        dev = self.device
        f = dict(dtype=torch.float32, device=dev)
        p = self.params
        g = {k: torch.empty_like(v) for k, v in p.items()}
        buf = {"xn": torch.empty(R, N_IN, **f), "z1": torch.empty(R, N_HID, **f), "h1": torch.empty(R, N_HID, **f),
               "z2": torch.empty(R, N_HID, **f), "h2": torch.empty(R, N_HID, **f), "y": torch.empty(R, N_OUT, **f),
               "dy": torch.empty(R, N_OUT, **f), "dh": torch.empty(R, N_HID, **f), "dh2": torch.empty(R, N_HID, **f),
               "scratch_wq": torch.empty(N_HID * N_IN + N_HID * N_HID + N_OUT * N_HID, **f),
               "loss": torch.zeros(1, **f), "status": torch.zeros(1, dtype=torch.int32, device=dev)}
        a = NbWsTrain()
        a.rows = R
        a.x, a.t = ptr(x.contiguous()), ptr(t.contiguous())
        a.in_mean, a.in_inv_std, a.out_scale = ptr(self.in_mean), ptr(self.in_inv_std), ptr(self.out_scale)
        for k in p:
            setattr(a, k, ptr(p[k]))
            setattr(a, "g_" + k, ptr(g[k]))
        for k, v in buf.items():
            setattr(a, k, ptr(v))
        _lib.check("nb_ws_grads", lib.nb_ws_grads(C.byref(a), C.c_void_p(_lib.stream_handle(dev))))
        if int(buf["status"].item()):
            raise RuntimeError("nb_ws_grads: a tensor-core wait timed out")
        return g, float(buf["loss"].item())

    def fit(self, features: torch.Tensor, lam: torch.Tensor, epochs: int = 30, batch: int = 4096,
            lr: float = 2e-3, weight_decay: float = 1e-5, seed: int = 0, log=None, group=None) -> list[float]:
        """Adam on minibatches (nb_ws_grads + nb_ws_adam) of (features [R, 27], lambda [R, 3]) samples,
        regressing the ratios y = lambda * w / prior of the rows with a prior; normalisation from the
        data.  With a torch.distributed process group every rank holds its own shard of the samples
        (the same number of minibatches per epoch on every rank) and the gradients are averaged over
        the ranks before each update (data parallel; NCCL over NVLink on GPUs)."""
        lib = _lib.load()
        x, t = ratio_targets(features, lam)
        batch = max(1, min(batch, x.shape[0]))
        self.set_normalisation(x, t, group)
        n_batches = x.shape[0] // batch
        if group is not None:
            import torch.distributed as dist

            nbt = torch.tensor([n_batches], device=x.device)
            dist.all_reduce(nbt, op=dist.ReduceOp.MIN, group=group)
            n_batches = int(nbt.item())
        m1 = {k: torch.zeros_like(v) for k, v in self.params.items()}
        m2 = {k: torch.zeros_like(v) for k, v in self.params.items()}
        gen = torch.Generator(device=x.device).manual_seed(seed)
        step, losses = 0, []
        stream = C.c_void_p(_lib.stream_handle(self.device))
        for ep in range(epochs):
            perm = torch.randperm(x.shape[0], generator=gen, device=x.device)
            tot, nb = 0.0, 0
            for bi in range(n_batches):
                idx = perm[bi * batch:(bi + 1) * batch]
                g, loss = self.grads(x[idx], t[idx])
                if group is not None:
                    allreduce_mean(g, group)
                step += 1
                cur_lr = lr * 0.5 * (1.0 + np.cos(np.pi * ep / max(epochs, 1)))
                for k, w in self.params.items():
                    _lib.check("nb_ws_adam", lib.nb_ws_adam(C.c_void_p(ptr(w)), C.c_void_p(ptr(g[k])),
                                                            C.c_void_p(ptr(m1[k])), C.c_void_p(ptr(m2[k])),
                                                            w.numel(), cur_lr, 0.9, 0.999, 1e-8, weight_decay, step,
                                                            stream))
                tot += loss
                nb += 1
            losses.append(tot / max(nb, 1))
            if log:
                log(f"epoch {ep}: loss {losses[-1]:.5f}")
        self._packed = None
        return losses

    # ------------------------------------------------------------ persistence
    def save(self, path: str) -> None:
        arrs = {k: v.detach().cpu().numpy() for k, v in self.params.items()}
        arrs.update(in_mean=self.in_mean.cpu().numpy(), in_inv_std=self.in_inv_std.cpu().numpy(),
                    out_scale=self.out_scale.cpu().numpy())
        np.savez(path, **arrs)

    @classmethod
    def load(cls, path: str, device="cuda") -> "WarmStartNet":
        d = np.load(path)
        net = cls(device=device)
        dev = torch.device(device)
        for k in net.params:
            net.params[k] = torch.from_numpy(d[k]).to(dev)
        net.in_mean = torch.from_numpy(d["in_mean"]).to(dev)
        net.in_inv_std = torch.from_numpy(d["in_inv_std"]).to(dev)
        net.out_scale = torch.from_numpy(d["out_scale"]).to(dev)
        return net


class WarmStart:
    """Per-solver warm-start state: set ``solver.warm_start = WarmStart(net, iterations=2)``.

    Each ``solver.step`` with contacts then computes the features of the
    published contacts from ``state_in``, runs the network, applies its
    predictions before ``iterations`` plain iterations (instead of the
    solver's own count) and keeps this substep's solved lambdas as the next
    substep's ``previous lambda`` feature (matched through the pipeline's
    contact matching, if enabled).  With ``net=None`` nothing is predicted and
    the step is the plain one; ``record=True`` keeps every substep's
    (features, solved lambda) pairs for training (``samples()``).
    """

    def __init__(self, net: WarmStartNet | None, iterations: int | None = 2, record: bool = False,
                 record_fraction: float = 1.0, seed: int = 0, gain=(1.0, 0.0), judge: str = "proxy"):
        self.net = net
        self.iterations = iterations
        # "proxy": a world falls back to no warm start when the prediction raises its largest penetration;
        # "none": every prediction is kept (the judge measurement of train_warmstart.judge_check)
        if judge not in ("proxy", "none"):
            raise ValueError("judge must be 'proxy' or 'none'")
        self.judge = judge
        # (normal, tangent) factors on the predictions; the tangential (friction) fit is poor
        # (R^2 ~0.4 against ~0.95 for the normal), and applying it raises penetration, so it is off
        self.gain = gain
        self.record = record
        self.record_fraction = record_fraction
        self.update_prev = True
        self._bufs = None
        self._records = []
        self._gen = None
        self._seed = seed

    def _alloc(self, model, contacts):
        cap = contacts.rigid_contact_max
        dev = model.device
        f = dict(dtype=torch.float32, device=dev)
        if self._bufs is None or self._bufs["cap"] != cap:
            self._bufs = {"cap": cap, "feat": torch.zeros(max(cap, 1), N_FEAT, **f),
                          "lam": torch.zeros(max(cap, 1), N_OUT, **f), "solved": torch.zeros(max(cap, 1), N_OUT, **f),
                          "prev": torch.zeros(max(cap, 1), N_OUT, **f), "impulse": torch.zeros(max(cap, 1), 6, **f),
                          "body_count": torch.zeros(max(model.body_count, 1), dtype=torch.int32, device=dev),
                          "fallback": torch.zeros(1, dtype=torch.int32, device=dev),
                          "status": torch.zeros(1, dtype=torch.int32, device=dev)}
        seg = contacts._seg
        if "impulse_scratch" not in seg:
            P5 = seg["rec"].shape[0]
            seg["impulse_scratch"] = torch.zeros((P5, 6), **f)
        return self._bufs

    def enabled(self) -> bool:
        """Whether the step applies predictions (and runs `iterations` instead of the solver's count)."""
        return self.net is not None

    def predict(self, features: torch.Tensor, count: torch.Tensor, out: torch.Tensor, status: torch.Tensor) -> None:
        """Contact-frame lambdas [cap, 3] of the published contacts (rows < count) into `out`."""
        self.net.infer(features, count, out, status, self.gain)

    def before_step(self, model, pipe, desc, state_in, contacts, dt: float, io) -> None:
        lib = _lib.load()
        b = self._alloc(model, contacts)
        stream = C.c_void_p(_lib.stream_handle(model.device))
        pub = pipe.public_struct(contacts)
        have_prev = contacts.rigid_contact_match_index is not None
        _lib.check("nb_ws_features", lib.nb_ws_features(
            C.byref(desc), C.c_void_p(ptr(state_in.body_q)), C.c_void_p(ptr(state_in.body_qd)), C.byref(pub),
            C.c_void_p(ptr(b["prev"]) if have_prev else None),
            C.c_void_p(ptr(contacts.rigid_contact_match_index) if have_prev else None),
            C.c_void_p(ptr(b["body_count"])), float(dt), C.c_void_p(ptr(b["feat"])), stream))
        if self.enabled():
            self.predict(b["feat"], contacts.rigid_contact_count, b["lam"], b["status"])
            io.ws_lambda = ptr(b["lam"])
            io.ws_capacity = contacts.rigid_contact_max
            io.ws_fallback = ptr(b["fallback"])
            io.ws_flags = NB_WS_KEEP_ALL if self.judge == "none" else 0
        # own impulse buffer (contacts without a force array): zero at allocation and kept zero by
        # nb_ws_targets, which clears the rows it reads; a solver-owned one is zeroed by the solver
        self._clear = not io.contact_impulse
        if self._clear:
            io.contact_impulse = ptr(b["impulse"])
            io.impulse_scratch = ptr(contacts._seg["impulse_scratch"])
            io.contact_impulse_capacity = contacts.rigid_contact_max
        self._impulse_ptr = io.contact_impulse
        self._stream = stream
        self._pub = pub

    def after_step(self, contacts) -> None:
        lib = _lib.load()
        b = self._bufs
        # the solved lambdas become the next substep's previous-lambda feature in place
        dest = b["prev"] if self.update_prev else b["solved"]
        _lib.check("nb_ws_targets", lib.nb_ws_targets(C.byref(self._pub), C.c_void_p(self._impulse_ptr),
                                                      C.c_void_p(ptr(dest)), 1 if self._clear else 0, self._stream))
        self._last = dest
        if self.record:
            n = min(int(contacts.rigid_contact_count.item()), contacts.rigid_contact_max)
            x, t = b["feat"][:n], dest[:n]
            if self.record_fraction < 1.0:
                if self._gen is None:
                    self._gen = torch.Generator(device=x.device).manual_seed(self._seed)
                keep = torch.rand(n, generator=self._gen, device=x.device) < self.record_fraction
                x, t = x[keep], t[keep]
            self._records.append((x.clone(), t.clone()))

    def samples(self) -> tuple[torch.Tensor, torch.Tensor]:
        """Recorded (features, lambda) rows; rows with a non-finite value are dropped."""
        x = torch.cat([r[0] for r in self._records]) if self._records else torch.zeros(0, N_FEAT)
        t = torch.cat([r[1] for r in self._records]) if self._records else torch.zeros(0, N_OUT)
        ok = torch.isfinite(x).all(1) & torch.isfinite(t).all(1)
        return x[ok].contiguous(), t[ok].contiguous()

    @property
    def fallback_count(self) -> int:
        return 0 if self._bufs is None else int(self._bufs["fallback"].item())


def kernel_timing(kind: str = "infer", rows: int = 111000, warmup: int = 3, reps: int = 20, seed: int = 0,
                  path: str | None = None) -> dict:
    """Mean CUDA-event time of the network's tensor-core kernels on random inputs: ``"infer"`` =
    nb_ws_infer on `rows` feature rows, ``"grads"`` = one nb_ws_grads call on `rows` samples.  The
    network is the committed C2 one unless `path` is given."""
    import os

    path = path or os.path.join(os.path.dirname(__file__), "data", "warmstart_c2.npz")
    net = WarmStartNet.load(path)
    dev = net.device
    g = torch.Generator(device="cpu").manual_seed(seed)
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
    if kind == "infer":
        feat = torch.randn(rows, N_FEAT, generator=g).to(dev)
        count = torch.tensor([rows], dtype=torch.int32, device=dev)
        out = torch.empty(rows, N_OUT, dtype=torch.float32, device=dev)
        status = torch.zeros(1, dtype=torch.int32, device=dev)
        for _ in range(warmup):
            net.infer(feat, count, out, status)
        torch.cuda.synchronize()
        ev[0].record()
        for _ in range(reps):
            net.infer(feat, count, out, status)
        ev[1].record()
        flops = 2.0 * (N_IN * N_HID + N_HID * N_HID + N_HID * N_OUT) * rows
    elif kind == "grads":
        x = torch.randn(rows, N_IN, generator=g).to(dev)
        t = torch.randn(rows, N_OUT, generator=g).to(dev)
        for _ in range(warmup):
            net.grads(x, t)
        torch.cuda.synchronize()
        ev[0].record()
        for _ in range(reps):
            net.grads(x, t)
        ev[1].record()
        flops = 3.0 * 2.0 * (N_IN * N_HID + N_HID * N_HID + N_HID * N_OUT) * rows
    else:
        raise ValueError("kind must be 'infer' or 'grads'")
    torch.cuda.synchronize()
    ms = ev[0].elapsed_time(ev[1]) / reps
    return {"kind": kind, "rows": rows, "ms": ms, "tflops": flops / (ms * 1e-3) / 1e12}


if __name__ == "__main__":
    import argparse
    import json

    ap = argparse.ArgumentParser(description="time the warm-start tensor-core kernels on random inputs")
    ap.add_argument("--kernel", default="infer", choices=["infer", "grads"])
    ap.add_argument("--rows", type=int, default=111000)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--reps", type=int, default=20)
    a = ap.parse_args()
    print(json.dumps(kernel_timing(a.kernel, a.rows, a.warmup, a.reps)))
