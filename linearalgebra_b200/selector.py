"""Learned precision selector for the mixed-precision LU-IR solve.

A 12 -> 64 -> 64 -> 4 MLP maps cheap matrix features to the factorization
precision class {FP8, BF16, FP32, FP64}.  Everything that computes runs in
libb200la.so: the features (b200la_selector_features: O(n^2) statistics of
A, no factorization), the network's forward pass, its training
(b200la_mlp_gradient: forward and backward in one kernel; b200la_mlp_adam),
and the selected solve (b200la_dsolve_selected), which tries the predicted
precision first; refinement failure escalates, so accuracy never depends on
the network.

Labels come from the method itself: each training system is solved at FP32,
then BF16 and FP8 while the previous one converged, and at FP64, each attempt
without escalation and timed; the label is the precision with the shortest
time among those whose refinement reached the tolerance within 10 iterations
(a GMRES-IR correction counts as one).  FP64 always converges, so every
system has a label.

Systems: A = U diag(sigma) V^T with U, V products of 8 seeded Householder
reflectors and sigma geometric from 1 to 1/kappa (the construction of
``workloads.conditioned``, applied on the device), n log-uniform in
[64, 4096], kappa log-uniform in [1e1, 1e12], x_true uniform in [-1, 1].

Weights are stored as JSON with a schema tag, the feature standardization and
a SHA-256 of the float32 parameter bytes (checked on load).

CLI (GPU):
    python -m linearalgebra_b200.selector label --start 0 --count 25000 --out shard0.npz
    python -m linearalgebra_b200.selector train --dataset shard0.npz,shard1.npz --out W.json
    python -m linearalgebra_b200.selector evaluate --weights W.json --systems 5000
"""
from __future__ import annotations

import argparse
import ctypes
import hashlib
import json
import math
import os
import sys
import time

import numpy as np
import torch

from . import _lib
from .api import MixedSolver, _ptr, _stream, refine_options, workspace

CLASSES = ("fp8", "bf16", "fp32", "fp64")
CLASS_PREC = (_lib.PREC_FP8, _lib.PREC_BF16, _lib.PREC_FP32, _lib.PREC_FP64)
PREC_CLASS = {p: i for i, p in enumerate(CLASS_PREC)}
N_FEATURES = 12
N_PARAMS = 5252
SCHEMA = "b200la-selector/2"
DEFAULT_WEIGHTS = os.path.join(os.path.dirname(os.path.abspath(__file__)), "selector_weights.json")
LABEL_ITERATIONS = 10
TOLERANCE = 1e-14


# ----------------------------------------------------------------------------
# systems
# ----------------------------------------------------------------------------
def conditioned_device(n: int, kappa: float, seed: int, device="cuda", reflectors: int = 8) -> torch.Tensor:
    """workloads.conditioned(n, kappa, seed) built on the device (same seeded
    reflectors and singular values; rank-1 updates in FP64)."""
    rng = np.random.default_rng(seed)
    sigma = kappa ** (-np.arange(n) / max(n - 1, 1))
    vu = torch.from_numpy(rng.standard_normal((reflectors, n))).to(device)
    vv = torch.from_numpy(rng.standard_normal((reflectors, n))).to(device)
    m = torch.diag(torch.from_numpy(sigma).to(device))

    def reflect_left(mat, vs):
        for v in reversed(list(vs)):
            beta = 2.0 / float(v @ v)
            mat -= beta * torch.outer(v, v @ mat)
        return mat

    m = reflect_left(m, vu)
    mt = reflect_left(m.T.contiguous(), vv)
    return mt.T.contiguous()


def sample_stream(count: int, seed: int, n_range=(64, 4096), kappa_range=(1e1, 1e12)):
    """(n, kappa, matrix seed) triples: n and kappa log-uniform."""
    rng = np.random.default_rng(seed)
    ns = np.rint(np.exp(rng.uniform(math.log(n_range[0]), math.log(n_range[1]), count))).astype(int)
    ks = 10.0 ** rng.uniform(math.log10(kappa_range[0]), math.log10(kappa_range[1]), count)
    seeds = rng.integers(0, 2 ** 31 - 1, count)
    return [(int(n), float(k), int(s)) for n, k, s in zip(ns, ks, seeds)]


def make_system(n: int, kappa: float, seed: int, device="cuda"):
    a = conditioned_device(n, kappa, seed, device)
    g = torch.Generator(device=device).manual_seed(seed)
    x_true = torch.rand(n, dtype=torch.float64, device=device, generator=g) * 2 - 1
    return a, a @ x_true, x_true


# ----------------------------------------------------------------------------
# device calls
# ----------------------------------------------------------------------------
class _Workspace:
    """One growing device workspace for the mixed-solver entry points."""

    def __init__(self):
        self.buf = None

    def get(self, n: int):
        lib = _lib.load()
        need = int(lib.b200la_dsolve_mixed_workspace_size(n, 1, None))
        if self.buf is None or self.buf.numel() < need:
            self.buf = workspace(need)
        return self.buf


_WS = _Workspace()
_STATS = {}


def features(a: torch.Tensor, stream=None) -> np.ndarray:
    """The 12 features (float32 numpy) of the square FP64 CUDA tensor a."""
    n = a.shape[0]
    f = (ctypes.c_float * N_FEATURES)()
    ws = _STATS.get(a.device)
    if ws is None:
        ws = _STATS[a.device] = torch.empty(16, dtype=torch.int64, device=a.device)
    _lib.check(_lib.load().b200la_selector_features(_ptr(a), n, f, _ptr(ws), 128, _stream(stream)))
    return np.frombuffer(f, dtype=np.float32).copy()


def condition_estimate(a: torch.Tensor, stream=None) -> float:
    """kappa_1 estimate of a from one FP32 LU (Hager / Higham)."""
    n = a.shape[0]
    k = ctypes.c_double(0)
    info = ctypes.c_int(0)
    ws = _WS.get(n)
    _lib.check(_lib.load().b200la_dcondition_estimate(_ptr(a), n, ctypes.byref(k), ctypes.byref(info), _ptr(ws),
                                                       ws.numel(), _stream(stream)),
               allow=(_lib.SUCCESS, _lib.SINGULAR))
    return float(k.value)


def attempt(a, b, precision: str, max_iterations: int = LABEL_ITERATIONS, escalate=False):
    """One mixed solve at `precision` (no escalation by default): dict with
    converged, iterations, gmres_iterations, backward_error, ms (wall)."""
    solver = MixedSolver(a.shape[0], 1, a.device, precision=precision, max_iterations=max_iterations,
                         escalate=escalate)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    x, res, st = solver(a, b)
    torch.cuda.synchronize()
    res["ms"] = (time.perf_counter() - t0) * 1e3
    res["status"] = st
    return x, res


def label_system(a, b):
    """(label class, {precision: outcome}) by the method itself: FP64, then
    FP32, BF16, FP8 while the previous low precision converged; the label is
    the fastest attempt that converged within LABEL_ITERATIONS."""
    out = {"fp64": attempt(a, b, "fp64")[1]}
    for p in ("fp32", "bf16", "fp8"):
        _, r = attempt(a, b, p)
        out[p] = r
        if not (r["converged"] and r["iterations"] <= LABEL_ITERATIONS):
            break
    ok = {p: r["ms"] for p, r in out.items() if r["converged"] and r["iterations"] <= LABEL_ITERATIONS}
    return CLASSES.index(min(ok, key=ok.get)), out


def generate(count: int, seed: int, log_every: int = 0, **stream_kw):
    """Label `count` systems of the seeded stream (see generate_systems)."""
    return generate_systems(sample_stream(count, seed, **stream_kw), log_every)


def generate_systems(systems, log_every: int = 0):
    """Label the given (n, kappa, seed) systems.  Returns a dict of numpy
    arrays: features [count, 12], labels, n, kappa, and per precision
    (columns fp8, bf16, fp32, fp64) convergence within the label's
    iterations and wall time (-1 / NaN where not attempted)."""
    count = len(systems)
    feats = np.zeros((count, N_FEATURES), np.float32)
    labels = np.zeros(count, np.int32)
    conv = np.full((count, 4), -1, np.int8)
    ms = np.full((count, 4), np.nan)
    t_start = time.time()
    for i, (n, kappa, s) in enumerate(systems):
        a, b, _ = make_system(n, kappa, s)
        feats[i] = features(a)
        labels[i], outs = label_system(a, b)
        for j, p in enumerate(CLASSES):
            if p in outs:
                conv[i, j] = int(outs[p]["converged"] and outs[p]["iterations"] <= LABEL_ITERATIONS)
                ms[i, j] = outs[p]["ms"]
        if log_every and (i + 1) % log_every == 0:
            print(f"[selector] labelled {i + 1}/{count} in {time.time() - t_start:.0f} s; "
                  f"class counts {np.bincount(labels[:i + 1], minlength=4).tolist()}", file=sys.stderr, flush=True)
    return {"features": feats, "labels": labels, "n": np.array([t[0] for t in systems]),
            "kappa": np.array([t[1] for t in systems]), "converged": conv, "ms": ms}


# ----------------------------------------------------------------------------
# network
# ----------------------------------------------------------------------------
def init_params(seed: int) -> np.ndarray:
    """He-uniform weights, zero biases (float32, the kernels' layout)."""
    rng = np.random.default_rng(seed)
    parts = []
    for fan_in, fan_out in ((12, 64), (64, 64), (64, 4)):
        bound = math.sqrt(6.0 / fan_in)
        parts.append(rng.uniform(-bound, bound, size=(fan_in, fan_out)).ravel())
        parts.append(np.zeros(fan_out))
    p = np.concatenate(parts).astype(np.float32)
    assert p.size == N_PARAMS
    return p


class Network:
    """Parameters (device float32: 5252 weights, then mean[12] and inverse
    std[12] of the features) and the kernels that use them."""

    def __init__(self, params: np.ndarray, mean: np.ndarray, inv_std: np.ndarray, device="cuda"):
        lib = _lib.load()
        assert lib.b200la_mlp_param_count() == N_PARAMS
        host = np.concatenate([np.asarray(params, np.float32), np.asarray(mean, np.float32),
                               np.asarray(inv_std, np.float32)])
        self.buf = torch.from_numpy(host).to(device)
        self.device = device
        self.meta: dict = {}

    @property
    def params(self) -> torch.Tensor:
        return self.buf[:N_PARAMS]

    @property
    def mean(self) -> np.ndarray:
        return self.buf[N_PARAMS:N_PARAMS + N_FEATURES].cpu().numpy()

    @property
    def inv_std(self) -> np.ndarray:
        return self.buf[N_PARAMS + N_FEATURES:].cpu().numpy()

    def standardize(self, f: np.ndarray) -> torch.Tensor:
        x = (np.asarray(f, np.float32) - self.mean) * self.inv_std
        return torch.from_numpy(np.ascontiguousarray(x, np.float32)).to(self.device)

    def probs(self, x_std: torch.Tensor, stream=None) -> torch.Tensor:
        """softmax(net(x)) for standardized features x [batch, 12] (device)."""
        x_std = x_std.contiguous()
        out = torch.empty(x_std.shape[0], 4, dtype=torch.float32, device=self.device)
        _lib.check(_lib.load().b200la_mlp_forward(_ptr(self.params), _ptr(x_std), x_std.shape[0], _ptr(out),
                                                  _stream(stream)))
        return out

    def predict(self, f: np.ndarray) -> np.ndarray:
        return self.probs(self.standardize(np.atleast_2d(f))).argmax(1).cpu().numpy()

    # ---- persistence -------------------------------------------------------
    def to_json(self, meta: dict | None = None) -> dict:
        p = self.params.cpu().numpy().astype(np.float32)
        return {"schema": SCHEMA, "classes": list(CLASSES), "layers": [12, 64, 64, 4],
                "sha256": hashlib.sha256(p.tobytes()).hexdigest(),
                "mean": [float(v) for v in self.mean], "inv_std": [float(v) for v in self.inv_std],
                "params": [float(v) for v in p], "meta": meta or {}}

    def save(self, path: str, meta: dict | None = None):
        with open(path, "w") as fh:
            json.dump(self.to_json(meta), fh)

    @classmethod
    def load(cls, path: str = DEFAULT_WEIGHTS, device="cuda") -> "Network":
        with open(path) as fh:
            d = json.load(fh)
        if d.get("schema") != SCHEMA:
            raise ValueError(f"{path}: schema {d.get('schema')!r}, expected {SCHEMA!r}")
        p = np.asarray(d["params"], np.float32)
        if p.size != N_PARAMS or hashlib.sha256(p.tobytes()).hexdigest() != d["sha256"]:
            raise ValueError(f"{path}: parameter checksum mismatch")
        net = cls(p, np.asarray(d["mean"]), np.asarray(d["inv_std"]), device)
        net.meta = d.get("meta", {})
        return net


def train(feats: np.ndarray, labels: np.ndarray, epochs: int = 300, batch: int = 512, lr: float = 3e-3,
          weight_decay: float = 1e-4, seed: int = 0, device="cuda", log_every: int = 0):
    """Train on the GPU with the library's kernels (mini-batch Adam on the
    mean cross-entropy).  Returns (Network, history of epoch mean losses)."""
    lib = _lib.load()
    feats = np.asarray(feats, np.float32)
    mean = feats.mean(0)
    std = feats.std(0)
    inv_std = np.where(std > 1e-6, 1.0 / np.maximum(std, 1e-6), 1.0).astype(np.float32)
    net = Network(init_params(seed), mean, inv_std, device)
    x_all = net.standardize(feats)
    y_all = torch.from_numpy(np.asarray(labels, np.int32)).to(device)
    grads = torch.zeros(N_PARAMS, dtype=torch.float32, device=device)
    m1 = torch.zeros_like(grads)
    m2 = torch.zeros_like(grads)
    loss = torch.zeros(1, dtype=torch.float32, device=device)
    g = torch.Generator(device="cpu").manual_seed(seed)
    count = feats.shape[0]
    step = 0
    history = []
    s = _stream(None)
    for ep in range(epochs):
        perm = torch.randperm(count, generator=g).to(device)
        xs, ys = x_all[perm].contiguous(), y_all[perm].contiguous()
        loss.zero_()
        for b0 in range(0, count, batch):
            bsz = min(batch, count - b0)
            step += 1
            _lib.check(lib.b200la_mlp_gradient(_ptr(net.params), _ptr(xs[b0:]), _ptr(ys[b0:]), bsz, _ptr(grads),
                                               _ptr(loss), s))
            _lib.check(lib.b200la_mlp_adam(_ptr(net.params), _ptr(grads), _ptr(m1), _ptr(m2), bsz, lr, 0.9, 0.999,
                                           1e-8, step, weight_decay, s))
        history.append(float(loss.item()) / count)
        if log_every and (ep + 1) % log_every == 0:
            print(f"[selector] epoch {ep + 1}: loss {history[-1]:.4f}", file=sys.stderr, flush=True)
    return net, history


# ----------------------------------------------------------------------------
# selected solve and evaluation
# ----------------------------------------------------------------------------
def solve_selected(net: Network, a: torch.Tensor, b: torch.Tensor, x: torch.Tensor | None = None,
                   tolerance: float = TOLERANCE, stream=None):
    """b200la_dsolve_selected: returns (x, result dict, predicted precision
    name, features)."""
    n = a.shape[0]
    if x is None:
        x = torch.empty_like(b)
    opts = refine_options("fp32", tolerance=tolerance)
    res = _lib.RefineResult()
    pred = ctypes.c_int(-1)
    f = (ctypes.c_float * N_FEATURES)()
    ws = _WS.get(n)
    st = _lib.load().b200la_dsolve_selected(_ptr(a), n, _ptr(b), _ptr(x), _ptr(net.buf), ctypes.byref(opts),
                                            ctypes.byref(res), ctypes.byref(pred), f, _ptr(ws), ws.numel(),
                                            _stream(stream))
    _lib.check(st, allow=(_lib.SUCCESS, _lib.NOT_CONVERGED, _lib.SINGULAR))
    d = res.as_dict()
    d["status"] = st
    return x, d, _lib.PREC_NAMES[pred.value], np.frombuffer(f, dtype=np.float32).copy()


STRATEGIES = ("selected", "fixed_fp32", "fp64")


def run_strategy(name: str, net: Network | None, a, b):
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    if name == "selected":
        x, r, pred, _ = solve_selected(net, a, b)
        r["predicted"] = pred
    else:
        prec = "fp32" if name == "fixed_fp32" else "fp64"
        solver = MixedSolver(a.shape[0], 1, a.device, precision=prec, escalate=True)
        x, r, st = solver(a, b)
        r["status"] = st
    torch.cuda.synchronize()
    r["ms"] = (time.perf_counter() - t0) * 1e3
    return x, r


def evaluate(net: Network, count: int, seed: int, strategies=STRATEGIES, warmup: int = 3, **stream_kw):
    """Run the strategies over a held-out seeded stream.  Returns a summary
    per strategy (total ms, solves/s, worst backward error, converged count,
    escalations) and per-system records."""
    systems = sample_stream(count, seed, **stream_kw)
    for (n, kappa, s) in systems[:warmup]:
        a, b, _ = make_system(n, kappa, s)
        for name in strategies:
            run_strategy(name, net, a, b)
    recs = []
    for (n, kappa, s) in systems:
        a, b, x_true = make_system(n, kappa, s)
        rec = {"n": n, "kappa": kappa}
        for name in strategies:
            x, r = run_strategy(name, net, a, b)
            fe = float((x - x_true).abs().max() / x_true.abs().max())
            rec[name] = {"ms": r["ms"], "eta": r["backward_error"], "converged": r["converged"],
                         "escalations": r["escalations"], "precision_used": r["precision_used"],
                         "forward_error": fe}
            if name == "selected":
                rec[name]["predicted"] = r["predicted"]
        recs.append(rec)
    summary = {}
    for name in strategies:
        ms = np.array([r[name]["ms"] for r in recs])
        eta = np.array([r[name]["eta"] for r in recs])
        summary[name] = {"total_ms": float(ms.sum()), "solves_per_s": float(len(recs) / (ms.sum() / 1e3)),
                         "worst_eta": float(eta.max()), "converged": int(sum(r[name]["converged"] for r in recs)),
                         "escalations": int(sum(r[name]["escalations"] for r in recs))}
    if "selected" in strategies:
        summary["selected"]["predicted"] = {c: int(sum(r["selected"]["predicted"] == c for r in recs))
                                            for c in CLASSES}
    return summary, recs


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    sub = ap.add_subparsers(dest="cmd", required=True)
    lab = sub.add_parser("label", help="label a slice of the seeded training stream into an npz shard")
    lab.add_argument("--systems", type=int, default=50000, help="length of the seeded stream")
    lab.add_argument("--seed", type=int, default=1)
    lab.add_argument("--start", type=int, default=0)
    lab.add_argument("--count", type=int, default=None)
    lab.add_argument("--out", required=True)
    t = sub.add_parser("train")
    t.add_argument("--systems", type=int, default=50000)
    t.add_argument("--seed", type=int, default=1)
    t.add_argument("--epochs", type=int, default=300)
    t.add_argument("--out", default=DEFAULT_WEIGHTS)
    t.add_argument("--dataset", default=None,
                   help="comma-separated npz shards to train on (else label --systems here)")
    e = sub.add_parser("evaluate")
    e.add_argument("--weights", default=DEFAULT_WEIGHTS)
    e.add_argument("--systems", type=int, default=5000)
    e.add_argument("--seed", type=int, default=2)
    e.add_argument("--out", default=None)
    args = ap.parse_args(argv)
    if args.cmd == "label":
        systems = sample_stream(args.systems, args.seed)
        end = len(systems) if args.count is None else min(len(systems), args.start + args.count)
        t0 = time.time()
        parts = []
        for c0 in range(args.start, end, 2500):
            parts.append(generate_systems(systems[c0:min(c0 + 2500, end)], log_every=500))
            d = {k: np.concatenate([p[k] for p in parts]) for k in parts[0]}
            d["label_seconds"] = np.array(time.time() - t0)
            d["stream"] = np.array([args.systems, args.seed, args.start, c0 + len(parts[-1]["labels"])])
            np.savez_compressed(args.out, **d)
        print(json.dumps({"systems": int(len(d["labels"])), "seconds": float(d["label_seconds"]),
                          "class_counts": np.bincount(d["labels"], minlength=4).tolist()}))
        return
    if args.cmd == "train":
        if args.dataset:
            shards = [dict(np.load(f)) for f in args.dataset.split(",")]
            d = {k: np.concatenate([sh[k] for sh in shards]) for k in ("features", "labels", "n", "kappa",
                                                                          "converged", "ms")}
            if d["ms"].shape[1] != len(CLASSES):
                raise ValueError("dataset shards predate the time-aware labels; label them again")
            d["label_seconds"] = np.array(sum(float(sh["label_seconds"]) for sh in shards))
        else:
            t0 = time.time()
            d = generate(args.systems, args.seed, log_every=1000)
            d["label_seconds"] = np.array(time.time() - t0)
        nval = max(1, len(d["labels"]) // 10)
        t1 = time.time()
        net, hist = train(d["features"][nval:], d["labels"][nval:], epochs=args.epochs, log_every=50)
        train_seconds = time.time() - t1
        pred = net.predict(d["features"][:nval])
        acc = float((pred == d["labels"][:nval]).mean())
        counts = np.bincount(d["labels"], minlength=4).tolist()
        meta = {"systems": int(len(d["labels"])), "seed": args.seed, "class_counts": counts,
                "validation_systems": int(nval), "validation_accuracy": acc, "final_loss": hist[-1],
                "epochs": args.epochs, "label_seconds": float(d.get("label_seconds", np.nan)),
                "train_seconds": train_seconds}
        net.save(args.out, meta)
        print(json.dumps(meta))
    else:
        net = Network.load(args.weights)
        summary, recs = evaluate(net, args.systems, args.seed)
        print(json.dumps(summary))
        if args.out:
            with open(args.out, "w") as fh:
                json.dump({"summary": summary, "systems": recs}, fh)


if __name__ == "__main__":
    main()
