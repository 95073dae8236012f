"""Batched solves of many independent systems of uneven order (16..512),
through b200la_dgesv_batched: one persistent kernel launch per batch,
optionally replayed as a CUDA graph.

* ``BatchedSolver(sizes)`` packs the batch layout (row-major matrices back to
  back, offsets per system), orders the systems largest first so the last
  CTAs get the smallest work, and owns the workspace.
* ``autotune(...)`` picks the panel width and the threads per system (a CTA
  of 256 threads solves 1, 2 or 4 systems at once) per order bucket of 64 by
  timing the candidates on a sample of the batch's own systems, and caches
  the choice on disk per device (``B200LA_TUNE_CACHE`` or
  ~/.cache/b200la/batched_tune.json).
* ``shard(sizes, world, rank)`` splits a batch across ranks with balanced
  sum(n^3) (greedy, largest first); ranks share nothing in the data path.
"""
from __future__ import annotations

import ctypes
import json
import os

import numpy as np
import torch

from . import _lib
from .api import _ptr, _stream, workspace

NB_BUCKETS = 8
NB_CHOICES = {_lib.PREC_FP32: (16, 32), _lib.PREC_FP64: (8, 16)}
GROUP_CHOICES = (64, 128, 256)  # threads that solve one system


def bucket_of(n: int) -> int:
    return min((int(n) - 1) // 64, NB_BUCKETS - 1)


def entry(nb: int, threads: int) -> int:
    """A bucket's table entry: panel width in bits 0-7, threads per system / 32
    in bits 8-15 (0 for a whole CTA of 256)."""
    return int(nb) | ((0 if threads >= 256 else threads // 32) << 8)


def entry_parts(e: int) -> tuple[int, int]:
    g = ((int(e) >> 8) & 0xFF) * 32
    return int(e) & 0xFF, (g if g in (64, 128) else 256)


def table_valid(prec: int, table) -> bool:
    arr = (ctypes.c_int32 * NB_BUCKETS)(*[int(v) for v in table])
    return bool(_lib.load().b200la_batched_table_valid(prec, arr))


def default_table(prec: int) -> list[int]:
    """Per bucket: the widest panel and the fewest threads per system whose
    shared-memory slice holds the bucket's largest order."""
    out = []
    for bk in range(NB_BUCKETS):
        chosen = None
        for g in GROUP_CHOICES:
            for nb in sorted(NB_CHOICES[prec], reverse=True):
                trial = [entry(NB_CHOICES[prec][-1], 256)] * NB_BUCKETS
                trial[bk] = entry(nb, g)
                if table_valid(prec, trial):
                    chosen = entry(nb, g)
                    break
            if chosen is not None:
                break
        out.append(chosen if chosen is not None else entry(NB_CHOICES[prec][0], 256))
    return out


def shard(sizes, world: int, rank: int) -> np.ndarray:
    """Indices of the systems rank `rank` of `world` solves: greedy
    largest-first assignment to the rank with the least sum(n^3) so far."""
    sizes = np.asarray(sizes)
    order = np.argsort(-sizes, kind="stable")
    load = np.zeros(world)
    owner = np.empty(len(sizes), dtype=np.int64)
    for i in order:
        r = int(np.argmin(load))
        owner[i] = r
        load[r] += float(sizes[i]) ** 3
    return np.nonzero(owner == rank)[0]


def _cache_path() -> str:
    return os.environ.get("B200LA_TUNE_CACHE",
                          os.path.join(os.path.expanduser("~"), ".cache", "b200la", "batched_tune.json"))


class BatchedSolver:
    def __init__(self, sizes, precision: str = "fp32", device=None, tolerance: float = 1e-14,
                 max_iterations: int = 10, nb_table=None):
        self.device = torch.device(device) if device is not None else torch.device("cuda")
        self.sizes_h = np.asarray(sizes, dtype=np.int64)
        if self.sizes_h.min() < 1 or self.sizes_h.max() > 512:
            raise ValueError("orders must lie in [1, 512]")
        self.count = len(self.sizes_h)
        self.prec = _lib.PREC_FP32 if precision == "fp32" else _lib.PREC_FP64
        sq = self.sizes_h ** 2
        self.offa_h = np.concatenate([[0], np.cumsum(sq)[:-1]]).astype(np.int64)
        self.offv_h = np.concatenate([[0], np.cumsum(self.sizes_h)[:-1]]).astype(np.int64)
        self.total_a = int(sq.sum())
        self.total_v = int(self.sizes_h.sum())
        order = np.argsort(-self.sizes_h, kind="stable").astype(np.int32)
        d = self.device
        self.sizes = torch.from_numpy(self.sizes_h.astype(np.int32)).to(d)
        self.offa = torch.from_numpy(self.offa_h).to(d)
        self.offv = torch.from_numpy(self.offv_h).to(d)
        self.order = torch.from_numpy(order).to(d)
        self.status = torch.empty(self.count, dtype=torch.int32, device=d)
        self.berr = torch.empty(self.count, dtype=torch.float64, device=d)
        self.tolerance = tolerance
        self.max_iterations = max_iterations
        if nb_table is None:
            nb_table = default_table(self.prec)
        self.set_nb_table(nb_table)
        lib = _lib.load()
        self.ws_bytes = int(lib.b200la_dgesv_batched_workspace_size(self.total_a, self.total_v, self.prec))
        self.ws = workspace(self.ws_bytes, d)
        self.graph = None

    def set_nb_table(self, table):
        self.nb_table_h = [int(v) for v in table]
        self.nb_table = torch.tensor(self.nb_table_h, dtype=torch.int32, device=self.device)

    def views(self, buf: torch.Tensor, i: int, matrix: bool):
        n = int(self.sizes_h[i])
        if matrix:
            o = int(self.offa_h[i])
            return buf[o:o + n * n].view(n, n)
        o = int(self.offv_h[i])
        return buf[o:o + n]

    def launch(self, a: torch.Tensor, b: torch.Tensor, x: torch.Tensor, stream=None):
        st = _lib.load().b200la_dgesv_batched(
            self.count, _ptr(self.sizes), _ptr(self.offa), _ptr(self.offv), _ptr(self.order), _ptr(a), _ptr(b),
            _ptr(x), self.total_a, self.total_v, self.prec, _ptr(self.nb_table), self.max_iterations,
            self.tolerance, _ptr(self.status), _ptr(self.berr), _ptr(self.ws), self.ws_bytes, _stream(stream))
        _lib.check(st)

    def capture(self, a, b, x):
        """Record one launch as a CUDA graph (after a warm-up launch)."""
        s = torch.cuda.Stream(self.device)
        s.wait_stream(torch.cuda.current_stream(self.device))
        with torch.cuda.stream(s):
            self.launch(a, b, x, s)
        torch.cuda.current_stream(self.device).wait_stream(s)
        torch.cuda.synchronize(self.device)
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g, stream=s):
            self.launch(a, b, x, s)
        self.graph = g
        return g

    def replay(self):
        self.graph.replay()

    # --- autotuning of the panel width and threads per system, per bucket --
    def autotune(self, a, b, x, sample_per_bucket: int = 48, use_cache: bool = True):
        """Per order bucket, time every valid (panel width, threads per
        system) pair on up to `sample_per_bucket` of the batch's own systems
        of that bucket and keep the fastest; cached per device and precision."""
        key = f"{torch.cuda.get_device_name(self.device)}|prec{self.prec}|v2"
        path = _cache_path()
        cache = {}
        if use_cache and os.path.exists(path):
            try:
                cache = json.load(open(path))
            except (OSError, ValueError):
                cache = {}
        if use_cache and key in cache:
            self.set_nb_table(cache[key]["nb_table"])
            return cache[key]
        table = default_table(self.prec)
        timings = {}
        buckets = np.array([bucket_of(n) for n in self.sizes_h])
        for bk in range(NB_BUCKETS):
            idx = np.nonzero(buckets == bk)[0][:sample_per_bucket]
            if len(idx) == 0:
                continue
            sub = BatchedSolver(self.sizes_h[idx], "fp32" if self.prec == _lib.PREC_FP32 else "fp64",
                                self.device, self.tolerance, self.max_iterations)
            sa = torch.cat([self.views(a, int(i), True).reshape(-1) for i in idx])
            sb = torch.cat([self.views(b, int(i), False) for i in idx])
            sx = torch.empty_like(sb)
            best = None
            for g in GROUP_CHOICES:
                for nb in NB_CHOICES[self.prec]:
                    trial = list(table)
                    trial[bk] = entry(nb, g)
                    if not table_valid(self.prec, trial):
                        continue
                    sub.set_nb_table(trial)
                    sub.launch(sa, sb, sx)
                    torch.cuda.synchronize(self.device)
                    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                    e0.record()
                    for _ in range(3):
                        sub.launch(sa, sb, sx)
                    e1.record()
                    torch.cuda.synchronize(self.device)
                    t = e0.elapsed_time(e1) / 3
                    timings[f"{bk}:nb{nb}:t{g}"] = t
                    if best is None or t < best[0]:
                        best = (t, entry(nb, g))
            if best is not None:
                table[bk] = best[1]
        self.set_nb_table(table)
        out = {"nb_table": table, "timings_ms": timings,
               "per_bucket": [{"panel_width": entry_parts(e)[0], "threads_per_system": entry_parts(e)[1]}
                              for e in table]}
        if use_cache:
            try:
                os.makedirs(os.path.dirname(path), exist_ok=True)
                cache[key] = out
                json.dump(cache, open(path, "w"), indent=1)
            except OSError:
                pass
        return out


def make_batch(count: int, seed: int, device="cuda", lo: int = 16, hi: int = 512):
    """The benchmark's batch: n uniform in [lo, hi], A iid N(0,1) with n*I added
    to every other system (diagonally dominant), x_true iid U[-1,1],
    b = A x_true.  Returns (sizes, a, b, x_true) with a, b packed as
    BatchedSolver lays them out."""
    rng = np.random.default_rng(seed)
    sizes = rng.integers(lo, hi + 1, size=count)
    sq = sizes.astype(np.int64) ** 2
    offa = np.concatenate([[0], np.cumsum(sq)[:-1]])
    offv = np.concatenate([[0], np.cumsum(sizes)[:-1]])
    g = torch.Generator(device=device)
    g.manual_seed(seed)
    a = torch.randn(int(sq.sum()), dtype=torch.float64, device=device, generator=g)
    x_true = torch.rand(int(sizes.sum()), dtype=torch.float64, device=device, generator=g) * 2 - 1
    b = torch.empty_like(x_true)
    dom = np.nonzero(np.arange(count) % 2 == 0)[0]
    diag_idx = np.concatenate([offa[i] + np.arange(sizes[i]) * (sizes[i] + 1) for i in dom])
    di = torch.from_numpy(diag_idx).to(device)
    a[di] += torch.from_numpy(np.repeat(sizes[dom], sizes[dom]).astype(np.float64)).to(device)
    for i in range(count):
        n = int(sizes[i])
        av = a[int(offa[i]):int(offa[i]) + n * n].view(n, n)
        b[int(offv[i]):int(offv[i]) + n] = av @ x_true[int(offv[i]):int(offv[i]) + n]
    return sizes, a, b, x_true
