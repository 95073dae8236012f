#!/usr/bin/env python
"""Benchmark of the B200 LU-solve path.

Workload (one "step"): solve one dense system A x = b of order n = 16384,
A iid N(0,1) with nothing added to the diagonal, x_true iid U[-1,1],
b = A x_true, nrhs = 1, FP64 result, from inputs resident in HBM.  The metric
is time-to-solution in seconds (lower is better).  The 2 GiB matrix is larger
than the 126 MB L2, so no L2 flush is needed between steps.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]

--impl b200 (default) prints one JSON line with the device-timed value, the
end-to-end value through the C ABI with host buffers, the roofline of the
dominant kernel (timed live with the library's launch recorder), the CPU
baseline (the reference's own NATIVE LU solve, bounded sample), the clocks
seen during the timed region, and the reference's own cuSOLVER (CUDA_BLAS)
LU solve of the same system as a GPU baseline.  --impl reference times the
reference's NATIVE CPU implementation alone on a bounded sample of the same
workload.  With
N > 1 (torchrun), each rank solves its own system (replicas: a single dense
LU has no data-parallel split); the value is the max over ranks.
"""
from __future__ import annotations

import argparse
import ctypes
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "LU solve sec at n=16384 & batched solves/s, mixed-IR vs FP64, bwd err<=1e-14"
N_DEFAULT = 16384
SEED = 16384
CPU_SAMPLE_N = 4096
EPS64 = 2.0 ** -52


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=5)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", choices=["b200", "reference"], default="b200")
    p.add_argument("--n", type=int, default=N_DEFAULT)
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--no-e2e", action="store_true")
    p.add_argument("--no-compare", action="store_true", help="skip timing the other method")
    p.add_argument("--method", choices=["mixed", "fp64"], default="mixed")
    p.add_argument("--precision", choices=["fp32", "tf32", "bf16", "fp16"], default="fp32")
    p.add_argument("--batch-count", type=int, default=20000)
    p.add_argument("--no-batched", action="store_true")
    p.add_argument("--inv-n", type=int, default=16384, help="order of the inversion / determinant measurement")
    p.add_argument("--no-inversion", action="store_true")
    p.add_argument("--no-multiplication", action="store_true")
    p.add_argument("--chol-n", type=int, default=16384, help="order of the Cholesky-mode solve measurement")
    p.add_argument("--no-cholesky", action="store_true")
    p.add_argument("--no-transpose", action="store_true")
    p.add_argument("--tp-n", type=int, default=16384, help="order of the square transpose measurement")
    p.add_argument("--no-side-workloads", "--no-configs", dest="no_side_workloads", action="store_true",
                   help="skip the n=512 solve, the BF16/FP16 and nrhs=64 solves at n=16384 and the "
                        "conditioning sweep at n=4096/8192")
    p.add_argument("--selector-systems", type=int, default=5000,
                   help="held-out systems of the precision selector's stream (0: skip)")
    return p.parse_args()


# ---------------------------------------------------------------------------
# distributed plumbing (replicas)
# ---------------------------------------------------------------------------
def dist_setup(args):
    import torch

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        import torch.distributed as dist

        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600),
                                device_id=torch.device("cuda", local))
    elif torch.cuda.is_available():
        torch.cuda.set_device(0)
    return world, rank, local


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def max_over_ranks(world, value: float) -> float:
    if world == 1:
        return value
    import torch
    import torch.distributed as dist
    t = torch.tensor([value], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


# ---------------------------------------------------------------------------
# clocks sampled during the timed region
# ---------------------------------------------------------------------------
class ClockSampler:
    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index: int):
        self.proc = None
        self.lines: list[str] = []
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200", "-i", str(device_index)],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except (OSError, ValueError):
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.lines:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 7:
                continue
            try:
                sm.append(float(parts[0]))
                smax = float(parts[1])
            except ValueError:
                continue
            for name, flag in zip(names, parts[3:7]):
                if flag.lower() == "active":
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


# ---------------------------------------------------------------------------
# measured FP64 peak (the denominator of the FP64 trailing-update roofline)
# ---------------------------------------------------------------------------
def measured_fp64_peak_tflops() -> float:
    import torch
    n = 8192
    a = torch.randn(n, n, dtype=torch.float64, device="cuda")
    b = torch.randn(n, n, dtype=torch.float64, device="cuda")
    for _ in range(2):
        torch.matmul(a, b)
    best = 0.0
    for _ in range(5):
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record()
        torch.matmul(a, b)
        e.record()
        e.synchronize()
        best = max(best, 2 * n ** 3 / (s.elapsed_time(e) * 1e-3) / 1e12)
    del a, b
    torch.cuda.empty_cache()
    return best


def measured_peaks() -> dict:
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            d = json.load(f)
        return {"hbm_gbs": d.get("hbm_gbs", 6650.0), "bf16_tflops": d.get("bf16_tflops", 1590.0),
                "source": "measured (MEASURED_PEAKS.json)"}
    return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "source": "fallback"}

# ---------------------------------------------------------------------------
# inversion / determinant (LU modes): this library vs the reference's
# CUDA_BLAS path (baseline/_ref) at the same order
# ---------------------------------------------------------------------------
def inversion_gemm_flops(n: int, nb: int = 512, sub: int = 64) -> int:
    """Flops of the inversion's GEMM updates (k_dmma_update launches) for
    order n: the block-row sub-updates and the big forward / backward ones."""
    fl = 0
    for b0 in range(0, n, nb):
        bw = min(nb, n - b0)
        k1 = b0 + bw
        for phase_cols in (k1, n):  # forward block row: k1 columns; backward: n
            for r0 in range(0, bw, sub):
                sw = min(sub, bw - r0)
                rows_left = bw - r0 - sw  # rows of the block still to update
                fl += 2 * rows_left * phase_cols * sw
        if k1 < n:
            fl += 2 * (n - k1) * k1 * bw  # forward: rows below, columns [0, k1)
        if b0 > 0:
            fl += 2 * b0 * n * bw  # backward: rows above, all columns
    return fl


def cuda_blas_inverse(lib_path, A, stream, steps):
    import torch
    lib = ctypes.CDLL(lib_path)
    lib.ref_cublas_dinverse_workspace_size.restype = ctypes.c_size_t
    lib.ref_cublas_dinverse_workspace_size.argtypes = [ctypes.c_int64]
    lib.ref_cublas_dinverse.argtypes = [ctypes.c_void_p, ctypes.c_int64, ctypes.c_void_p, ctypes.c_size_t,
                                        ctypes.c_void_p]
    lib.ref_cublas_ddeterminant_workspace_size.restype = ctypes.c_size_t
    lib.ref_cublas_ddeterminant_workspace_size.argtypes = [ctypes.c_int64]
    lib.ref_cublas_ddeterminant.argtypes = [ctypes.c_void_p, ctypes.c_int64, ctypes.c_void_p, ctypes.c_void_p,
                                            ctypes.c_size_t, ctypes.c_void_p]
    lib.ref_cublas_last_error.restype = ctypes.c_char_p
    n = A.shape[0]
    nb = int(lib.ref_cublas_dinverse_workspace_size(n))
    ws = torch.empty(max(nb, 256), dtype=torch.uint8, device=A.device)
    m = torch.empty_like(A)

    def inv_step():
        m.copy_(A)
        if lib.ref_cublas_dinverse(m.data_ptr(), n, ws.data_ptr(), nb, stream.cuda_stream) != 0:
            raise RuntimeError(lib.ref_cublas_last_error().decode())

    inv_step()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(steps):
        inv_step()
    e1.record(stream)
    torch.cuda.synchronize()
    t_inv = e0.elapsed_time(e1) / steps / 1e3
    res = (torch.mm(A, m) - torch.eye(n, dtype=A.dtype, device=A.device)).abs().max().item()
    del ws
    db = int(lib.ref_cublas_ddeterminant_workspace_size(n))
    dws = torch.empty(max(db, 256), dtype=torch.uint8, device=A.device)
    out = ctypes.c_double(0)
    m.copy_(A)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    if lib.ref_cublas_ddeterminant(m.data_ptr(), n, ctypes.addressof(out), dws.data_ptr(), db,
                                   stream.cuda_stream) != 0:
        raise RuntimeError(lib.ref_cublas_last_error().decode())
    t_det = time.perf_counter() - t0
    del m, dws
    torch.cuda.empty_cache()
    return {"inverse_s": t_inv, "inverse_residual": res, "determinant_s": t_det, "steps": steps,
            "what": "the reference's inversion / determinant<double,CUDA_BLAS> LU mode (cuSOLVER getrf, getrs "
                    "against the identity, the reference's transposes; determinant host-synchronous)"}


def run_inversion(args, world, rank, local):
    """inversion / determinant<double, B200> LU mode at order args.inv_n:
    each step restores m from A (device copy), factors and inverts in place."""
    import torch

    import linearalgebra_b200 as la
    from linearalgebra_b200 import _lib

    lib = _lib.load()
    n = args.inv_n
    dev = torch.device("cuda", local)
    gen = torch.Generator(device=dev)
    gen.manual_seed(SEED + 1 + rank)
    A = torch.randn(n, n, dtype=torch.float64, device=dev, generator=gen)
    m = torch.empty_like(A)
    piv = torch.empty(n, dtype=torch.int64, device=dev)
    nbytes = la.inversion.workspace_size(n, la.LU_LINEAR_SOLVER)
    ws = torch.empty(nbytes, dtype=torch.uint8, device=dev)
    stream = torch.cuda.current_stream(dev)

    def step():
        m.copy_(A)
        la.inversion.apply(m, piv, n, la.LU_LINEAR_SOLVER, ws, nbytes, stream)

    steps = 2
    step()
    torch.cuda.synchronize()
    lib.b200la_profile_start(sum(1 << c for c in CLASS_NAMES))
    step()
    torch.cuda.synchronize()
    breakdown = {}
    for c, name in CLASS_NAMES.items():
        t_ms, cnt = ctypes.c_double(0), ctypes.c_int64(0)
        lib.b200la_profile_stop(c, ctypes.addressof(t_ms), ctypes.addressof(cnt))
        if cnt.value:
            breakdown[name] = {"ms": round(t_ms.value, 3), "launches": int(cnt.value)}
    lib.b200la_profile_start(1 << 10)
    barrier(world)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(steps):
        step()
    e1.record(stream)
    torch.cuda.synchronize()
    barrier(world)
    k_ms, k_n = ctypes.c_double(0), ctypes.c_int64(0)
    lib.b200la_profile_stop(10, ctypes.addressof(k_ms), ctypes.addressof(k_n))
    t_inv = max_over_ranks(world, e0.elapsed_time(e1) / steps) / 1e3
    res = (torch.mm(A, m) - torch.eye(n, dtype=A.dtype, device=dev)).abs().max().item()
    xnorm = torch.linalg.matrix_norm(m, ord=float("inf")).item()
    anorm = torch.linalg.matrix_norm(A, ord=float("inf")).item()
    gflops = inversion_gemm_flops(n)
    peak = measured_fp64_peak_tflops()
    achieved = gflops * steps / (k_ms.value * 1e-3) / 1e12 if k_ms.value else None

    # determinant, LU mode (factor + diagonal product), host-synchronous
    m.copy_(A)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    d = la.det(m, piv)
    t_det = time.perf_counter() - t0

    out = {"n": n, "inverse_s": t_inv, "steps": steps,
           "residual_max_abs_AX_minus_I": res,
           "residual_bound_2n_eps_normA_normX": 2 * n * EPS64 * anorm * xnorm,
           "determinant_s": t_det, "log_abs_det": d["log_abs"], "det_sign": d["sign"],
           "roofline": {"kernel": "inversion_gemm (k_dmma_update, DMMA m8n8k4)", "bound": "fp64",
                        "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                        "frac": achieved / peak if achieved else None,
                        "peak_source": "cuBLAS DGEMM 8192^3 via torch.matmul, best of 5, measured in this run",
                        "flops_per_step": gflops, "launches": int(k_n.value),
                        "share_of_step": (k_ms.value / steps / 1e3) / t_inv if t_inv else None},
           "breakdown_one_step": breakdown}
    del m, ws
    torch.cuda.empty_cache()
    path = os.path.join(ROOT, "baseline", "_ref", "libref_cublas.so")
    if rank == 0 and world == 1 and os.path.exists(path):
        out["cuda_blas"] = cuda_blas_inverse(path, A, stream, steps)
        out["speedup_vs_cuda_blas"] = out["cuda_blas"]["inverse_s"] / t_inv
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        import numpy as np
        from oracle import Oracle, available
        kind = "reference" if available("reference") else "port"
        o = Oracle(kind)
        ns = 768
        a = np.random.default_rng(ns).standard_normal((ns, ns))
        t0 = time.perf_counter()
        o.getri(a)
        t = time.perf_counter() - t0
        out["cpu_baseline"] = {"value": t * (n / ns) ** 3, "unit": "s", "cores": 1, "kind": kind,
                               "sample": f"inversion<double,NATIVE> LU mode at n={ns} ({t:.2f} s) scaled by "
                                         f"(n/{ns})^3 to n={n}; 1 thread"}
    del A
    torch.cuda.empty_cache()
    return out


# ---------------------------------------------------------------------------
# Cholesky modes of linear_solver: this library vs the reference's CUDA_BLAS
# path (cuSOLVER potrf + potrs, baseline/_ref) at the same order
# ---------------------------------------------------------------------------
def cholesky_update_flops(n: int, nb: int = 64) -> int:
    """Algorithmic flops of the trailing updates (k_chol_syrk): for each full
    block, 2 * 64 per entry of the trailing lower triangle."""
    fl = 0
    for k in range(0, n, nb):
        below = n - k - nb
        if below > 0:
            fl += 2 * nb * below * (below + 1) // 2
    return fl


def cuda_blas_cholesky(lib_path, A, b, stream, steps):
    import torch
    lib = ctypes.CDLL(lib_path)
    lib.ref_cublas_dcholesky_solve_workspace_size.restype = ctypes.c_size_t
    lib.ref_cublas_dcholesky_solve_workspace_size.argtypes = [ctypes.c_int64]
    lib.ref_cublas_dcholesky_solve.argtypes = [ctypes.c_void_p, ctypes.c_int64, ctypes.c_void_p, ctypes.c_void_p,
                                               ctypes.c_size_t, ctypes.c_void_p]
    lib.ref_cublas_last_error.restype = ctypes.c_char_p
    n = A.shape[0]
    nb = int(lib.ref_cublas_dcholesky_solve_workspace_size(n))
    ws = torch.empty(max(nb, 256), dtype=torch.uint8, device=A.device)
    m, x = torch.empty_like(A), torch.empty_like(b)

    def step():
        m.copy_(A)
        x.copy_(b)
        if lib.ref_cublas_dcholesky_solve(m.data_ptr(), n, x.data_ptr(), ws.data_ptr(), nb, stream.cuda_stream) != 0:
            raise RuntimeError(lib.ref_cublas_last_error().decode())

    step()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(steps):
        step()
    e1.record(stream)
    torch.cuda.synchronize()
    t = e0.elapsed_time(e1) / steps / 1e3
    r = (torch.mv(A, x) - b).abs().max().item()
    eta = r / (torch.linalg.matrix_norm(A, ord=float("inf")).item() * x.abs().max().item() + b.abs().max().item())
    del m, x, ws
    torch.cuda.empty_cache()
    return {"s": t, "backward_error": eta, "steps": steps,
            "what": "the reference's linear_solver<double,CUDA_BLAS> CHOLESKY mode (cuSOLVER potrf + potrs)"}


def run_cholesky(args, world, rank, local):
    """linear_solver<double, B200> CHOLESKY mode at order args.chol_n: each
    step restores m and x (device copies), factors (bit-identical to the
    reference's NATIVE factor) and solves in place."""
    import torch

    import linearalgebra_b200 as la
    from linearalgebra_b200 import _lib

    lib = _lib.load()
    n = args.chol_n
    dev = torch.device("cuda", local)
    gen = torch.Generator(device=dev)
    gen.manual_seed(SEED + 2 + rank)
    R = torch.randn(n, n, dtype=torch.float64, device=dev, generator=gen)
    A = torch.mm(R, R.t())
    A.diagonal().add_(float(n))
    del R
    b = torch.randn(n, dtype=torch.float64, device=dev, generator=gen)
    m, x = torch.empty_like(A), torch.empty_like(b)
    piv = torch.empty(n, dtype=torch.int64, device=dev)
    nbytes = la.linear_solver.workspace_size(n, la.CHOLESKY_LINEAR_SOLVER)
    ws = torch.empty(max(nbytes, 256), dtype=torch.uint8, device=dev)
    stream = torch.cuda.current_stream(dev)

    def step():
        m.copy_(A)
        x.copy_(b)
        la.linear_solver.apply(m, piv, n, x, la.CHOLESKY_LINEAR_SOLVER, ws, nbytes, stream)

    steps = 3
    step()
    torch.cuda.synchronize()
    lib.b200la_profile_start(sum(1 << c for c in CLASS_NAMES))
    step()
    torch.cuda.synchronize()
    breakdown = {}
    for c, name in CLASS_NAMES.items():
        t_ms, cnt = ctypes.c_double(0), ctypes.c_int64(0)
        lib.b200la_profile_stop(c, ctypes.addressof(t_ms), ctypes.addressof(cnt))
        if cnt.value:
            breakdown[name] = {"ms": round(t_ms.value, 3), "launches": int(cnt.value)}
    lib.b200la_profile_start(1 << 12)
    barrier(world)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(steps):
        step()
    e1.record(stream)
    torch.cuda.synchronize()
    barrier(world)
    k_ms, k_n = ctypes.c_double(0), ctypes.c_int64(0)
    lib.b200la_profile_stop(12, ctypes.addressof(k_ms), ctypes.addressof(k_n))
    t = max_over_ranks(world, e0.elapsed_time(e1) / steps) / 1e3
    r = (torch.mv(A, x) - b).abs().max().item()
    eta = r / (torch.linalg.matrix_norm(A, ord=float("inf")).item() * x.abs().max().item() + b.abs().max().item())
    fl = cholesky_update_flops(n)
    # every product of the update is rounded on its own (the reference's
    # compiled loop), so it runs as a DMUL and a DADD on the FP64 pipe, not
    # as fused or tensor-core work: its bound is half the FP64 peak
    peak = measured_fp64_peak_tflops() / 2
    achieved = fl * steps / (k_ms.value * 1e-3) / 1e12 if k_ms.value else None
    out = {"n": n, "s": t, "steps": steps, "backward_error": eta,
           "roofline": {"kernel": "k_chol_syrk (trailing lower-triangle update, FP64 pipe)", "bound": "fp64_unfused",
                        "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                        "frac": achieved / peak if achieved else None,
                        "peak_source": "half of cuBLAS DGEMM 8192^3 (torch.matmul, best of 5, measured in this run): "
                                       "one separately rounded multiply and one add per term",
                        "flops_per_step": fl, "launches": int(k_n.value),
                        "share_of_step": (k_ms.value / steps / 1e3) / t if t else None},
           "breakdown_one_step": breakdown}
    del m, x, ws
    torch.cuda.empty_cache()
    path = os.path.join(ROOT, "baseline", "_ref", "libref_cublas.so")
    if rank == 0 and world == 1 and os.path.exists(path):
        out["cuda_blas"] = cuda_blas_cholesky(path, A, b, stream, steps)
        out["speedup_vs_cuda_blas"] = out["cuda_blas"]["s"] / t
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        import numpy as np
        from oracle import Oracle, available
        from linearalgebra_b200.workloads import spd_matrix
        kind = "reference" if available("reference") else "port"
        o = Oracle(kind)
        ns = 3072
        a = spd_matrix(ns, seed=ns)
        bb = np.ones(ns)
        t0 = time.perf_counter()
        o.gesv(a, bb, 3)
        tc = time.perf_counter() - t0
        out["cpu_baseline"] = {"value": tc * (n / ns) ** 3, "unit": "s", "cores": 1, "kind": kind,
                               "sample": f"linear_solver<double,NATIVE> CHOLESKY mode at n={ns} ({tc:.2f} s) "
                                         f"scaled by (n/{ns})^3 to n={n}; 1 thread"}
    del A, b
    torch.cuda.empty_cache()
    return out


# ---------------------------------------------------------------------------
# transpose: in place (square: one read and one write per element) and out of
# place, vs the reference's CUDA_BLAS transpose (geam into scratch + copy)
# ---------------------------------------------------------------------------
def run_transpose(args, world, rank, local):
    import torch

    import linearalgebra_b200 as la
    from linearalgebra_b200 import api

    dev = torch.device("cuda", local)
    stream = torch.cuda.current_stream(dev)
    pk = measured_peaks()
    peak, peak_src = pk["hbm_gbs"], pk["source"]
    n = args.tp_n
    m = torch.randn(n, n, dtype=torch.float64, device=dev)
    dst = torch.empty_like(m)

    def timed(fn, steps=5):
        fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(steps):
            fn()
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / steps / 1e3

    # an even number of in-place transposes leaves m as it was
    t_sq = timed(lambda: api.transpose.apply(n, n, m, None, 0, stream), steps=6)
    t_out = timed(lambda: la.transpose_out(m, dst, stream))
    rows, cols = n // 2, n * 2
    r = torch.randn(rows, cols, dtype=torch.float64, device=dev)
    nb = api.transpose.workspace_size(rows, cols)
    ws = torch.empty(nb, dtype=torch.uint8, device=dev)
    state = {"shape": (rows, cols)}

    def rect():
        rr, cc = state["shape"]
        api.transpose.apply(rr, cc, r, ws, nb, stream)
        state["shape"] = (cc, rr)

    t_rect = timed(rect, steps=4)
    sq_bytes = 16 * n * n
    out = {"square": {"n": n, "s": t_sq, "bytes": sq_bytes, "gbs": sq_bytes / t_sq / 1e9},
           "out_of_place": {"n": n, "s": t_out, "bytes": sq_bytes, "gbs": sq_bytes / t_out / 1e9},
           "rectangular_in_place": {"rows": rows, "columns": cols, "s": t_rect, "bytes": 32 * rows * cols,
                                    "gbs": 32 * rows * cols / t_rect / 1e9,
                                    "note": "transpose into the workspace, then one device copy back"},
           "roofline": {"kernel": f"k_transpose_square (in place, n={n} FP64)", "bound": "hbm",
                        "achieved": sq_bytes / t_sq / 1e9, "peak": peak, "unit": "GB/s",
                        "frac": sq_bytes / t_sq / 1e9 / peak, "peak_source": peak_src},
           "dtype": "f64"}
    del r, ws
    path = os.path.join(ROOT, "baseline", "_ref", "libref_cublas.so")
    if rank == 0 and world == 1 and os.path.exists(path):
        lib = ctypes.CDLL(path)
        lib.ref_cublas_dtranspose_workspace_size.restype = ctypes.c_size_t
        lib.ref_cublas_dtranspose_workspace_size.argtypes = [ctypes.c_int64, ctypes.c_int64]
        lib.ref_cublas_dtranspose.argtypes = [ctypes.c_int64, ctypes.c_int64, ctypes.c_void_p, ctypes.c_void_p,
                                              ctypes.c_size_t, ctypes.c_void_p]
        rb = int(lib.ref_cublas_dtranspose_workspace_size(n, n))
        rws = torch.empty(max(rb, 256), dtype=torch.uint8, device=dev)

        def ref_step():
            if lib.ref_cublas_dtranspose(n, n, m.data_ptr(), rws.data_ptr(), rb, stream.cuda_stream) != 0:
                raise RuntimeError("reference transpose failed")

        t_ref = timed(ref_step, steps=6)
        out["cuda_blas"] = {"s": t_ref, "what": "the reference's transpose<double,CUDA_BLAS> (cuBLAS geam into "
                                                f"scratch, device copy back), n={n} in place"}
        out["speedup_vs_cuda_blas"] = t_ref / t_sq
        del rws
    del m, dst
    torch.cuda.empty_cache()
    return out


# ---------------------------------------------------------------------------
# multiplication: FP64 general product on the tensor cores vs measured cuBLAS
# DGEMM, and batched_matrix_multiplication vs the reference's CUDA kernel
# ---------------------------------------------------------------------------
def run_multiplication(args, world, rank, local):
    import torch

    import linearalgebra_b200 as la

    dev = torch.device("cuda", local)
    stream = torch.cuda.current_stream(dev)
    out = {}

    def timed(fn, steps):
        fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(steps):
            fn()
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / steps / 1e3

    n = 8192
    gen = torch.Generator(device=dev)
    gen.manual_seed(SEED + 2 + rank)
    a = torch.randn(n, n, dtype=torch.float64, device=dev, generator=gen)
    b = torch.randn(n, n, dtype=torch.float64, device=dev, generator=gen)
    c = torch.empty_like(a)
    t = timed(lambda: la.gemm(False, False, 1.0, a, b, 0.0, c, stream), 3)
    peak = measured_fp64_peak_tflops()
    out["general_fp64"] = {"shape": f"{n}x{n}x{n} NN, alpha 1, beta 0", "s": t,
                           "tflops": 2 * n ** 3 / t / 1e12, "measured_dgemm_tflops": peak,
                           "frac_of_dgemm": 2 * n ** 3 / t / 1e12 / peak,
                           "note": "bit-identical to the reference NATIVE loop (fma chain in k order)"}
    del a, b, c
    torch.cuda.empty_cache()

    path = os.path.join(ROOT, "baseline", "_ref", "libref_cublas.so")
    ref = None
    if rank == 0 and world == 1 and os.path.exists(path):
        ref = ctypes.CDLL(path)
        for nm in ("ref_cublas_dgemm_batched", "ref_cublas_sgemm_batched"):
            getattr(ref, nm).argtypes = [ctypes.c_int64, ctypes.c_int64] + [ctypes.c_void_p] * 4
    for dtype, tag in ((torch.float64, "d"), (torch.float32, "s")):
        dim, count = 256, 1000
        a = torch.randn(count, dim, dim, dtype=dtype, device=dev, generator=gen)
        b = torch.randn(count, dim, dim, dtype=dtype, device=dev, generator=gen)
        c = torch.empty_like(a)
        t = timed(lambda: la.batched_matrix_multiplication(dim, count, a, b, c, stream), 3)
        entry = {"dim": dim, "count": count, "s": t, "tflops": 2 * dim ** 3 * count / t / 1e12}
        if ref is not None:
            rc = torch.empty_like(a)
            fn = getattr(ref, f"ref_cublas_{tag}gemm_batched")
            tr = timed(lambda: fn(dim, count, a.data_ptr(), b.data_ptr(), rc.data_ptr(), stream.cuda_stream), 3)
            entry["reference_kernel_s"] = tr
            entry["speedup_vs_reference_kernel"] = tr / t
            entry["bit_identical_to_reference_kernel"] = bool(torch.equal(c, rc))
        out[f"batched_{'fp64' if tag == 'd' else 'fp32'}"] = entry
        del a, b, c
        torch.cuda.empty_cache()
    return out


# ---------------------------------------------------------------------------
# CPU: the reference's own NATIVE linear_solver (oracle/_ref), single thread
# ---------------------------------------------------------------------------
def cpu_reference_solve_seconds(n: int, repeats: int = 1):
    import numpy as np

    from linearalgebra_b200.workloads import system
    from oracle import Oracle, available

    kind = "reference" if available("reference") else "port"
    orc = Oracle(kind)
    a, _, b = system(n, seed=SEED)
    times = []
    for _ in range(repeats):
        t0 = time.perf_counter()
        _, _, x = orc.gesv(a, b)
        times.append(time.perf_counter() - t0)
    eta = Oracle("port").backward_error(a, x, b) if available("port") else None
    return kind, statistics.median(times), eta


def cpu_model():
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


# ---------------------------------------------------------------------------
# GPU baseline: the reference's own CUDA_BLAS LU solve (cuSOLVER), when built
# ---------------------------------------------------------------------------
def cusolver_reference_seconds(A, b, stream, steps: int = 2):
    """linear_solver<double, CUDA_BLAS> LU mode from baseline/_ref on the same
    system, timed with CUDA events on `stream` (each step restores A and b
    by device copies, as the FP64 arm does)."""
    import torch

    path = os.path.join(ROOT, "baseline", "_ref", "libref_cublas.so")
    if not os.path.exists(path):
        return {"unavailable": "baseline/_ref/libref_cublas.so is not built (needs the reference sources)"}
    lib = ctypes.CDLL(path)
    lib.ref_cublas_dgesv_workspace_size.restype = ctypes.c_size_t
    lib.ref_cublas_dgesv_workspace_size.argtypes = [ctypes.c_int64]
    lib.ref_cublas_dgesv.restype = ctypes.c_int
    lib.ref_cublas_dgesv.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64, ctypes.c_void_p,
                                     ctypes.c_void_p, ctypes.c_size_t, ctypes.c_void_p]
    lib.ref_cublas_last_error.restype = ctypes.c_char_p
    n = A.shape[0]
    nbytes = int(lib.ref_cublas_dgesv_workspace_size(n))
    ws = torch.empty(max(nbytes, 256), dtype=torch.uint8, device=A.device)
    m = torch.empty_like(A)
    xx = torch.empty_like(b)
    piv = torch.empty(n, dtype=torch.int64, device=A.device)

    def step():
        m.copy_(A)
        xx.copy_(b)
        if lib.ref_cublas_dgesv(m.data_ptr(), piv.data_ptr(), n, xx.data_ptr(), ws.data_ptr(), nbytes,
                                stream.cuda_stream) != 0:
            raise RuntimeError(lib.ref_cublas_last_error().decode())

    step()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(steps):
        step()
    e1.record(stream)
    torch.cuda.synchronize()
    r = b - A @ xx
    eta = (r.abs().max() / (A.abs().sum(1).max() * xx.abs().max() + b.abs().max())).item()
    out = {"value": e0.elapsed_time(e1) / steps / 1e3, "unit": "s", "backward_error": eta, "steps": steps,
           "what": "the reference's linear_solver<double,CUDA_BLAS> LU mode (cuSOLVER getrf/getrs with the "
                   "reference's row/column-major transposes and host pivot round trip), same system"}
    del m, xx, piv, ws
    torch.cuda.empty_cache()
    return out


# ---------------------------------------------------------------------------
# B200 arm
# ---------------------------------------------------------------------------
# DRAM bytes (ncu dram__bytes_read.sum + dram__bytes_write.sum) per algorithmic
# byte of the dominant kernels, from one capture each on a smaller case
# (profiles/): the persistent tensor-core update at n=4096 (the M=3328,
# N=3072 launch beside the panels: 55.0 of 81.8 MB; its last tiles' C writes
# were still in L2 when the launch ended) and the FP64 trailing update (DMMA
# band kernel) at n=4096 (rest=3712: 168.8 of 220.5 MB).  Traffic grows with
# the C tile bytes, so it scales to a full launch by the algorithmic bytes.
TRAFFIC_PER_ALGORITHMIC_BYTE = {5: 0.673, 2: 0.766}

CLASS_NAMES = {0: "panel", 1: "laswp_u12", 2: "trailing", 3: "solve", 4: "gemm", 5: "tc_update",
               6: "residual", 7: "batched", 8: "operand_prep", 9: "selector", 10: "inversion_gemm",
               11: "inversion_aux", 12: "cholesky_update", 13: "cholesky_aux", 14: "transpose"}


def algorithmic_work(n: int, method: str, nb_out: int = 256):
    """Per-step algorithmic flops / bytes of the kernel classes that have a
    roofline, for one solve of order n (nrhs = 1)."""
    work = {}
    if method == "fp64":
        fl = sum(2 * (n - k - min(64, n - k)) ** 2 * min(64, n - k) for k in range(0, n, 64))
        work[2] = {"bound": "fp64", "flops": fl, "bytes": 16 * sum((n - k - 64) ** 2 for k in range(0, n, 64) if n - k > 64)}
    else:
        fl, by = 0, 0
        for K in range(0, n, nb_out):
            rest = n - min(K + nb_out, n)
            if rest > 0:
                fl += 2 * rest * rest * nb_out
                by += 8 * rest * rest
        work[5] = {"bound": "hbm", "flops": fl, "bytes": by}
        work[6] = {"bound": "hbm", "flops": 2 * n * n, "bytes": 8 * n * n}
    return work


def batched_roofline(sizes, status, seconds, prec, dev) -> dict:
    """Both ceilings of the batched solve.  Compute: 2 n^3 / 3 per system
    against the CUDA cores' nominal FP32 (FP64: half) rate at the maximum SM
    clock.  Memory: the algorithmic bytes per system, (c + 2) (8 + e) n^2 for
    c corrections and factor elements of e bytes (A read once for the copy
    and once per solve for the residual, the factor written once and read
    once per solve), against the measured HBM copy bandwidth."""
    import numpy as np
    import torch

    es = 4 if prec == "fp32" else 8
    st = np.asarray(status)
    corr = np.maximum(np.where(st >= 1000, st - 1000, st), 0).astype(np.float64)
    n = np.asarray(sizes, dtype=np.float64)
    flops = float((2.0 * n ** 3 / 3).sum())
    nbytes = float(((corr + 2) * (8 + es) * n * n).sum())
    sms = torch.cuda.get_device_properties(dev).multi_processor_count
    simt_peak = sms * (128 if prec == "fp32" else 64) * 2 * 1965e6 / 1e12
    pk = measured_peaks()
    tflops = flops / seconds / 1e12
    gbs = nbytes / seconds / 1e9
    return {"bound": "latency (both fractions low)" if max(tflops / simt_peak, gbs / pk["hbm_gbs"]) < 0.5
            else ("simt" if tflops / simt_peak >= gbs / pk["hbm_gbs"] else "hbm"),
            "tflops": tflops, "simt_peak_tflops": simt_peak, "simt_frac": tflops / simt_peak,
            "simt_peak_source": f"nominal: {sms} SMs x {128 if prec == 'fp32' else 64} FMA/clk x 1965 MHz",
            "gbs": gbs, "hbm_peak_gbs": pk["hbm_gbs"], "hbm_frac": gbs / pk["hbm_gbs"],
            "hbm_peak_source": pk["source"], "algorithmic_bytes_per_batch": nbytes, "flops_per_batch": flops}


def run_batched(args, world, rank, local):
    """Config 4: 20,000 uneven systems (n uniform in [16, 512], half
    diagonally dominant), FP32 factors + FP64 refinement to eta <= 1e-14 in one
    persistent launch replayed as a CUDA graph; beside it the batched plain
    FP64 LU and a loop of single-system mixed solves (sampled)."""
    import numpy as np
    import torch

    import linearalgebra_b200 as la
    from linearalgebra_b200.batched import BatchedSolver, make_batch, shard

    dev = torch.device("cuda", local)
    count = args.batch_count
    sizes, a, b, x_true = make_batch(count, seed=SEED, device=dev)
    mine = shard(sizes, world, rank)
    if len(mine) < count:  # this rank's shard, repacked
        offa = np.concatenate([[0], np.cumsum(sizes.astype(np.int64) ** 2)[:-1]])
        offv = np.concatenate([[0], np.cumsum(sizes)[:-1]])
        a = torch.cat([a[int(offa[i]):int(offa[i]) + int(sizes[i]) ** 2] for i in mine])
        b = torch.cat([b[int(offv[i]):int(offv[i]) + int(sizes[i])] for i in mine])
        sizes = sizes[mine]
    out = {}
    x = torch.empty_like(b)
    for prec in ("fp32", "fp64"):
        solver = BatchedSolver(sizes, prec, dev, tolerance=1e-14, max_iterations=10 if prec == "fp32" else 2)
        tune = solver.autotune(a, b, x) if prec == "fp32" else {"nb_table": solver.nb_table_h}
        solver.capture(a, b, x)
        for _ in range(max(1, args.warmup)):
            solver.replay()
        torch.cuda.synchronize(dev)
        barrier(world)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        reps = max(1, min(args.steps, 3))
        e0.record()
        for _ in range(reps):
            solver.replay()
        e1.record()
        torch.cuda.synchronize(dev)
        t = max_over_ranks(world, e0.elapsed_time(e1) / reps / 1e3)
        berr = solver.berr.max().item()
        st = solver.status.cpu().numpy()
        out[prec] = {"solves_per_s": count / t, "ms_per_batch": t * 1e3, "max_backward_error": berr,
                     "converged": int(((st >= 0) & (st < 1000)).sum() + (st >= 1000).sum()),
                     "escalated_to_fp64": int((st >= 1000).sum()), "not_converged": int((st == -1000000).sum()),
                     "max_corrections": int(np.where(st >= 1000, st - 1000, st).max()),
                     "singular": int(((st < 0) & (st != -1000000)).sum()), "nb_table": tune["nb_table"]}
        out[prec]["roofline"] = batched_roofline(sizes, st, t, prec, dev)
        del solver
    # a loop of single-system solves through the one-system mixed solver (sampled)
    if rank == 0:
        rng = np.random.default_rng(1)
        idx = rng.choice(len(sizes), size=min(100, len(sizes)), replace=False)
        offa = np.concatenate([[0], np.cumsum(sizes.astype(np.int64) ** 2)[:-1]])
        offv = np.concatenate([[0], np.cumsum(sizes)[:-1]])
        solvers = {}
        torch.cuda.synchronize(dev)
        t0 = time.perf_counter()
        for i in idx:
            n = int(sizes[i])
            if n not in solvers:
                solvers[n] = la.MixedSolver(n, 1, dev, precision="fp32", tolerance=1e-14)
            av = a[int(offa[i]):int(offa[i]) + n * n]
            bv = b[int(offv[i]):int(offv[i]) + n]
            solvers[n](av, bv)
        torch.cuda.synchronize(dev)
        # exclude the one-time workspace allocations: time a second pass
        t0 = time.perf_counter()
        for i in idx:
            n = int(sizes[i])
            av = a[int(offa[i]):int(offa[i]) + n * n]
            bv = b[int(offv[i]):int(offv[i]) + n]
            solvers[n](av, bv)
        torch.cuda.synchronize(dev)
        tl = (time.perf_counter() - t0) / len(idx)
        out["loop_single"] = {"solves_per_s": 1.0 / tl, "sample": f"{len(idx)} systems of the batch, "
                              "b200la_dsolve_mixed one at a time (FP32 factors, FP64 refinement to 1e-14), "
                              "workspaces preallocated, host wall clock"}
        out["speedup_vs_loop"] = out["fp32"]["solves_per_s"] / out["loop_single"]["solves_per_s"]
        out["speedup_vs_batched_fp64"] = out["fp32"]["solves_per_s"] / out["fp64"]["solves_per_s"]
    out["count"] = count
    out["systems_this_rank"] = int(len(sizes))
    out["data"] = ("synthetic: n uniform in [16,512], A iid N(0,1) + n*I on every other system, "
                   f"x_true iid U[-1,1] (seed {SEED})")
    out["flops_per_batch"] = float(sum(2.0 * int(n) ** 3 / 3 for n in sizes))
    return out


# ---------------------------------------------------------------------------
# n = 512: plain FP64 LU + solve (latency-bound), beside the
# mixed solve and the reference's NATIVE CPU solve of the same system
# ---------------------------------------------------------------------------
def run_n512(args, local, fp64_peak):
    import numpy as np
    import torch

    import linearalgebra_b200 as la
    from linearalgebra_b200 import _lib
    from linearalgebra_b200.workloads import system
    from oracle import Oracle

    lib = _lib.load()
    n = 512
    dev = torch.device("cuda", local)
    stream = torch.cuda.current_stream(dev)
    sp = stream.cuda_stream
    a, x_true, b = system(n, seed=512)
    A = torch.from_numpy(a).to(dev)
    B = torch.from_numpy(b).to(dev)
    m, x = torch.empty_like(A), torch.empty_like(B)
    piv = torch.empty(n, dtype=torch.int64, device=dev)
    nbytes = lib.b200la_dgesv_workspace_size(n, la.LU_LINEAR_SOLVER)
    ws = torch.empty(nbytes, dtype=torch.uint8, device=dev)

    def step():
        m.copy_(A)
        x.copy_(B)
        _lib.check(lib.b200la_dgesv(m.data_ptr(), piv.data_ptr(), n, x.data_ptr(), la.LU_LINEAR_SOLVER,
                                    ws.data_ptr(), nbytes, sp))

    def timed(fn, reps=50):
        for _ in range(5):
            fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(reps):
            fn()
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / reps / 1e3

    t64 = timed(step)
    port = Oracle("port")
    eta64 = port.backward_error(a, x.cpu().numpy(), b)
    flops = 2 * n ** 3 / 3 + 2 * n * n
    solver = la.MixedSolver(n, 1, dev, precision="fp32", tolerance=1e-14)
    xm = torch.empty_like(B)
    res = {}

    def mstep():
        _, r, _ = solver(A, B, xm, stream)
        res.update(r)

    tm = timed(mstep, reps=20)
    etam = port.backward_error(a, xm.cpu().numpy(), b)
    kind, tcpu, etacpu = cpu_reference_solve_seconds(n, repeats=5)
    return {"n": n, "workload": "A iid N(0,1), x_true iid U[-1,1], b = A x_true (numpy seed 512), nrhs=1",
            "fp64_lu_solve_s": t64, "fp64_backward_error": eta64,
            "fp64_tflops": flops / t64 / 1e12, "fp64_frac_of_measured_dgemm": flops / t64 / 1e12 / fp64_peak,
            "mixed_fp32_ir_s": tm, "mixed_backward_error": etam, "mixed_iterations": res.get("iterations"),
            "reference_native_cpu_s": tcpu, "reference_native_backward_error": etacpu,
            "reference_kind": kind, "bound_10_n_eps": 10 * n * EPS64,
            "note": "device time per solve incl. the 2 MiB device copies restoring A and b; latency-bound "
                    "(the FP64 fraction is of measured cuBLAS DGEMM 8192^3)"}


# ---------------------------------------------------------------------------
# n = 16384, the rest: BF16 and FP16 factorizations and nrhs = 64
# ---------------------------------------------------------------------------
def run_n16384_more(args, A, b, stream, local):
    import torch

    import linearalgebra_b200 as la
    from linearalgebra_b200 import _lib

    lib = _lib.load()
    n = A.shape[0]
    dev = A.device
    sp = stream.cuda_stream
    anorm = A.abs().sum(1).max()

    def eta_of(xx, bb):
        r = bb - A @ xx
        if r.dim() == 1:
            return (r.abs().max() / (anorm * xx.abs().max() + bb.abs().max())).item()
        return ((r.abs().amax(0)) / (anorm * xx.abs().amax(0) + bb.abs().amax(0))).max().item()

    def timed(fn, reps=2):
        fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(reps):
            fn()
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / reps / 1e3

    out = {}
    x = torch.empty_like(b)
    for prec in ("bf16", "fp16"):
        solver = la.MixedSolver(n, 1, dev, precision=prec, tolerance=1e-14)
        res = {}

        def st(solver=solver, res=res):
            _, r, _ = solver(A, b, x, stream)
            res.update(r)

        t = timed(st)
        out[prec] = {"s": t, "backward_error": eta_of(x, b),
                     **{k: res[k] for k in ("precision_used", "iterations", "gmres_iterations", "escalations",
                                            "converged", "factor_ms", "refine_ms")}}
        del solver
        torch.cuda.empty_cache()
    # nrhs = 64: mixed FP32 LU-IR and the plain FP64 LU + multi-RHS solve
    nrhs = 64
    g = torch.Generator(device=dev)
    g.manual_seed(SEED + 64)
    xt = torch.rand(n, nrhs, dtype=torch.float64, device=dev, generator=g) * 2 - 1
    B = A @ xt
    X = torch.empty_like(B)
    solver = la.MixedSolver(n, nrhs, dev, precision="fp32", tolerance=1e-14)
    res = {}

    def st64():
        _, r, _ = solver(A, B, X, stream)
        res.update(r)

    t = timed(st64)
    out["nrhs64_mixed_fp32"] = {"s": t, "backward_error_max_over_columns": eta_of(X, B),
                                "forward_error": ((X - xt).abs().max() / xt.abs().max()).item(),
                                **{k: res[k] for k in ("precision_used", "iterations", "gmres_iterations",
                                                       "escalations", "converged", "factor_ms", "refine_ms")}}
    del solver
    torch.cuda.empty_cache()
    m = torch.empty_like(A)
    piv = torch.empty(n, dtype=torch.int64, device=dev)
    fb = lib.b200la_dgetrf_workspace_size(n)
    sb = lib.b200la_dgetrs_workspace_size(n, nrhs)
    ws = torch.empty(max(fb, sb), dtype=torch.uint8, device=dev)

    def st_fp64():
        m.copy_(A)
        X.copy_(B)
        _lib.check(lib.b200la_dgetrf_async(m.data_ptr(), n, piv.data_ptr(), ws.data_ptr(), fb, sp))
        _lib.check(lib.b200la_dgetrs(m.data_ptr(), piv.data_ptr(), n, nrhs, X.data_ptr(), nrhs, ws.data_ptr(),
                                     sb, sp))

    t64 = timed(st_fp64)
    out["nrhs64_fp64"] = {"s": t64, "backward_error_max_over_columns": eta_of(X, B),
                          "what": "plain FP64 LU (bit-identical factors) + 64-column triangular solves"}
    out["nrhs64_speedup_mixed_vs_fp64"] = t64 / out["nrhs64_mixed_fp32"]["s"]
    del m, ws, B, X, xt
    torch.cuda.empty_cache()
    return out


# ---------------------------------------------------------------------------
# conditioning sweep, n in {4096, 8192}, kappa 1e2 .. 1e10,
# FP8-E4M3 / BF16 / FP32 factorizations against the FP64 oracle solution
# ---------------------------------------------------------------------------
KAPPAS = (1e2, 1e4, 1e6, 1e8, 1e10)
SWEEP_PRECISIONS = ("fp8", "bf16", "fp32")


def run_conditioning_sweep(args, local):
    import torch

    import linearalgebra_b200 as la
    from linearalgebra_b200 import _lib
    from linearalgebra_b200.selector import conditioned_device

    lib = _lib.load()
    dev = torch.device("cuda", local)
    stream = torch.cuda.current_stream(dev)
    sp = stream.cuda_stream
    rows = []
    for n in (4096, 8192):
        solvers = {p: la.MixedSolver(n, 1, dev, precision=p, tolerance=1e-14) for p in SWEEP_PRECISIONS}
        m = torch.empty(n, n, dtype=torch.float64, device=dev)
        piv = torch.empty(n, dtype=torch.int64, device=dev)
        nbytes = lib.b200la_dgesv_workspace_size(n, la.LU_LINEAR_SOLVER)
        ws = torch.empty(nbytes, dtype=torch.uint8, device=dev)
        for ki, kappa in enumerate(KAPPAS):
            seed = 3000 + 10 * ki + n
            A = conditioned_device(n, kappa, seed, device=dev)
            g = torch.Generator(device=dev)
            g.manual_seed(seed)
            xt = torch.rand(n, dtype=torch.float64, device=dev, generator=g) * 2 - 1
            b = A @ xt
            anorm = A.abs().sum(1).max()
            # the FP64 oracle solution: plain FP64 LU, factors bit-identical to the reference's
            m.copy_(A)
            x64 = b.clone()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            _lib.check(lib.b200la_dgesv(m.data_ptr(), piv.data_ptr(), n, x64.data_ptr(), la.LU_LINEAR_SOLVER,
                                        ws.data_ptr(), nbytes, sp))
            e1.record(stream)
            torch.cuda.synchronize()

            def errs(xx):
                r = b - A @ xx
                return ((r.abs().max() / (anorm * xx.abs().max() + b.abs().max())).item(),
                        ((xx - xt).abs().max() / xt.abs().max()).item(),
                        ((xx - x64).abs().max() / x64.abs().max()).item())

            eta64, fwd64, _ = errs(x64)
            row = {"n": n, "kappa": kappa, "seed": seed,
                   "fp64_oracle": {"ms": e0.elapsed_time(e1), "backward_error": eta64, "forward_error": fwd64}}
            for prec in SWEEP_PRECISIONS:
                x = torch.empty_like(b)
                if ki == 0:
                    solvers[prec](A, b, x, stream)  # warm-up of this order and precision
                torch.cuda.synchronize()
                s0, s1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                s0.record(stream)
                _, r, status = solvers[prec](A, b, x, stream)
                s1.record(stream)
                torch.cuda.synchronize()
                eta, fwd, fwd_o = errs(x)
                row[prec] = {"ms": s0.elapsed_time(s1), "status": int(status),
                             "precision_used": _lib.PREC_NAMES.get(r["precision_used"], r["precision_used"]),
                             "iterations": r["iterations"], "gmres_iterations": r["gmres_iterations"],
                             "escalations": r["escalations"], "converged": r["converged"],
                             "backward_error": eta, "forward_error": fwd, "forward_error_vs_fp64_oracle": fwd_o}
            rows.append(row)
            del A, b, xt, x64
        del solvers, m, ws
        torch.cuda.empty_cache()
    return {"construction": "A = U diag(sigma) V^T, U and V products of 8 seeded Householder reflectors, sigma "
                            "geometric from 1 to 1/kappa; x_true iid U[-1,1]; tolerance eta <= 1e-14; "
                            "escalation on (FP8 -> BF16 -> FP32 -> FP64)",
            "fp8_scaling": "power-of-two scale per row of L21 and per column of U12 (finer than per 128x128 block)",
            "rows": rows}


# ---------------------------------------------------------------------------
# the learned precision selector on the held-out stream of systems
# ---------------------------------------------------------------------------
def run_selector(args):
    from linearalgebra_b200 import selector

    net = selector.Network.load()
    summary, recs = selector.evaluate(net, args.selector_systems, seed=2)
    best_fixed = max(("fixed_fp32", "fp64"), key=lambda k: summary[k]["solves_per_s"])
    return {"systems": args.selector_systems, "stream_seed": 2,
            "stream": "n log-uniform in [64, 4096], kappa log-uniform in [1e1, 1e12] (Householder construction)",
            "summary": summary, "best_fixed_policy": best_fixed,
            "selected_vs_best_fixed": summary["selected"]["solves_per_s"] / summary[best_fixed]["solves_per_s"],
            "timing": "host wall clock per solve, synchronized, matrices built on the device beforehand",
            "weights_meta": net.meta}


def run_b200(args, world, rank, local):
    import numpy as np
    import torch

    import linearalgebra_b200 as la
    from linearalgebra_b200 import _lib

    lib = _lib.load()
    n = args.n
    dev = torch.device("cuda", local)
    gen = torch.Generator(device=dev)
    gen.manual_seed(SEED + rank)
    A = torch.randn(n, n, dtype=torch.float64, device=dev, generator=gen)
    x_true = torch.rand(n, dtype=torch.float64, device=dev, generator=gen) * 2 - 1
    b = A @ x_true
    x = torch.empty_like(b)
    stream = torch.cuda.current_stream(dev)
    sp = stream.cuda_stream
    peaks = measured_peaks()

    # ---- the FP64 comparison arm: plain FP64 LU + solve (the reference's algorithm)
    m = torch.empty_like(A)
    xf = torch.empty_like(b)
    piv = torch.empty(n, dtype=torch.int64, device=dev)
    ws_bytes = lib.b200la_dgesv_workspace_size(n, la.LU_LINEAR_SOLVER)
    ws = torch.empty(ws_bytes, dtype=torch.uint8, device=dev)

    def step_fp64():
        m.copy_(A)
        xf.copy_(b)
        _lib.check(lib.b200la_dgesv(m.data_ptr(), piv.data_ptr(), n, xf.data_ptr(),
                                    la.LU_LINEAR_SOLVER, ws.data_ptr(), ws_bytes, sp))

    # ---- the headline arm: mixed-precision LU-IR to eta <= 1e-14
    solver = la.MixedSolver(n, 1, dev, precision=args.precision, tolerance=1e-14)
    last = {}

    def step_mixed():
        _, res, st = solver(A, b, x, stream)
        last.update(res)
        last["status"] = st

    step = step_mixed if args.method == "mixed" else step_fp64
    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()

    # ---- per-class breakdown of one untimed step (picks the roofline kernel)
    lib.b200la_profile_start(sum(1 << c for c in CLASS_NAMES))
    step()
    torch.cuda.synchronize()
    breakdown = {}
    for c, name in CLASS_NAMES.items():
        t_ms, cnt = ctypes.c_double(0), ctypes.c_int64(0)
        lib.b200la_profile_stop(c, ctypes.addressof(t_ms), ctypes.addressof(cnt))
        if cnt.value:
            breakdown[name] = {"ms": round(t_ms.value, 3), "launches": int(cnt.value)}
    work = algorithmic_work(n, args.method)
    roof_cls = max(work, key=lambda c: breakdown.get(CLASS_NAMES[c], {"ms": 0})["ms"])

    # ---- timed region
    clocks = ClockSampler(local)
    launches0 = lib.b200la_launch_count()
    lib.b200la_profile_start(1 << roof_cls)
    barrier(world)
    torch.cuda.synchronize()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    for _ in range(args.steps):
        step()
    ev1.record(stream)
    torch.cuda.synchronize()
    barrier(world)
    elapsed_ms = ev0.elapsed_time(ev1)
    k_ms, k_n = ctypes.c_double(0), ctypes.c_int64(0)
    lib.b200la_profile_stop(roof_cls, ctypes.addressof(k_ms), ctypes.addressof(k_n))
    launches = lib.b200la_launch_count() - launches0
    clk = clocks.stop()
    ms_per_step = max_over_ranks(world, elapsed_ms / args.steps)

    # accuracy of the last solve, checked on the device in FP64
    xs = x if args.method == "mixed" else xf
    r = b - A @ xs
    eta = (r.abs().max() / (A.abs().sum(1).max() * xs.abs().max() + b.abs().max())).item()
    fwd = ((xs - x_true).abs().max() / x_true.abs().max()).item()

    # ---- roofline of the dominant kernel class, timed live over the region
    w = work[roof_cls]
    secs = k_ms.value * 1e-3
    if w["bound"] == "fp64":
        achieved = w["flops"] * args.steps / secs / 1e12 if secs else None
        peak, unit = measured_fp64_peak_tflops(), "TFLOP/s"
        peak_src = ("cuBLAS DGEMM 8192^3 via torch.matmul, best of 5, measured in this run "
                    "(MEASURED_PEAKS.json holds no FP64 figure)")
    else:
        achieved = w["bytes"] * args.steps / secs / 1e9 if secs else None
        peak, unit = peaks["hbm_gbs"], "GB/s"
        peak_src = peaks["source"]
    roofline = {
        "kernel": CLASS_NAMES[roof_cls], "bound": w["bound"], "achieved": achieved, "peak": peak,
        "unit": unit, "frac": achieved / peak if achieved else None,
        "traffic": (w["bytes"] * args.steps / max(1, k_n.value) * TRAFFIC_PER_ALGORITHMIC_BYTE[roof_cls]
                    if roof_cls in TRAFFIC_PER_ALGORITHMIC_BYTE else None),
        "traffic_note": "bytes per launch: the ncu DRAM/algorithmic ratio of a smaller capture (profiles/) "
                        "times this run's algorithmic bytes per launch",
        "peak_source": peak_src, "launches": int(k_n.value),
        "avg_launch_ms": k_ms.value / max(1, k_n.value),
        "share_of_step": (k_ms.value / args.steps) / ms_per_step if ms_per_step else None,
        "algorithmic_per_step": {"flops": w["flops"], "bytes": w["bytes"]},
        "tensor_tflops": (w["flops"] * args.steps / secs / 1e12) if (secs and w["bound"] == "hbm") else None,
    }

    # ---- the panel chain's latency roofline: per-column time of the panel
    # kernels in this step against the measured floor of their per-column
    # exchange (cluster barrier, keys and pivot row through distributed
    # shared memory, two block barriers), 64- and 32-column forms
    panel_roofline = None
    if "panel" in breakdown:
        fws = torch.empty(256, dtype=torch.uint8, device=dev)
        floors = {}
        for width in (64, 32):
            v = ctypes.c_double(0)
            elem = 8 if args.method == "fp64" else 4
            if lib.b200la_panel_exchange_floor(elem, width, 2048, ctypes.addressof(v), fws.data_ptr(), 256,
                                               sp) == 0:
                floors[width] = v.value / 1e3
        us_col = breakdown["panel"]["ms"] * 1e3 / n
        floor = min(floors.values()) if floors else None
        panel_roofline = {
            "kernel": "k_panel_cluster (per-column pivot exchange inside one 16-CTA cluster) and k_panel (grid)",
            "bound": "latency", "unit": "us per column",
            "achieved": us_col, "floor": floor, "floors_by_width": floors,
            "frac": floor / us_col if floor else None,
            "launches": breakdown["panel"]["launches"],
            "note": "achieved = the step's panel-class time (CUDA events around each panel launch, so it includes "
                    "waiting for SMs held by the concurrent trailing update) / n columns; floor = "
                    "b200la_panel_exchange_floor, device-timed, exchange only"}
        del fws

    # ---- the other arm, timed the same way (fewer steps)
    other = {}
    if not args.no_compare:
        ostep = step_fp64 if args.method == "mixed" else step_mixed
        ostep()
        torch.cuda.synchronize()
        o0, o1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ksteps = max(1, min(args.steps, 2))
        o0.record(stream)
        for _ in range(ksteps):
            ostep()
        o1.record(stream)
        torch.cuda.synchronize()
        o_ms = max_over_ranks(world, o0.elapsed_time(o1) / ksteps)
        ox = xf if args.method == "mixed" else x
        rr = b - A @ ox
        oeta = (rr.abs().max() / (A.abs().sum(1).max() * ox.abs().max() + b.abs().max())).item()
        other = {"method": "fp64_lu" if args.method == "mixed" else "mixed_ir", "s": o_ms / 1e3,
                 "backward_error": oeta, "steps": ksteps}

    # ---- end to end through the C ABI from pinned host buffers
    e2e = None
    if not args.no_e2e:
        hA = A.cpu().pin_memory()
        hb = b.cpu().pin_memory()
        hx = torch.empty(n, dtype=torch.float64).pin_memory()
        dA = torch.empty_like(A)
        db = torch.empty_like(b)
        e_steps = max(1, min(args.steps, 3))
        torch.cuda.synchronize()
        barrier(world)
        s0, s1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s0.record(stream)
        for _ in range(e_steps):
            dA.copy_(hA, non_blocking=True)
            db.copy_(hb, non_blocking=True)
            if args.method == "mixed":
                solver(dA, db, x, stream)
                hx.copy_(x, non_blocking=True)
            else:
                m.copy_(dA)
                xf.copy_(db)
                _lib.check(lib.b200la_dgesv(m.data_ptr(), piv.data_ptr(), n, xf.data_ptr(),
                                            la.LU_LINEAR_SOLVER, ws.data_ptr(), ws_bytes, sp))
                hx.copy_(xf, non_blocking=True)
        s1.record(stream)
        torch.cuda.synchronize()
        barrier(world)
        e2e_s = max_over_ranks(world, s0.elapsed_time(s1) / e_steps) / 1e3
        e2e = {"value": e2e_s, "unit": "s", "h2d_bytes_per_step": 8 * n * n + 8 * n,
               "d2h_bytes_per_step": 8 * n, "steps": e_steps}
        del hA, hb, hx, dA, db

    cusolver = None
    if rank == 0 and world == 1 and not args.no_compare:
        cusolver = cusolver_reference_seconds(A, b, stream)

    batched = None
    if not args.no_batched:
        del m, xf, ws
        torch.cuda.empty_cache()
        batched = run_batched(args, world, rank, local)

    inversion = None
    if not args.no_inversion:
        if batched is None:
            del m, xf, ws
            torch.cuda.empty_cache()
        inversion = run_inversion(args, world, rank, local)

    multiplication = None
    if not args.no_multiplication:
        multiplication = run_multiplication(args, world, rank, local)

    cholesky = None
    if not args.no_cholesky:
        cholesky = run_cholesky(args, world, rank, local)

    transpose = None
    if not args.no_transpose:
        transpose = run_transpose(args, world, rank, local)

    side = {}
    if rank == 0 and world == 1 and not args.no_side_workloads:
        fp64_peak = measured_fp64_peak_tflops()
        side["solve_n512"] = run_n512(args, local, fp64_peak)
        side["mixed_n16384_bf16_fp16_nrhs64"] = run_n16384_more(args, A, b, stream, local)
        side["conditioning_sweep_n4096_n8192"] = run_conditioning_sweep(args, local)
    if rank == 0 and world == 1 and args.selector_systems > 0:
        side["precision_selector"] = run_selector(args)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        kind, t, ceta = cpu_reference_solve_seconds(CPU_SAMPLE_N)
        scale = (n / CPU_SAMPLE_N) ** 3
        cpu = {"value": t * scale, "unit": "s", "cores": 1, "kind": kind,
               "sample": f"one linear_solver<double,NATIVE> LU solve at n={CPU_SAMPLE_N} "
                         f"({t:.2f} s, eta={ceta:.1e}) scaled by (n/{CPU_SAMPLE_N})^3 = {scale:.0f} "
                         f"to n={n}; 1 thread of {os.cpu_count()} ({cpu_model()}); the reference "
                         "has no threading"}

    if rank == 0:
        line = {
            "metric": METRIC,
            "value": ms_per_step / 1e3,
            "unit": "s",
            "n_gpus": world,
            "steps": args.steps,
            "warmup": args.warmup,
            "ms_per_step": ms_per_step,
            "higher_is_better": False,
            "scaling": "weak",
            "vs_baseline": None,
            "dtype": "f64" if args.method == "fp64" else f"{args.precision}+f64",
            "data": f"synthetic: A iid N(0,1) (torch generator seed {SEED}+rank), x_true iid U[-1,1], b = A x_true",
            "config": arm_config(n, args.method, args.precision, world),
            "accuracy": {"backward_error": eta, "forward_error": fwd, "target": 1e-14,
                         "refinement": {k: last[k] for k in ("precision_used", "iterations", "gmres_iterations",
                                                             "escalations", "converged", "factor_ms", "refine_ms")}
                         if last else None},
            "compare": other,
            "speedup_vs_fp64_lu": (other["s"] / (ms_per_step / 1e3)) if other and args.method == "mixed" else None,
            "roofline": roofline,
            "panel_roofline": panel_roofline,
            "cpu_baseline": cpu,
            "cusolver_baseline": cusolver,
            "e2e": e2e,
            "gpu_launches": int(launches),
            "breakdown_one_step": breakdown,
            "batched": batched,
            "inversion": inversion,
            "multiplication": multiplication,
            "cholesky": cholesky,
            "transpose": transpose,
            **side,
            "clocks": clk,
            "peaks": peaks,
        }
        print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------
# reference arm: the reference's NATIVE CPU LU solve (oracle/_ref)
# ---------------------------------------------------------------------------
def arm_config(n: int, method: str, precision: str, world: int) -> dict:
    """The `config` of the JSON line, shared by both arms."""
    method_desc = (f"mixed-precision LU-IR ({precision} factorization on tcgen05, FP64 "
                   "refinement to backward error <= 1e-14)" if method == "mixed"
                   else "plain FP64 blocked LU + solve")
    return {"workload": f"dense LU solve n={n} nrhs=1, {method_desc}",
            "n": n, "nrhs": 1, "method": method,
            "precision": precision if method == "mixed" else "fp64",
            "step": ("solve from A, b resident in HBM (A left unchanged)" if method == "mixed"
                     else "restore A and b (device copies, 2 GiB), factor, solve"),
            "l2": "inputs (2 GiB) larger than L2; no flush",
            "parallelism": "replicas" if world > 1 else "single GPU"}


def run_reference(args, world, rank):
    """Every timed step is one full linear_solver<double, NATIVE> LU solve of
    order n (A iid N(0,1), x_true iid U[-1,1], b = A x_true) by the
    reference's own build (oracle/_ref).  The reference is single-threaded,
    so it uses the host's threads the only way it can: the K steps run as K
    independent solves in concurrent threads (each on its own copy of A and
    b, made before the clock starts; at most as many at once as host memory
    holds).  value = wall time of all K solves / K: seconds of host time per
    n=16384 solve with every host thread busy."""
    if rank != 0:
        return
    import numpy as np
    from concurrent.futures import ThreadPoolExecutor

    from linearalgebra_b200.workloads import system
    from oracle import Oracle, available

    if not (available("reference") or available("port")):
        print(json.dumps({"impl": "reference", "unavailable": "CPU reference build missing"}))
        return
    kind = "reference" if available("reference") else "port"
    orc = Oracle(kind)
    fn = getattr(orc.lib, f"{orc._pre}dgesv")
    n = args.n
    for _ in range(args.warmup):
        cpu_reference_solve_seconds(1024)
    a, x_true, b = system(n, seed=SEED)
    try:
        avail = os.sysconf("SC_PAGE_SIZE") * os.sysconf("SC_AVPHYS_PAGES")
    except (ValueError, OSError):
        avail = 64 << 30
    ws_fn = getattr(orc.lib, "ref_dgetrf_workspace_size", None)
    if ws_fn is not None:
        ws_fn.restype = ctypes.c_size_t
        ws_fn.argtypes = [ctypes.c_int64]
        ws_bytes = int(ws_fn(n))
    else:
        ws_bytes = 8 * n * n + (64 << 20)
    per_solve = 8 * n * n + ws_bytes + 16 * n  # the copy of A, the reference's workspace, x and pivots
    threads = len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else os.cpu_count()
    concurrent = max(1, min(args.steps, int(0.8 * avail // per_solve)))
    ms = [np.empty_like(a) for _ in range(concurrent)]
    xs = [np.empty_like(b) for _ in range(concurrent)]
    pivs = [np.empty(n, dtype=np.int64) for _ in range(concurrent)]
    times = [0.0] * args.steps
    etas = [None] * args.steps

    def one(i):
        slot = i % concurrent
        m, x, piv = ms[slot], xs[slot], pivs[slot]
        np.copyto(m, a)
        np.copyto(x, b)
        t0 = time.perf_counter()
        st = fn(m.ctypes.data, piv.ctypes.data, n, x.ctypes.data, 1)
        times[i] = time.perf_counter() - t0
        if st < 0:
            raise RuntimeError(f"reference gesv failed ({st})")
        if i < concurrent:
            etas[i] = float(np.abs(b - a @ x).max() / (np.abs(a).sum(1).max() * np.abs(x).max() + np.abs(b).max()))

    t0 = time.perf_counter()
    with ThreadPoolExecutor(max_workers=concurrent) as ex:
        list(ex.map(one, range(args.steps)))
    wall = time.perf_counter() - t0
    value = wall / args.steps
    eta = max(e for e in etas if e is not None)
    sample = (f"{args.steps} full linear_solver<double,NATIVE> LU solves at n={n} (A iid N(0,1), numpy seed {SEED}), "
              f"{concurrent} at a time in threads on {threads} host threads ({cpu_model()}); "
              f"value = wall {wall:.1f} s / {args.steps}; each solve alone-in-thread took "
              f"{min(times):.1f}..{max(times):.1f} s (median {statistics.median(times):.1f} s, "
              f"input copies excluded); max eta {eta:.2e}; warm-up: {args.warmup} solves at n=1024")
    line = {
        "metric": METRIC, "impl": "reference", "value": value, "unit": "s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": value * 1e3, "higher_is_better": False, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64",
        "data": f"synthetic: A iid N(0,1), x_true iid U[-1,1], b = A x_true (numpy seed {SEED})",
        "config": arm_config(n, args.method, args.precision, world),
        "reference_solve": {"what": "linear_solver<double,NATIVE> LU mode, the reference's own sources "
                                    "(oracle/_ref, LINALG_HAS_LU_PIVOTING=1)",
                            "per_solve_s": times, "median_per_solve_s": statistics.median(times),
                            "concurrent_solves": concurrent, "host_threads": threads, "wall_s": wall,
                            "backward_error": eta},
        "cpu_baseline": {"value": value, "unit": "s", "cores": min(concurrent, threads), "kind": kind,
                         "sample": sample},
        "e2e": {"value": value, "unit": "s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def main():
    args = parse()
    if args.impl == "reference":
        world = int(os.environ.get("WORLD_SIZE", "1"))
        rank = int(os.environ.get("RANK", "0"))
        run_reference(args, world, rank)
        return
    world, rank, local = dist_setup(args)
    try:
        run_b200(args, world, rank, local)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
