"""Parity of the B200 LU path with the reference (GPU).

The FP64/FP32 factorization performs the reference's arithmetic operation for
operation, so factors and pivots are compared bit for bit against the golden
fixtures (produced by the reference's own NATIVE build) and against the CPU
oracle.  Solutions are compared through the normwise backward error
eta = ||b - A x||_inf / (||A||_inf ||x||_inf + ||b||_inf) <= 10 n eps64 and
against the reference's solution.
"""
import hashlib

import numpy as np
import pytest
import torch

import linearalgebra_b200 as la
from linearalgebra_b200.workloads import (
    KNOWN_ANSWER_INFO,
    known_answer_matrices,
    random_matrix,
    system,
)

pytestmark = pytest.mark.gpu

EPS64 = np.finfo(np.float64).eps
LU_SIZES = (1, 2, 3, 17, 63, 64, 65, 130, 200)


def sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def dev(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def gpu_getrf(a):
    m = dev(a)
    piv, info = la.getrf(m)
    torch.cuda.synchronize()
    return m.cpu().numpy(), piv.cpu().numpy(), info


@pytest.mark.parametrize("n", LU_SIZES)
@pytest.mark.parametrize("dt", ["f64", "f32"])
def test_lu_bitwise_vs_golden(golden, n, dt):
    a = random_matrix(n, seed=1000 + n, dtype=np.float64 if dt == "f64" else np.float32)
    assert sha(a) == str(golden[f"lu_{dt}_{n}_a_sha"])
    lu, piv, info = gpu_getrf(a)
    assert np.array_equal(piv, golden[f"lu_{dt}_{n}_piv"])
    assert info == int(golden[f"lu_{dt}_{n}_info"])
    assert np.array_equal(lu, golden[f"lu_{dt}_{n}_lu"])


@pytest.mark.parametrize("name", sorted(KNOWN_ANSWER_INFO))
@pytest.mark.parametrize("dt,npdt", [("f64", np.float64), ("f32", np.float32)])
def test_lu_known_answers(golden, name, dt, npdt):
    a = known_answer_matrices(npdt)[name]
    m = dev(a)
    piv = torch.full((a.shape[0],), -1, dtype=torch.int64, device="cuda")
    ws = la.api.workspace(la.lu_decomposition.workspace_size(a.shape[0], m.dtype))
    ok, info = la.lu_decomposition.apply(m, a.shape[0], piv, ws, ws.numel())
    assert info == KNOWN_ANSWER_INFO[name]
    assert ok == (info == 0)
    assert np.array_equal(piv.cpu().numpy(), golden[f"ka_{name}_{dt}_piv"])
    assert np.array_equal(m.cpu().numpy(), golden[f"ka_{name}_{dt}_lu"])
    assert np.all(np.isfinite(m.cpu().numpy()))


@pytest.mark.parametrize("n", [257, 1000, 1500])
def test_lu_bitwise_vs_oracle(port, n):
    a = random_matrix(n, seed=4242 + n)
    lu_o, piv_o, info_o = port.getrf(a)
    lu, piv, info = gpu_getrf(a)
    assert info == info_o == 0
    assert np.array_equal(piv, piv_o)
    assert np.array_equal(lu, lu_o)


@pytest.mark.parametrize("n", [300, 1500])
def test_lu_grid_panel_path_bitwise(port, monkeypatch, n):
    """The grid-wide panel kernel (used when a panel does not fit in one
    thread-block cluster) gives the same bits as the cluster one."""
    monkeypatch.setenv("B200LA_FORCE_GRID_PANEL", "1")
    a = random_matrix(n, seed=31 + n)
    lu_o, piv_o, _ = port.getrf(a)
    lu, piv, _ = gpu_getrf(a)
    assert np.array_equal(piv, piv_o)
    assert np.array_equal(lu, lu_o)


@pytest.mark.parametrize("n", [100, 700, 2500, 6200])
@pytest.mark.parametrize("dt", [np.float64, np.float32])
def test_lu_cluster_panel_bitwise(port, n, dt):
    """The cluster panel (every panel up to ~6,400 FP64 / ~13,000 FP32 rows)
    gives the oracle's pivots and factors bit for bit."""
    a = random_matrix(n, seed=91 + n, dtype=dt)
    lu_o, piv_o, _ = port.getrf(a)
    lu, piv, _ = gpu_getrf(a)
    assert np.array_equal(piv, piv_o)
    assert np.array_equal(lu, lu_o)


@pytest.mark.parametrize("force_grid", ["0", "1"])
def test_lu_lookahead_bitwise(port, monkeypatch, force_grid):
    """The FP64 look-ahead (next panel on a side stream beside the rest of
    the trailing update; grid panels on fewer CTAs there) changes only the
    schedule: the factors equal the oracle's and the run without it."""
    monkeypatch.setenv("B200LA_FORCE_GRID_PANEL", force_grid)
    n = 1500
    a = random_matrix(n, seed=77 + n)
    lu_o, piv_o, _ = port.getrf(a)
    lu, piv, _ = gpu_getrf(a)
    assert np.array_equal(piv, piv_o)
    assert np.array_equal(lu, lu_o)
    monkeypatch.setenv("B200LA_LU_LOOKAHEAD", "0")
    lu0, piv0, _ = gpu_getrf(a)
    assert np.array_equal(piv0, piv) and np.array_equal(lu0, lu)


def test_lu_lookahead_neutral_large():
    """n = 7000 (grid panels while more than ~6200 rows remain, cluster
    panels after): look-ahead on and off give identical bits."""
    import os
    a = random_matrix(7000, seed=7000)
    lu, piv, _ = gpu_getrf(a)
    os.environ["B200LA_LU_LOOKAHEAD"] = "0"
    try:
        lu0, piv0, _ = gpu_getrf(a)
    finally:
        del os.environ["B200LA_LU_LOOKAHEAD"]
    assert np.array_equal(piv0, piv) and np.array_equal(lu0, lu)


def wide_exponent_matrix(n, seed, kind):
    """N(0,1) entries scaled by 2^e with e spread over most of the FP64
    range: 'wide' (|e| <= 900, products over- and underflow), 'subnormal'
    (a tenth of the entries scaled into the subnormal range), 'zeros' (a
    third exact zeros, some -0)."""
    rng = np.random.default_rng(seed)
    a = rng.standard_normal((n, n))
    if kind == "wide":
        a *= np.exp2(rng.integers(-900, 900, size=(n, n)).astype(np.float64))
    elif kind == "subnormal":
        mask = rng.random((n, n)) < 0.1
        a[mask] *= 2.0 ** -1060
    else:
        mask = rng.random((n, n))
        a[mask < 0.33] = 0.0
        a[(mask >= 0.33) & (mask < 0.4)] = -0.0
        a += np.eye(n)
    return a


@pytest.mark.parametrize("kind", ["wide", "subnormal", "zeros"])
def test_lu_bitwise_special_values(port, kind):
    """The FP64 trailing update runs on the FP64 tensor cores (DMMA chains,
    delta from zero in k order): its bits must equal the reference's fma loop
    also where products overflow, underflow into subnormals, or vanish."""
    n = 450
    a = wide_exponent_matrix(n, seed=99, kind=kind)
    lu_o, piv_o, info_o = port.getrf(a)
    lu, piv, info = gpu_getrf(a)
    assert info == info_o
    assert np.array_equal(piv, piv_o)
    same = (lu.view(np.uint64) == lu_o.view(np.uint64)) | (np.isnan(lu) & np.isnan(lu_o))
    assert same.all(), int((~same).sum())


def test_lu_float32_bitwise_vs_oracle(port):
    a = random_matrix(700, seed=11, dtype=np.float32)
    lu_o, piv_o, _ = port.getrf(a)
    lu, piv, _ = gpu_getrf(a)
    assert np.array_equal(piv, piv_o)
    assert np.array_equal(lu, lu_o)


def test_n512_solve_parity(port, golden):
    """n=512 plain FP64 LU + solve: same pivots, same factors, eta <= 10 n eps."""
    n = 512
    a, x_true, b = system(n, seed=512)
    m, x = dev(a), dev(b)
    piv = la.gesv(m, x)
    torch.cuda.synchronize()
    assert np.array_equal(piv.cpu().numpy(), golden["n512_piv"])
    assert sha(m.cpu().numpy()) == str(golden["n512_lu_sha"])
    xs = x.cpu().numpy()
    eta = port.backward_error(a, xs, b)
    assert eta <= 10 * n * EPS64, eta
    x_ref = golden["n512_x"]
    assert port.backward_error(a, x_ref, b) <= 10 * n * EPS64
    assert np.max(np.abs(xs - x_ref)) / np.max(np.abs(x_ref)) < 1e-11


def test_upfront_mode_reuses_pivots(port):
    n = 300
    a, _, b = system(n, seed=21)
    m = dev(a)
    piv, info = la.getrf(m)
    x = dev(b)
    la.gesv(m, x, pivot=piv, type=la.LU_UPFRONT_LINEAR_SOLVER)
    torch.cuda.synchronize()
    assert port.backward_error(a, x.cpu().numpy(), b) <= 10 * n * EPS64


def test_singular_system_leaves_rhs_unchanged():
    a = known_answer_matrices(np.float64)["rank_def"]
    b = np.array([1.0, 2.0, 3.0])
    m, x = dev(a), dev(b)
    la.gesv(m, x)
    torch.cuda.synchronize()
    assert np.array_equal(x.cpu().numpy(), b)


@pytest.mark.parametrize("nrhs", [1, 3, 64, 70])
def test_getrs_multi_rhs(port, nrhs):
    n = 333
    a, x_true, b = system(n, seed=5, nrhs=nrhs)
    m = dev(a)
    piv, _ = la.getrf(m)
    x = dev(b.reshape(n, nrhs) if nrhs > 1 else b)
    la.getrs(m, piv, x)
    torch.cuda.synchronize()
    xs = x.cpu().numpy().reshape(n, nrhs)
    bb = b.reshape(n, nrhs)
    for j in range(nrhs):
        assert port.backward_error(a, xs[:, j], bb[:, j]) <= 10 * n * EPS64


def test_panel_spans_many_ctas(port):
    """n large enough that the panel kernel runs on every SM with several
    rows per CTA, and a singular trailing column appears mid-matrix."""
    n = 2500
    a = random_matrix(n, seed=99)
    a[:, 1700] = 0.0
    lu_o, piv_o, info_o = port.getrf(a)
    lu, piv, info = gpu_getrf(a)
    assert info == info_o == 1701
    assert np.array_equal(piv, piv_o)
    assert np.array_equal(lu, lu_o)


def test_nan_never_wins_pivot_search(port):
    a = random_matrix(70, seed=1)
    a[5, 3] = np.nan
    a[40, 0] = np.nan
    lu_o, piv_o, info_o = port.getrf(a)
    lu, piv, info = gpu_getrf(a)
    assert np.array_equal(piv, piv_o)
    assert np.array_equal(lu, lu_o, equal_nan=True)


def test_large_factorization_properties():
    """n = 8192 (beyond oracle reach): pivots in range, P L U reconstructs
    sampled rows of A to FP64 accuracy, eta of the solve within bound."""
    n = 8192
    torch.manual_seed(0)
    a = torch.randn(n, n, dtype=torch.float64, device="cuda")
    x_true = torch.rand(n, dtype=torch.float64, device="cuda") * 2 - 1
    b = a @ x_true
    m = a.clone()
    x = b.clone()
    piv = la.gesv(m, x)
    torch.cuda.synchronize()
    p = piv.cpu().numpy()
    assert np.all((p >= np.arange(1, n + 1)) & (p <= n))
    r = b - a @ x
    eta = (r.abs().max() / (a.abs().sum(1).max() * x.abs().max() + b.abs().max())).item()
    assert eta <= 10 * n * EPS64, eta
    # reconstruct rows of P A from L U
    perm = np.arange(n)
    for i in range(n):
        q = p[i] - 1
        perm[i], perm[q] = perm[q], perm[i]
    rows = torch.tensor(np.sort(np.random.default_rng(0).choice(n, 64, replace=False)), device="cuda")
    cols = torch.arange(n, device="cuda")
    L = torch.where(cols[None, :] < rows[:, None], m[rows], torch.zeros((), dtype=m.dtype, device="cuda"))
    L[torch.arange(64, device="cuda"), rows] = 1.0
    U = torch.triu(m)
    pa = a[torch.from_numpy(perm).cuda()[rows]]
    err = (L @ U - pa).abs().max().item()
    assert err <= 1e-10 * n, err
