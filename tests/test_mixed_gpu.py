"""Mixed-precision LU with FP64 iterative refinement (GPU): every
factorization precision reaches the requested normwise backward error on the
benchmark's matrix classes, and the answer agrees with the FP64 oracle."""
import numpy as np
import pytest
import torch

import linearalgebra_b200 as la
from linearalgebra_b200.workloads import conditioned, system

pytestmark = pytest.mark.gpu

EPS64 = np.finfo(np.float64).eps


def dev(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def eta_of(a, x, b):
    r = b - a @ x
    return np.abs(r).max() / (np.abs(a).sum(1).max() * np.abs(x).max() + np.abs(b).max())


@pytest.mark.parametrize("precision", ["fp32", "tf32", "bf16", "fp16", "fp8"])
@pytest.mark.parametrize("n", [300, 1100])
def test_mixed_reaches_fp64_accuracy(port, precision, n):
    a, x_true, b = system(n, seed=70 + n)
    x, res, st = la.solve_mixed(dev(a), dev(b), precision=precision, tolerance=1e-14)
    torch.cuda.synchronize()
    assert st == 0 and res["converged"] == 1, res
    xs = x.cpu().numpy()
    assert port.backward_error(a, xs, b) <= 1e-14
    # against the FP64 oracle's solution (forward error, conditioning-scaled)
    _, _, x_ref = port.gesv(a, b)
    assert np.abs(xs - x_ref).max() / np.abs(x_ref).max() < 1e-9


@pytest.mark.parametrize("precision", ["bf16", "fp16", "fp8"])
def test_mixed_low_precision_at_4096(precision):
    """The low-precision factorizations at n = 4096 (the conditioning
    sweep's order; kappa = 1e2 by the sweep's Householder construction): the
    refined solution reaches eta <= 1e-14 and agrees with the plain FP64 LU
    solve (bit-identical to the reference's) to the conditioning."""
    from linearalgebra_b200 import selector
    n = 4096
    a, b, _ = selector.make_system(n, 1e2, 4096)
    x, res, st = la.solve_mixed(a, b, precision=precision, tolerance=1e-14)
    torch.cuda.synchronize()
    assert st == 0 and res["converged"] == 1, res
    x64, res64, st64 = la.solve_mixed(a, b, precision="fp64", tolerance=1e-14)
    torch.cuda.synchronize()
    assert st64 == 0, res64
    anorm = a.abs().sum(1).max()
    eta = ((b - a @ x).abs().max() / (anorm * x.abs().max() + b.abs().max())).item()
    assert eta <= 1e-14, eta
    diff = ((x - x64).abs().max() / x64.abs().max()).item()
    assert diff < 1e-10, diff  # measured 1e-13..7e-13 for this system class


def test_mixed_64_column_panels(port, monkeypatch):
    """64-column cluster panels (B200LA_MIXED_PANEL_WIDTH=64) instead of the
    default 32-column ones: same accuracy."""
    monkeypatch.setenv("B200LA_MIXED_PANEL_WIDTH", "64")
    n = 1100
    a, _, b = system(n, seed=1132)
    x, res, st = la.solve_mixed(dev(a), dev(b), precision="fp32", tolerance=1e-14)
    torch.cuda.synchronize()
    assert st == 0 and res["converged"] == 1 and res["escalations"] == 0, res
    assert port.backward_error(a, x.cpu().numpy(), b) <= 1e-14


def test_mixed_at_headline_order_agrees_with_fp64_lu():
    """n = 16384, A iid N(0,1) (the benchmark's system): the mixed solve
    (FP32 factors, FP64 refinement) reaches eta <= 1e-14 and agrees with the
    plain FP64 LU solve (the reference's algorithm, bit-identical factors)
    to well within what the conditioning allows."""
    from linearalgebra_b200 import _lib
    n = 16384
    g = torch.Generator(device="cuda").manual_seed(16384)
    A = torch.randn(n, n, dtype=torch.float64, device="cuda", generator=g)
    x_true = torch.rand(n, dtype=torch.float64, device="cuda", generator=g) * 2 - 1
    b = A @ x_true
    x, res, st = la.solve_mixed(A, b, precision="fp32", tolerance=1e-14)
    assert st == 0 and res["converged"] == 1, res
    lib = _lib.load()
    m = A.clone()
    x64 = b.clone()
    piv = torch.empty(n, dtype=torch.int64, device="cuda")
    nbytes = lib.b200la_dgesv_workspace_size(n, 1)
    ws = torch.empty(nbytes, dtype=torch.uint8, device="cuda")
    _lib.check(lib.b200la_dgesv(m.data_ptr(), piv.data_ptr(), n, x64.data_ptr(), 1, ws.data_ptr(), nbytes,
                                torch.cuda.current_stream().cuda_stream))
    del m, ws
    anorm = A.abs().sum(1).max()

    def eta(xx):
        return ((b - A @ xx).abs().max() / (anorm * xx.abs().max() + b.abs().max())).item()

    assert eta(x) <= 1e-14
    assert eta(x64) <= 10 * n * EPS64
    # both solutions are backward stable; their difference is bounded by
    # cond(A) times their backward errors (cond_inf of this class is ~1e5-1e6)
    diff = ((x - x64).abs().max() / x64.abs().max()).item()
    assert diff < 1e-7, diff
    fwd = ((x - x_true).abs().max() / x_true.abs().max()).item()
    assert fwd < 1e-7, fwd


def test_mixed_fp32_takes_few_iterations():
    a, _, b = system(2048, seed=5)
    _, res, st = la.solve_mixed(dev(a), dev(b), precision="fp32")
    assert st == 0 and res["precision_used"] == la._lib.PREC_FP32
    assert res["iterations"] <= 6 and res["escalations"] == 0, res


@pytest.mark.parametrize("n,nrhs", [(700, 64), (701, 5), (1500, 64)])
def test_mixed_multi_rhs(n, nrhs):
    # the one-launch multi-right-hand-side solves: 128-row blocks, a ragged
    # last block, an order that is not a multiple of four (scalar tile loads)
    a, x_true, b = system(n, seed=8, nrhs=nrhs)
    x, res, st = la.solve_mixed(dev(a), dev(b), precision="fp32")
    torch.cuda.synchronize()
    assert st == 0 and res["escalations"] == 0, res
    assert res["iterations"] <= 8, res
    xs = x.cpu().numpy()
    for j in range(nrhs):
        assert eta_of(a, xs[:, j], b[:, j]) <= 1e-14, j


@pytest.mark.parametrize("kappa", [1e4, 1e8])
def test_mixed_conditioned_gmres_or_escalation(kappa):
    n = 1024
    a = conditioned(n, kappa, seed=3)
    x_true = np.random.default_rng(1).uniform(-1, 1, n)
    b = a @ x_true
    x, res, st = la.solve_mixed(dev(a), dev(b), precision="bf16", tolerance=1e-14)
    torch.cuda.synchronize()
    assert st == 0 and res["converged"] == 1, res
    assert eta_of(a, x.cpu().numpy(), b) <= 1e-14


def test_mixed_fp64_precision_is_plain_lu():
    a, _, b = system(600, seed=2)
    x, res, st = la.solve_mixed(dev(a), dev(b), precision="fp64")
    assert st == 0 and res["precision_used"] == la._lib.PREC_FP64
    assert eta_of(a, x.cpu().numpy(), b) <= 1e-14


def test_mixed_singular_reports_info():
    a = np.zeros((130, 130))
    a[np.arange(130), np.arange(130)] = 1.0
    a[:, 77] = 0.0
    b = np.ones(130)
    x, res, st = la.solve_mixed(dev(a), dev(b), precision="fp32", escalate=False)
    assert st == la._lib.SINGULAR and res["info"] == 78


def test_mixed_fp8_well_conditioned_without_escalation():
    """FP8-E4M3 updates (per-row / per-column power-of-two scales) on a
    well-conditioned system: GMRES-IR on the FP8-updated factors converges
    to FP64 accuracy without leaving FP8."""
    n = 1024
    a = conditioned(n, 1e1, seed=11)
    b = a @ np.random.default_rng(2).uniform(-1, 1, n)
    x, res, st = la.solve_mixed(dev(a), dev(b), precision="fp8", escalate=False)
    torch.cuda.synchronize()
    assert st == 0 and res["converged"] == 1 and res["precision_used"] == la._lib.PREC_FP8, res
    assert eta_of(a, x.cpu().numpy(), b) <= 1e-14


def test_mixed_fp8_escalation_chain_reaches_fp64():
    """kappa = 1e12 defeats every low precision: FP8 -> BF16 -> FP32 -> FP64."""
    n = 512
    a = conditioned(n, 1e12, seed=11)
    b = a @ np.random.default_rng(3).uniform(-1, 1, n)
    x, res, st = la.solve_mixed(dev(a), dev(b), precision="fp8", max_iterations=10)
    torch.cuda.synchronize()
    assert st == 0 and res["converged"] == 1, res
    assert res["precision_used"] == la._lib.PREC_FP64 and res["escalations"] == 3, res
    assert eta_of(a, x.cpu().numpy(), b) <= 1e-14


@pytest.mark.parametrize("width", ["32", "64"])
def test_mixed_nested_lookahead_is_neutral(monkeypatch, width):
    """Inside a block, the next panel's interchanges, U12 and update applied
    by the next panel kernel itself (the FP32 32-column cluster kernel) or by
    two kernels before it, and the rest of the block on a second stream: the
    same arithmetic, so the refined solution is bit-identical with the nesting
    switched off.  Width 64 mixes 64-column panels (not fused) with a narrow
    last panel after a 64-column one (not fused either)."""
    monkeypatch.setenv("B200LA_MIXED_PANEL_WIDTH", width)
    n = 1100
    a, _, b = system(n, seed=1100)
    da, db = dev(a), dev(b)
    out = {}
    for flag in ("1", "0"):
        monkeypatch.setenv("B200LA_MIXED_NESTED", flag)
        x, res, st = la.solve_mixed(da, db, precision="fp32")
        torch.cuda.synchronize()
        assert st == 0 and res["converged"] == 1 and res["gmres_iterations"] == 0, res
        out[flag] = (x.cpu().numpy(), res)
    assert out["1"][1]["iterations"] == out["0"][1]["iterations"]
    assert np.array_equal(out["1"][0], out["0"][0])


@pytest.mark.parametrize("precision", ["fp32", "tf32", "fp8"])
@pytest.mark.parametrize("n", [777, 1300, 2048])
def test_mixed_lookahead_is_neutral(monkeypatch, precision, n):
    """The look-ahead (next block's panels on a second stream beside the
    rest of the tensor-core update, interchanges right of the block deferred)
    performs the same operations.  Plain refinement is deterministic, so the
    solution is bit-identical with the look-ahead switched off; GMRES-IR sums
    its dot products with atomics, so there both runs must converge and agree
    to the conditioning."""
    a, _, b = system(n, seed=90 + n)
    da, db = dev(a), dev(b)
    out = {}
    for flag in ("1", "0"):
        monkeypatch.setenv("B200LA_MIXED_LOOKAHEAD", flag)
        x, res, st = la.solve_mixed(da, db, precision=precision)
        torch.cuda.synchronize()
        assert st == 0 and res["converged"] == 1, res
        out[flag] = (x.cpu().numpy(), res)
    x1, r1 = out["1"]
    x0, r0 = out["0"]
    if r1["gmres_iterations"] == 0 and r0["gmres_iterations"] == 0 and r1["escalations"] == 0:
        assert r1["iterations"] == r0["iterations"]
        assert np.array_equal(x1, x0)
    else:
        assert eta_of(a, x1, b) <= 1e-14 and eta_of(a, x0, b) <= 1e-14
        assert np.abs(x1 - x0).max() / np.abs(x0).max() < 1e-8
