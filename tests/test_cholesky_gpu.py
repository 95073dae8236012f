"""cholesky_decomposition and the Cholesky modes of linear_solver on the GPU
against the oracle.

The factor kernels keep the reference's own order of operations per entry
(the sequential dot product, rounded as the reference's compiled loops round
it, then the subtraction and the square root or division), so the factors
(lower and upper), info and the partial state a non-positive pivot leaves are
compared bit for bit.  The solve runs blocked triangular substitutions, not
the reference's sequential rows, so its x is held to the backward error
  eta = ||A x - b||_inf / (||A||_inf ||x||_inf + ||b||_inf) <= 10 n eps.
"""
import hashlib
import os

import numpy as np
import pytest
import torch

import linearalgebra_b200 as la
from linearalgebra_b200 import api
from linearalgebra_b200.workloads import spd_matrix

pytestmark = pytest.mark.gpu

SIZES = (1, 2, 3, 17, 63, 64, 65, 127, 130, 200, 257, 1000)
TYPES = [("f64", np.float64), ("f32", np.float32)]


def sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def dev(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


@pytest.fixture(scope="module")
def cg():
    return np.load(os.path.join(os.path.dirname(__file__), "golden", "cholesky_golden.npz"))


def gpu_potrf(a, upper=False):
    m = dev(a)
    info = la.potrf(m, upper=upper)
    return m.cpu().numpy(), info


@pytest.mark.parametrize("n", SIZES)
@pytest.mark.parametrize("dt,npdt", TYPES)
def test_cholesky_factor_bitwise(port, n, dt, npdt):
    a = spd_matrix(n, seed=7000 + n, dtype=npdt)
    for upper in (False, True):
        f, info = gpu_potrf(a, upper)
        f_ref, info_ref = port.potrf(a, upper)
        assert info == info_ref == 0
        assert np.array_equal(f, f_ref), (n, upper, np.abs(f - f_ref).max())


@pytest.mark.parametrize("dt,npdt", TYPES)
def test_cholesky_factor_matches_golden(cg, dt, npdt):
    for n in (17, 65, 200):
        a = spd_matrix(n, seed=7000 + n, dtype=npdt)
        for tag, upper in (("lower", False), ("upper", True)):
            f, _ = gpu_potrf(a, upper)
            assert sha(f) == str(cg[f"chol_{dt}_{n}_{tag}_sha"]), (n, tag)


@pytest.mark.parametrize("dt,npdt", TYPES)
@pytest.mark.parametrize("n,fail_row", [(100, 70), (100, 5), (300, 0), (300, 64), (300, 250)])
def test_cholesky_not_positive_definite_state(port, cg, dt, npdt, n, fail_row):
    """info = failing row + 1 and the matrix holds exactly what the reference
    leaves: the rows before the failing one factored, the rest as given."""
    a = spd_matrix(n, seed=7100 + fail_row, dtype=npdt, fail_row=fail_row)
    f, info = gpu_potrf(a)
    f_ref, info_ref = port.potrf(a)
    assert info == info_ref == fail_row + 1
    assert np.array_equal(f, f_ref)
    key = f"cholfail_{dt}_{n}_{fail_row}_m"
    if key in cg:
        assert np.array_equal(f, cg[key])
    fu, info_u = gpu_potrf(a, upper=True)
    assert info_u == info and np.array_equal(fu, port.potrf(a, True)[0])


@pytest.mark.parametrize("n,seed", [(10, 100), (12, 312), (21, 111), (45, 345), (70, 370), (95, 7095)])
def test_cholesky_pivot_rounding(port, cg, n, seed):
    """Inputs on which the reference build's pivot dot products round
    differently from its other dot products (for double: no half vector)."""
    a = spd_matrix(n, seed=seed)
    f, info = gpu_potrf(a)
    assert info == 0
    assert sha(f) == str(cg[f"pivot_{n}_{seed}_sha"])
    assert np.array_equal(f, port.potrf(a)[0])


@pytest.mark.parametrize("dt,npdt", TYPES)
def test_cholesky_sweep_bitwise(port, dt, npdt):
    for n in range(1, 97, 5):
        for seed in (300 + n, 90 + n):
            a = spd_matrix(n, seed=seed, dtype=npdt)
            assert np.array_equal(gpu_potrf(a)[0], port.potrf(a)[0]), (n, seed)


def test_cholesky_lookahead_neutral(port, monkeypatch):
    """The look-ahead schedule (next block's kernels beside the trailing
    update) gives the same bits as the plain sequence, also when a late
    block is not positive definite."""
    for fail_row in (-1, 1400):
        a = spd_matrix(1500, seed=15, fail_row=fail_row)
        monkeypatch.delenv("B200LA_LU_LOOKAHEAD", raising=False)
        f1, i1 = gpu_potrf(a)
        monkeypatch.setenv("B200LA_LU_LOOKAHEAD", "0")
        f0, i0 = gpu_potrf(a)
        monkeypatch.delenv("B200LA_LU_LOOKAHEAD")
        assert i0 == i1 == fail_row + 1
        assert np.array_equal(f0, f1)
        if fail_row >= 0:
            assert np.array_equal(f1, port.potrf(a)[0])


def test_cholesky_large_bitwise(port):
    n = 2500
    a = spd_matrix(n, seed=2500)
    f, info = gpu_potrf(a)
    f_ref, _ = port.potrf(a)
    assert info == 0
    assert np.array_equal(f, f_ref), np.abs(f - f_ref).max()


@pytest.mark.parametrize("n", [1, 2, 64, 65, 257, 1000, 3000])
@pytest.mark.parametrize("dt,npdt", TYPES)
def test_cholesky_linear_solver(port, n, dt, npdt):
    """Mode 3 factors (bitwise, lower) and solves; mode 4 solves with the
    given factor."""
    a = spd_matrix(n, seed=7000 + n, dtype=npdt)
    b = np.random.default_rng(8000 + n).standard_normal(n).astype(npdt)
    m, x = dev(a), dev(b)
    la.gesv(m, x, type=la.CHOLESKY_LINEAR_SOLVER)
    torch.cuda.synchronize()
    mf = m.cpu().numpy()
    if n <= 1000:
        assert np.array_equal(mf, port.potrf(a)[0])
    eps = np.finfo(npdt).eps
    assert port.backward_error(a, x.cpu().numpy(), b) <= 10 * n * eps
    x4 = dev(b)
    la.gesv(m, x4, type=la.CHOLESKY_UPFRONT_LINEAR_SOLVER)
    torch.cuda.synchronize()
    assert port.backward_error(a, x4.cpu().numpy(), b) <= 10 * n * eps
    assert np.array_equal(m.cpu().numpy(), mf), "mode 4 leaves the factor alone"


def test_cholesky_solve_matches_golden_solution(cg):
    for n in (17, 130, 200):
        a = spd_matrix(n, seed=7000 + n)
        b = cg[f"chol_f64_{n}_b"]
        x = dev(b)
        la.gesv(dev(a), x, type=la.CHOLESKY_LINEAR_SOLVER)
        torch.cuda.synchronize()
        x_ref = cg[f"chol_f64_{n}_x"]
        assert np.abs(x.cpu().numpy() - x_ref).max() <= 1e-12 * np.abs(x_ref).max()


@pytest.mark.parametrize("dt,npdt", TYPES)
def test_cholesky_solver_not_positive_definite_leaves_x(dt, npdt):
    a = spd_matrix(300, seed=7164, dtype=npdt, fail_row=164)
    b = np.ones(300, dtype=npdt)
    x = dev(b)
    la.gesv(dev(a), x, type=la.CHOLESKY_LINEAR_SOLVER)
    torch.cuda.synchronize()
    assert np.array_equal(x.cpu().numpy(), b)


def test_cholesky_decomposition_api():
    n = 70
    a = spd_matrix(n, seed=3)
    m = dev(a)
    ws_bytes = api.cholesky_decomposition.workspace_size(n)
    ws = api.workspace(ws_bytes, m.device)
    ok, info = api.cholesky_decomposition.apply(m, n, la.LOWER_TRIANGULAR, ws, ws.numel())
    assert ok and info == 0
    f = m.cpu().numpy()
    assert np.abs(f @ f.T - a).max() <= 1e-12 * np.abs(a).max()
    bad = dev(spd_matrix(n, seed=3, fail_row=9))
    ok, info = api.cholesky_decomposition.apply(bad, n, la.LOWER_TRIANGULAR, ws, ws.numel())
    assert not ok and info == 10
    with pytest.raises(la.B200InvalidArgument):
        api.cholesky_decomposition.apply(m, n, "X", ws, ws.numel())
    with pytest.raises(la.B200InvalidArgument):
        api.cholesky_decomposition.apply(m, n, la.LOWER_TRIANGULAR, ws, 0)


def test_linear_solver_rejects_unknown_mode():
    m, x = dev(np.eye(4)), dev(np.ones(4))
    with pytest.raises(la.B200InvalidArgument):
        la.gesv(m, x, type=7)
