"""inversion in its Cholesky modes on the GPU against the oracle.

CHOLESKY factors m with the bit-exact blocked Cholesky and inverts it,
CHOLESKY_UPFRONT inverts the lower factor given in m (its upper triangle is
not read), both as A^-1 = U^-1 L^-1 with U = L^T by two GEMM-blocked back
substitutions.  The reference forms L^-1 column by column and then the dot
products of its rows (inversion_native.cpp:306-410), an order no blocked
computation reproduces, so the inverse is held to rounding-level agreement
with the oracle's (bit-identical to the reference's, pinned by
tests/test_oracle.py):
  max|X - X_ref| <= 4 (n+1) eps kappa_inf(A) max|X_ref|
  max|A X - I|   <= 4 (n+1) eps ||A||_inf ||X||_inf
and must be exactly symmetric, as the reference's is.  A non-positive pivot
leaves the partial factor in m, bit for bit, with info = its 1-based row.
This file is collected last so that a failure here does not hide the other
tests.
"""
import hashlib

import numpy as np
import pytest
import torch

import linearalgebra_b200 as la
from linearalgebra_b200.workloads import spd_matrix, spd_product

pytestmark = pytest.mark.gpu

TYPES = [("f64", np.float64), ("f32", np.float32)]


def sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def gpu_inverse(a, mode):
    m = torch.from_numpy(np.ascontiguousarray(a)).cuda()
    _, info = la.inverse(m, type=mode)
    torch.cuda.synchronize()
    return m.cpu().numpy(), info


def check_inverse(a, x, x_ref):
    a64 = a.astype(np.float64)
    x64 = x.astype(np.float64)
    n = a.shape[0]
    eps = np.finfo(a.dtype).eps
    kappa = np.linalg.norm(a64, np.inf) * np.linalg.norm(np.linalg.inv(a64), np.inf)
    fwd = np.abs(x64 - x_ref.astype(np.float64)).max()
    assert fwd <= 4 * (n + 1) * eps * kappa * np.abs(x_ref).max(), (n, fwd, kappa)
    res = np.abs(a64 @ x64 - np.eye(n)).max()
    assert res <= 4 * (n + 1) * eps * np.linalg.norm(a64, np.inf) * np.linalg.norm(x64, np.inf), (n, res)


@pytest.mark.parametrize("n", (1, 2, 3, 17, 63, 64, 65, 130, 257))
@pytest.mark.parametrize("dt,npdt", TYPES)
def test_cholesky_inverse_vs_oracle(port, inverse_golden, n, dt, npdt):
    a = spd_matrix(n, seed=9000 + n, dtype=npdt)
    x_ref, _, st = port.getri(a, mode=la.CHOLESKY_LINEAR_SOLVER)
    assert st == 0 and sha(x_ref) == str(inverse_golden[f"cholinv_{dt}_{n}_inv_sha"])
    x, info = gpu_inverse(a, la.CHOLESKY_LINEAR_SOLVER)
    assert info == 0
    assert np.array_equal(x, x.T)
    check_inverse(a, x, x_ref)


@pytest.mark.parametrize("n", (511, 512, 513, 1000))
@pytest.mark.parametrize("dt,npdt", TYPES)
def test_cholesky_inverse_block_edges(port, n, dt, npdt):
    """Orders around the 512-row substitution block; odd orders (rows not
    16-byte aligned: the element-wise copy paths)."""
    a = spd_matrix(n, seed=9200 + n, dtype=npdt)
    x_ref, _, _ = port.getri(a, mode=la.CHOLESKY_LINEAR_SOLVER)
    x, info = gpu_inverse(a, la.CHOLESKY_LINEAR_SOLVER)
    assert info == 0 and np.array_equal(x, x.T)
    check_inverse(a, x, x_ref)


@pytest.mark.parametrize("n", (3, 198))
@pytest.mark.parametrize("dt,npdt", TYPES)
def test_cholesky_inverse_reference_test_case(n, dt, npdt):
    """Testing/Cxx/TestInversion.cxx, CHOLESKY_LINEAR_SOLVER: A = R R^T,
    ||A^-1 A - I||_max <= 5e-12 (double) / 2e-4 (float)."""
    a = spd_product(n, seed=6000 + n, dtype=npdt)
    x, info = gpu_inverse(a, la.CHOLESKY_LINEAR_SOLVER)
    assert info == 0
    err = np.abs(x.astype(np.float64) @ a.astype(np.float64) - np.eye(n)).max()
    assert err <= (5e-12 if npdt == np.float64 else 2e-4)


@pytest.mark.parametrize("dt,npdt", TYPES)
def test_cholesky_upfront_reads_only_the_lower_factor(port, dt, npdt):
    """CHOLESKY_UPFRONT on the oracle's lower factor (the same bits as the
    library's) with junk above the diagonal gives the same bits as
    CHOLESKY on the matrix."""
    n = 300
    a = spd_matrix(n, seed=9300, dtype=npdt)
    x, _ = gpu_inverse(a, la.CHOLESKY_LINEAR_SOLVER)
    f, info = port.potrf(a)
    assert info == 0
    f = f + np.triu(np.full((n, n), 3.0, dtype=npdt), 1)
    x4, info4 = gpu_inverse(f, la.CHOLESKY_UPFRONT_LINEAR_SOLVER)
    assert info4 == 0 and np.array_equal(x4, x)


@pytest.mark.parametrize("n,fr", [(100, 70), (130, 3), (700, 600)])
@pytest.mark.parametrize("dt,npdt", TYPES)
def test_cholesky_inverse_not_positive_definite_leaves_factor(port, n, fr, dt, npdt):
    a = spd_matrix(n, seed=9100 + fr, dtype=npdt, fail_row=fr)
    m, info = gpu_inverse(a, la.CHOLESKY_LINEAR_SOLVER)
    f_ref, info_ref = port.potrf(a)
    assert info == info_ref == fr + 1
    assert np.array_equal(m, f_ref)
