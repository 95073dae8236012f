"""inversion and determinant (LU modes) on the GPU against the oracle.

The determinant is the product of U's diagonal in index order over factors
that are bit-identical to the reference's, so its magnitude is compared bit
for bit with the golden fixtures (the reference's NATIVE value); the pivot
sign is checked against numpy.  The inverse comes from GEMM-blocked
substitutions, not the reference's sequential row loops, so it is held to
rounding-level agreement:
  max|X - X_ref| <= 2 n eps kappa_inf(A) max|X_ref|      (forward error)
  max|A X - I|   <= 2 n eps ||A||_inf ||X||_inf            (residual)
with X_ref the oracle's inverse (bit-identical to the reference's, pinned by
tests/test_oracle.py), plus the reference inversion test's own bound on its
R R^T matrices.
"""
import hashlib

import numpy as np
import pytest
import torch

import linearalgebra_b200 as la
from linearalgebra_b200 import api
from linearalgebra_b200.workloads import determinant_known_answers, random_matrix, spd_product

pytestmark = pytest.mark.gpu

INV_SIZES = (1, 2, 3, 17, 64, 65, 130, 257)
TYPES = [("f64", np.float64), ("f32", np.float32)]


def sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def dev(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def gpu_inverse(a, mode=la.LU_LINEAR_SOLVER, pivot=None):
    m = dev(a)
    piv = None if pivot is None else dev(pivot)
    piv, info = la.inverse(m, piv, type=mode)
    torch.cuda.synchronize()
    return m.cpu().numpy(), piv.cpu().numpy(), info


def check_inverse(a, x, x_ref):
    a64 = a.astype(np.float64)
    x64 = x.astype(np.float64)
    n = a.shape[0]
    eps = np.finfo(a.dtype).eps
    kappa = np.linalg.norm(a64, np.inf) * np.linalg.norm(np.linalg.inv(a64), np.inf)
    fwd = np.abs(x64 - x_ref.astype(np.float64)).max()
    assert fwd <= 2 * n * eps * kappa * np.abs(x_ref).max(), (n, fwd, kappa)
    res = np.abs(a64 @ x64 - np.eye(n)).max()
    assert res <= 2 * n * eps * np.linalg.norm(a64, np.inf) * np.linalg.norm(x64, np.inf), (n, res)


@pytest.mark.parametrize("n", INV_SIZES)
@pytest.mark.parametrize("dt,npdt", TYPES)
def test_inverse_vs_oracle(port, inverse_golden, n, dt, npdt):
    a = random_matrix(n, seed=5000 + n, dtype=npdt)
    x_ref, piv_ref, _ = port.getri(a)
    assert sha(x_ref) == str(inverse_golden[f"inv_{dt}_{n}_inv_sha"])
    x, piv, info = gpu_inverse(a)
    assert info == 0
    assert np.array_equal(piv, piv_ref)
    check_inverse(a, x, x_ref)


@pytest.mark.parametrize("n", (255, 256, 511, 513, 1000))
@pytest.mark.parametrize("dt,npdt", TYPES)
def test_inverse_block_edges(port, n, dt, npdt):
    """Orders around the 256-row substitution block and the 128 GEMM tile,
    odd orders (unaligned rows: the element-wise copy path)."""
    a = random_matrix(n, seed=5100 + n, dtype=npdt)
    x_ref, piv_ref, _ = port.getri(a)
    x, piv, info = gpu_inverse(a)
    assert info == 0 and np.array_equal(piv, piv_ref)
    check_inverse(a, x, x_ref)


@pytest.mark.parametrize("n", (3, 198))
@pytest.mark.parametrize("dt,npdt", TYPES)
def test_inverse_reference_test_case(n, dt, npdt):
    """Testing/Cxx/TestInversion.cxx: A = R R^T, ||A^-1 A - I||_max <= 5e-12
    (double) / 2e-4 (float), dimension 128+24+16+12+8+4+3+2+1 = 198 and 3."""
    a = spd_product(n, seed=6000 + n, dtype=npdt)
    x, _, info = gpu_inverse(a)
    assert info == 0
    err = np.abs(x.astype(np.float64) @ a.astype(np.float64) - np.eye(n)).max()
    assert err <= (5e-12 if npdt == np.float64 else 2e-4)


@pytest.mark.parametrize("dt,npdt", TYPES)
def test_inverse_upfront_and_null_pivot_agree(dt, npdt):
    """LU_UPFRONT on the library's own factors, and LU mode with the pivots
    kept in the workspace, give the same bits as LU mode."""
    n = 300
    a = random_matrix(n, seed=5300, dtype=npdt)
    x, piv, _ = gpu_inverse(a)
    m = dev(a)
    gpiv, _ = la.getrf(m)
    lu = m.cpu().numpy()
    x_up, _, info = gpu_inverse(lu, mode=la.LU_UPFRONT_LINEAR_SOLVER, pivot=gpiv.cpu().numpy())
    assert info == 0 and np.array_equal(x_up, x)
    m2 = dev(a)
    nb = la.inversion.workspace_size(n, la.LU_LINEAR_SOLVER, m2.dtype)
    ws = api.workspace(nb)
    la.inversion.apply(m2, None, n, la.LU_LINEAR_SOLVER, ws, ws.numel())
    torch.cuda.synchronize()
    assert np.array_equal(m2.cpu().numpy(), x)


@pytest.mark.parametrize("dt,npdt", TYPES)
def test_inverse_singular_leaves_factors(inverse_golden, dt, npdt):
    a = np.array([[1, 2, 3], [2, 4, 5], [4, 8, 1]], dtype=npdt)
    m, piv, info = gpu_inverse(a)
    assert info == 2
    assert np.array_equal(m, inverse_golden[f"sing_{dt}_m"])
    assert np.array_equal(piv, inverse_golden[f"sing_{dt}_piv"])


def test_inverse_large_residual():
    """n = 4096: a property check at a size the oracle does not reach."""
    n = 4096
    a = random_matrix(n, seed=5400)
    m = dev(a)
    la.inverse(m)
    a_t = dev(a)
    r = torch.mm(a_t, m) - torch.eye(n, dtype=torch.float64, device="cuda")
    res = r.abs().max().item()
    bound = 2 * n * np.finfo(np.float64).eps * np.linalg.norm(a, np.inf) * torch.linalg.matrix_norm(
        m, ord=float("inf")).item()
    assert res <= bound, (res, bound)


@pytest.mark.parametrize("n", INV_SIZES)
@pytest.mark.parametrize("dt,npdt", TYPES)
def test_determinant_bitwise(inverse_golden, n, dt, npdt):
    a = random_matrix(n, seed=5000 + n, dtype=npdt)
    m = dev(a)
    r = la.det(m)
    assert not r["singular"]
    assert np.array_equal(np.array(r["product"], dtype=npdt), inverse_golden[f"inv_{dt}_{n}_det"])
    assert np.array_equal(r["pivot"].cpu().numpy(), inverse_golden[f"inv_{dt}_{n}_piv"])
    sign, logdet = np.linalg.slogdet(a.astype(np.float64))
    assert r["sign"] * np.sign(r["product"]) == sign  # pivot parity times the diagonal's sign
    assert abs(r["log_abs"] - logdet) <= 1e-10 * max(1.0, abs(logdet)) * (1e5 if npdt == np.float32 else 1)
    if np.isfinite(r["product"]) and r["product"] != 0:
        assert r["det"] == r["sign"] * r["product"]
    # LU_UPFRONT on the factors just written
    up = la.det(m, pivot=r["pivot"], type=la.LU_UPFRONT_LINEAR_SOLVER)
    assert np.array_equal(np.array(up["product"], dtype=npdt), np.array(r["product"], dtype=npdt))
    assert up["sign"] == r["sign"]


@pytest.mark.parametrize("dt,npdt", TYPES)
def test_determinant_known_answers(inverse_golden, dt, npdt):
    """Testing/Cxx/TestDeterminant.cxx LU cases: diagonal matrices, the
    identity, a singular diagonal (0)."""
    for name, (diag, expected) in determinant_known_answers().items():
        r = la.det(dev(np.diag(np.array(diag, dtype=npdt))))
        assert r["det"] == expected, name
        assert np.array_equal(np.array(r["product"], dtype=npdt), inverse_golden[f"det_{name}_{dt}"])
        assert r["singular"] == (expected == 0.0)


def test_determinant_sign_of_a_swap():
    """[[0, 1], [1, 0]]: one row interchange, det -1 (the reference's NATIVE
    product is +1; this backend applies the pivot sign like CUDA_BLAS)."""
    r = la.det(dev(np.array([[0.0, 1.0], [1.0, 0.0]])))
    assert r["product"] == 1.0 and r["sign"] == -1 and r["det"] == -1.0


def test_determinant_overflow_keeps_log():
    n = 512
    a = random_matrix(n, seed=5500) * 1e3
    r = la.det(dev(a))
    assert np.isinf(r["product"])
    assert abs(r["log_abs"] - np.linalg.slogdet(a)[1]) < 1e-8 * abs(r["log_abs"])


def test_invalid_arguments_raise():
    m = dev(np.eye(4))
    piv = torch.zeros(4, dtype=torch.int64, device="cuda")
    ws = api.workspace(la.inversion.workspace_size(4, la.LU_LINEAR_SOLVER))
    for mode in (5, 0):  # not a linear_solver_type
        with pytest.raises(la.B200Error):
            la.inversion.apply(m, piv, 4, mode, ws, ws.numel())
    for mode in (5, 0):
        with pytest.raises(la.B200Error):
            la.determinant.apply(m, piv, 4, mode, ws, ws.numel())
    lib = la._lib.load()
    assert lib.b200la_dinverse(None, piv.data_ptr(), 4, 1, ws.data_ptr(), ws.numel(), None) == -1
    assert lib.b200la_ddeterminant(None, piv.data_ptr(), 4, 1, None, None, None, ws.data_ptr(),
                                   ws.numel(), None) == -1
    with pytest.raises(la.B200InvalidArgument):
        la.inversion.apply(m, piv, 0, la.LU_LINEAR_SOLVER, ws, ws.numel())
    with pytest.raises(la.B200InvalidArgument):
        la.inversion.apply(m, None, 4, la.LU_UPFRONT_LINEAR_SOLVER, ws, ws.numel())
    with pytest.raises(la.B200InvalidArgument):
        la.inversion.apply(m, piv, 4, la.LU_LINEAR_SOLVER, ws, 16)
    with pytest.raises(la.B200InvalidArgument):
        la.determinant.apply(m, None, 4, la.LU_UPFRONT_LINEAR_SOLVER, ws, ws.numel())


@pytest.mark.parametrize("dt,npdt", TYPES)
def test_determinant_cholesky_modes(port, dt, npdt):
    """CHOLESKY: the lower factor's diagonal product in index order, bit for
    bit (NATIVE's value, sqrt(det A)); CHOLESKY_UPFRONT on the given factor;
    0 when the matrix is not positive definite."""
    from linearalgebra_b200.workloads import spd_matrix
    for n in (1, 17, 70, 130, 300):
        a = spd_matrix(n, seed=300 + n, dtype=npdt)
        m = dev(a)
        nbytes = la.determinant.workspace_size(n, la.CHOLESKY_LINEAR_SOLVER, m.dtype)
        ws = api.workspace(nbytes)
        prod, sign, log_abs, singular = la.determinant.parts(m, None, n, la.CHOLESKY_LINEAR_SOLVER, ws, ws.numel())
        d_ref, f_ref, _ = port.det(a, mode=3)
        assert np.array_equal(np.array(prod, dtype=npdt), np.array(d_ref)) and sign == 1 and not singular
        assert np.array_equal(m.cpu().numpy(), f_ref)
        l64 = np.log(np.diag(f_ref).astype(np.float64))
        assert abs(log_abs - 2 * l64.sum()) <= 1e-9 * max(1.0, abs(log_abs))
        prod4, _, _, _ = la.determinant.parts(m, None, n, la.CHOLESKY_UPFRONT_LINEAR_SOLVER, ws, ws.numel())
        assert np.array_equal(np.array(prod4, dtype=npdt), np.array(d_ref))
        assert la.determinant.apply(dev(a), None, n, la.CHOLESKY_LINEAR_SOLVER, ws, ws.numel()) == \
            pytest.approx(float(d_ref) ** 2, rel=1e-12)
    bad = dev(spd_matrix(100, seed=5, dtype=npdt, fail_row=60))
    ws = api.workspace(la.determinant.workspace_size(100, la.CHOLESKY_LINEAR_SOLVER, bad.dtype))
    prod, _, _, singular = la.determinant.parts(bad, None, 100, la.CHOLESKY_LINEAR_SOLVER, ws, ws.numel())
    assert prod == 0 and singular

