"""triangular_solver and multiplication on the B200 (GPU), against the
reference's known-answer cases and the golden fixtures."""
import numpy as np
import pytest
import torch

import linearalgebra_b200 as la
from linearalgebra_b200.workloads import triangular_cases

pytestmark = pytest.mark.gpu


def dev(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


@pytest.mark.parametrize("dtype,tol", [(np.float64, 1e-12), (np.float32, 1e-5)])
def test_trsm_known_answers(golden, dtype, tol):
    stream = torch.cuda.Stream()  # non-default stream, as the reference's GPU test
    for key, case in triangular_cases(dtype).items():
        upper, transpose, unit, n, nrhs, lda, ldb, ldx, a, b, expected = case
        da, db = dev(a), dev(b)
        dx = torch.full((n, ldx), -123.0, dtype=da.dtype, device="cuda")
        with torch.cuda.stream(stream):
            la.triangular_solver.apply(upper, transpose, unit, n, nrhs, da, lda, db, ldb, dx, ldx,
                                       None, 0, stream)
        stream.synchronize()
        x = dx.cpu().numpy()
        np.testing.assert_allclose(x[:, :nrhs], expected[:, :nrhs], rtol=0, atol=tol, err_msg=key)
        assert np.all(x[:, nrhs:] == -123.0), key  # padding untouched
        assert np.array_equal(da.cpu().numpy(), a, equal_nan=True)  # A preserved
        assert np.array_equal(db.cpu().numpy(), b)  # B preserved
        if dtype == np.float64:
            ref = golden[f"trsm_{key}_x"]
            np.testing.assert_allclose(x[:, :nrhs], ref[:, :nrhs], rtol=0, atol=1e-13, err_msg=key)


def test_trsm_large_multi_block(port):
    n, nrhs = 1000, 5
    rng = np.random.default_rng(3)
    a = rng.standard_normal((n, n)) * 0.01
    a[np.arange(n), np.arange(n)] = 2.0
    b = rng.standard_normal((n, nrhs))
    for upper in (False, True):
        for transpose in (False, True):
            for unit in (False, True):
                x_ref = np.zeros((n, nrhs))
                port.trsm(upper, transpose, unit, n, nrhs, a, n, b, nrhs, x_ref, nrhs)
                x = la.trsm(upper, transpose, unit, dev(a), dev(b))
                torch.cuda.synchronize()
                np.testing.assert_allclose(x.cpu().numpy(), x_ref, rtol=0, atol=1e-11)


def test_trsm_invalid_arguments():
    a = torch.eye(4, dtype=torch.float64, device="cuda")
    b = torch.ones(4, 2, dtype=torch.float64, device="cuda")
    with pytest.raises(ValueError):
        la.triangular_solver.apply(False, False, False, 4, 2, a, 4, b, 2, b, 2, None, 0)
    with pytest.raises(ValueError):
        la.triangular_solver.apply(False, False, False, 4, 2, a, 3, b, 2,
                                   torch.empty_like(b), 2, None, 0)
    with pytest.raises(ValueError):
        la.triangular_solver.apply(False, False, False, 0, 2, a, 4, b, 2,
                                   torch.empty_like(b), 2, None, 0)


def test_gemm_golden(golden):
    keys = sorted({k.rsplit("_", 1)[0] for k in golden.files if k.startswith("gemm_") and k.endswith("_a")})
    for key in keys:
        _, m, n, k, tt = key.split("_")
        m, n, k = int(m), int(n), int(k)
        ta, tb = bool(int(tt[0])), bool(int(tt[1]))
        a, b, c0 = golden[key + "_a"], golden[key + "_b"], golden[key + "_c0"]
        for alpha, beta in ((1.0, 0.0), (2.5, -0.5), (0.0, 2.0)):
            dc = dev(c0)
            la.gemm(ta, tb, alpha, dev(a), dev(b), beta, dc)
            torch.cuda.synchronize()
            ref = golden[f"{key}_{alpha}_{beta}_c"]
            got = dc.cpu().numpy()
            if not tb:
                # the reference updates c one depth index at a time: same
                # fused operations in the same order
                assert np.array_equal(got, ref), (key, alpha, beta)
            else:
                np.testing.assert_allclose(got, ref, rtol=1e-13, atol=1e-13)


def test_gemm_beta_zero_ignores_nan_and_large_shapes():
    rows, cols, depth = 300, 200, 129
    a = torch.randn(rows, depth, dtype=torch.float64, device="cuda")
    b = torch.randn(depth, cols, dtype=torch.float64, device="cuda")
    c = torch.full((rows, cols), float("nan"), dtype=torch.float64, device="cuda")
    la.gemm(False, False, 1.0, a, b, 0.0, c)
    torch.cuda.synchronize()
    assert torch.isfinite(c).all()
    assert torch.allclose(c, a @ b, rtol=1e-12, atol=1e-12)
    c2 = torch.randn(rows, cols, dtype=torch.float64, device="cuda")
    c3 = c2.clone()
    la.gemm(True, True, -0.5, a.t().contiguous(), b.t().contiguous(), 2.0, c2)
    torch.cuda.synchronize()
    assert torch.allclose(c2, -0.5 * (a @ b) + 2.0 * c3, rtol=1e-12, atol=1e-12)


def test_gemm_float32():
    a = torch.randn(150, 70, dtype=torch.float32, device="cuda")
    b = torch.randn(70, 90, dtype=torch.float32, device="cuda")
    c = torch.zeros(150, 90, dtype=torch.float32, device="cuda")
    la.gemm(False, False, 1.0, a, b, 0.0, c)
    torch.cuda.synchronize()
    ref = a.double() @ b.double()
    assert (c.double() - ref).abs().max().item() < 1e-4


@pytest.mark.parametrize("ta", [False, True])
@pytest.mark.parametrize("alpha,beta", [(1.0, 0.0), (1.0, 1.0), (-0.75, 0.5), (3.0, -2.0)])
def test_gemm_fp64_tensor_core_path_bitwise(port, ta, alpha, beta):
    """FP64 multiplication with op(b) = b runs on the FP64 tensor cores; it
    must keep the reference's bits (beta c, then fma(alpha a_ik, b_kj, c) in
    k order) on sizes that cross the 128 tile and 32-deep stage edges, with
    odd strides (the element-wise copy path) and wide exponents."""
    rng = np.random.default_rng(7)
    for (m, n, k) in ((300, 257, 513), (128, 128, 32), (129, 65, 33), (1, 1, 1)):
        a = rng.standard_normal((k, m) if ta else (m, k)) * np.exp2(rng.integers(-40, 40, size=(k, m) if ta else (m, k)))
        b = rng.standard_normal((k, n))
        c0 = rng.standard_normal((m, n))
        ref = c0.copy()
        port.gemm(int(ta), 0, m, n, k, alpha, a, a.shape[1], b, n, beta, ref, n)
        dc = dev(c0)
        la.gemm(ta, False, alpha, dev(a), dev(b), beta, dc)
        torch.cuda.synchronize()
        assert np.array_equal(dc.cpu().numpy(), ref), (m, n, k, ta, alpha, beta)


@pytest.mark.parametrize("dim,count", [(1, 3), (5, 7), (64, 2), (65, 3), (130, 2), (257, 1)])
@pytest.mark.parametrize("dtype", [np.float64, np.float32])
def test_batched_multiplication_bitwise(port, dim, count, dtype):
    """batched_matrix_multiplication: each entry a sum of products from zero
    in k order (the reference kernel's fma chain), bit for bit against the
    oracle's restatement."""
    rng = np.random.default_rng(dim * 10 + count)
    a = rng.standard_normal((count, dim, dim)).astype(dtype)
    b = rng.standard_normal((count, dim, dim)).astype(dtype)
    ref = port.gemm_batched(a, b)
    got = la.gemm_batched(dev(a), dev(b))
    torch.cuda.synchronize()
    assert np.array_equal(got.cpu().numpy(), ref)


def test_batched_multiplication_matches_reference_kernel():
    """Against the reference's own CUDA kernel (multiplication_batched_cublas.cu,
    built into baseline/_ref by baseline/Makefile) on the same inputs."""
    import ctypes
    import os
    path = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "baseline", "_ref",
                        "libref_cublas.so")
    if not os.path.exists(path):
        pytest.skip("baseline/_ref/libref_cublas.so is not built")
    lib = ctypes.CDLL(path)
    for name in ("ref_cublas_dgemm_batched", "ref_cublas_sgemm_batched"):
        getattr(lib, name).argtypes = [ctypes.c_int64, ctypes.c_int64] + [ctypes.c_void_p] * 4
    for dtype, name in ((torch.float64, "ref_cublas_dgemm_batched"), (torch.float32, "ref_cublas_sgemm_batched")):
        for dim, count in ((48, 5), (200, 3)):
            a = torch.randn(count, dim, dim, dtype=dtype, device="cuda")
            b = torch.randn(count, dim, dim, dtype=dtype, device="cuda")
            ref = torch.empty_like(a)
            assert getattr(lib, name)(dim, count, a.data_ptr(), b.data_ptr(), ref.data_ptr(), None) == 0
            got = la.gemm_batched(a, b)
            torch.cuda.synchronize()
            assert torch.equal(got, ref), (dtype, dim, count)


def test_batched_multiplication_invalid_arguments():
    a = torch.zeros(2, 4, 4, dtype=torch.float64, device="cuda")
    with pytest.raises(la.B200InvalidArgument):
        la.batched_matrix_multiplication(0, 2, a, a, a)
    with pytest.raises(la.B200InvalidArgument):
        la.batched_matrix_multiplication(4, 0, a, a, a)
    lib = la._lib.load()
    assert lib.b200la_dgemm_batched(4, 2, None, a.data_ptr(), a.data_ptr(), None) == -1
