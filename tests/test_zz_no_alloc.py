"""The allocation-free linear solve, b200la_dgesv_noalloc (GPU).

It serves callers that cannot allocate device memory -- a host-language
binding or plugin host that is handed only the matrix, pivot and
right-hand-side pointers, or a service that forbids allocation after start-up
-- by keeping the solve's scratch in a fixed device array inside the library.
These tests call it through the C ABI and compare it with the workspace entry
point b200la_dgesv on the same inputs, on two calls in a row (the shared
scratch keeps the previous call's contents, so the second call checks that
everything that must start cleared is cleared).  This file is collected last
so that a failure here does not hide the other tests.
"""
import numpy as np
import pytest
import torch

from linearalgebra_b200 import _lib
from linearalgebra_b200.workloads import known_answer_matrices, system

pytestmark = pytest.mark.gpu

EPS64 = np.finfo(np.float64).eps


def _dev(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def _with_workspace(a, b, mode=1, pivot=None):
    lib = _lib.load()
    n = a.shape[0]
    m, x = _dev(a), _dev(b)
    piv = torch.empty(n, dtype=torch.int64, device="cuda") if pivot is None else _dev(pivot)
    nbytes = lib.b200la_dgesv_workspace_size(n, mode)
    ws = torch.empty(nbytes, dtype=torch.uint8, device="cuda")
    st = lib.b200la_dgesv(m.data_ptr(), piv.data_ptr(), n, x.data_ptr(), mode, ws.data_ptr(),
                          nbytes, torch.cuda.current_stream().cuda_stream)
    _lib.check(st)
    torch.cuda.synchronize()
    return m.cpu().numpy(), piv.cpu().numpy(), x.cpu().numpy()


def _no_alloc(a, b, mode=1, pivot=None):
    lib = _lib.load()
    n = a.shape[0]
    m, x = _dev(a), _dev(b)
    piv = torch.empty(n, dtype=torch.int64, device="cuda") if pivot is None else _dev(pivot)
    st = lib.b200la_dgesv_noalloc(m.data_ptr(), piv.data_ptr(), n, x.data_ptr(), mode,
                                  torch.cuda.current_stream().cuda_stream)
    _lib.check(st)
    torch.cuda.synchronize()
    return m.cpu().numpy(), piv.cpu().numpy(), x.cpu().numpy()


def test_no_alloc_matches_workspace_entry_point_twice(port):
    for call, (n, seed) in enumerate(((512, 7), (1000, 8))):
        a, _, b = system(n, seed=seed)
        m1, p1, x1 = _with_workspace(a, b)
        m2, p2, x2 = _no_alloc(a, b)
        assert np.array_equal(p2, p1), f"call {call}: pivots differ"
        assert np.array_equal(m2, m1), f"call {call}: factors differ"
        np.testing.assert_allclose(x2, x1, rtol=0, atol=1e-12 * np.abs(x1).max())
        assert port.backward_error(a, x2, b) <= 10 * n * EPS64


def test_no_alloc_singular_then_regular_and_upfront():
    # a singular system leaves x unchanged and must not leak its status into
    # the next call through the shared scratch
    z = known_answer_matrices(np.float64)["rank_def"]
    zb = np.array([1.0, 2.0, 3.0])
    _, _, xz = _no_alloc(z, zb)
    assert np.array_equal(xz, zb)
    a, _, b = system(300, seed=9)
    m1, p1, x1 = _with_workspace(a, b)
    m2, p2, x2 = _no_alloc(a, b)
    assert np.array_equal(p2, p1) and np.array_equal(m2, m1)
    np.testing.assert_allclose(x2, x1, rtol=0, atol=1e-12 * np.abs(x1).max())
    # LU_UPFRONT with the factors and pivots of the previous call
    _, _, x3 = _with_workspace(m1, b, mode=2, pivot=p1)
    _, _, x4 = _no_alloc(m1, b, mode=2, pivot=p1)
    np.testing.assert_allclose(x4, x3, rtol=0, atol=1e-12 * np.abs(x3).max())


def test_no_alloc_cholesky_modes_twice(port):
    """The Cholesky modes (no pivot array): same factor and solution as the
    workspace entry point, on two calls in a row."""
    from linearalgebra_b200.workloads import spd_matrix
    lib = _lib.load()
    for call, n in enumerate((300, 700)):
        a = spd_matrix(n, seed=40 + n)
        b = np.random.default_rng(n).standard_normal(n)
        m1, _, x1 = _with_workspace(a, b, mode=3)
        m, x = _dev(a), _dev(b)
        _lib.check(lib.b200la_dgesv_noalloc(m.data_ptr(), None, n, x.data_ptr(), 3,
                                            torch.cuda.current_stream().cuda_stream))
        torch.cuda.synchronize()
        m2, x2 = m.cpu().numpy(), x.cpu().numpy()
        assert np.array_equal(m2, m1), f"call {call}: factors differ"
        np.testing.assert_allclose(x2, x1, rtol=0, atol=1e-12 * np.abs(x1).max())
        assert port.backward_error(a, x2, b) <= 10 * n * EPS64
        x = _dev(b)
        _lib.check(lib.b200la_dgesv_noalloc(m.data_ptr(), None, n, x.data_ptr(), 4,
                                            torch.cuda.current_stream().cuda_stream))
        torch.cuda.synchronize()
        np.testing.assert_allclose(x.cpu().numpy(), x1, rtol=0, atol=1e-12 * np.abs(x1).max())


def test_no_alloc_failed_cholesky_leaves_x_and_next_call_unaffected():
    """A non-positive-definite matrix in mode 3 leaves x unchanged; the next
    call, which finds the failed call's status and factor state in the
    shared scratch, still matches b200la_dgesv."""
    from linearalgebra_b200.workloads import spd_matrix
    lib = _lib.load()
    s = torch.cuda.current_stream().cuda_stream
    n = 400
    bad = spd_matrix(n, seed=77, fail_row=200)  # the pivot of row 200 is not positive
    b = np.random.default_rng(3).standard_normal(n)
    m, x = _dev(bad), _dev(b)
    _lib.check(lib.b200la_dgesv_noalloc(m.data_ptr(), None, n, x.data_ptr(), 3, s))
    torch.cuda.synchronize()
    assert np.array_equal(x.cpu().numpy(), b), "x changed although the factorization failed"
    for call, nn in enumerate((400, 650)):
        a = spd_matrix(nn, seed=78 + call)
        bb = np.random.default_rng(4 + call).standard_normal(nn)
        m1, _, x1 = _with_workspace(a, bb, mode=3)
        m2, x2 = _dev(a), _dev(bb)
        _lib.check(lib.b200la_dgesv_noalloc(m2.data_ptr(), None, nn, x2.data_ptr(), 3, s))
        torch.cuda.synchronize()
        assert np.array_equal(m2.cpu().numpy(), m1), f"call {call}: factors differ"
        np.testing.assert_allclose(x2.cpu().numpy(), x1, rtol=0, atol=1e-12 * np.abs(x1).max())


def test_no_alloc_rejects_orders_beyond_its_scratch():
    lib = _lib.load()
    p = torch.empty(8, dtype=torch.float64, device="cuda").data_ptr()
    st = lib.b200la_dgesv_noalloc(p, p, 16385, p, 1, None)
    assert st == _lib.INVALID_ARGUMENT
    assert "16384" in _lib.last_error()
    st = lib.b200la_dgesv_noalloc(None, p, 16, p, 1, None)
    assert st == _lib.INVALID_ARGUMENT
