"""transpose (include/matrix_operation/transpose.h) without a GPU: the oracle
against numpy and the reference's NATIVE build, the C ABI's workspace sizes
and argument checks."""
import os

import numpy as np
import pytest

from linearalgebra_b200 import _lib
from oracle import REF_LIB, Oracle

SHAPES = [(1, 1), (2, 2), (5, 5), (64, 64), (65, 65), (130, 129), (1, 9), (7, 1), (100, 300), (300, 100)]


@pytest.mark.parametrize("shape", SHAPES)
@pytest.mark.parametrize("dt", [np.float64, np.float32])
def test_port_transpose(port, shape, dt):
    a = np.random.default_rng(sum(shape)).standard_normal(shape).astype(dt)
    t = port.transpose(a)
    assert t.shape == (shape[1], shape[0])
    assert np.array_equal(t, a.T)


@pytest.mark.skipif(not os.path.exists(REF_LIB), reason="reference build not present")
@pytest.mark.parametrize("shape", SHAPES + [(1000, 1100)])
def test_port_transpose_equals_reference_build(port, shape):
    """Non-square orders stay below rows * rows * columns = 2^31: the
    reference's cycle-following transpose indexes with int and faults above
    that (transpose_native.cpp, (n * a) % mn1)."""
    ref = Oracle("reference")
    for dt in (np.float64, np.float32):
        a = np.random.default_rng(7).standard_normal(shape).astype(dt)
        assert np.array_equal(port.transpose(a), ref.transpose(a))


def test_transpose_workspace_sizes():
    lib = _lib.load()
    for f, size in ((lib.b200la_dtranspose_workspace_size, 8), (lib.b200la_stranspose_workspace_size, 4)):
        assert f(4096, 4096) == 0
        assert f(1, 1) == 0
        assert f(100, 300) >= 100 * 300 * size
        assert f(0, 5) == 0 and f(5, -1) == 0


def test_transpose_rejects_bad_arguments_without_device():
    lib = _lib.load()
    p = 1 << 20
    assert lib.b200la_dtranspose(4, 4, None, None, 0, None) == _lib.INVALID_ARGUMENT
    assert "m must not be null" in _lib.last_error()
    assert lib.b200la_dtranspose(0, 4, p, None, 0, None) == _lib.INVALID_ARGUMENT
    assert "rows and columns must be positive" in _lib.last_error()
    assert lib.b200la_stranspose(4, -2, p, None, 0, None) == _lib.INVALID_ARGUMENT
    assert lib.b200la_dtranspose(4, 8, p, None, 0, None) == _lib.WORKSPACE_TOO_SMALL
    assert lib.b200la_dtranspose(4, 8, p, p + 4096, 16, None) == _lib.WORKSPACE_TOO_SMALL
    assert lib.b200la_dtranspose_out(4, 8, p, p + 64, None) == _lib.INVALID_ARGUMENT
    assert "overlap" in _lib.last_error()
    assert lib.b200la_dtranspose_out(4, 8, None, p, None) == _lib.INVALID_ARGUMENT
    assert lib.b200la_stranspose_out(4, 0, p, p + 4096, None) == _lib.INVALID_ARGUMENT
