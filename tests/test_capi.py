"""C-ABI checks that need no GPU: the library loads, exports every symbol
include/b200la.h declares, sizes its workspaces on the host, and rejects
invalid arguments before touching a device."""
import ctypes

import pytest

from linearalgebra_b200 import _lib


def test_library_exports_every_declared_symbol():
    lib = _lib.load()
    declared = _lib.declared_symbols()
    assert len(declared) >= 20
    missing = [s for s in declared if not hasattr(lib, s)]
    assert not missing, missing
    # every declared function has a ctypes signature in the binding
    assert set(declared) <= set(_lib.SIGNATURES), set(declared) - set(_lib.SIGNATURES)


def test_workspace_sizes_are_host_side_and_consistent():
    lib = _lib.load()
    for n in (1, 64, 512, 16384):
        d = lib.b200la_dgetrf_workspace_size(n)
        s = lib.b200la_sgetrf_workspace_size(n)
        assert d > 0 and s > 0 and s <= d
        assert lib.b200la_dgesv_workspace_size(n, 1) >= d + 8 * n
        assert lib.b200la_dgesv_workspace_size(n, 2) == lib.b200la_dgesv_workspace_size(n, 1)
        assert lib.b200la_dgetrs_workspace_size(n, 64) >= 8 * n * 64
    for mode in (3, 4):  # Cholesky modes share the LU plan's status and solve buffers
        assert lib.b200la_dgesv_workspace_size(16, mode) == lib.b200la_dgesv_workspace_size(16, 1)
    assert lib.b200la_dgesv_workspace_size(16, 5) == 0
    for f in (lib.b200la_dpotrf, lib.b200la_spotrf):
        info = ctypes.c_int(7)
        assert f(None, 4, 0, None, 0, ctypes.addressof(info), None) == _lib.INVALID_ARGUMENT
        assert f(1 << 20, 0, 0, 1 << 20, 1 << 20, None, None) == _lib.INVALID_ARGUMENT
        assert f(1 << 20, 8, 2, 1 << 20, 1 << 20, None, None) == _lib.INVALID_ARGUMENT
        assert f(1 << 20, 8, 0, 1 << 20, 16, None, None) == _lib.WORKSPACE_TOO_SMALL
    assert lib.b200la_dgesv_workspace_size(0, 1) == 0


def test_inversion_modes_host_side():
    """inversion takes all four linear_solver_type modes; the Cholesky ones
    need no pivot array and the same workspace as the LU ones."""
    lib = _lib.load()
    for n in (1, 64, 513):
        for f in (lib.b200la_dinverse_workspace_size, lib.b200la_sinverse_workspace_size):
            sizes = [f(n, mode) for mode in (1, 2, 3, 4)]
            assert sizes[0] > 0 and len(set(sizes)) == 1
            assert f(n, 0) == 0 and f(n, 5) == 0
    p = 1 << 20
    for mode in (3, 4):
        assert lib.b200la_dinverse(p, None, 4, mode, p, 16, None) == _lib.WORKSPACE_TOO_SMALL
        assert lib.b200la_sinverse(p, None, 4, mode, p, 16, None) == _lib.WORKSPACE_TOO_SMALL
    assert lib.b200la_dinverse(p, None, 4, 5, p, 1 << 20, None) == _lib.INVALID_ARGUMENT
    assert "unsupported linear_solver_type" in _lib.last_error()
    assert lib.b200la_dinverse(p, None, 4, 2, p, 1 << 20, None) == _lib.INVALID_ARGUMENT


def test_cholesky_ir_checks_host_side():
    """b200la_dsolve_mixed_spd factorizes in FP32 or FP64 only, and checks its
    arguments and workspace like b200la_dsolve_mixed before any device work."""
    lib = _lib.load()
    p = 1 << 20
    o = _lib.RefineOptions()
    lib.b200la_refine_default_options(ctypes.byref(o))
    need = lib.b200la_dsolve_mixed_workspace_size(64, 1, ctypes.byref(o))
    assert need > 0
    for prec in (_lib.PREC_TF32, _lib.PREC_BF16, _lib.PREC_FP16, _lib.PREC_FP8):
        o.precision = prec
        assert lib.b200la_dsolve_mixed_spd(p, 64, 1, p, 1, p, 1, ctypes.byref(o), None, p, need,
                                           None) == _lib.INVALID_ARGUMENT
        assert "FP32 or FP64" in _lib.last_error()
    o.precision = _lib.PREC_FP32
    assert lib.b200la_dsolve_mixed_spd(None, 64, 1, p, 1, p, 1, ctypes.byref(o), None, p, need,
                                       None) == _lib.INVALID_ARGUMENT
    assert lib.b200la_dsolve_mixed_spd(p, 64, 1, p, 1, p, 1, ctypes.byref(o), None, p, 16,
                                       None) == _lib.WORKSPACE_TOO_SMALL


def test_status_strings():
    lib = _lib.load()
    for st in (0, 1, 2, -1, -2, -3, -4, -5):
        assert lib.b200la_status_string(st)
    assert lib.b200la_version() >= 100


def test_invalid_arguments_rejected_without_device():
    lib = _lib.load()
    info = ctypes.c_int(0)
    st = lib.b200la_dgetrf(None, 4, None, None, 0, ctypes.addressof(info), None)
    assert st == _lib.INVALID_ARGUMENT
    assert "must not be null" in _lib.last_error()
    st = lib.b200la_dgetrf(1 << 20, 0, 1 << 20, 1 << 20, 1 << 20, None, None)
    assert st == _lib.INVALID_ARGUMENT and "lda must be positive" in _lib.last_error()
    st = lib.b200la_dgetrf(1 << 20, 8, 1 << 20, 1 << 20, 16, None, None)
    assert st == _lib.WORKSPACE_TOO_SMALL
    # triangular_solver argument checks (src/common/triangular_solver_checks.h)
    p = 1 << 20
    assert lib.b200la_dtrsm(0, 0, 0, 0, 1, p, 1, p + 64, 1, p + 128, 1, None, 0, None) == _lib.INVALID_ARGUMENT
    assert lib.b200la_dtrsm(0, 0, 0, 4, 1, p, 4, p, 1, p + 128, 1, None, 0, None) == _lib.INVALID_ARGUMENT
    assert "distinct" in _lib.last_error()
    assert lib.b200la_dtrsm(0, 0, 0, 4, 2, p, 3, p + 64, 2, p + 128, 2, None, 0, None) == _lib.INVALID_ARGUMENT
    assert "row stride" in _lib.last_error()
    # multiplication argument checks
    assert lib.b200la_dgemm(0, 0, 0, 1, 1, 1.0, p, 1, p, 1, 0.0, p, 1, None, 0, None) == _lib.INVALID_ARGUMENT
    assert lib.b200la_dgemm(0, 0, 1, 1, 1, 1.0, None, 1, p, 1, 0.0, p, 1, None, 0, None) == _lib.INVALID_ARGUMENT
    # linear_solver: an unknown mode is rejected; the Cholesky modes need no pivot array
    assert lib.b200la_dgesv(p, p, 4, p, 5, p, 1 << 20, None) == _lib.INVALID_ARGUMENT
    assert "unsupported linear_solver_type" in _lib.last_error()
    assert lib.b200la_dgesv(p, None, 4, p, 1, p, 1 << 20, None) == _lib.INVALID_ARGUMENT
    assert lib.b200la_dgesv(p, None, 4, p, 3, p, 16, None) == _lib.WORKSPACE_TOO_SMALL


def test_python_errors_map_to_exceptions():
    with pytest.raises(ValueError):
        _lib.check(_lib.INVALID_ARGUMENT)
    with pytest.raises(_lib.B200Error):
        _lib.check(_lib.CUDA_ERROR)
    assert _lib.check(_lib.SINGULAR, allow=(_lib.SUCCESS, _lib.SINGULAR)) == _lib.SINGULAR


def test_no_alloc_scratch_covers_its_largest_order():
    lib = _lib.load()
    # the allocation-free solve carves the same plan as b200la_dgesv from a
    # fixed 1 MiB device array, for orders up to 16384
    for mode in (1, 2, 3, 4):
        for n in (1, 129, 4096, 16384):
            size = lib.b200la_dgesv_workspace_size(n, mode)
            assert 0 < size <= 1 << 20, (mode, n, size)


def test_batched_table_rules_and_workspace_host_side():
    """b200la_batched_table_valid (host only): panel widths the kernel is
    built for (FP32 16/32, FP64 8/16), every bucket's largest order fitting
    its group's shared memory and factor scratch; the workspace holds one
    2 MiB factor slot per CTA: min(total_v, 192) slots."""
    from linearalgebra_b200 import _lib
    from linearalgebra_b200.batched import default_table, entry, table_valid

    lib = _lib.load()
    for prec in (_lib.PREC_FP32, _lib.PREC_FP64):
        assert table_valid(prec, default_table(prec))
    whole_cta = [entry(32, 256)] * 8
    assert table_valid(_lib.PREC_FP32, whole_cta)
    assert not table_valid(_lib.PREC_FP32, [entry(24, 256)] * 8)   # no kernel for width 24
    assert not table_valid(_lib.PREC_FP64, whole_cta)              # FP64 goes up to width 16
    assert table_valid(_lib.PREC_FP64, [entry(16, 256)] * 8)
    # a 512-order system does not fit a 64-thread group's quarter of the CTA
    assert not table_valid(_lib.PREC_FP32, [entry(32, 64)] * 8)
    slot = 512 * 512 * 8
    small = lib.b200la_dgesv_batched_workspace_size(10 * 16 * 16, 10 * 16, _lib.PREC_FP32)
    large = lib.b200la_dgesv_batched_workspace_size(20000 * 300 * 300, 20000 * 300, _lib.PREC_FP32)
    # the count is bounded by total_v (every system has at least one row)
    assert 160 * slot <= small < 161 * slot
    assert 192 * slot <= large < 193 * slot
