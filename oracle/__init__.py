"""CPU oracles for the LU-solve path.

TEST INFRASTRUCTURE ONLY.  Only tests/, ``__graft_entry__.smoke()`` and the
CPU-baseline leg of ``bench.py`` import this package, and only as the thing
results are checked against (or, for the baseline leg, timed beside the GPU).
The B200 library never imports it.

Two CPU implementations are exposed with one numpy-facing interface:

* ``Oracle("port")``      -- liboracle.so, the plain-C restatement of the
  reference's NATIVE algorithm (lu_oracle_impl.h cites each reference line);
* ``Oracle("reference")`` -- oracle/_ref/libref_native.so, the reference's own
  NATIVE sources compiled by oracle/Makefile (present wherever it was built;
  the built file travels with the repository snapshot).
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
PORT_LIB = os.path.join(HERE, "liboracle.so")
REF_LIB = os.path.join(HERE, "_ref", "libref_native.so")

_i64 = ctypes.c_int64
_p = ctypes.c_void_p
_int = ctypes.c_int

LU_LINEAR_SOLVER = 1
LU_UPFRONT_LINEAR_SOLVER = 2


def build(ref_root: str | None = None) -> None:
    """Compile liboracle.so (always) and oracle/_ref (when the reference
    sources are present)."""
    cmd = ["make", "-s", "-f", os.path.join(HERE, "Makefile")]
    if ref_root:
        cmd.append(f"REF={ref_root}")
    subprocess.run(cmd, check=True)


def available(kind: str) -> bool:
    return os.path.exists(PORT_LIB if kind == "port" else REF_LIB)


def _ptr(a: np.ndarray) -> int:
    return a.ctypes.data


class Oracle:
    """numpy interface over one of the two CPU builds.  Every method works on
    row-major C-contiguous arrays and mirrors the reference call it restates."""

    def __init__(self, kind: str = "port"):
        if kind not in ("port", "reference"):
            raise ValueError(kind)
        path = PORT_LIB if kind == "port" else REF_LIB
        if not os.path.exists(path):
            raise FileNotFoundError(f"{path} is not built (run make -f oracle/Makefile)")
        self.kind = kind
        self.lib = ctypes.CDLL(path)
        pre = "or_" if kind == "port" else "ref_"
        self._pre = pre
        for t in ("d", "s"):
            f = getattr(self.lib, f"{pre}{t}getrf")
            f.argtypes = [_p, _i64, _p, _p]
            f.restype = _int
            f = getattr(self.lib, f"{pre}{t}gesv")
            f.argtypes = [_p, _p, _i64, _p, _int]
            f.restype = _int
            f = getattr(self.lib, f"{pre}{t}trsm")
            f.argtypes = [_int, _int, _int, _i64, _i64, _p, _i64, _p, _i64, _p, _i64]
            f.restype = _int
            f = getattr(self.lib, f"{pre}{t}gemm")
            ct = ctypes.c_double if t == "d" else ctypes.c_float
            f.argtypes = [_int, _int, _i64, _i64, _i64, ct, _p, _i64, _p, _i64, ct, _p, _i64]
            f.restype = _int
            if kind == "port":
                f = getattr(self.lib, f"or_{t}gemm_batched")
                f.argtypes = [_i64, _i64, _p, _p, _p]
                f.restype = _int
            f = getattr(self.lib, f"{pre}{t}potrf")
            f.argtypes = [_p, _i64, _int, _p]
            f.restype = _int
            f = getattr(self.lib, f"{pre}{t}transpose")
            f.argtypes = [_i64, _i64, _p] + ([_p] if kind == "port" else [])
            f.restype = _int
            f = getattr(self.lib, f"{pre}{t}getri")
            f.argtypes = [_p, _p, _i64, _int]
            f.restype = _int
            f = getattr(self.lib, f"{pre}{t}det")
            if kind == "port":
                f.argtypes = [_p, _p, _i64, _int, _p]
                f.restype = ct
            else:
                f.argtypes = [_p, _p, _i64, _int, _p]
                f.restype = _int
        if kind == "port":
            self.lib.or_backward_error.argtypes = [_p, _i64, _i64, _p, _p]
            self.lib.or_backward_error.restype = ctypes.c_double
            self.lib.or_dmin_pivot_gap.argtypes = [_p, _i64]
            self.lib.or_dmin_pivot_gap.restype = ctypes.c_double

    @staticmethod
    def _t(a: np.ndarray) -> str:
        if a.dtype == np.float64:
            return "d"
        if a.dtype == np.float32:
            return "s"
        raise TypeError(a.dtype)

    def getrf(self, a: np.ndarray):
        """In-place LU of a copy of ``a``; returns (lu, pivot[int64, 1-based], info)."""
        m = np.ascontiguousarray(a).copy()
        n = m.shape[0]
        piv = np.full(n, -1, dtype=np.int64)
        info = ctypes.c_int(-1)
        st = getattr(self.lib, f"{self._pre}{self._t(m)}getrf")(
            _ptr(m), n, _ptr(piv), ctypes.addressof(info))
        if st < 0:
            raise ValueError(f"getrf rejected its arguments (status {st})")
        return m, piv, int(info.value)

    def gesv(self, a: np.ndarray, x: np.ndarray, mode: int = LU_LINEAR_SOLVER, pivot=None):
        """linear_solver LU modes on copies; returns (m, pivot, x)."""
        m = np.ascontiguousarray(a).copy()
        xx = np.ascontiguousarray(x).copy()
        n = m.shape[0]
        piv = np.full(n, -1, dtype=np.int64) if pivot is None else np.ascontiguousarray(pivot, dtype=np.int64).copy()
        st = getattr(self.lib, f"{self._pre}{self._t(m)}gesv")(_ptr(m), _ptr(piv), n, _ptr(xx), mode)
        if st < 0:
            raise ValueError(f"gesv rejected its arguments (status {st})")
        return m, piv, xx

    def trsm(self, upper, transpose, unit, n, nrhs, a, lda, b, ldb, x, ldx):
        """triangular_solver on caller arrays (x written in place)."""
        st = getattr(self.lib, f"{self._pre}{self._t(a)}trsm")(
            int(upper), int(transpose), int(unit), n, nrhs, _ptr(a), lda, _ptr(b), ldb, _ptr(x), ldx)
        if st < 0:
            raise ValueError(f"trsm rejected its arguments (status {st})")
        return x

    def gemm(self, ta, tb, rows, cols, depth, alpha, a, lda, b, ldb, beta, c, ldc):
        st = getattr(self.lib, f"{self._pre}{self._t(a)}gemm")(
            int(ta), int(tb), rows, cols, depth, alpha, _ptr(a), lda, _ptr(b), ldb, beta, _ptr(c), ldc)
        if st < 0:
            raise ValueError(f"gemm rejected its arguments (status {st})")
        return c

    def potrf(self, a: np.ndarray, upper: bool = False):
        """cholesky_decomposition (lower, or upper) of a copy; returns
        (factor, info): info 0, or the 1-based index of the first
        non-positive pivot."""
        m = np.ascontiguousarray(a).copy()
        info = ctypes.c_int(-1)
        st = getattr(self.lib, f"{self._pre}{self._t(m)}potrf")(_ptr(m), m.shape[0], int(upper),
                                                              ctypes.addressof(info))
        if st < 0:
            raise ValueError(f"potrf rejected its arguments (status {st})")
        return m, int(info.value)

    def transpose(self, a: np.ndarray) -> np.ndarray:
        """transpose::apply on a copy of the row-major 2-D array a; returns
        the (columns, rows) result."""
        m = np.ascontiguousarray(a).copy()
        rows, cols = m.shape
        f = getattr(self.lib, f"{self._pre}{self._t(m)}transpose")
        if self.kind == "port":
            scratch = np.empty(rows * cols, dtype=m.dtype)
            st = f(rows, cols, _ptr(m), _ptr(scratch))
        else:
            st = f(rows, cols, _ptr(m))
        if st < 0:
            raise ValueError(f"transpose rejected its arguments (status {st})")
        return m.reshape(cols, rows)

    def gemm_batched(self, a: np.ndarray, b: np.ndarray) -> np.ndarray:
        """c_i = a_i b_i for (count, dim, dim) arrays, the reference CUDA
        kernel's arithmetic (port build only: the reference has no CPU
        version)."""
        if self.kind != "port":
            raise NotImplementedError("the reference has no CPU batched multiplication")
        a = np.ascontiguousarray(a)
        b = np.ascontiguousarray(b)
        c = np.empty_like(a)
        st = getattr(self.lib, f"or_{self._t(a)}gemm_batched")(a.shape[1], a.shape[0], _ptr(a), _ptr(b), _ptr(c))
        if st < 0:
            raise ValueError(f"gemm_batched rejected its arguments (status {st})")
        return c

    def getri(self, a: np.ndarray, mode: int = LU_LINEAR_SOLVER, pivot=None):
        """inversion on copies, all four modes (1, 2: LU; 3, 4: Cholesky);
        returns (m, pivot, status): m holds the inverse, or the factors when
        mode 1 met an exact zero pivot (the partial Cholesky factor when mode
        3 met a non-positive one; status is then that 1-based index)."""
        m = np.ascontiguousarray(a).copy()
        n = m.shape[0]
        piv = np.full(n, -1, dtype=np.int64) if pivot is None else np.ascontiguousarray(pivot, dtype=np.int64).copy()
        st = getattr(self.lib, f"{self._pre}{self._t(m)}getri")(_ptr(m), _ptr(piv), n, mode)
        if st < 0:
            raise ValueError(f"inversion rejected its arguments (status {st})")
        return m, piv, int(st)

    def det(self, a: np.ndarray, mode: int = LU_LINEAR_SOLVER, pivot=None):
        """determinant on a copy; returns (value, m, pivot): the reference's
        value (the factor's diagonal product: U's without the pivot sign in
        the LU modes, L's in the Cholesky modes; 0 when mode 1 met an exact
        zero pivot or mode 3 a non-positive one) and the factored matrix."""
        m = np.ascontiguousarray(a).copy()
        n = m.shape[0]
        piv = np.full(n, -1, dtype=np.int64) if pivot is None else np.ascontiguousarray(pivot, dtype=np.int64).copy()
        f = getattr(self.lib, f"{self._pre}{self._t(m)}det")
        if self.kind == "port":
            st = ctypes.c_int(-1)
            val = f(_ptr(m), _ptr(piv), n, mode, ctypes.addressof(st))
            status = st.value
        else:
            out = np.zeros(1, dtype=m.dtype)
            status = f(_ptr(m), _ptr(piv), n, mode, _ptr(out))
            val = out[0]
        if status < 0:
            raise ValueError(f"determinant rejected its arguments (status {status})")
        return m.dtype.type(val), m, piv

    # --- metrics (port build only) ---
    def backward_error(self, a: np.ndarray, x: np.ndarray, b: np.ndarray) -> float:
        a = np.ascontiguousarray(a, dtype=np.float64)
        x = np.ascontiguousarray(x, dtype=np.float64)
        b = np.ascontiguousarray(b, dtype=np.float64)
        return float(self.lib.or_backward_error(_ptr(a), a.shape[0], a.shape[1], _ptr(x), _ptr(b)))

    def min_pivot_gap(self, a: np.ndarray) -> float:
        a = np.ascontiguousarray(a, dtype=np.float64)
        return float(self.lib.or_dmin_pivot_gap(_ptr(a), a.shape[0]))
