"""Python mirror of the reference's operator interface for the LU-solve path,
over the C ABI.

The reference's API is ``op<T, Backend>::apply(...)`` / ``workspace_size(...)``
(include/matrix_operation/{lu_decomposition,linear_solver,triangular_solver,
multiplication}.h).  Here ``T`` is the tensors' dtype (float64 or float32) and
the backend is always the B200 one.  Arguments keep the reference's names,
order and meaning; device buffers are torch CUDA tensors (row-major,
contiguous where the reference expects a packed matrix); ``stream`` is a
``torch.cuda.Stream`` or ``None`` for the current stream.  Errors raise like
the reference's LINALG_CHECK (ValueError subclasses for invalid arguments).

``inversion`` and ``determinant`` (include/matrix_operation/{inversion,
determinant}.h) follow the same pattern for their LU modes.

Convenience wrappers (``getrf``, ``gesv``, ``getrs``, ``trsm``, ``gemm``,
``inverse``, ``det``) allocate the workspace with torch and return results.
"""
from __future__ import annotations

import ctypes

import torch

from . import _lib

LU_LINEAR_SOLVER = _lib.LU_LINEAR_SOLVER
LU_UPFRONT_LINEAR_SOLVER = _lib.LU_UPFRONT_LINEAR_SOLVER
CHOLESKY_LINEAR_SOLVER = _lib.CHOLESKY_LINEAR_SOLVER
CHOLESKY_UPFRONT_LINEAR_SOLVER = _lib.CHOLESKY_UPFRONT_LINEAR_SOLVER
LOWER_TRIANGULAR = "L"
UPPER_TRIANGULAR = "U"


def _prefix(dtype: torch.dtype) -> str:
    if dtype == torch.float64:
        return "d"
    if dtype == torch.float32:
        return "s"
    raise TypeError(f"unsupported dtype {dtype}: the LU path is float64/float32")


def _stream(stream) -> int:
    if stream is None:
        return torch.cuda.current_stream().cuda_stream
    if isinstance(stream, int):
        return stream
    return stream.cuda_stream


def _ptr(t) -> int:
    if t is None:
        return 0
    if isinstance(t, int):
        return t
    return t.data_ptr()


def workspace(nbytes: int, device=None) -> torch.Tensor:
    """A device byte buffer of at least `nbytes` (at least 256 bytes)."""
    return torch.empty(max(int(nbytes), 256), dtype=torch.uint8,
                       device=device if device is not None else "cuda")


class lu_decomposition:
    """lu_decomposition<T, B200> (include/matrix_operation/lu_decomposition.h:15-54)."""

    @staticmethod
    def workspace_size(lda: int, dtype=torch.float64) -> int:
        return int(getattr(_lib.load(), f"b200la_{_prefix(dtype)}getrf_workspace_size")(lda))

    @staticmethod
    def apply(m: torch.Tensor, lda: int, pivot: torch.Tensor, workspace: torch.Tensor,
              workspace_size: int, stream=None):
        """Factor m in place; returns (ok, info) like the reference's bool and
        host info.  Synchronizes the stream."""
        info = ctypes.c_int(-1)
        f = getattr(_lib.load(), f"b200la_{_prefix(m.dtype)}getrf")
        st = f(_ptr(m), lda, _ptr(pivot), _ptr(workspace), workspace_size,
               ctypes.addressof(info), _stream(stream))
        _lib.check(st, allow=(_lib.SUCCESS, _lib.SINGULAR))
        return st == _lib.SUCCESS, int(info.value)


class cholesky_decomposition:
    """cholesky_decomposition<T, B200> (include/matrix_operation/cholesky_decomposition.h)."""

    @staticmethod
    def workspace_size(lda: int, type: str = LOWER_TRIANGULAR, dtype=torch.float64) -> int:
        return int(getattr(_lib.load(), f"b200la_{_prefix(dtype)}getrf_workspace_size")(lda))

    @staticmethod
    def apply(C: torch.Tensor, lda: int, type: str, workspace: torch.Tensor, workspace_size: int,
              stream=None):
        """Factor C in place (type "L" or "U"); returns (ok, info) like the
        reference's bool and info.  Synchronizes the stream."""
        if type not in (LOWER_TRIANGULAR, UPPER_TRIANGULAR):
            raise _lib.B200InvalidArgument(_lib.INVALID_ARGUMENT, "Unsupported enum type!")
        info = ctypes.c_int(-1)
        f = getattr(_lib.load(), f"b200la_{_prefix(C.dtype)}potrf")
        st = f(_ptr(C), lda, 1 if type == UPPER_TRIANGULAR else 0, _ptr(workspace), workspace_size,
               ctypes.addressof(info), _stream(stream))
        _lib.check(st, allow=(_lib.SUCCESS, _lib.SINGULAR))
        return st == _lib.SUCCESS, int(info.value)


class linear_solver:
    """linear_solver<T, B200>, LU and Cholesky modes (include/matrix_operation/linear_solver.h:26-65)."""

    @staticmethod
    def workspace_size(lda: int, type: int = LU_LINEAR_SOLVER, dtype=torch.float64) -> int:
        return int(getattr(_lib.load(), f"b200la_{_prefix(dtype)}gesv_workspace_size")(lda, type))

    @staticmethod
    def apply(m, pivot, lda: int, x, type: int, workspace, workspace_size: int, stream=None):
        f = getattr(_lib.load(), f"b200la_{_prefix(m.dtype)}gesv")
        _lib.check(f(_ptr(m), _ptr(pivot), lda, _ptr(x), type, _ptr(workspace), workspace_size,
                     _stream(stream)))


class triangular_solver:
    """triangular_solver<T, B200> (include/matrix_operation/triangular_solver.h:20-38)."""

    @staticmethod
    def workspace_size(n: int, nrhs: int, dtype=torch.float64) -> int:
        return int(getattr(_lib.load(), f"b200la_{_prefix(dtype)}trsm_workspace_size")(n, nrhs))

    @staticmethod
    def apply(upper: bool, transpose: bool, unit_diagonal: bool, n: int, nrhs: int, a, lda: int,
              b, ldb: int, x, ldx: int, workspace, workspace_size: int, stream=None):
        f = getattr(_lib.load(), f"b200la_{_prefix(a.dtype)}trsm")
        _lib.check(f(int(upper), int(transpose), int(unit_diagonal), n, nrhs, _ptr(a), lda,
                     _ptr(b), ldb, _ptr(x), ldx, _ptr(workspace), workspace_size, _stream(stream)))


class multiplication:
    """multiplication<T, B200> (include/matrix_operation/multiplication.h:15-114)."""

    @staticmethod
    def workspace_size(rows: int, columns: int, depth: int, dtype=torch.float64) -> int:
        return int(getattr(_lib.load(), f"b200la_{_prefix(dtype)}gemm_workspace_size")(rows, columns, depth))

    @staticmethod
    def apply(transpose_a: bool, transpose_b: bool, rows: int, columns: int, depth: int,
              alpha, a, lda: int, b, ldb: int, beta, c, ldc: int, workspace=None,
              workspace_size: int = 0, stream=None):
        f = getattr(_lib.load(), f"b200la_{_prefix(c.dtype)}gemm")
        _lib.check(f(int(transpose_a), int(transpose_b), rows, columns, depth, float(alpha),
                     _ptr(a), lda, _ptr(b), ldb, float(beta), _ptr(c), ldc, _ptr(workspace),
                     workspace_size, _stream(stream)))


def batched_matrix_multiplication(dim: int, count: int, a, b, c, stream=None):
    """c_i = a_i b_i for `count` packed dim x dim matrices
    (include/matrix_operation/multiplication_batched.h).  Asynchronous."""
    f = getattr(_lib.load(), f"b200la_{_prefix(c.dtype)}gemm_batched")
    _lib.check(f(dim, count, _ptr(a), _ptr(b), _ptr(c), _stream(stream)))


class transpose:
    """transpose<T, B200> (include/matrix_operation/transpose.h): the row-major
    rows x columns matrix m becomes its columns x rows transpose in place."""

    @staticmethod
    def workspace_size(rows: int, columns: int, dtype=torch.float64) -> int:
        return int(getattr(_lib.load(), f"b200la_{_prefix(dtype)}transpose_workspace_size")(rows, columns))

    @staticmethod
    def apply(rows: int, columns: int, m, workspace=None, workspace_size: int = 0, stream=None):
        f = getattr(_lib.load(), f"b200la_{_prefix(m.dtype)}transpose")
        _lib.check(f(rows, columns, _ptr(m), _ptr(workspace), workspace_size, _stream(stream)))


def transpose_in_place(m: torch.Tensor, stream=None) -> torch.Tensor:
    """Transpose the contiguous 2-D tensor m in its own storage; returns the
    (columns, rows) view of that storage."""
    rows, cols = m.shape
    nbytes = transpose.workspace_size(rows, cols, m.dtype)
    ws = workspace(nbytes, m.device) if nbytes else None
    transpose.apply(rows, cols, m, ws, nbytes, stream)
    return m.view(cols, rows)


def transpose_out(src: torch.Tensor, dst: torch.Tensor | None = None, stream=None) -> torch.Tensor:
    """dst = src^T for a contiguous 2-D src (the column-major copy of a
    row-major matrix, and back)."""
    rows, cols = src.shape
    if dst is None:
        dst = torch.empty(cols, rows, dtype=src.dtype, device=src.device)
    f = getattr(_lib.load(), f"b200la_{_prefix(src.dtype)}transpose_out")
    _lib.check(f(rows, cols, _ptr(src), _ptr(dst), _stream(stream)))
    return dst


class inversion:
    """inversion<T, B200>, LU and Cholesky modes (include/matrix_operation/inversion.h:15-53)."""

    @staticmethod
    def workspace_size(lda: int, type: int = LU_LINEAR_SOLVER, dtype=torch.float64) -> int:
        return int(getattr(_lib.load(), f"b200la_{_prefix(dtype)}inverse_workspace_size")(lda, type))

    @staticmethod
    def apply(m, pivot, lda: int, type: int, workspace, workspace_size: int, stream=None):
        """Invert m in place (asynchronous).  pivot may be None in LU mode and
        is not used by the Cholesky modes."""
        f = getattr(_lib.load(), f"b200la_{_prefix(m.dtype)}inverse")
        _lib.check(f(_ptr(m), _ptr(pivot), lda, type, _ptr(workspace), workspace_size, _stream(stream)))


class determinant:
    """determinant<T, B200>, LU and Cholesky modes (include/matrix_operation/determinant.h)."""

    @staticmethod
    def workspace_size(lda: int, type: int = LU_LINEAR_SOLVER, dtype=torch.float64) -> int:
        return int(getattr(_lib.load(), f"b200la_{_prefix(dtype)}determinant_workspace_size")(lda, type))

    @staticmethod
    def parts(m, pivot, lda: int, type: int, workspace, workspace_size: int, stream=None):
        """(product, sign, log_abs, singular): the factor's diagonal product
        in index order (the reference's NATIVE value: U's in the LU modes,
        the Cholesky factor's, i.e. sqrt(det A), in the Cholesky modes), the
        pivot sign (1 in the Cholesky modes), log|det A|, and whether the
        factorization failed (product 0)."""
        ct = ctypes.c_double if m.dtype == torch.float64 else ctypes.c_float
        product, sign, log_abs = ct(0), ctypes.c_int(1), ctypes.c_double(0)
        f = getattr(_lib.load(), f"b200la_{_prefix(m.dtype)}determinant")
        st = f(_ptr(m), _ptr(pivot), lda, type, ctypes.addressof(product), ctypes.addressof(sign),
               ctypes.addressof(log_abs), _ptr(workspace), workspace_size, _stream(stream))
        _lib.check(st, allow=(_lib.SUCCESS, _lib.SINGULAR))
        return product.value, sign.value, log_abs.value, st == _lib.SINGULAR

    @staticmethod
    def apply(m, pivot, lda: int, type: int, workspace, workspace_size: int, stream=None) -> float:
        """det(A): sign * product in the LU modes, product squared in the
        Cholesky modes (0 when the factorization failed)."""
        product, sign, _, _ = determinant.parts(m, pivot, lda, type, workspace, workspace_size, stream)
        if type in (CHOLESKY_LINEAR_SOLVER, CHOLESKY_UPFRONT_LINEAR_SOLVER):
            return product * product
        return 0.0 if product == 0 else (-product if sign < 0 else product)


# ----------------------------------------------------------------------------
# convenience wrappers
# ----------------------------------------------------------------------------
def getrf(m: torch.Tensor, stream=None):
    """In-place LU of the square row-major CUDA tensor m.
    Returns (pivot[int64, 1-based], info)."""
    n = m.shape[0]
    assert m.is_contiguous() and m.shape == (n, n)
    piv = torch.empty(n, dtype=torch.int64, device=m.device)
    nbytes = lu_decomposition.workspace_size(n, m.dtype)
    ws = workspace(nbytes, m.device)
    _, info = lu_decomposition.apply(m, n, piv, ws, ws.numel(), stream)
    return piv, info


def gesv(m: torch.Tensor, x: torch.Tensor, pivot: torch.Tensor | None = None,
         type: int = LU_LINEAR_SOLVER, stream=None):
    """linear_solver in place on (m, x): LU modes (pivot filled or, in
    LU_UPFRONT mode, read) and Cholesky modes (m's lower triangle factored
    or, in CHOLESKY_UPFRONT mode, read; pivot unused).  Returns the pivot
    tensor."""
    n = m.shape[0]
    if pivot is None:
        pivot = torch.empty(n, dtype=torch.int64, device=m.device)
    nbytes = linear_solver.workspace_size(n, type, m.dtype)
    ws = workspace(nbytes, m.device)
    linear_solver.apply(m, pivot, n, x, type, ws, ws.numel(), stream)
    return pivot


def potrf(m: torch.Tensor, upper: bool = False, stream=None):
    """cholesky_decomposition in place on m; returns info (0 or the 1-based
    index of the first non-positive pivot)."""
    n = m.shape[0]
    ws = workspace(cholesky_decomposition.workspace_size(n, dtype=m.dtype), m.device)
    _, info = cholesky_decomposition.apply(m, n, UPPER_TRIANGULAR if upper else LOWER_TRIANGULAR, ws,
                                           ws.numel(), stream)
    return info


def getrs(lu: torch.Tensor, pivot: torch.Tensor, x: torch.Tensor, stream=None):
    """Solve with existing factors, x (n x nrhs, row-major) in place."""
    n = lu.shape[0]
    nrhs = 1 if x.dim() == 1 else x.shape[1]
    ldx = 1 if x.dim() == 1 else x.stride(0)
    lib = _lib.load()
    nbytes = lib.b200la_dgetrs_workspace_size(n, nrhs)
    ws = workspace(nbytes, lu.device)
    _lib.check(lib.b200la_dgetrs(_ptr(lu), _ptr(pivot), n, nrhs, _ptr(x), ldx, _ptr(ws),
                                 ws.numel(), _stream(stream)))
    return x


def inverse(m: torch.Tensor, pivot: torch.Tensor | None = None, type: int = LU_LINEAR_SOLVER,
            stream=None):
    """inversion in place on m, any of the four modes.  Returns (pivot,
    info): info is the factorization's LAPACK info (nonzero: m holds the
    factors -- the partial Cholesky factor in CHOLESKY mode -- not the
    inverse).  Synchronizes the stream to read it."""
    n = m.shape[0]
    if pivot is None:
        pivot = torch.empty(n, dtype=torch.int64, device=m.device)
    nbytes = inversion.workspace_size(n, type, m.dtype)
    ws = workspace(nbytes, m.device)
    inversion.apply(m, pivot, n, type, ws, ws.numel(), stream)
    info = ctypes.c_int(0)
    _lib.check(_lib.load().b200la_workspace_status(_ptr(ws), ctypes.addressof(info), _stream(stream)),
               allow=(_lib.SUCCESS, _lib.SINGULAR))
    return pivot, int(info.value)


def det(m: torch.Tensor, pivot: torch.Tensor | None = None, type: int = LU_LINEAR_SOLVER, stream=None):
    """determinant, any of the four modes (m factored in place in the LU and
    CHOLESKY modes).  Returns a dict with det (signed), product, sign,
    log_abs, singular and the pivot tensor."""
    n = m.shape[0]
    if pivot is None:
        pivot = torch.empty(n, dtype=torch.int64, device=m.device)
    nbytes = determinant.workspace_size(n, type, m.dtype)
    ws = workspace(nbytes, m.device)
    product, sign, log_abs, singular = determinant.parts(m, pivot, n, type, ws, ws.numel(), stream)
    value = 0.0 if product == 0 else (-product if sign < 0 else product)
    return {"det": value, "product": product, "sign": sign, "log_abs": log_abs, "singular": singular,
            "pivot": pivot}


def gemm_batched(a: torch.Tensor, b: torch.Tensor, stream=None) -> torch.Tensor:
    """(count, dim, dim) tensors -> their products, one per matrix."""
    c = torch.empty_like(a)
    batched_matrix_multiplication(a.shape[1], a.shape[0], a, b, c, stream)
    return c


def trsm(upper, transpose, unit, a, b, x=None, stream=None):
    n = a.shape[0]
    nrhs = b.shape[1]
    if x is None:
        x = torch.empty_like(b)
    triangular_solver.apply(upper, transpose, unit, n, nrhs, a, a.stride(0), b, b.stride(0),
                            x, x.stride(0), None, 0, stream)
    return x


def gemm(transpose_a, transpose_b, alpha, a, b, beta, c, stream=None):
    rows, cols = c.shape
    depth = a.shape[0] if transpose_a else a.shape[1]
    multiplication.apply(transpose_a, transpose_b, rows, cols, depth, alpha, a, a.stride(0),
                         b, b.stride(0), beta, c, c.stride(0), None, 0, stream)
    return c


# ----------------------------------------------------------------------------
# mixed-precision LU-IR (extension; no reference counterpart)
# ----------------------------------------------------------------------------
PRECISIONS = {"fp64": _lib.PREC_FP64, "fp32": _lib.PREC_FP32, "tf32": _lib.PREC_TF32,
              "bf16": _lib.PREC_BF16, "fp16": _lib.PREC_FP16, "fp8": _lib.PREC_FP8}


def refine_options(precision="fp32", tolerance=1e-14, max_iterations=50, gmres_restart=30, escalate=True):
    o = _lib.RefineOptions()
    _lib.load().b200la_refine_default_options(ctypes.byref(o))
    o.precision = PRECISIONS[precision] if isinstance(precision, str) else int(precision)
    o.tolerance = tolerance
    o.max_iterations = max_iterations
    o.gmres_restart = gmres_restart
    o.escalate = int(bool(escalate))
    return o


class MixedSolver:
    """Reusable workspace + call of b200la_dsolve_mixed (spd: the Cholesky-IR,
    b200la_dsolve_mixed_spd) for one (n, nrhs, options)."""

    def __init__(self, n, nrhs=1, device=None, spd=False, **opts):
        self.n, self.nrhs = n, nrhs
        self.entry = "b200la_dsolve_mixed_spd" if spd else "b200la_dsolve_mixed"
        self.opts = refine_options(**opts)
        lib = _lib.load()
        self.nbytes = int(lib.b200la_dsolve_mixed_workspace_size(n, nrhs, ctypes.byref(self.opts)))
        self.ws = workspace(self.nbytes, device)

    def __call__(self, a, b, x=None, stream=None):
        n, nrhs = self.n, self.nrhs
        if x is None:
            x = torch.empty_like(b)
        ldb = 1 if b.dim() == 1 else b.stride(0)
        ldx = 1 if x.dim() == 1 else x.stride(0)
        res = _lib.RefineResult()
        st = getattr(_lib.load(), self.entry)(_ptr(a), n, nrhs, _ptr(b), ldb, _ptr(x), ldx,
                                              ctypes.byref(self.opts), ctypes.byref(res), _ptr(self.ws),
                                              self.nbytes, _stream(stream))
        _lib.check(st, allow=(_lib.SUCCESS, _lib.NOT_CONVERGED, _lib.SINGULAR))
        return x, res.as_dict(), st


def solve_mixed(a, b, precision="fp32", spd=False, **opts):
    """Mixed-precision LU-IR solve of a x = b (FP64 CUDA tensors, a row-major
    n x n, b n or n x nrhs); spd: the Cholesky-IR for a symmetric positive
    definite a (precision fp32 or fp64).  Returns (x, result dict, status)."""
    nrhs = 1 if b.dim() == 1 else b.shape[1]
    solver = MixedSolver(a.shape[0], nrhs, a.device, spd=spd, precision=precision, **opts)
    return solver(a, b)
