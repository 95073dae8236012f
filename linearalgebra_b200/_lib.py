"""ctypes binding of libb200la.so (the C ABI in include/b200la.h).

The library is the only compute path: if it is missing or no sm_100 device is
present, every call raises.  There is no CPU fallback.
"""
from __future__ import annotations

import ctypes
import os
import re

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libb200la.so")
HEADER = os.path.join(os.path.dirname(HERE), "include", "b200la.h")

SUCCESS = 0
SINGULAR = 1
NOT_CONVERGED = 2
INVALID_ARGUMENT = -1
WORKSPACE_TOO_SMALL = -2
CUDA_ERROR = -3
DEVICE_TIMEOUT = -4
NOT_SUPPORTED = -5

LU_LINEAR_SOLVER = 1
LU_UPFRONT_LINEAR_SOLVER = 2
CHOLESKY_LINEAR_SOLVER = 3
CHOLESKY_UPFRONT_LINEAR_SOLVER = 4

_i64 = ctypes.c_int64
_i32 = ctypes.c_int
_sz = ctypes.c_size_t
_p = ctypes.c_void_p
_d = ctypes.c_double
_f = ctypes.c_float

# name -> (restype, argtypes)
SIGNATURES: dict[str, tuple] = {
    "b200la_last_error": (ctypes.c_char_p, []),
    "b200la_status_string": (ctypes.c_char_p, [_i32]),
    "b200la_version": (_i32, []),
    "b200la_launch_count": (_i64, []),
    "b200la_profile_start": (None, [_i32]),
    "b200la_profile_stop": (_i32, [_i32, _p, _p]),
    "b200la_dgetrf_workspace_size": (_sz, [_i64]),
    "b200la_sgetrf_workspace_size": (_sz, [_i64]),
    "b200la_dgetrf": (_i32, [_p, _i64, _p, _p, _sz, _p, _p]),
    "b200la_sgetrf": (_i32, [_p, _i64, _p, _p, _sz, _p, _p]),
    "b200la_dgetrf_async": (_i32, [_p, _i64, _p, _p, _sz, _p]),
    "b200la_sgetrf_async": (_i32, [_p, _i64, _p, _p, _sz, _p]),
    "b200la_workspace_status": (_i32, [_p, _p, _p]),
    "b200la_test_wait_expiry": (_i32, [_p, _i64, _p, ctypes.c_uint64, _p, _sz, _p]),
    "b200la_panel_exchange_floor": (_i32, [_i32, _i32, _i32, _p, _p, _sz, _p]),
    "b200la_dgesv_workspace_size": (_sz, [_i64, _i32]),
    "b200la_sgesv_workspace_size": (_sz, [_i64, _i32]),
    "b200la_dgesv": (_i32, [_p, _p, _i64, _p, _i32, _p, _sz, _p]),
    "b200la_sgesv": (_i32, [_p, _p, _i64, _p, _i32, _p, _sz, _p]),
    "b200la_dgesv_noalloc": (_i32, [_p, _p, _i64, _p, _i32, _p]),
    "b200la_dgetrs_workspace_size": (_sz, [_i64, _i64]),
    "b200la_dgetrs": (_i32, [_p, _p, _i64, _i64, _p, _i64, _p, _sz, _p]),
    "b200la_dinverse_workspace_size": (_sz, [_i64, _i32]),
    "b200la_sinverse_workspace_size": (_sz, [_i64, _i32]),
    "b200la_dinverse": (_i32, [_p, _p, _i64, _i32, _p, _sz, _p]),
    "b200la_sinverse": (_i32, [_p, _p, _i64, _i32, _p, _sz, _p]),
    "b200la_ddeterminant_workspace_size": (_sz, [_i64, _i32]),
    "b200la_sdeterminant_workspace_size": (_sz, [_i64, _i32]),
    "b200la_ddeterminant": (_i32, [_p, _p, _i64, _i32, _p, _p, _p, _p, _sz, _p]),
    "b200la_sdeterminant": (_i32, [_p, _p, _i64, _i32, _p, _p, _p, _p, _sz, _p]),
    "b200la_dtrsm_workspace_size": (_sz, [_i64, _i64]),
    "b200la_strsm_workspace_size": (_sz, [_i64, _i64]),
    "b200la_dtrsm": (_i32, [_i32, _i32, _i32, _i64, _i64, _p, _i64, _p, _i64, _p, _i64, _p, _sz, _p]),
    "b200la_strsm": (_i32, [_i32, _i32, _i32, _i64, _i64, _p, _i64, _p, _i64, _p, _i64, _p, _sz, _p]),
    "b200la_dgemm_workspace_size": (_sz, [_i64, _i64, _i64]),
    "b200la_sgemm_workspace_size": (_sz, [_i64, _i64, _i64]),
    "b200la_dgemm": (_i32, [_i32, _i32, _i64, _i64, _i64, _d, _p, _i64, _p, _i64, _d, _p, _i64, _p, _sz, _p]),
    "b200la_sgemm": (_i32, [_i32, _i32, _i64, _i64, _i64, _f, _p, _i64, _p, _i64, _f, _p, _i64, _p, _sz, _p]),
    "b200la_dpotrf": (_i32, [_p, _i64, _i32, _p, _sz, _p, _p]),
    "b200la_spotrf": (_i32, [_p, _i64, _i32, _p, _sz, _p, _p]),
    "b200la_dgemm_batched": (_i32, [_i64, _i64, _p, _p, _p, _p]),
    "b200la_sgemm_batched": (_i32, [_i64, _i64, _p, _p, _p, _p]),
    "b200la_dtranspose_workspace_size": (_sz, [_i64, _i64]),
    "b200la_stranspose_workspace_size": (_sz, [_i64, _i64]),
    "b200la_dtranspose": (_i32, [_i64, _i64, _p, _p, _sz, _p]),
    "b200la_stranspose": (_i32, [_i64, _i64, _p, _p, _sz, _p]),
    "b200la_dtranspose_out": (_i32, [_i64, _i64, _p, _p, _p]),
    "b200la_stranspose_out": (_i32, [_i64, _i64, _p, _p, _p]),
    "b200la_refine_default_options": (None, [_p]),
    "b200la_dsolve_mixed_workspace_size": (_sz, [_i64, _i64, _p]),
    "b200la_dsolve_mixed": (_i32, [_p, _i64, _i64, _p, _i64, _p, _i64, _p, _p, _p, _sz, _p]),
    "b200la_dsolve_mixed_spd": (_i32, [_p, _i64, _i64, _p, _i64, _p, _i64, _p, _p, _p, _sz, _p]),
    "b200la_dgesv_batched_workspace_size": (_sz, [_i64, _i64, _i32]),
    "b200la_batched_table_valid": (_i32, [_i32, _p]),
    "b200la_dgesv_batched": (_i32, [_i64, _p, _p, _p, _p, _p, _p, _p, _i64, _i64, _i32, _p, _i32, _d, _p, _p,
                                    _p, _sz, _p]),
    "b200la_tc_update_workspace_size": (_sz, []),
    "b200la_sgemm_tc_update": (_i32, [_i32, _i32, _p, _i64, _i64, _i64, _i64, _p, _p, _p, _p, _p, _sz, _p]),
    "b200la_sgemm_tc_update_fp8": (_i32, [_p, _i64, _i64, _i64, _i64, _p, _p, _p, _p, _p, _sz, _p]),
    "b200la_mlp_param_count": (_i32, []),
    "b200la_mlp_forward": (_i32, [_p, _p, _i64, _p, _p]),
    "b200la_mlp_gradient": (_i32, [_p, _p, _p, _i64, _p, _p, _p]),
    "b200la_mlp_adam": (_i32, [_p, _p, _p, _p, _i64, _f, _f, _f, _f, _i32, _f, _p]),
    "b200la_matrix_stats": (_i32, [_p, _i64, _p, _p]),
    "b200la_selector_features": (_i32, [_p, _i64, _p, _p, _sz, _p]),
    "b200la_dcondition_estimate": (_i32, [_p, _i64, _p, _p, _p, _sz, _p]),
    "b200la_dsolve_selected": (_i32, [_p, _i64, _p, _p, _p, _p, _p, _p, _p, _p, _sz, _p]),
}


PREC_FP64, PREC_FP32, PREC_TF32, PREC_BF16, PREC_FP16, PREC_FP8 = 0, 1, 2, 3, 4, 5
PREC_NAMES = {PREC_FP64: "fp64", PREC_FP32: "fp32", PREC_TF32: "tf32", PREC_BF16: "bf16", PREC_FP16: "fp16",
              PREC_FP8: "fp8"}


class RefineOptions(ctypes.Structure):
    _fields_ = [("precision", ctypes.c_int), ("max_iterations", ctypes.c_int),
                ("tolerance", ctypes.c_double), ("gmres_restart", ctypes.c_int),
                ("escalate", ctypes.c_int)]


class RefineResult(ctypes.Structure):
    _fields_ = [("precision_used", ctypes.c_int), ("info", ctypes.c_int), ("converged", ctypes.c_int),
                ("iterations", ctypes.c_int), ("gmres_iterations", ctypes.c_int),
                ("escalations", ctypes.c_int), ("backward_error", ctypes.c_double),
                ("factor_ms", ctypes.c_double), ("refine_ms", ctypes.c_double)]

    def as_dict(self):
        return {f: getattr(self, f) for f, _ in self._fields_}


class B200Error(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"[{status}] {message}")
        self.status = status


class B200InvalidArgument(B200Error, ValueError):
    pass


_lib = None


def declared_symbols() -> list[str]:
    """Every b200la_* function declared in include/b200la.h."""
    text = open(HEADER).read()
    return sorted(set(re.findall(r"\b(b200la_[a-z0-9_]+)\s*\(", text)))


def load() -> ctypes.CDLL:
    """Load libb200la.so (once).  Raises if it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(
            f"{LIB_PATH} is missing: build it with `python -m linearalgebra_b200.build` "
            "(there is no fallback implementation)")
    lib = ctypes.CDLL(LIB_PATH)
    for name, (res, args) in SIGNATURES.items():
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    _lib = lib
    return lib


def last_error() -> str:
    msg = load().b200la_last_error()
    return msg.decode() if msg else ""


def check(status: int, allow=(SUCCESS,)) -> int:
    """Raise for error statuses; return non-error statuses in `allow`."""
    if status in allow:
        return status
    msg = last_error()
    if status in (INVALID_ARGUMENT, WORKSPACE_TOO_SMALL):
        raise B200InvalidArgument(status, msg)
    raise B200Error(status, msg)
