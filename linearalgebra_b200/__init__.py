"""B200-native (sm_100a) backend for LinearAlgebra's LU-solve path.

Host-side Python mirror of the reference's operator interface over the C ABI
of libb200la.so (include/b200la.h).  The CUDA library is the only compute
path; importing works without it, the first call raises if it is missing.
"""
from . import workloads  # noqa: F401
from ._lib import B200Error, B200InvalidArgument  # noqa: F401
from .api import (  # noqa: F401
    CHOLESKY_LINEAR_SOLVER,
    CHOLESKY_UPFRONT_LINEAR_SOLVER,
    LOWER_TRIANGULAR,
    LU_LINEAR_SOLVER,
    LU_UPFRONT_LINEAR_SOLVER,
    UPPER_TRIANGULAR,
    MixedSolver,
    batched_matrix_multiplication,
    cholesky_decomposition,
    det,
    determinant,
    gemm,
    gemm_batched,
    gesv,
    getrf,
    getrs,
    inverse,
    inversion,
    linear_solver,
    lu_decomposition,
    multiplication,
    potrf,
    solve_mixed,
    transpose,
    transpose_in_place,
    transpose_out,
    triangular_solver,
    trsm,
)
