"""Seeded synthetic inputs for the LU-solve path.

Every input the tests and the benchmark use is built here from an explicit
seed with numpy's PCG64 generator, so the same seed gives the same matrix on
any x86 host.  Right-hand sides are formed as b = A x_true with the products
summed in 80-bit extended precision and rounded once, which makes b
independent of the host's BLAS build.

Workloads (n, distributions and constructions follow the reference project's
benchmark definitions for this path):

* ``system(n, seed)``          A iid N(0,1) (no diagonal shift), x_true iid
                               U[-1,1], b = A x_true;
* ``conditioned(n, kappa, seed)`` A = U diag(sigma) V^T with U, V products of 8
                               seeded Householder reflectors and sigma
                               geometric from 1 down to 1/kappa;
* ``batch_sizes(count, seed)`` orders n uniform in [16, 512] for the batched
                               solver, half of them made diagonally dominant.
"""
from __future__ import annotations

import math

import numpy as np


def random_matrix(n: int, seed: int, dtype=np.float64) -> np.ndarray:
    """Row-major n x n matrix with iid N(0,1) entries."""
    rng = np.random.default_rng(seed)
    return rng.standard_normal((n, n)).astype(dtype)


def matvec_exact(a: np.ndarray, x: np.ndarray) -> np.ndarray:
    """b = A x with the products summed in extended precision, rounded once."""
    a = np.asarray(a)
    x = np.asarray(x)
    ld = np.longdouble
    if x.ndim == 1:
        return (a.astype(ld) * x.astype(ld)[None, :]).sum(axis=1).astype(np.float64)
    out = np.empty((a.shape[0], x.shape[1]), dtype=np.float64)
    al = a.astype(ld)
    for j in range(x.shape[1]):
        out[:, j] = (al * x[:, j].astype(ld)[None, :]).sum(axis=1).astype(np.float64)
    return out


def system(n: int, seed: int, nrhs: int = 1):
    """A iid N(0,1), x_true iid U[-1,1] (n, or n x nrhs), b = A x_true."""
    rng = np.random.default_rng(seed)
    a = rng.standard_normal((n, n))
    shape = (n,) if nrhs == 1 else (n, nrhs)
    x_true = rng.uniform(-1.0, 1.0, size=shape)
    b = matvec_exact(a, x_true)
    return a, x_true, b


def householder_vectors(n: int, count: int, rng: np.random.Generator) -> np.ndarray:
    return rng.standard_normal((count, n))


def apply_reflectors_left(m: np.ndarray, vs: np.ndarray) -> np.ndarray:
    """(H_1 ... H_k) m with H = I - 2 v v^T / (v^T v), applied right to left."""
    for v in vs[::-1]:
        beta = 2.0 / float(v @ v)
        m -= beta * np.outer(v, v @ m)
    return m


def conditioned(n: int, kappa: float, seed: int, reflectors: int = 8) -> np.ndarray:
    """A = U diag(sigma) V^T, sigma_i = kappa^(-i/(n-1)); U, V orthogonal
    products of `reflectors` seeded Householder reflectors each."""
    rng = np.random.default_rng(seed)
    sigma = kappa ** (-np.arange(n) / max(n - 1, 1))
    vu = householder_vectors(n, reflectors, rng)
    vv = householder_vectors(n, reflectors, rng)
    m = np.diag(sigma)
    m = apply_reflectors_left(m, vu)  # U diag(sigma)
    # (U S) V^T = ((V (U S)^T))^T
    mt = apply_reflectors_left(np.ascontiguousarray(m.T), vv)
    return np.ascontiguousarray(mt.T)


def batch_sizes(count: int, seed: int, lo: int = 16, hi: int = 512) -> np.ndarray:
    rng = np.random.default_rng(seed)
    return rng.integers(lo, hi + 1, size=count)


def known_answer_matrices(dtype=np.float64) -> dict[str, np.ndarray]:
    """Closed-form LU cases with exact expected status:

    zero_col   first column zero            -> info 1
    rank_def   column 1 zero after one step -> info 2
    zeros2     2x2 zero matrix              -> info 1
    tiny_eye   1e-8 * I                     -> info 0 (no absolute threshold)
    subnormal  [[t, 1], [t/2, 1]], t subnormal -> finite multipliers, info 0
    """
    fin = np.finfo(dtype)
    t = math.ldexp(1.0, fin.minexp - 4)
    return {
        "zero_col": np.array([[0, 1, 2], [0, 3, 4], [0, 5, 7]], dtype=dtype),
        "rank_def": np.array([[1, 2, 3], [2, 4, 5], [4, 8, 1]], dtype=dtype),
        "zeros2": np.zeros((2, 2), dtype=dtype),
        "tiny_eye": np.array([[1e-8, 0], [0, 1e-8]], dtype=dtype),
        "subnormal": np.array([[t, 1], [t / 2, 1]], dtype=dtype),
    }


KNOWN_ANSWER_INFO = {"zero_col": 1, "rank_def": 2, "zeros2": 1, "tiny_eye": 0, "subnormal": 0}


def spd_product(n: int, seed: int, dtype=np.float64) -> np.ndarray:
    """A = R R^T with R unit lower triangular, R[i][j] = 0.4 U[0,1) below the
    diagonal: the construction of the reference's inversion test
    (Testing/Cxx/TestInversion.cxx:46-68), seeded here."""
    rng = np.random.default_rng(seed)
    r = np.tril(0.4 * rng.random((n, n)), -1) + np.eye(n)
    r = r.astype(dtype)
    return (r.astype(np.float64) @ r.T.astype(np.float64)).astype(dtype)


def spd_matrix(n: int, seed: int, dtype=np.float64, fail_row: int = -1) -> np.ndarray:
    """A = R R^T + n I with R iid N(0,1) (symmetric positive definite; the
    product summed in float64, then cast).  fail_row >= 0: that diagonal
    entry set to -1, so the leading block of that order is positive
    definite and the Cholesky pivot of that row is not."""
    rng = np.random.default_rng(seed)
    r = rng.standard_normal((n, n))
    a = r @ r.T + n * np.eye(n)
    if fail_row >= 0:
        a[fail_row, fail_row] = -1.0
    return a.astype(dtype)


def determinant_known_answers() -> dict[str, tuple[list[float], float]]:
    """Diagonal matrices and their determinants, the LU-mode cases of the
    reference's determinant test (Testing/Cxx/TestDeterminant.cxx:84-127):
    name -> (diagonal, determinant)."""
    return {
        "diag2": ([2.0, 3.0], 6.0),
        "diag3": ([2.0, 3.0, 4.0], 24.0),
        "diag4": ([1.0, 2.0, 3.0, 5.0], 30.0),
        "eye1": ([1.0], 1.0),
        "eye4": ([1.0] * 4, 1.0),
        "singular": ([1.0, 0.0, 1.0], 0.0),
    }

TRIANGULAR_SHAPES = ((1, 1), (5, 3), (17, 7), (35, 1), (35, 9), (65, 2))


def triangular_case(upper: bool, transpose: bool, unit: bool, n: int, nrhs: int, dtype=np.float64):
    """Known-answer triangular system: padded strides lda=n+2, ldb=nrhs+1,
    ldx=nrhs+3; the unread triangle (and the diagonal when unit) hold NaN;
    the selected triangle holds 2+0.02 i on the diagonal and
    0.01 sin(i n + j + 1) off it; X_expected[i, j] = sin(i nrhs + j + 1) and
    B = op(A) X_expected."""
    lda, ldb, ldx = n + 2, nrhs + 1, nrhs + 3
    a = np.full((n, lda), np.nan, dtype=dtype)
    for i in range(n):
        for j in range(n):
            if (j >= i) if upper else (j <= i):
                if i == j:
                    a[i, j] = np.nan if unit else 2.0 + 0.02 * i
                else:
                    a[i, j] = 0.01 * math.sin(i * n + j + 1)
    expected = np.full((n, ldx), -123.0, dtype=dtype)
    for i in range(n):
        for j in range(nrhs):
            expected[i, j] = math.sin(i * nrhs + j + 1)
    b = np.full((n, ldb), -123.0, dtype=dtype)
    for i in range(n):
        for j in range(nrhs):
            s = 0.0
            for k in range(n):
                row, col = (k, i) if transpose else (i, k)
                if (col < row) if upper else (col > row):
                    continue
                coef = 1.0 if (unit and row == col) else float(a[row, col])
                s += coef * float(expected[k, j])
            b[i, j] = s
    return lda, ldb, ldx, a, b, expected


def triangular_cases(dtype=np.float64):
    out = {}
    for n, nrhs in TRIANGULAR_SHAPES:
        for upper in (False, True):
            for transpose in (False, True):
                for unit in (False, True):
                    lda, ldb, ldx, a, b, e = triangular_case(upper, transpose, unit, n, nrhs, dtype)
                    key = f"{n}_{nrhs}_{int(upper)}{int(transpose)}{int(unit)}"
                    out[key] = (upper, transpose, unit, n, nrhs, lda, ldb, ldx, a, b, e)
    return out
