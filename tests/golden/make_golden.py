"""Generate the golden fixtures for the LU-solve path from the reference's own
NATIVE build (oracle/_ref/libref_native.so, built by oracle/Makefile from the
reference sources).

Run from the repository root, where the reference build exists:

    make -f oracle/Makefile && python tests/golden/make_golden.py

Writes tests/golden/lu_golden.npz (LU, solve, triangular solver, GEMM),
tests/golden/inverse_golden.npz (inversion in its LU and Cholesky modes, and
the determinant; `--inverse` writes that one and the next) and
tests/golden/cholesky_golden.npz (Cholesky factor and the Cholesky modes of
linear_solver; `--cholesky` writes only that one).  Every input is seeded (numpy PCG64) or a closed-form
known-answer matrix; each array's name says what it is.
"""
from __future__ import annotations

import hashlib
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from oracle import Oracle  # noqa: E402
from linearalgebra_b200.workloads import (  # noqa: E402
    determinant_known_answers,
    known_answer_matrices,
    random_matrix,
    spd_matrix,
    spd_product,
    system,
    triangular_cases,
)

LU_SIZES = (1, 2, 3, 17, 63, 64, 65, 130, 200)

OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "lu_golden.npz")
OUT_INV = os.path.join(os.path.dirname(os.path.abspath(__file__)), "inverse_golden.npz")
OUT_CHOL = os.path.join(os.path.dirname(os.path.abspath(__file__)), "cholesky_golden.npz")
CHOL_SIZES = (1, 2, 3, 17, 63, 64, 65, 130, 200)
PIVOT_CASES = ((10, 100), (12, 312), (21, 111), (45, 345), (70, 370), (95, 7095))
INV_SIZES = (1, 2, 3, 17, 64, 65, 130, 257)
CHOLINV_SIZES = (1, 2, 3, 17, 63, 64, 65, 130, 257)


def sha(a: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def main() -> None:
    ref = Oracle("reference")
    out: dict[str, np.ndarray] = {}

    # 1. seeded LU cases (float64 and float32): inputs regenerated from the
    #    seed by linearalgebra_b200.workloads; the fixture holds the
    #    reference's factors.
    for n in LU_SIZES:
        for dt in ("f64", "f32"):
            a = random_matrix(n, seed=1000 + n, dtype=np.float64 if dt == "f64" else np.float32)
            lu, piv, info = ref.getrf(a)
            out[f"lu_{dt}_{n}_a_sha"] = np.array(sha(a))
            out[f"lu_{dt}_{n}_lu"] = lu
            out[f"lu_{dt}_{n}_piv"] = piv
            out[f"lu_{dt}_{n}_info"] = np.array(info)

    # 2. known-answer matrices (zero pivots, tiny scale, subnormal pivot)
    for dt, npdt in (("f64", np.float64), ("f32", np.float32)):
        for name, aa in known_answer_matrices(npdt).items():
            lu, piv, info = ref.getrf(aa)
            out[f"ka_{name}_{dt}_a"] = aa
            out[f"ka_{name}_{dt}_lu"] = lu
            out[f"ka_{name}_{dt}_piv"] = piv
            out[f"ka_{name}_{dt}_info"] = np.array(info)

    # 3. the n=512 plain FP64 LU + solve workload: A ~ N(0,1), x_true ~ U[-1,1]
    a, x_true, b = system(512, seed=512)
    m, piv, x = ref.gesv(a, b)
    out["n512_a_sha"] = np.array(sha(a))
    out["n512_b_sha"] = np.array(sha(b))
    out["n512_lu_sha"] = np.array(sha(m))
    out["n512_piv"] = piv
    out["n512_x"] = x
    out["n512_lu_diag"] = np.diag(m).copy()

    # 4. triangular solver known-answer cases (reference outputs)
    for key, case in triangular_cases(np.float64).items():
        upper, transpose, unit, n, nrhs, lda, ldb, ldx, a_t, b_t, expected = case
        x = np.full((n, ldx), -123.0)
        ref.trsm(upper, transpose, unit, n, nrhs, a_t, lda, b_t, ldb, x, ldx)
        out[f"trsm_{key}_x"] = x

    # 5. GEMM cases, all four transpose combinations, alpha/beta variants
    rng = np.random.default_rng(77)
    for (m_, n_, k_) in ((7, 5, 3), (65, 33, 64), (40, 24, 33)):
        for ta in (0, 1):
            for tb in (0, 1):
                a_ = rng.standard_normal((k_, m_) if ta else (m_, k_))
                b_ = rng.standard_normal((n_, k_) if tb else (k_, n_))
                c0 = rng.standard_normal((m_, n_))
                key = f"gemm_{m_}_{n_}_{k_}_{ta}{tb}"
                out[key + "_a"] = a_
                out[key + "_b"] = b_
                out[key + "_c0"] = c0
                for alpha, beta in ((1.0, 0.0), (2.5, -0.5), (0.0, 2.0)):
                    c = c0.copy()
                    ref.gemm(ta, tb, m_, n_, k_, alpha, a_, a_.shape[1], b_, b_.shape[1], beta, c, n_)
                    out[f"{key}_{alpha}_{beta}_c"] = c

    np.savez_compressed(OUT, **out)
    print(f"wrote {OUT}: {len(out)} arrays, {os.path.getsize(OUT)} bytes")


def inverse_main() -> None:
    """Inversion and determinant fixtures.  The large inverses are stored as
    SHA-256 digests of their bytes (the oracle must reproduce them bit for
    bit); the small ones, the pivots and the determinants in full."""
    ref = Oracle("reference")
    out: dict[str, np.ndarray] = {}
    for dt, npdt in (("f64", np.float64), ("f32", np.float32)):
        # 1. seeded N(0,1) matrices, LU mode
        for n in INV_SIZES:
            a = random_matrix(n, seed=5000 + n, dtype=npdt)
            inv, piv, _ = ref.getri(a, mode=1)
            d, lu, dpiv = ref.det(a, mode=1)
            assert np.array_equal(piv, dpiv)
            key = f"inv_{dt}_{n}"
            out[key + "_a_sha"] = np.array(sha(a))
            out[key + "_inv_sha"] = np.array(sha(inv))
            out[key + "_piv"] = piv
            out[key + "_det"] = np.array(d)
            out[key + "_absmax"] = np.array(np.abs(inv).max())
            if n <= 17:
                out[key + "_inv"] = inv
            # LU_UPFRONT on the reference's own factors gives the same inverse
            inv2, _, _ = ref.getri(lu, mode=2, pivot=piv)
            assert sha(inv2) == sha(inv)
        # 2. the reference inversion test's construction (A = R R^T), n = 3, 198
        for n in (3, 198):
            a = spd_product(n, seed=6000 + n, dtype=npdt)
            inv, piv, _ = ref.getri(a, mode=1)
            out[f"spd_{dt}_{n}_a_sha"] = np.array(sha(a))
            out[f"spd_{dt}_{n}_inv_sha"] = np.array(sha(inv))
            out[f"spd_{dt}_{n}_piv"] = piv
        # 3. determinant known answers (diagonal matrices, a singular one)
        for name, (diag, _) in determinant_known_answers().items():
            a = np.diag(np.array(diag, dtype=npdt))
            d, _, _ = ref.det(a, mode=1)
            out[f"det_{name}_{dt}"] = np.array(d)
        # 4. singular LU mode: the inverse call leaves the factors
        a = np.array([[1, 2, 3], [2, 4, 5], [4, 8, 1]], dtype=npdt)
        m, piv, _ = ref.getri(a, mode=1)
        out[f"sing_{dt}_m"] = m
        out[f"sing_{dt}_piv"] = piv
        # 5. Cholesky modes: mode 3 factors and inverts, mode 4 inverts the
        # reference's own lower factor (same bits); a non-positive pivot
        # leaves the partial factor
        for n in CHOLINV_SIZES:
            a = spd_matrix(n, seed=9000 + n, dtype=npdt)
            inv, _, _ = ref.getri(a, mode=3)
            f, info = ref.potrf(a)
            assert info == 0
            inv4, _, _ = ref.getri(f, mode=4)
            assert sha(inv4) == sha(inv)
            key = f"cholinv_{dt}_{n}"
            out[key + "_a_sha"] = np.array(sha(a))
            out[key + "_inv_sha"] = np.array(sha(inv))
            out[key + "_absmax"] = np.array(np.abs(inv).max())
            if n <= 17:
                out[key + "_inv"] = inv
        for n, fr in ((100, 70), (130, 3)):
            a = spd_matrix(n, seed=9100 + fr, dtype=npdt, fail_row=fr)
            m, _, _ = ref.getri(a, mode=3)
            f, info = ref.potrf(a)
            assert info == fr + 1 and np.array_equal(m, f)
            out[f"cholinvfail_{dt}_{n}_{fr}_a_sha"] = np.array(sha(a))
            out[f"cholinvfail_{dt}_{n}_{fr}_m_sha"] = np.array(sha(m))
            out[f"cholinvfail_{dt}_{n}_{fr}_info"] = np.array(info)
    np.savez_compressed(OUT_INV, **out)
    print(f"wrote {OUT_INV}: {len(out)} arrays, {os.path.getsize(OUT_INV)} bytes")


def cholesky_main() -> None:
    """Cholesky fixtures: factors (SHA-256 of the bytes, full up to n=17),
    info, the Cholesky solve, and the state left by a non-positive pivot."""
    ref = Oracle("reference")
    out: dict[str, np.ndarray] = {}
    for dt, npdt in (("f64", np.float64), ("f32", np.float32)):
        for n in CHOL_SIZES:
            a = spd_matrix(n, seed=7000 + n, dtype=npdt)
            key = f"chol_{dt}_{n}"
            out[key + "_a_sha"] = np.array(sha(a))
            for up, tag in ((0, "lower"), (1, "upper")):
                f, info = ref.potrf(a, upper=bool(up))
                assert info == 0
                out[f"{key}_{tag}_sha"] = np.array(sha(f))
                if n <= 17:
                    out[f"{key}_{tag}"] = f
            b = np.random.default_rng(8000 + n).standard_normal(n).astype(npdt)
            m, _, x = ref.gesv(a, b, 3)
            out[key + "_b"] = b
            out[key + "_x"] = x
            _, _, x4 = ref.gesv(m, b, 4)
            out[key + "_x_upfront"] = x4
        for n, fr in ((100, 70), (100, 5)):
            a = spd_matrix(n, seed=7100 + fr, dtype=npdt, fail_row=fr)
            f, info = ref.potrf(a)
            out[f"cholfail_{dt}_{n}_{fr}_a_sha"] = np.array(sha(a))
            out[f"cholfail_{dt}_{n}_{fr}_m"] = f
            out[f"cholfail_{dt}_{n}_{fr}_info"] = np.array(info)
    # inputs whose pivot dot products round differently in the pivot call
    # site of the reference build than in its other call sites
    for n, seed in PIVOT_CASES:
        a = spd_matrix(n, seed=seed)
        f, info = ref.potrf(a)
        assert info == 0
        out[f"pivot_{n}_{seed}_sha"] = np.array(sha(f))
    np.savez_compressed(OUT_CHOL, **out)
    print(f"wrote {OUT_CHOL}: {len(out)} arrays, {os.path.getsize(OUT_CHOL)} bytes")


if __name__ == "__main__":
    args = sys.argv[1:]
    if "--cholesky" in args:
        cholesky_main()
    else:
        if "--inverse" not in args:
            main()
        inverse_main()
        cholesky_main()
