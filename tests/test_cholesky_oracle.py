"""CPU checks of the oracle's Cholesky restatement (no GPU): factors, info and
the Cholesky modes of linear_solver against the golden fixtures produced by
the reference's NATIVE build (tests/golden/make_golden.py --cholesky), and
against that build directly when it is present."""
import hashlib
import os

import numpy as np
import pytest

from linearalgebra_b200.workloads import spd_matrix
from oracle import REF_LIB, Oracle

CHOL_SIZES = (1, 2, 3, 17, 63, 64, 65, 130, 200)
TYPES = [("f64", np.float64), ("f32", np.float32)]
CHOLESKY_LINEAR_SOLVER = 3
CHOLESKY_UPFRONT_LINEAR_SOLVER = 4


def sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


@pytest.fixture(scope="module")
def cg():
    return np.load(os.path.join(os.path.dirname(__file__), "golden", "cholesky_golden.npz"))


@pytest.mark.parametrize("n", CHOL_SIZES)
@pytest.mark.parametrize("dt,npdt", TYPES)
def test_port_cholesky_matches_golden_bitwise(port, cg, n, dt, npdt):
    key = f"chol_{dt}_{n}"
    a = spd_matrix(n, seed=7000 + n, dtype=npdt)
    assert sha(a) == str(cg[key + "_a_sha"])
    for upper, tag in ((False, "lower"), (True, "upper")):
        f, info = port.potrf(a, upper=upper)
        assert info == 0
        assert sha(f) == str(cg[f"{key}_{tag}_sha"]), tag
        if f"{key}_{tag}" in cg:
            assert np.array_equal(f, cg[f"{key}_{tag}"])
        tri = np.triu(f, 1) if not upper else np.tril(f, -1)
        assert not tri.any(), "the other triangle is zeroed"


@pytest.mark.parametrize("n", CHOL_SIZES)
@pytest.mark.parametrize("dt,npdt", TYPES)
def test_port_cholesky_solve_matches_golden_bitwise(port, cg, n, dt, npdt):
    key = f"chol_{dt}_{n}"
    a = spd_matrix(n, seed=7000 + n, dtype=npdt)
    b = cg[key + "_b"]
    m, _, x = port.gesv(a, b, CHOLESKY_LINEAR_SOLVER)
    assert np.array_equal(x, cg[key + "_x"])
    assert sha(m) == str(cg[f"{key}_lower_sha"])
    _, _, x4 = port.gesv(m, b, CHOLESKY_UPFRONT_LINEAR_SOLVER)
    assert np.array_equal(x4, cg[key + "_x_upfront"])
    if npdt == np.float64:
        assert port.backward_error(a, x, b) <= 10 * n * np.finfo(np.float64).eps


@pytest.mark.parametrize("dt,npdt", TYPES)
@pytest.mark.parametrize("fail_row", [70, 5])
def test_port_cholesky_not_positive_definite(port, cg, dt, npdt, fail_row):
    """info is the 1-based failing row; the matrix keeps the reference's
    partial state; the Cholesky linear_solver leaves x untouched."""
    key = f"cholfail_{dt}_100_{fail_row}"
    a = spd_matrix(100, seed=7100 + fail_row, dtype=npdt, fail_row=fail_row)
    assert sha(a) == str(cg[key + "_a_sha"])
    f, info = port.potrf(a)
    assert info == int(cg[key + "_info"]) == fail_row + 1
    assert np.array_equal(f, cg[key + "_m"])
    b = np.ones(100, dtype=npdt)
    m, _, x = port.gesv(a, b, CHOLESKY_LINEAR_SOLVER)
    assert np.array_equal(x, b)
    assert np.array_equal(m, f)


PIVOT_CASES = ((10, 100), (12, 312), (21, 111), (45, 345), (70, 370), (95, 7095))


def test_port_cholesky_pivot_rounding_golden(port, cg):
    """Inputs on which the reference build's pivot dot products (its
    dot(a_i, a_i, i) call site: for double, no half vector) round
    differently from its other call sites."""
    for n, seed in PIVOT_CASES:
        f, info = port.potrf(spd_matrix(n, seed=seed))
        assert info == 0 and sha(f) == str(cg[f"pivot_{n}_{seed}_sha"]), (n, seed)


@pytest.mark.skipif(not os.path.exists(REF_LIB), reason="reference build not present")
@pytest.mark.parametrize("dt", [np.float64, np.float32])
def test_port_cholesky_sweep_equals_reference_build(port, dt):
    ref = Oracle("reference")
    for n in range(1, 97):
        for seed in (300 + n, 90 + n):
            a = spd_matrix(n, seed=seed, dtype=dt)
            assert np.array_equal(port.potrf(a)[0], ref.potrf(a)[0]), (n, seed)


@pytest.mark.skipif(not os.path.exists(REF_LIB), reason="reference build not present")
@pytest.mark.parametrize("n", [4, 65, 129, 257])
def test_port_cholesky_equals_reference_build(port, n):
    ref = Oracle("reference")
    for npdt in (np.float64, np.float32):
        a = spd_matrix(n, seed=90 + n, dtype=npdt)
        for upper in (False, True):
            assert sha(port.potrf(a, upper)[0]) == sha(ref.potrf(a, upper)[0])
        b = np.random.default_rng(n).standard_normal(n).astype(npdt)
        for mode in (CHOLESKY_LINEAR_SOLVER,):
            mp, _, xp = port.gesv(a, b, mode)
            mr, _, xr = ref.gesv(a, b, mode)
            assert np.array_equal(mp, mr) and np.array_equal(xp, xr)
            assert np.array_equal(port.gesv(mp, b, 4)[2], ref.gesv(mr, b, 4)[2])


@pytest.mark.parametrize("dt,npdt", TYPES)
def test_port_cholesky_determinant(port, cg, dt, npdt):
    """determinant CHOLESKY modes: the product of the lower factor's diagonal
    in index order (determinant.cpp cholesky_determinant, not squared)."""
    for n in (1, 17, 65, 200):
        a = spd_matrix(n, seed=7000 + n, dtype=npdt)
        d, f, _ = port.det(a, mode=CHOLESKY_LINEAR_SOLVER)
        assert sha(f) == str(cg[f"chol_{dt}_{n}_lower_sha"])
        expect = f[0, 0]
        with np.errstate(over="ignore"):  # FP32 at n = 200 overflows to inf, as the reference's product does
            for i in range(1, n):
                expect = npdt(expect * f[i, i])
        assert d == expect
        d4, _, _ = port.det(f, mode=CHOLESKY_UPFRONT_LINEAR_SOLVER)
        assert np.array_equal(np.array(d4), np.array(d))
    bad = spd_matrix(100, seed=7170, dtype=npdt, fail_row=70)
    assert port.det(bad, mode=CHOLESKY_LINEAR_SOLVER)[0] == 0


@pytest.mark.skipif(not os.path.exists(REF_LIB), reason="reference build not present")
def test_port_cholesky_determinant_equals_reference_build(port):
    ref = Oracle("reference")
    for npdt in (np.float64, np.float32):
        for n in (3, 70, 129):
            a = spd_matrix(n, seed=300 + n, dtype=npdt)
            for mode in (CHOLESKY_LINEAR_SOLVER,):
                dp, fp, _ = port.det(a, mode=mode)
                dr, fr, _ = ref.det(a, mode=mode)
                assert np.array_equal(np.array(dp), np.array(dr)) and np.array_equal(fp, fr)
                assert np.array_equal(np.array(port.det(fp, mode=4)[0]), np.array(ref.det(fr, mode=4)[0]))

