"""CPU checks of the oracle (no GPU): the plain-C restatement against the
golden fixtures produced by the reference's own NATIVE build, and against
that build directly when it is present."""
import hashlib
import os

import numpy as np
import pytest

from linearalgebra_b200.workloads import (
    KNOWN_ANSWER_INFO,
    known_answer_matrices,
    random_matrix,
    spd_matrix,
    system,
    triangular_cases,
)
from oracle import REF_LIB, Oracle

LU_SIZES = (1, 2, 3, 17, 63, 64, 65, 130, 200)
EPS64 = np.finfo(np.float64).eps


def sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


@pytest.mark.parametrize("n", LU_SIZES)
@pytest.mark.parametrize("dt", ["f64", "f32"])
def test_port_lu_matches_golden_bitwise(port, golden, n, dt):
    a = random_matrix(n, seed=1000 + n, dtype=np.float64 if dt == "f64" else np.float32)
    assert sha(a) == str(golden[f"lu_{dt}_{n}_a_sha"]), "seeded generator drifted"
    lu, piv, info = port.getrf(a)
    assert np.array_equal(piv, golden[f"lu_{dt}_{n}_piv"])
    assert np.array_equal(lu, golden[f"lu_{dt}_{n}_lu"])
    assert info == int(golden[f"lu_{dt}_{n}_info"])


@pytest.mark.parametrize("name", sorted(KNOWN_ANSWER_INFO))
@pytest.mark.parametrize("dt,npdt", [("f64", np.float64), ("f32", np.float32)])
def test_port_known_answers(port, golden, name, dt, npdt):
    a = known_answer_matrices(npdt)[name]
    lu, piv, info = port.getrf(a)
    assert info == KNOWN_ANSWER_INFO[name]
    assert info == int(golden[f"ka_{name}_{dt}_info"])
    assert np.array_equal(piv, golden[f"ka_{name}_{dt}_piv"])
    np.testing.assert_array_equal(lu, golden[f"ka_{name}_{dt}_lu"])
    assert np.all(np.isfinite(lu))
    n = a.shape[0]
    assert np.all((piv >= np.arange(1, n + 1)) & (piv <= n))
    # P L U reconstructs A (reference test tolerance: 16 eps)
    L = np.tril(lu.astype(np.float64), -1) + np.eye(n)
    U = np.triu(lu.astype(np.float64))
    r = L @ U
    for i in range(n - 1, -1, -1):
        p = piv[i] - 1
        if p != i:
            r[[i, p]] = r[[p, i]]
    tol = 16 * np.finfo(npdt).eps
    if name == "subnormal":
        tol = np.finfo(npdt).tiny
    assert np.max(np.abs(r - a)) <= tol


def test_port_n512_solve_matches_golden(port, golden):
    a, x_true, b = system(512, seed=512)
    assert sha(a) == str(golden["n512_a_sha"])
    assert sha(b) == str(golden["n512_b_sha"])
    m, piv, x = port.gesv(a, b)
    assert np.array_equal(piv, golden["n512_piv"])
    assert sha(m) == str(golden["n512_lu_sha"])
    assert np.array_equal(x, golden["n512_x"])
    eta = port.backward_error(a, x, b)
    assert eta <= 10 * 512 * EPS64
    assert port.min_pivot_gap(a) > 1e-9


def test_port_upfront_mode_reuses_factors(port):
    a, _, b = system(100, seed=3)
    m, piv, x1 = port.gesv(a, b)
    _, _, x2 = port.gesv(m, b, mode=2, pivot=piv)
    assert np.array_equal(x1, x2)


def test_port_singular_leaves_x(port):
    a = known_answer_matrices(np.float64)["rank_def"]
    b = np.array([1.0, 2.0, 3.0])
    _, _, x = port.gesv(a, b)
    assert np.array_equal(x, b)


@pytest.mark.parametrize("key", sorted(triangular_cases(np.float64)))
def test_port_trsm_known_answers(port, golden, key):
    upper, transpose, unit, n, nrhs, lda, ldb, ldx, a, b, expected = triangular_cases(np.float64)[key]
    a0, b0 = a.copy(), b.copy()
    x = np.full((n, ldx), -123.0)
    port.trsm(upper, transpose, unit, n, nrhs, a, lda, b, ldb, x, ldx)
    assert np.array_equal(x, golden[f"trsm_{key}_x"])
    np.testing.assert_allclose(x[:, :nrhs], expected[:, :nrhs], rtol=0, atol=1e-13)
    assert np.all(x[:, nrhs:] == -123.0)
    assert np.array_equal(a0, a, equal_nan=True) and np.array_equal(b0, b)


def test_port_trsm_rejects_bad_arguments(port):
    a = np.eye(4)
    b = np.ones((4, 2))
    x = np.zeros((4, 2))
    with pytest.raises(ValueError):
        port.trsm(0, 0, 0, 0, 2, a, 4, b, 2, x, 2)
    with pytest.raises(ValueError):
        port.trsm(0, 0, 0, 4, 2, a, 3, b, 2, x, 2)
    with pytest.raises(ValueError):
        port.trsm(0, 0, 0, 4, 2, a, 4, b, 2, b, 2)


def test_port_gemm_matches_golden(port, golden):
    keys = sorted({k.rsplit("_", 1)[0] for k in golden.files if k.startswith("gemm_") and k.endswith("_a")})
    assert keys
    for key in keys:
        _, m, n, k, tt = key.split("_")
        m, n, k = int(m), int(n), int(k)
        ta, tb = int(tt[0]), int(tt[1])
        a, b, c0 = golden[key + "_a"], golden[key + "_b"], golden[key + "_c0"]
        for alpha, beta in ((1.0, 0.0), (2.5, -0.5), (0.0, 2.0)):
            c = c0.copy()
            port.gemm(ta, tb, m, n, k, alpha, a, a.shape[1], b, b.shape[1], beta, c, n)
            assert np.array_equal(c, golden[f"{key}_{alpha}_{beta}_c"]), (key, alpha, beta)


@pytest.mark.skipif(not os.path.exists(REF_LIB), reason="reference build not present")
@pytest.mark.parametrize("n", [1, 5, 64, 65, 129, 257, 300])
def test_port_equals_reference_build(port, n):
    ref = Oracle("reference")
    for npdt in (np.float64, np.float32):
        a = random_matrix(n, seed=77 + n, dtype=npdt)
        lp, pp, ip = port.getrf(a)
        lr, pr, ir = ref.getrf(a)
        assert np.array_equal(pp, pr) and np.array_equal(lp, lr) and ip == ir
        x = np.random.default_rng(n).uniform(-1, 1, n).astype(npdt)
        b = (a.astype(np.float64) @ x.astype(np.float64)).astype(npdt)
        assert np.array_equal(port.gesv(a, b)[2], ref.gesv(a, b)[2])


def test_backward_error_metric(port):
    a, x_true, b = system(64, seed=9)
    assert port.backward_error(a, x_true, b) < 4 * EPS64
    assert port.backward_error(a, x_true + 1e-6, b) > 1e-8


# ---- inversion / determinant ------------------------------------------------
INV_SIZES = (1, 2, 3, 17, 64, 65, 130, 257)
INV_TYPES = [("f64", np.float64), ("f32", np.float32)]


@pytest.mark.parametrize("n", INV_SIZES)
@pytest.mark.parametrize("dt,npdt", INV_TYPES)
def test_port_inverse_matches_golden_bitwise(port, inverse_golden, n, dt, npdt):
    g = inverse_golden
    key = f"inv_{dt}_{n}"
    a = random_matrix(n, seed=5000 + n, dtype=npdt)
    assert sha(a) == str(g[key + "_a_sha"])
    inv, piv, st = port.getri(a, mode=1)
    assert st == 0
    assert np.array_equal(piv, g[key + "_piv"])
    assert sha(inv) == str(g[key + "_inv_sha"])
    if key + "_inv" in g:
        assert np.array_equal(inv, g[key + "_inv"])
    d, lu, dpiv = port.det(a, mode=1)
    assert np.array_equal(dpiv, piv)
    assert np.array_equal(np.array(d), g[key + "_det"])
    # LU_UPFRONT on the factors: same inverse, same determinant
    inv2, _, _ = port.getri(lu, mode=2, pivot=piv)
    assert sha(inv2) == sha(inv)
    d2, _, _ = port.det(lu, mode=2, pivot=piv)
    assert np.array_equal(np.array(d2), np.array(d))


@pytest.mark.parametrize("n", (3, 198))
@pytest.mark.parametrize("dt,npdt", INV_TYPES)
def test_port_inverse_spd_case(port, inverse_golden, n, dt, npdt):
    """The reference inversion test's construction: golden bits and its
    acceptance bound ||A^-1 A - I||_max <= 5e-12 (double) / 2e-4 (float)."""
    from linearalgebra_b200.workloads import spd_product
    a = spd_product(n, seed=6000 + n, dtype=npdt)
    assert sha(a) == str(inverse_golden[f"spd_{dt}_{n}_a_sha"])
    inv, piv, _ = port.getri(a, mode=1)
    assert sha(inv) == str(inverse_golden[f"spd_{dt}_{n}_inv_sha"])
    assert np.array_equal(piv, inverse_golden[f"spd_{dt}_{n}_piv"])
    err = np.abs(inv.astype(np.float64) @ a.astype(np.float64) - np.eye(n)).max()
    assert err <= (5e-12 if npdt == np.float64 else 2e-4)


@pytest.mark.parametrize("dt,npdt", INV_TYPES)
def test_port_determinant_known_answers(port, inverse_golden, dt, npdt):
    from linearalgebra_b200.workloads import determinant_known_answers
    for name, (diag, expected) in determinant_known_answers().items():
        d, _, _ = port.det(np.diag(np.array(diag, dtype=npdt)), mode=1)
        assert d == expected, name
        assert np.array_equal(np.array(d), inverse_golden[f"det_{name}_{dt}"]), name


@pytest.mark.parametrize("dt,npdt", INV_TYPES)
def test_port_singular_inverse_leaves_factors(port, inverse_golden, dt, npdt):
    a = np.array([[1, 2, 3], [2, 4, 5], [4, 8, 1]], dtype=npdt)
    m, piv, st = port.getri(a, mode=1)
    assert st == 2
    assert np.array_equal(m, inverse_golden[f"sing_{dt}_m"])
    assert np.array_equal(piv, inverse_golden[f"sing_{dt}_piv"])
    lu, lpiv, _ = port.getrf(a)
    assert np.array_equal(m, lu) and np.array_equal(piv, lpiv)


CHOLINV_SIZES = (1, 2, 3, 17, 63, 64, 65, 130, 257)


@pytest.mark.parametrize("n", CHOLINV_SIZES)
@pytest.mark.parametrize("dt,npdt", INV_TYPES)
def test_port_cholesky_inverse_matches_golden_bitwise(port, inverse_golden, n, dt, npdt):
    """inversion's CHOLESKY modes (inversion_native.cpp:306-410): mode 3
    factors and inverts, mode 4 inverts the given lower factor; both give
    the reference build's bits, and the result is symmetric."""
    g = inverse_golden
    key = f"cholinv_{dt}_{n}"
    a = spd_matrix(n, seed=9000 + n, dtype=npdt)
    assert sha(a) == str(g[key + "_a_sha"])
    inv, _, st = port.getri(a, mode=3)
    assert st == 0
    assert sha(inv) == str(g[key + "_inv_sha"])
    if key + "_inv" in g:
        assert np.array_equal(inv, g[key + "_inv"])
    assert np.array_equal(inv, inv.T)
    f, info = port.potrf(a)
    assert info == 0
    # the upper triangle of a mode-4 input is not read
    f_junk = f + np.triu(np.full((n, n), 7.0, dtype=npdt), 1)
    inv4, _, st4 = port.getri(f_junk, mode=4)
    assert st4 == 0 and sha(inv4) == sha(inv)
    err = np.abs(inv.astype(np.float64) @ a.astype(np.float64) - np.eye(n)).max()
    assert err <= (1e-12 if npdt == np.float64 else 1e-4)


@pytest.mark.parametrize("n,fr", [(100, 70), (130, 3)])
@pytest.mark.parametrize("dt,npdt", INV_TYPES)
def test_port_cholesky_inverse_failed_pivot_leaves_factor(port, inverse_golden, n, fr, dt, npdt):
    key = f"cholinvfail_{dt}_{n}_{fr}"
    a = spd_matrix(n, seed=9100 + fr, dtype=npdt, fail_row=fr)
    assert sha(a) == str(inverse_golden[key + "_a_sha"])
    m, _, st = port.getri(a, mode=3)
    assert st == fr + 1 == int(inverse_golden[key + "_info"])
    assert sha(m) == str(inverse_golden[key + "_m_sha"])
    assert np.array_equal(m, port.potrf(a)[0])


def test_port_inverse_rejects_bad_mode(port):
    with pytest.raises(ValueError):
        port.getri(np.eye(3), mode=5)
    with pytest.raises(ValueError):
        port.det(np.eye(3), mode=5)


@pytest.mark.skipif(not os.path.exists(REF_LIB), reason="reference build not present")
@pytest.mark.parametrize("n", [5, 66, 129])
def test_port_inverse_equals_reference_build(port, n):
    ref = Oracle("reference")
    for npdt in (np.float64, np.float32):
        a = random_matrix(n, seed=88 + n, dtype=npdt)
        assert sha(port.getri(a)[0]) == sha(ref.getri(a)[0])
        assert np.array_equal(np.array(port.det(a)[0]), np.array(ref.det(a)[0]))
        s = spd_matrix(n, seed=77 + n, dtype=npdt)
        assert sha(port.getri(s, mode=3)[0]) == sha(ref.getri(s, mode=3)[0])
        f = port.potrf(s)[0]
        assert sha(port.getri(f, mode=4)[0]) == sha(ref.getri(f, mode=4)[0])
