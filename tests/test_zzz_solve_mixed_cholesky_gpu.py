"""Mixed-precision Cholesky-IR (b200la_dsolve_mixed_spd) on the GPU.

The FP32 Cholesky factor of a symmetric positive definite A, used in LU form
(L D^-1, D L^T, identity permutation) by the FP64 refinement of the mixed LU
solve, must reach the requested normwise backward error and agree with the
FP64 Cholesky solve of the oracle (bit-identical to the reference's NATIVE
solve) to what the conditioning allows.  A matrix that is not positive
definite ends the FP32 attempt with info = the failing row and escalates to
the plain FP64 LU.  This file is collected last so that a failure here does
not hide the other tests.
"""
import numpy as np
import pytest
import torch

import linearalgebra_b200 as la
from linearalgebra_b200.workloads import spd_matrix, spd_product

pytestmark = pytest.mark.gpu


def dev(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def eta_of(a, x, b):
    r = b - a @ x
    return np.abs(r).max() / (np.abs(a).sum(1).max() * np.abs(x).max() + np.abs(b).max())


@pytest.mark.parametrize("n", (300, 1100, 2048))
def test_cholesky_ir_reaches_fp64_accuracy(port, n):
    a = spd_matrix(n, seed=9400 + n)
    x_true = np.random.default_rng(n).uniform(-1, 1, n)
    b = a @ x_true
    x, res, st = la.solve_mixed(dev(a), dev(b), precision="fp32", spd=True)
    torch.cuda.synchronize()
    assert st == 0 and res["converged"] == 1, res
    assert res["precision_used"] == la._lib.PREC_FP32 and res["escalations"] == 0, res
    assert res["iterations"] <= 6, res
    xs = x.cpu().numpy()
    assert eta_of(a, xs, b) <= 1e-14
    _, _, x_ref = port.gesv(a, b, la.CHOLESKY_LINEAR_SOLVER)
    # each solution is within 2 kappa eta of x_true (eta's denominator holds ||b||)
    kappa = np.linalg.cond(a, np.inf)
    assert np.abs(xs - x_ref).max() <= 4e-14 * kappa * np.abs(x_ref).max()


@pytest.mark.parametrize("n,nrhs", [(701, 5), (700, 64)])
def test_cholesky_ir_multi_rhs(n, nrhs):
    a = spd_matrix(n, seed=9500 + n)
    b = a @ np.random.default_rng(nrhs).uniform(-1, 1, (n, nrhs))
    x, res, st = la.solve_mixed(dev(a), dev(b), precision="fp32", spd=True)
    torch.cuda.synchronize()
    assert st == 0 and res["converged"] == 1 and res["escalations"] == 0, res
    xs = x.cpu().numpy()
    for j in range(nrhs):
        assert eta_of(a, xs[:, j], b[:, j]) <= 1e-14, j


def test_cholesky_ir_reference_test_matrix():
    """A = R R^T with R unit lower (Testing/Cxx/TestInversion.cxx's
    construction; kappa_inf about 5e5 at n = 198): still FP32."""
    n = 198
    a = spd_product(n, seed=6000 + n)
    b = a @ np.random.default_rng(1).uniform(-1, 1, n)
    x, res, st = la.solve_mixed(dev(a), dev(b), precision="fp32", spd=True)
    torch.cuda.synchronize()
    assert st == 0 and res["converged"] == 1, res
    assert eta_of(a, x.cpu().numpy(), b) <= 1e-14


@pytest.mark.parametrize("n,fr", [(300, 250), (1100, 5)])
def test_cholesky_ir_not_positive_definite(n, fr):
    """The FP32 Cholesky stops at row fr; with escalation the plain FP64 LU
    solves the (symmetric, indefinite) system, without it the call reports
    the failing row."""
    a = spd_matrix(n, seed=9600 + fr, fail_row=fr)
    b = a @ np.random.default_rng(fr).uniform(-1, 1, n)
    x, res, st = la.solve_mixed(dev(a), dev(b), precision="fp32", spd=True)
    torch.cuda.synchronize()
    assert st == 0 and res["converged"] == 1, res
    assert res["precision_used"] == la._lib.PREC_FP64 and res["escalations"] == 1, res
    assert eta_of(a, x.cpu().numpy(), b) <= 1e-14
    _, res1, st1 = la.solve_mixed(dev(a), dev(b), precision="fp32", spd=True, escalate=False)
    torch.cuda.synchronize()
    assert st1 == la._lib.SINGULAR and res1["info"] == fr + 1, res1
