"""Batched solver of many uneven systems in one launch (GPU)."""
import numpy as np
import pytest
import torch

from linearalgebra_b200 import _lib
from linearalgebra_b200.batched import BatchedSolver, make_batch


def test_make_batch_layout():
    sizes, a, b, x_true = make_batch(10, seed=3)
    solver = BatchedSolver(sizes, "fp32")
    assert a.numel() == solver.total_a and b.numel() == solver.total_v
    # even-indexed systems carry n*I (diagonally dominant)
    A0 = solver.views(a, 0, True)
    assert float(A0.diagonal().abs().min()) > 0.5 * int(sizes[0])

pytestmark = pytest.mark.gpu


def host_views(solver, a, b, x, i):
    return (solver.views(a, i, True).cpu().numpy(), solver.views(b, i, False).cpu().numpy(),
            solver.views(x, i, False).cpu().numpy())


@pytest.mark.parametrize("precision", ["fp32", "fp64"])
def test_batched_matches_oracle(port, precision):
    rng = np.random.default_rng(5)
    sizes = rng.integers(16, 513, size=120)
    sizes[:3] = [512, 16, 17]  # the extremes
    solver = BatchedSolver(sizes, precision)
    a = torch.randn(solver.total_a, dtype=torch.float64, device="cuda")
    xt = torch.rand(solver.total_v, dtype=torch.float64, device="cuda") * 2 - 1
    b = torch.empty_like(xt)
    for i in range(solver.count):
        b[int(solver.offv_h[i]):int(solver.offv_h[i]) + int(sizes[i])] = solver.views(a, i, True) @ solver.views(xt, i, False)
    x = torch.empty_like(b)
    solver.launch(a, b, x)
    torch.cuda.synchronize()
    status = solver.status.cpu().numpy()
    berr = solver.berr.cpu().numpy()
    assert np.all(status >= 0), status[status < 0]
    tol = 1e-14 if precision == "fp32" else 1e-14
    assert berr.max() <= tol, berr.max()
    for i in list(range(6)) + list(rng.choice(solver.count, 10, replace=False)):
        A, B, X = host_views(solver, a, b, x, int(i))
        assert port.backward_error(A, X, B) <= 1e-14
        _, _, xr = port.gesv(A, B)
        # both solutions have normwise backward error <= 1e-14, so they can
        # differ by about kappa_inf(A) * 2e-14 relative to |x|
        kappa = np.linalg.cond(A, np.inf)
        fe = np.abs(X - xr).max() / np.abs(xr).max()
        assert fe <= 4 * kappa * 1e-14, (fe, kappa)


@pytest.mark.parametrize("threads", [64, 128, 256])
def test_batched_group_sizes_match_oracle(port, threads):
    """Every threads-per-system choice (a CTA solving 4, 2 or 1 systems at
    once) and both panel widths give solutions at eta <= 1e-14."""
    from linearalgebra_b200.batched import entry, table_valid
    rng = np.random.default_rng(threads)
    sizes = np.concatenate([rng.integers(1, 129, size=40), [1, 2, 3, 31, 32, 33, 64, 65, 127, 128]])
    for nb in (16, 32, 7):
        table = [entry(nb, threads)] * 2 + [entry(16, 256)] * 6
        if not table_valid(_lib.PREC_FP32, table):
            continue
        solver = BatchedSolver(sizes, "fp32", nb_table=table)
        a = torch.randn(solver.total_a, dtype=torch.float64, device="cuda")
        b = torch.randn(solver.total_v, dtype=torch.float64, device="cuda")
        x = torch.empty_like(b)
        solver.launch(a, b, x)
        torch.cuda.synchronize()
        st = solver.status.cpu().numpy()
        assert np.all(st >= 0), (nb, st)
        assert solver.berr.max().item() <= 1e-14
        for i in range(0, solver.count, 7):
            A, B, X = host_views(solver, a, b, x, i)
            assert port.backward_error(A, X, B) <= 1e-14


def test_batched_unsorted_order_is_safe(port):
    """An order that is not largest first (a larger system after a smaller
    one in a chunk) is solved with the whole CTA instead of overflowing a
    group's shared memory."""
    sizes = np.array([20, 500, 30, 480, 100, 512, 17, 256])
    solver = BatchedSolver(sizes, "fp32")
    solver.order = torch.arange(len(sizes), dtype=torch.int32, device="cuda")
    a = torch.randn(solver.total_a, dtype=torch.float64, device="cuda")
    b = torch.randn(solver.total_v, dtype=torch.float64, device="cuda")
    x = torch.empty_like(b)
    solver.launch(a, b, x)
    torch.cuda.synchronize()
    assert np.all(solver.status.cpu().numpy() >= 0)
    for i in range(len(sizes)):
        A, B, X = host_views(solver, a, b, x, i)
        assert port.backward_error(A, X, B) <= 1e-14


def test_batched_singular_and_graph(tmp_path, monkeypatch):
    monkeypatch.setenv("B200LA_TUNE_CACHE", str(tmp_path / "tune.json"))
    sizes = np.array([40, 300, 33, 129])
    solver = BatchedSolver(sizes, "fp32")
    a = torch.randn(solver.total_a, dtype=torch.float64, device="cuda")
    # system 2: column 7 zero -> exactly singular U
    v = solver.views(a, 2, True)
    v[:, 7] = 0.0
    b = torch.randn(solver.total_v, dtype=torch.float64, device="cuda")
    x = torch.zeros_like(b)
    solver.capture(a, b, x)
    x.zero_()
    solver.replay()
    torch.cuda.synchronize()
    st = solver.status.cpu().numpy()
    assert st[2] == -8, st
    assert st[0] >= 0 and st[1] >= 0 and st[3] >= 0
    x1 = x.clone()
    solver.replay()
    torch.cuda.synchronize()
    assert torch.equal(x1, x)
    entry = solver.autotune(a, b, x, sample_per_bucket=2)
    assert len(entry["nb_table"]) == 8
    assert all(p["panel_width"] in (16, 32) and p["threads_per_system"] in (64, 128, 256)
               for p in entry["per_bucket"])
    assert (tmp_path / "tune.json").exists()
    again = solver.autotune(a, b, x)  # from the cache
    assert again["nb_table"] == entry["nb_table"]
