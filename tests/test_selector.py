"""Learned precision selector: the CPU oracle of the network (finite
differences), the seeded system stream and device construction, the weights
file format (CPU); the CUDA forward / gradient / Adam kernels against the
oracle, training on the GPU, the features, and the selected solve's accuracy
and gain over the method without the network (GPU)."""
import json
import os

import numpy as np
import pytest
import torch

from linearalgebra_b200 import selector as sel
from linearalgebra_b200.workloads import conditioned
from oracle import selector_oracle as orc


# ---------------------------------------------------------------------------
# CPU
# ---------------------------------------------------------------------------
def test_oracle_gradient_matches_finite_differences():
    rng = np.random.default_rng(0)
    p = orc.init_params(3).astype(np.float64)
    p[orc.N_PARAMS - 4:] = rng.normal(size=4) * 0.1  # nonzero output bias
    x = rng.normal(size=(9, 12))
    y = rng.integers(0, 4, 9)
    _, g = orc.loss_and_grad(p, x, y)
    idx = rng.choice(orc.N_PARAMS, 60, replace=False)
    h = 1e-6
    for i in idx:
        e = np.zeros_like(p)
        e[i] = h
        fd = (orc.loss_and_grad(p + e, x, y)[0] - orc.loss_and_grad(p - e, x, y)[0]) / (2 * h)
        assert abs(fd - g[i]) <= 1e-6 * max(1.0, abs(fd)), (i, fd, g[i])


def test_oracle_forward_is_a_distribution():
    rng = np.random.default_rng(1)
    probs, _ = orc.forward(orc.init_params(0), rng.normal(size=(50, 12)))
    assert probs.shape == (50, 4) and np.allclose(probs.sum(1), 1.0) and (probs >= 0).all()


def test_param_layout_matches_oracle():
    assert sel.N_PARAMS == orc.N_PARAMS == 5252
    p = sel.init_params(0)
    parts = orc.unpack(p)
    assert np.all(parts["b1"] == 0) and np.all(parts["b2"] == 0) and np.all(parts["b3"] == 0)
    assert np.abs(parts["W1"]).max() <= np.sqrt(6 / 12) and np.abs(parts["W2"]).max() <= np.sqrt(6 / 64)


def test_sample_stream_is_seeded_and_in_range():
    a = sel.sample_stream(2000, 5)
    assert a == sel.sample_stream(2000, 5)
    ns = np.array([t[0] for t in a])
    ks = np.array([t[1] for t in a])
    assert ns.min() >= 64 and ns.max() <= 4096 and ks.min() >= 1e1 and ks.max() <= 1e12
    # log-uniform: the median of log n sits near the middle of the range
    assert abs(np.median(np.log(ns)) - 0.5 * (np.log(64) + np.log(4096))) < 0.2


def test_device_construction_matches_numpy_generator():
    a = sel.conditioned_device(130, 1e6, 17, device="cpu").numpy()
    b = conditioned(130, 1e6, 17)
    assert np.abs(a - b).max() <= 1e-13
    s = np.linalg.svd(a, compute_uv=False)
    assert abs(s[0] / s[-1] / 1e6 - 1) < 1e-6


def test_weights_file_round_trip_and_checksum(tmp_path):
    net = sel.Network(sel.init_params(4), np.zeros(12), np.ones(12), device="cpu")
    path = str(tmp_path / "w.json")
    net.save(path, {"note": "test"})
    back = sel.Network.load(path, device="cpu")
    assert torch.equal(back.params, net.params)
    d = json.load(open(path))
    d["params"][7] += 1.0
    json.dump(d, open(path, "w"))
    with pytest.raises(ValueError, match="checksum"):
        sel.Network.load(path, device="cpu")
    d["schema"] = "other/0"
    json.dump(d, open(path, "w"))
    with pytest.raises(ValueError, match="schema"):
        sel.Network.load(path, device="cpu")


def test_committed_weights_load():
    if not os.path.exists(sel.DEFAULT_WEIGHTS):
        pytest.skip("no trained weights file")
    net = sel.Network.load(device="cpu")
    meta = json.load(open(sel.DEFAULT_WEIGHTS))["meta"]
    assert meta["systems"] >= 1000 and np.isfinite(net.params.numpy()).all()


def test_committed_label_data_are_the_methods_outcomes():
    """The committed training shards hold, per system, the measured time and
    convergence of each attempted precision (FP8 and BF16 only after the one
    above converged); FP64 always converged, and each label is the fastest
    attempt that did."""
    import glob
    files = sorted(glob.glob(os.path.join(os.path.dirname(sel.__file__), "selector_data", "*.npz")))
    if not files:
        pytest.skip("no label data")
    for f in files:
        d = np.load(f)
        ms, conv, lab = d["ms"], d["converged"].astype(bool), d["labels"]
        assert ms.shape[1] == len(sel.CLASSES) and d["features"].shape[1] == 12
        assert d["n"].min() >= 64 and d["n"].max() <= 4096
        assert d["kappa"].min() >= 10 * (1 - 1e-9) and d["kappa"].max() <= 1e12 * (1 + 1e-9)
        assert conv[:, 3].all() and not np.isnan(ms[:, 2:]).any()
        ok = conv & ~np.isnan(ms)
        assert np.array_equal(np.where(ok, ms, np.inf).argmin(1), lab)


# ---------------------------------------------------------------------------
# GPU
# ---------------------------------------------------------------------------
gpu = pytest.mark.gpu


def _dev(a, dtype=torch.float32):
    return torch.from_numpy(np.ascontiguousarray(a)).to("cuda", dtype)


@gpu
def test_forward_kernel_matches_oracle():
    rng = np.random.default_rng(2)
    p = orc.init_params(5)
    p[-4:] = rng.normal(size=4).astype(np.float32)
    x = rng.normal(size=(1000, 12)).astype(np.float32)
    net = sel.Network(p, np.zeros(12), np.ones(12))
    got = net.probs(_dev(x)).cpu().numpy()
    ref, _ = orc.forward(p, x)
    assert np.abs(got - ref).max() <= 1e-5


@gpu
@pytest.mark.parametrize("batch", [1, 127, 128, 1000])
def test_gradient_kernel_matches_oracle(batch):
    from linearalgebra_b200 import _lib
    rng = np.random.default_rng(batch)
    p = orc.init_params(6)
    p[-4:] = rng.normal(size=4).astype(np.float32)
    x = rng.normal(size=(batch, 12)).astype(np.float32)
    y = rng.integers(0, 4, batch).astype(np.int32)
    dp, dx, dy = _dev(p), _dev(x), torch.from_numpy(y).cuda()
    grads = torch.zeros(5252, device="cuda")
    loss = torch.zeros(1, device="cuda")
    _lib.check(_lib.load().b200la_mlp_gradient(dp.data_ptr(), dx.data_ptr(), dy.data_ptr(), batch,
                                               grads.data_ptr(), loss.data_ptr(), None))
    ref_loss, ref_g = orc.loss_and_grad(p, x, y)
    g = grads.cpu().numpy()
    assert abs(loss.item() - ref_loss) <= 1e-4 * max(1.0, ref_loss)
    assert np.abs(g - ref_g).max() <= 1e-4 * max(1.0, np.abs(ref_g).max())


@gpu
def test_adam_kernel_matches_oracle():
    from linearalgebra_b200 import _lib
    rng = np.random.default_rng(3)
    p = orc.init_params(7)
    g = rng.normal(size=5252).astype(np.float32)
    m1 = rng.normal(size=5252).astype(np.float32) * 0.1
    m2 = np.abs(rng.normal(size=5252)).astype(np.float32) * 0.01
    dp, dg, d1, d2 = _dev(p), _dev(g), _dev(m1), _dev(m2)
    _lib.check(_lib.load().b200la_mlp_adam(dp.data_ptr(), dg.data_ptr(), d1.data_ptr(), d2.data_ptr(), 64,
                                           1e-3, 0.9, 0.999, 1e-8, 5, 1e-4, None))
    rp, r1, r2 = orc.adam_step(p, g, m1, m2, 64, 1e-3, 0.9, 0.999, 1e-8, 5, 1e-4)
    assert np.abs(dp.cpu().numpy() - rp).max() <= 1e-6
    assert np.abs(d1.cpu().numpy() - r1).max() <= 1e-6 and np.abs(d2.cpu().numpy() - r2).max() <= 1e-7
    assert float(dg.abs().max()) == 0.0  # gradients cleared


@gpu
def test_training_on_gpu_learns_a_separable_rule():
    rng = np.random.default_rng(4)
    x = rng.normal(size=(4000, 12)).astype(np.float32)
    y = (np.digitize(x[:, 3] + 0.5 * x[:, 7], [-1.0, 0.0, 1.0])).astype(np.int32)
    net, hist = sel.train(x[:3000], y[:3000], epochs=40, batch=256, lr=3e-3)
    assert hist[-1] < 0.5 * hist[0]
    acc = (net.predict(x[3000:]) == y[3000:]).mean()
    assert acc > 0.9, acc


@gpu
def test_matrix_stats_match_numpy():
    from linearalgebra_b200 import _lib
    rng = np.random.default_rng(8)
    n = 333
    a = rng.normal(size=(n, n))
    a[np.arange(0, n, 3), np.arange(0, n, 3)] += 3 * n  # some dominant rows
    da = _dev(a, torch.float64)
    out = torch.zeros(16, dtype=torch.int64, device="cuda")
    _lib.check(_lib.load().b200la_matrix_stats(da.data_ptr(), n, out.data_ptr(), None))
    w = out.cpu().numpy()
    d = w.view(np.float64)
    ab = np.abs(a)
    rs, cs, dg = ab.sum(1), ab.sum(0), np.abs(np.diag(a))
    off = rs - dg
    assert np.isclose(d[0], rs.max(), rtol=1e-13) and d[1] == ab.max()
    assert np.isclose(d[2], (a * a).sum(), rtol=1e-12)
    assert np.isclose(d[3], (1 / (1 + dg / off)).max(), rtol=1e-12)
    assert w[4] == int((dg / off >= 1).sum())
    assert np.isclose(d[5], cs.max(), rtol=1e-13) and np.isclose(d[6], rs.min(), rtol=1e-13)
    assert d[7] == dg.min() and d[8] == dg.max() and np.isclose(d[9], ab.sum(), rtol=1e-12)
    assert np.isclose(d[10], cs.min(), rtol=1e-13) and np.isclose(d[11], dg.sum(), rtol=1e-12)
    f = sel.features(da)
    assert np.isfinite(f).all() and abs(f[0] - np.log2(n) / 12) < 1e-6
    assert abs(f[6] - (dg / off >= 1).mean()) < 1e-6


@gpu
@pytest.mark.parametrize("kappa", [1e2, 1e6, 1e10])
def test_condition_estimate(kappa):
    n = 300
    a = conditioned(n, kappa, seed=21)
    est = sel.condition_estimate(_dev(a, torch.float64))
    exact = orc.condition_1(a)
    if kappa * 2.0 ** -24 < 1:
        # accurate FP32 factors: Hager's estimate is a lower bound of
        # ||A||_1 ||A^-1||_1, usually within a small factor
        assert exact / 30 <= est <= exact * 1.5, (est, exact)
    else:
        # kappa u32 >> 1: the FP32 factors' inverse is far from A^-1, the
        # estimate only has to flag the ill-conditioning
        assert est >= 1e8, (est, exact)


@gpu
def test_labels_are_the_fastest_converged_attempt():
    for (n, kappa, s) in [(300, 1e2, 3), (900, 1e11, 4)]:
        a, b, _ = sel.make_system(n, kappa, s)
        label, outs = sel.label_system(a, b)
        ok = {p: r["ms"] for p, r in outs.items() if r["converged"] and r["iterations"] <= sel.LABEL_ITERATIONS}
        assert "fp64" in ok and sel.CLASSES[label] == min(ok, key=ok.get)


@gpu
def test_selected_solve_reaches_tolerance_for_every_prediction():
    """Accuracy never depends on the network: a network that always says FP8
    and one that always says FP64 both end at eta <= 1e-14."""
    for cls in (0, 3):
        p = np.zeros(5252, np.float32)
        p[-4 + cls] = 10.0  # output bias selects the class
        net = sel.Network(p, np.zeros(12), np.ones(12))
        for (n, kappa, s) in [(200, 1e3, 1), (700, 1e11, 2)]:
            a, b, _ = sel.make_system(n, kappa, s)
            x, r, pred, _ = sel.solve_selected(net, a, b)
            assert pred == sel.CLASSES[cls]
            assert r["converged"] == 1 and r["backward_error"] <= 1e-14, (cls, n, kappa, r)


@gpu
def test_trained_selector_gains_over_fixed_fp32():
    """The committed network against the method without it on a held-out
    seeded stream: every strategy reaches eta <= 1e-14 and the selected
    solve spends less time than fixed-FP32 refinement with escalation."""
    if not os.path.exists(sel.DEFAULT_WEIGHTS):
        pytest.skip("no trained weights file")
    net = sel.Network.load()
    summary, _ = sel.evaluate(net, 60, seed=12345, strategies=("selected", "fixed_fp32"),
                              n_range=(64, 1024))
    for name in ("selected", "fixed_fp32"):
        assert summary[name]["converged"] == 60 and summary[name]["worst_eta"] <= 1e-14, summary
    assert summary["selected"]["total_ms"] < summary["fixed_fp32"]["total_ms"], summary
