"""CPU oracle for the learned precision selector's network (test
infrastructure only: the tests compare the CUDA forward, gradient and Adam
kernels against it; nothing in the library calls it).

The reference has no selector, so there is no reference file to follow; this
is a float64 numpy statement of the same network and optimizer:

    h1 = relu(x W1 + b1), h2 = relu(h1 W2 + b2), logits = h2 W3 + b3,
    p = softmax(logits), loss = -sum_b log p[b, y_b]

Parameter vector layout (5252 floats): W1[12][64] | b1[64] | W2[64][64] |
b2[64] | W3[64][4] | b3[4], row-major.

Adam: Kingma & Ba, ICLR 2015, on the batch-mean gradient plus an L2 term
(g + wd * params), bias-corrected moments.
"""
from __future__ import annotations

import numpy as np

N_IN, N_H, N_OUT = 12, 64, 4
SHAPES = [("W1", (N_IN, N_H)), ("b1", (N_H,)), ("W2", (N_H, N_H)), ("b2", (N_H,)),
          ("W3", (N_H, N_OUT)), ("b3", (N_OUT,))]
N_PARAMS = sum(int(np.prod(s)) for _, s in SHAPES)
assert N_PARAMS == 5252


def unpack(params: np.ndarray) -> dict[str, np.ndarray]:
    out, off = {}, 0
    p = np.asarray(params, dtype=np.float64)
    for name, shape in SHAPES:
        size = int(np.prod(shape))
        out[name] = p[off:off + size].reshape(shape)
        off += size
    return out


def pack(parts: dict[str, np.ndarray]) -> np.ndarray:
    return np.concatenate([np.asarray(parts[name], dtype=np.float64).ravel() for name, _ in SHAPES])


def init_params(seed: int) -> np.ndarray:
    """He-uniform weights, zero biases."""
    rng = np.random.default_rng(seed)
    parts = {}
    for name, shape in SHAPES:
        if name.startswith("W"):
            bound = np.sqrt(6.0 / shape[0])
            parts[name] = rng.uniform(-bound, bound, size=shape)
        else:
            parts[name] = np.zeros(shape)
    return pack(parts).astype(np.float32)


def forward(params: np.ndarray, x: np.ndarray):
    """Returns (probs, cache)."""
    w = unpack(params)
    x = np.asarray(x, dtype=np.float64)
    z1 = x @ w["W1"] + w["b1"]
    h1 = np.maximum(z1, 0.0)
    z2 = h1 @ w["W2"] + w["b2"]
    h2 = np.maximum(z2, 0.0)
    logits = h2 @ w["W3"] + w["b3"]
    m = logits.max(axis=1, keepdims=True)
    e = np.exp(logits - m)
    probs = e / e.sum(axis=1, keepdims=True)
    return probs, (x, z1, h1, z2, h2)


def loss_and_grad(params: np.ndarray, x: np.ndarray, labels: np.ndarray):
    """Summed cross-entropy over the batch and its gradient (not divided by
    the batch size, like the device kernel)."""
    w = unpack(params)
    probs, (x, z1, h1, z2, h2) = forward(params, x)
    y = np.asarray(labels, dtype=np.int64)
    bsz = x.shape[0]
    loss = float(-np.log(np.maximum(probs[np.arange(bsz), y], 1e-30)).sum())
    dl = probs.copy()
    dl[np.arange(bsz), y] -= 1.0
    g = {"W3": h2.T @ dl, "b3": dl.sum(0)}
    dh2 = (dl @ w["W3"].T) * (z2 > 0)
    g["W2"] = h1.T @ dh2
    g["b2"] = dh2.sum(0)
    dh1 = (dh2 @ w["W2"].T) * (z1 > 0)
    g["W1"] = x.T @ dh1
    g["b1"] = dh1.sum(0)
    return loss, pack(g)


def adam_step(params, grads, m1, m2, batch, lr, beta1, beta2, eps, step, weight_decay):
    """One Adam step on grads / batch; returns (params, m1, m2)."""
    p = np.asarray(params, dtype=np.float64)
    g = np.asarray(grads, dtype=np.float64) / batch + weight_decay * p
    m1 = beta1 * np.asarray(m1, dtype=np.float64) + (1 - beta1) * g
    m2 = beta2 * np.asarray(m2, dtype=np.float64) + (1 - beta2) * g * g
    mh = m1 / (1 - beta1 ** step)
    vh = m2 / (1 - beta2 ** step)
    return p - lr * mh / (np.sqrt(vh) + eps), m1, m2


def condition_1(a: np.ndarray) -> float:
    """Exact ||A||_1 ||A^-1||_1 (for checking the device condition estimate)."""
    return float(np.abs(a).sum(0).max() * np.abs(np.linalg.inv(a)).sum(0).max())
