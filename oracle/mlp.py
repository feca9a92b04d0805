"""TEST INFRASTRUCTURE ONLY: a numpy statement of the strategy-selector MLP (forward, loss and
backward), the CPU oracle that the device kernels' gradients are checked against.

Network (include/pmb.h, PMB_SELECTOR_*): x[24] -> relu(W1 x + b1)[64] -> relu(W2 h1 + b2)[64]
-> W3 h2 + b3 [5]; outputs 0-3 are strategy scores (shared-memory hash, global hash, sort,
partitioned; softmax cross-entropy), output 4 predicts log2(group count) (squared error weighted
by wreg). Per-sample weights sw scale both terms; the
loss is their mean over the batch. Parameters are laid out W1, b1, W2, b2, W3, b3 (row-major, a
row per output unit). The selector has no counterpart in the reference, so nothing here is pinned
to reference vectors; the test pins this statement to finite differences instead.
"""

from __future__ import annotations

import numpy as np

NF, NH, NS = 24, 64, 4
NO = NS + 1
SIZES = [NH * NF, NH, NH * NH, NH, NO * NH, NO]
N_PARAMS = sum(SIZES)


def unpack(p: np.ndarray):
    p = np.asarray(p, dtype=np.float64)
    out, o = [], 0
    for s in SIZES:
        out.append(p[o:o + s])
        o += s
    W1, b1, W2, b2, W3, b3 = out
    return W1.reshape(NH, NF), b1, W2.reshape(NH, NH), b2, W3.reshape(NO, NH), b3


def forward(p: np.ndarray, X: np.ndarray) -> np.ndarray:
    W1, b1, W2, b2, W3, b3 = unpack(p)
    X = np.asarray(X, dtype=np.float64)
    h1 = np.maximum(X @ W1.T + b1, 0.0)
    h2 = np.maximum(h1 @ W2.T + b2, 0.0)
    return h2 @ W3.T + b3


def loss_and_grad(p, X, cls, y, sw=None, wreg: float = 0.25):
    W1, b1, W2, b2, W3, b3 = unpack(p)
    X = np.asarray(X, dtype=np.float64)
    B = X.shape[0]
    sw = np.ones(B) if sw is None else np.asarray(sw, dtype=np.float64)
    a1 = X @ W1.T + b1
    h1 = np.maximum(a1, 0.0)
    a2 = h1 @ W2.T + b2
    h2 = np.maximum(a2, 0.0)
    o = h2 @ W3.T + b3
    z = o[:, :NS] - o[:, :NS].max(axis=1, keepdims=True)
    e = np.exp(z)
    prob = e / e.sum(axis=1, keepdims=True)
    r = o[:, NS] - y
    w = sw / B
    loss = float(np.sum(w * (-np.log(np.maximum(prob[np.arange(B), cls], 1e-30)) + wreg * r * r)))
    dout = np.zeros_like(o)
    dout[:, :NS] = prob
    dout[np.arange(B), cls] -= 1.0
    dout[:, NS] = wreg * 2.0 * r
    dout *= w[:, None]
    gW3 = dout.T @ h2
    gb3 = dout.sum(0)
    dh2 = (dout @ W3) * (a2 > 0)
    gW2 = dh2.T @ h1
    gb2 = dh2.sum(0)
    dh1 = (dh2 @ W2) * (a1 > 0)
    gW1 = dh1.T @ X
    gb1 = dh1.sum(0)
    grad = np.concatenate([gW1.ravel(), gb1, gW2.ravel(), gb2, gW3.ravel(), gb3])
    return loss, grad


def adam_step(p, g, m, v, step: int, lr: float):
    m = 0.9 * m + 0.1 * g
    v = 0.999 * v + 0.001 * g * g
    c1, c2 = 1 - 0.9 ** step, 1 - 0.999 ** step
    return p - lr * (m / c1) / (np.sqrt(v / c2) + 1e-8), m, v
