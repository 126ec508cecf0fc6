"""CPU FP64 restatement of the planner cost model's network, loss and gradients (the checker of the device kernels
in crd_b200/csrc/mlp.cu). Test infrastructure only.

Network: a1 = relu(W1 x + b1), a2 = relu(W2 a1 + b2), y = W3 a2 + b3; loss = mean((y - t)^2). Parameters are one
flat array [W1 (H x D)][b1 (H)][W2 (H x H)][b2 (H)][W3 (H)][b3 (1)], weights row-major (out x in).
The reference has no learned planner (its per-level board is measured offline,
include/crd/hesap/fft/detail/level_plans_gen.hpp:33-148), so this oracle is pinned by finite differences, not by
reference vectors.
"""

from __future__ import annotations

import numpy as np


def unpack(p: np.ndarray, d: int, h: int):
    p = np.asarray(p, dtype=np.float64)
    i = 0
    W1 = p[i:i + h * d].reshape(h, d); i += h * d
    b1 = p[i:i + h]; i += h
    W2 = p[i:i + h * h].reshape(h, h); i += h * h
    b2 = p[i:i + h]; i += h
    W3 = p[i:i + h]; i += h
    b3 = p[i]; i += 1
    assert i == p.size
    return W1, b1, W2, b2, W3, b3


def forward(p, x, d, h):
    W1, b1, W2, b2, W3, b3 = unpack(p, d, h)
    x = np.asarray(x, dtype=np.float64)
    z1 = x @ W1.T + b1
    a1 = np.maximum(z1, 0.0)
    z2 = a1 @ W2.T + b2
    a2 = np.maximum(z2, 0.0)
    y = a2 @ W3 + b3
    return y, (x, z1, a1, z2, a2)


def loss_and_grad(p, x, t, d, h):
    W1, b1, W2, b2, W3, b3 = unpack(p, d, h)
    y, (x, z1, a1, z2, a2) = forward(p, x, d, h)
    t = np.asarray(t, dtype=np.float64)
    n = y.shape[0]
    e = y - t
    loss = float(np.mean(e * e))
    dy = 2.0 * e / n
    gW3 = dy @ a2
    gb3 = dy.sum()
    dz2 = np.outer(dy, W3) * (z2 > 0)
    gW2 = dz2.T @ a1
    gb2 = dz2.sum(axis=0)
    dz1 = (dz2 @ W2) * (z1 > 0)
    gW1 = dz1.T @ x
    gb1 = dz1.sum(axis=0)
    g = np.concatenate([gW1.ravel(), gb1, gW2.ravel(), gb2, gW3, [gb3]])
    return loss, g


def adam(p, g, m, v, step, lr, b1=0.9, b2=0.999, eps=1e-8):
    m = b1 * m + (1 - b1) * g
    v = b2 * v + (1 - b2) * g * g
    mh = m / (1 - b1 ** step)
    vh = v / (1 - b2 ** step)
    return p - lr * mh / (np.sqrt(vh) + eps), m, v
