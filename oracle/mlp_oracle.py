"""CPU restatement of the mixed-batch planner's cost model (test
infrastructure only: the library trains and runs the model with its own CUDA
kernels; this module exists to check those kernels' forward pass and
gradients).

Network: x (F) -> W1, b1 -> ReLU (H) -> W2, b2 -> ReLU (H) -> W3, b3 -> y (P).
Loss: mean over the masked entries of (y - target)^2.  Parameters are one
flat vector: W1 (F x H), b1 (H), W2 (H x H), b2 (H), W3 (H x P), b3 (P),
row-major, in that order (the layout of include/rsgpu.h's
rsgpu_model_get_params).  Arithmetic in float64.
"""
from __future__ import annotations

import numpy as np

F, H, P = 11, 32, 6


def unpack(w):
    w = np.asarray(w, np.float64)
    o = 0
    W1 = w[o:o + F * H].reshape(F, H); o += F * H
    b1 = w[o:o + H]; o += H
    W2 = w[o:o + H * H].reshape(H, H); o += H * H
    b2 = w[o:o + H]; o += H
    W3 = w[o:o + H * P].reshape(H, P); o += H * P
    b3 = w[o:o + P]; o += P
    assert o == w.size
    return W1, b1, W2, b2, W3, b3


def param_count():
    return F * H + H + H * H + H + H * P + P


def forward(w, x):
    W1, b1, W2, b2, W3, b3 = unpack(w)
    x = np.asarray(x, np.float64)
    z1 = x @ W1 + b1
    a1 = np.maximum(z1, 0)
    z2 = a1 @ W2 + b2
    a2 = np.maximum(z2, 0)
    return a2 @ W3 + b3


def loss_and_grad(w, x, t, mask):
    W1, b1, W2, b2, W3, b3 = unpack(w)
    x = np.asarray(x, np.float64)
    t = np.asarray(t, np.float64)
    m = np.asarray(mask, np.float64)
    cnt = m.sum()
    z1 = x @ W1 + b1
    a1 = np.maximum(z1, 0)
    z2 = a1 @ W2 + b2
    a2 = np.maximum(z2, 0)
    y = a2 @ W3 + b3
    err = (y - t) * m
    loss = float((err ** 2).sum() / cnt)
    dy = 2.0 * err / cnt
    gW3 = a2.T @ dy
    gb3 = dy.sum(0)
    dz2 = (dy @ W3.T) * (z2 > 0)
    gW2 = a1.T @ dz2
    gb2 = dz2.sum(0)
    dz1 = (dz2 @ W2.T) * (z1 > 0)
    gW1 = x.T @ dz1
    gb1 = dz1.sum(0)
    g = np.concatenate([gW1.ravel(), gb1, gW2.ravel(), gb2, gW3.ravel(), gb3])
    return loss, g


def init(seed, scale=1.0):
    """Seeded parameters for tests (not the library's initializer)."""
    rng = np.random.default_rng(seed)
    w = np.zeros(param_count())
    o = 0
    for fan_in, n in [(F, F * H), (None, H), (H, H * H), (None, H), (H, H * P), (None, P)]:
        if fan_in:
            w[o:o + n] = rng.uniform(-1, 1, n) * scale / np.sqrt(fan_in)
        else:
            w[o:o + n] = rng.uniform(-0.1, 0.1, n)
        o += n
    return w
