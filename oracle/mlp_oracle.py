"""numpy restatement of the rank-predictor MLP (TEST INFRASTRUCTURE ONLY): forward pass,
mean-squared-error gradient and one Adam step, in float64, with the parameter layout of the
CUDA kernels (W1[64x8] b1[64] W2[64x64] b2[64] W3[1x64] b3[1], row-major, contiguous) and
tanh-form GELU (Hendrycks & Gimpel 2016). No reference counterpart: the reference grows the
sample count adaptively only."""
from __future__ import annotations

import numpy as np

IN, H = 8, 64
SIZES = [H * IN, H, H * H, H, H, 1]
NPARAM = sum(SIZES)


def unpack(p):
    p = np.asarray(p, dtype=np.float64)
    o = np.cumsum([0] + SIZES)
    W1 = p[o[0]:o[1]].reshape(H, IN)
    b1 = p[o[1]:o[2]]
    W2 = p[o[2]:o[3]].reshape(H, H)
    b2 = p[o[3]:o[4]]
    W3 = p[o[4]:o[5]].reshape(1, H)
    b3 = p[o[5]:o[6]]
    return W1, b1, W2, b2, W3, b3


def gelu(x):
    c = np.sqrt(2 / np.pi)
    t = np.tanh(c * (x + 0.044715 * x ** 3))
    d = 0.5 * (1 + t) + 0.5 * x * (1 - t * t) * c * (1 + 3 * 0.044715 * x * x)
    return 0.5 * x * (1 + t), d


def forward(p, x):
    W1, b1, W2, b2, W3, b3 = unpack(p)
    a1 = x @ W1.T + b1
    h1, _ = gelu(a1)
    a2 = h1 @ W2.T + b2
    h2, _ = gelu(a2)
    return (h2 @ W3.T + b3)[:, 0]


def grad(p, x, t):
    """d/dp of mean((forward(p, x) - t)^2) and the summed squared error."""
    W1, b1, W2, b2, W3, b3 = unpack(p)
    n = len(x)
    a1 = x @ W1.T + b1
    h1, d1 = gelu(a1)
    a2 = h1 @ W2.T + b2
    h2, d2 = gelu(a2)
    y = (h2 @ W3.T + b3)[:, 0]
    e = y - t
    dy = 2 * e / n
    gW3 = dy @ h2
    gb3 = np.array([dy.sum()])
    da2 = (dy[:, None] * W3) * d2
    gW2 = da2.T @ h1
    gb2 = da2.sum(0)
    da1 = (da2 @ W2) * d1
    gW1 = da1.T @ x
    gb1 = da1.sum(0)
    g = np.concatenate([gW1.ravel(), gb1, gW2.ravel(), gb2, gW3.ravel(), gb3])
    return g, float((e * e).sum())


def adam(p, g, m, v, t, lr, b1=0.9, b2=0.999, eps=1e-8):
    m = b1 * m + (1 - b1) * g
    v = b2 * v + (1 - b2) * g * g
    mh = m / (1 - b1 ** t)
    vh = v / (1 - b2 ** t)
    return p - lr * mh / (np.sqrt(vh) + eps), m, v
