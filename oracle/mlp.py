"""numpy restatement of the router network's forward pass and of the
mean-squared-error gradient (TEST INFRASTRUCTURE ONLY), the checker of the
library's fjb_mlp_forward / fjb_mlp_gradient kernels.  FP64 arithmetic on
the FP32 parameters; packing as csrc/router.cuh states it:
mu[12] sd[12] W1[64][12] b1[64] W2[64][64] b2[64] w3[64] b3; the output adds
the fixed skip X[:, 9] + X[:, 10] + X[:, 11] (the log10 Schwarz x density
bound), so the parameters model the gap below that bound."""

from __future__ import annotations

import numpy as np

F, H = 12, 64


def unpack(p):
    p = np.asarray(p, np.float64)
    o = 0
    out = {}
    for name, size in (("mu", F), ("sd", F), ("W1", H * F), ("b1", H), ("W2", H * H),
                       ("b2", H), ("w3", H), ("b3", 1)):
        out[name] = p[o:o + size]
        o += size
    out["W1"] = out["W1"].reshape(H, F)
    out["W2"] = out["W2"].reshape(H, H)
    return out


def forward(p, X):
    q = unpack(p)
    xn = (np.asarray(X, np.float64) - q["mu"]) / q["sd"]
    h1 = np.tanh(xn @ q["W1"].T + q["b1"])
    h2 = np.tanh(h1 @ q["W2"].T + q["b2"])
    skip = np.asarray(X, np.float64)[:, 9:12].sum(1)
    return skip + h2 @ q["w3"] + q["b3"][0], (xn, h1, h2)


def gradient(p, X, T):
    """d mean((y - T)^2) / d params, packed like p (mu, sd entries zero)."""
    q = unpack(p)
    y, (xn, h1, h2) = forward(p, X)
    n = len(X)
    dy = 2.0 * (y - np.asarray(T, np.float64)) / n
    g_w3 = dy @ h2
    g_b3 = dy.sum()
    da2 = (dy[:, None] * q["w3"][None, :]) * (1 - h2 * h2)
    g_W2 = da2.T @ h1
    g_b2 = da2.sum(0)
    da1 = (da2 @ q["W2"]) * (1 - h1 * h1)
    g_W1 = da1.T @ xn
    g_b1 = da1.sum(0)
    return np.concatenate([np.zeros(2 * F), g_W1.ravel(), g_b1, g_W2.ravel(), g_b2, g_w3, [g_b3]])
