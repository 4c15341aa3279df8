"""CPU oracle of the learned warm-start network -- TEST INFRASTRUCTURE ONLY.

FP64 numpy forward and backward pass of the per-edge network the product
runs on the tensor cores (6 -> 64 -> 64 -> 1, SiLU; parameter layout as
tf_mlp_param_count / tf_mlp_init describe it: W1[64][16] with inputs 6..15
zero, b1[64], W2[64][64], b2[64], W3[64], b3).  The product feeds the tensor
cores BF16 weights and activations; `forward(..., bf16=True)` rounds the same
operands to BF16 so the comparison isolates accumulation order.  The network
has no counterpart in the reference (its CG starts from the previous
solution, Discretization.hpp:1536), so this oracle checks the product's own
kernels: gradients against the analytic backward pass written out here.
"""
from __future__ import annotations

import numpy as np

H, IN, INP = 64, 6, 16
OFF_W1, OFF_B1 = 0, H * INP
OFF_W2 = OFF_B1 + H
OFF_B2 = OFF_W2 + H * H
OFF_W3 = OFF_B2 + H
OFF_B3 = OFF_W3 + H
N_PARAM = OFF_B3 + 1


def bf16(x):
    """Round to the nearest BF16 value (ties to even), returned as float64."""
    a = np.asarray(x, dtype=np.float32)
    u = a.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return r.astype(np.uint32).view(np.float32).astype(np.float64)


def unpack(p):
    p = np.asarray(p, dtype=np.float64)
    return (p[OFF_W1:OFF_B1].reshape(H, INP), p[OFF_B1:OFF_W2], p[OFF_W2:OFF_B2].reshape(H, H),
            p[OFF_B2:OFF_W3], p[OFF_W3:OFF_B3], p[OFF_B3])


def silu(z):
    return z / (1.0 + np.exp(-z))


def dsilu(z):
    s = 1.0 / (1.0 + np.exp(-z))
    return s * (1.0 + z * (1.0 - s))


def forward(p, X, bf16_ops=True):
    """(y, cache) for inputs X[n, 6]."""
    W1, b1, W2, b2, W3, b3 = unpack(p)
    r = bf16 if bf16_ops else (lambda a: np.asarray(a, dtype=np.float64))
    Xp = np.zeros((len(X), INP))
    Xp[:, :IN] = X
    x0 = r(Xp)
    z1 = x0 @ r(W1).T + b1
    h1 = r(silu(z1))
    z2 = h1 @ r(W2).T + b2
    h2 = r(silu(z2))
    y = h2 @ r(W3) + b3
    return y, (x0, z1, h1, z2, h2, r(W2), r(W3))


def gradient(p, X, t, w=None):
    """(gradient of sum w (y - t)^2 / n, loss), FP64 backward pass."""
    n = len(X)
    w = np.ones(n) if w is None else np.asarray(w, dtype=np.float64)
    y, (x0, z1, h1, z2, h2, W2, W3) = forward(p, X)
    e = y - np.asarray(t, dtype=np.float64)
    loss = float(np.sum(w * e * e) / n)
    dy = 2.0 * w * e / n
    d2 = np.outer(dy, W3) * dsilu(z2)
    d1 = (d2 @ W2) * dsilu(z1)
    g = np.zeros(N_PARAM)
    g[OFF_W1:OFF_B1] = (d1.T @ x0).ravel()
    g[OFF_B1:OFF_W2] = d1.sum(0)
    g[OFF_W2:OFF_B2] = (d2.T @ h1).ravel()
    g[OFF_B2:OFF_W3] = d2.sum(0)
    g[OFF_W3:OFF_B3] = h2.T @ dy
    g[OFF_B3] = dy.sum()
    return g, loss
