"""float64 CPU restatement of the fusion cost model's network -- TEST INFRASTRUCTURE ONLY.

The learned cost model has no counterpart in the reference (its fuser is the plain greedy one,
core/jitk/graph.cpp:319-365); this module is the checker for the GPU network in
bohrium_b200/csrc/ve_cuda/mlp.cu: the same MLP F -> 64 -> 64 -> 1 with ReLU, the same flat
parameter layout (W1[H][F], b1[H], W2[H][H], b2[H], W3[H], b3) and the same loss, the mean
squared error over the rows. Its gradient is pinned by central finite differences in
tests/test_oracle.py; the GPU gradient is compared with it in tests/test_costmodel_gpu.py.
"""
from __future__ import annotations

import numpy as np

F = 16
H = 64
OFF_W1 = 0
OFF_B1 = OFF_W1 + H * F
OFF_W2 = OFF_B1 + H
OFF_B2 = OFF_W2 + H * H
OFF_W3 = OFF_B2 + H
OFF_B3 = OFF_W3 + H
NPARAMS = OFF_B3 + 1


def unpack(p: np.ndarray):
    p = np.asarray(p, dtype=np.float64)
    return (p[OFF_W1:OFF_B1].reshape(H, F), p[OFF_B1:OFF_W2], p[OFF_W2:OFF_B2].reshape(H, H),
            p[OFF_B2:OFF_W3], p[OFF_W3:OFF_B3], p[OFF_B3])


def forward(p: np.ndarray, X: np.ndarray) -> np.ndarray:
    W1, b1, W2, b2, W3, b3 = unpack(p)
    X = np.asarray(X, dtype=np.float64)
    h1 = np.maximum(X @ W1.T + b1, 0.0)
    h2 = np.maximum(h1 @ W2.T + b2, 0.0)
    return h2 @ W3 + b3


def loss_and_grad(p: np.ndarray, X: np.ndarray, t: np.ndarray):
    """(loss, gradient) of L = mean((y - t)^2), the gradient in the flat parameter layout."""
    W1, b1, W2, b2, W3, b3 = unpack(p)
    X = np.asarray(X, dtype=np.float64)
    t = np.asarray(t, dtype=np.float64)
    z1 = X @ W1.T + b1
    h1 = np.maximum(z1, 0.0)
    z2 = h1 @ W2.T + b2
    h2 = np.maximum(z2, 0.0)
    y = h2 @ W3 + b3
    e = y - t
    n = X.shape[0]
    dy = 2.0 * e / n
    g = np.zeros(NPARAMS)
    g[OFF_W3:OFF_B3] = dy @ h2
    g[OFF_B3] = dy.sum()
    dz2 = np.outer(dy, W3) * (z2 > 0)
    g[OFF_W2:OFF_B2] = (dz2.T @ h1).reshape(-1)
    g[OFF_B2:OFF_W3] = dz2.sum(axis=0)
    dz1 = (dz2 @ W2) * (z1 > 0)
    g[OFF_W1:OFF_B1] = (dz1.T @ X).reshape(-1)
    g[OFF_B1:OFF_W2] = dz1.sum(axis=0)
    return float(np.mean(e * e)), g
