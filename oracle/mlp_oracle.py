"""FP64 CPU restatement of the learned per-shape SDF network (3-64-64-1, SiLU) —
TEST INFRASTRUCTURE ONLY (gradient check of the CUDA training kernels).

The network is not in the reference; its oracle is this forward/backward pass in
FP64 (numpy) over the parameter layout of the CUDA code: W1[64][3], b1[64],
W2[64][64] (row = output unit), b2[64], w3[64], b3, padding to 4484. The loss is
the mean squared error over the points. `finite_difference_check` pins the
backward pass against central differences of the forward pass.
"""
from __future__ import annotations

import numpy as np

NP = 4484
W1, B1, W2, B2, W3, B3 = 0, 192, 256, 4352, 4416, 4480


def unpack(p):
    p = np.asarray(p, np.float64)
    return (p[W1:B1].reshape(64, 3), p[B1:W2], p[W2:B2].reshape(64, 64), p[B2:W3], p[W3:B3], p[B3])


def silu(x):
    return x / (1.0 + np.exp(-x))


def dsilu(x):
    s = 1.0 / (1.0 + np.exp(-x))
    return s * (1.0 + x * (1.0 - s))


def forward(p, u):
    """Network output for points u (n x 3)."""
    w1, b1, w2, b2, w3, b3 = unpack(p)
    h1 = u @ w1.T + b1
    a1 = silu(h1)
    h2 = a1 @ w2.T + b2
    a2 = silu(h2)
    return a2 @ w3 + b3


def loss_and_grad(p, pts):
    """Mean squared error of the network over pts (n x 4: x, y, z, target) and its gradient
    with respect to the 4484 parameters (padding entries zero)."""
    pts = np.asarray(pts, np.float64)
    u, t = pts[:, :3], pts[:, 3]
    n = len(pts)
    w1, b1, w2, b2, w3, b3 = unpack(p)
    h1 = u @ w1.T + b1
    a1 = silu(h1)
    h2 = a1 @ w2.T + b2
    a2 = silu(h2)
    y = a2 @ w3 + b3
    r = y - t
    loss = float(np.mean(r * r))
    dy = 2.0 * r / n
    g = np.zeros(NP)
    g[B3] = dy.sum()
    g[W3:B3] = a2.T @ dy
    dh2 = np.outer(dy, w3) * dsilu(h2)
    g[B2:W3] = dh2.sum(0)
    g[W2:B2] = (dh2.T @ a1).ravel()
    dh1 = (dh2 @ w2) * dsilu(h1)
    g[B1:W2] = dh1.sum(0)
    g[W1:B1] = (dh1.T @ u).ravel()
    return loss, g, y


def finite_difference_check(p, pts, idx, eps=1e-6):
    """Largest relative difference between the analytic gradient and central differences
    of the loss at parameter indices idx."""
    _, g, _ = loss_and_grad(p, pts)
    worst = 0.0
    for k in idx:
        q = np.array(p, np.float64)
        q[k] += eps
        lp, _, _ = loss_and_grad(q, pts)
        q[k] -= 2 * eps
        lm, _, _ = loss_and_grad(q, pts)
        fd = (lp - lm) / (2 * eps)
        worst = max(worst, abs(fd - g[k]) / max(abs(fd), abs(g[k]), 1e-12))
    return worst


def random_params(rng, scale=1.0):
    p = np.zeros(NP)
    p[W1:B1] = rng.uniform(-1, 1, 192) * np.sqrt(6 / 67) * scale
    p[B1:W2] = rng.normal(0, 0.1, 64)
    p[W2:B2] = rng.uniform(-1, 1, 4096) * np.sqrt(6 / 128) * scale
    p[B2:W3] = rng.normal(0, 0.1, 64)
    p[W3:B3] = rng.uniform(-1, 1, 64) * np.sqrt(6 / 65) * scale
    p[B3] = 0.05
    return p
