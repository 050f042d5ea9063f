"""CPU oracle of the warm-start network (test infrastructure only: the
checker of the GPU training and inference kernels, never run by the
product path).

The network has no counterpart in the reference; it is this project's
learned warm start of the bundle multipliers.  Layout and arithmetic follow
the GPU kernels (parallel_biqbin_maxcut_b200/csrc/warm.h, warm.cu):

    features x (F = 14) -> h1 = relu(x W1 + b1) (H = 32)
                        -> h2 = relu(h1 W2 + b2) (H)
                        -> z = h2 . w3 + b3,  gamma = softplus(z)
    loss = mean over the rows of (gamma - y)^2

parameters, one flat float vector: W1[F][H], b1[H], W2[H][H], b2[H], w3[H], b3.
Everything here is float64, so it checks the float32 kernels to float32
accuracy."""
from __future__ import annotations

import numpy as np

F, H = 14, 32
OFF_W1 = 0
OFF_B1 = OFF_W1 + F * H
OFF_W2 = OFF_B1 + H
OFF_B2 = OFF_W2 + H * H
OFF_W3 = OFF_B2 + H
OFF_B3 = OFF_W3 + H
NPARAM = OFF_B3 + 1


def unpack(p):
    p = np.asarray(p, dtype=np.float64)
    return (p[OFF_W1:OFF_B1].reshape(F, H), p[OFF_B1:OFF_W2], p[OFF_W2:OFF_B2].reshape(H, H), p[OFF_B2:OFF_W3],
            p[OFF_W3:OFF_B3], p[OFF_B3])


def softplus(z):
    return np.where(z > 20.0, z, np.log1p(np.exp(np.minimum(z, 20.0))))


def forward(p, X):
    """(gamma, cache) for rows X (N x F)."""
    W1, b1, W2, b2, w3, b3 = unpack(p)
    X = np.asarray(X, dtype=np.float64)
    a1 = X @ W1 + b1
    h1 = np.maximum(a1, 0.0)
    a2 = h1 @ W2 + b2
    h2 = np.maximum(a2, 0.0)
    z = h2 @ w3 + b3
    return softplus(z), (X, h1, h2, z)


def loss_and_grad(p, X, y):
    """Mean squared error of softplus(z) against y and its gradient with
    respect to the flat parameter vector."""
    W1, b1, W2, b2, w3, b3 = unpack(p)
    g, (X, h1, h2, z) = forward(p, X)
    N = X.shape[0]
    e = g - np.asarray(y, dtype=np.float64)
    loss = float(np.mean(e * e))
    dz = 2.0 * e / N / (1.0 + np.exp(-z))
    gw3 = h2.T @ dz
    gb3 = dz.sum()
    dh2 = np.outer(dz, w3) * (h2 > 0)
    gW2 = h1.T @ dh2
    gb2 = dh2.sum(axis=0)
    dh1 = (dh2 @ W2.T) * (h1 > 0)
    gW1 = X.T @ dh1
    gb1 = dh1.sum(axis=0)
    grad = np.concatenate([gW1.ravel(), gb1, gW2.ravel(), gb2, gw3, [gb3]])
    return loss, grad


def numeric_grad(p, X, y, idx, h=1e-6):
    """Central differences of the loss for the parameters in idx."""
    p = np.asarray(p, dtype=np.float64)
    out = np.zeros(len(idx))
    for q, i in enumerate(idx):
        pp, pm = p.copy(), p.copy()
        pp[i] += h
        pm[i] -= h
        out[q] = (loss_and_grad(pp, X, y)[0] - loss_and_grad(pm, X, y)[0]) / (2 * h)
    return out


def bf16(a):
    """Round float32 values to bfloat16 (nearest, ties to even) and back."""
    u = np.asarray(a, dtype=np.float32).view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return r.astype(np.uint32).view(np.float32)


def features(X, L, cuts, values, viol3, gap, parent_gamma=None):
    """The per-cut features the GPU computes (csrc/warm_body.cuh), float64:
    the violation v, v / viol3, viol3, the signed X entries of the cut's
    inequality s_ij X_ij + s_ik X_ik + s_jk X_jk <= 1 (sorted), the signed
    objective entries s L / scale (sorted; scale = mean |L_ij|, i != j),
    n / 128, log(1 + m) / 10, log(1 + gap / scale), and the parent's final
    multiplier of the same cut / scale with a flag 1 (parent_gamma[c] >= 0),
    or 0, 0 (parent_gamma None or < 0).  cuts: m x 4 (type, i, j, k)."""
    X = np.asarray(X, dtype=np.float64)
    L = np.asarray(L, dtype=np.float64)
    n = X.shape[0]
    m = len(cuts)
    off = np.abs(L).sum() - np.abs(np.diag(L)).sum()
    sc = off / (n * (n - 1)) if n > 1 and off > 0 else 1.0
    signs = {1: (-1, -1, -1), 2: (-1, 1, 1), 3: (1, -1, 1), 4: (1, 1, -1)}
    out = np.zeros((m, F))
    for c, (t, i, j, k) in enumerate(cuts):
        s = signs[int(t)]
        xs = sorted([s[0] * X[i, j], s[1] * X[i, k], s[2] * X[j, k]])
        ls = sorted([s[0] * L[i, j] / sc, s[1] * L[i, k] / sc, s[2] * L[j, k] / sc])
        v = values[c]
        pg = -1.0 if parent_gamma is None else float(parent_gamma[c])
        out[c] = [v, v / viol3 if viol3 > 1e-12 else 0.0, viol3, *xs, *ls, n / 128.0, np.log1p(m) / 10.0,
                  np.log1p(max(gap, 0.0) / sc), pg / sc if pg >= 0 else 0.0, 1.0 if pg >= 0 else 0.0]
    return out
