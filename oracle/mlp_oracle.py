"""CPU FP64 oracle of the surrogate MLP (test infrastructure only).

The reference has no learned surrogate; this restates, in float64 NumPy, the network the GPU
kernels train: 1280 -> 512 -> 512 -> 10 linear layers (weights row-major out x in, as
torch.nn.Linear), exact GELU (z/2 * (1 + erf(z / sqrt 2))), log-rate outputs, and the Poisson
negative log-likelihood L = (1/M) * sum(exp(z) - y * z) (the log y! term is constant). The
backward pass is the textbook chain rule; `numeric_grad` checks it by central differences.
"""

from __future__ import annotations

import numpy as np
from scipy.special import erf

SQRT1_2 = 0.7071067811865476
INV_SQRT_2PI = 0.3989422804014327


def gelu(z):
    return 0.5 * z * (1.0 + erf(z * SQRT1_2))


def gelu_grad(z):
    return 0.5 * (1.0 + erf(z * SQRT1_2)) + z * np.exp(-0.5 * z * z) * INV_SQRT_2PI


def forward(params, X):
    """params: [(W1, b1), (W2, b2), (W3, b3)] float64; returns (log-rates, cache)."""
    cache = [X]
    h = X
    zs = []
    for li, (W, b) in enumerate(params):
        z = h @ W.T + b
        zs.append(z)
        if li < len(params) - 1:
            h = gelu(z)
            cache.append(h)
    return zs[-1], (cache, zs)


def loss(params, X, Y):
    z, _ = forward(params, X)
    return float(np.sum(np.exp(z) - Y * z) / X.shape[0])


def loss_and_grads(params, X, Y):
    """Poisson NLL and its gradients [(dW1, db1), ...] in float64."""
    M = X.shape[0]
    z, (hs, zs) = forward(params, X)
    L = float(np.sum(np.exp(z) - Y * z) / M)
    dz = (np.exp(z) - Y) / M
    grads = [None] * len(params)
    for li in range(len(params) - 1, -1, -1):
        W, _ = params[li]
        grads[li] = (dz.T @ hs[li], dz.sum(0))
        if li > 0:
            dz = (dz @ W) * gelu_grad(zs[li - 1])
    return L, grads


def numeric_grad(params, X, Y, li, which, idx, eps=1e-6):
    """Central difference of the loss in one parameter entry (which: 0 weight, 1 bias)."""
    p = [(W.copy(), b.copy()) for W, b in params]
    arr = p[li][which]
    old = arr[idx]
    arr[idx] = old + eps
    lp = loss(p, X, Y)
    arr[idx] = old - eps
    lm = loss(p, X, Y)
    return (lp - lm) / (2 * eps)


def bf16_round(x):
    """Round float32 values to bfloat16 (nearest even), returned as float64."""
    u = np.asarray(x, np.float32).view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return r.astype(np.uint32).view(np.float32).astype(np.float64)
