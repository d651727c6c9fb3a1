"""FP64 reference of the step-proposer network (test infrastructure only):
forward pass and gradients of the mean squared error, with the weights
rounded to BF16 exactly as the device kernels use them (round to nearest,
ties to even, from the FP32 master copy)."""
from __future__ import annotations

import numpy as np


def bf16(a):
    """Round float32 values to bfloat16 (returned as float64)."""
    b = np.asarray(a, dtype=np.float32).view(np.uint32).astype(np.uint64)
    lsb = (b >> 16) & 1
    r = ((b + 0x7FFF + lsb) >> 16) << 16
    return r.astype(np.uint32).view(np.float32).astype(np.float64)


def unpack(P):
    P = np.asarray(P)
    if P.dtype != np.float64:
        P = P.astype(np.float32)
    o = 0
    W1 = P[o:o + 128 * 24].reshape(128, 24); o += 128 * 24
    b1 = P[o:o + 128]; o += 128
    W2 = P[o:o + 128 * 128].reshape(128, 128); o += 128 * 128
    b2 = P[o:o + 128]; o += 128
    W3 = P[o:o + 128]; o += 128
    b3 = P[o:o + 1]
    return W1, b1, W2, b2, W3, b3


def forward(P, mean, inv_std, X, rounding=True):
    W1, b1, W2, b2, W3, b3 = unpack(P)
    r = bf16 if rounding else (lambda a: np.asarray(a, np.float64))
    W1, W2, W3 = r(W1), r(W2), r(W3)
    xn = (np.asarray(X, np.float64) - mean.astype(np.float64)) * inv_std.astype(np.float64)
    z1 = xn @ W1.T + b1
    h1 = np.maximum(z1, 0)
    z2 = h1 @ W2.T + b2
    h2 = np.maximum(z2, 0)
    out = h2 @ W3 + b3[0]
    return out, (xn, z1, h1, z2, h2)


def grad(P, mean, inv_std, X, y, rounding=True):
    """Gradient of mean((out - y)^2) with respect to the FP32 parameter
    vector (through the BF16-rounded weights), and the loss."""
    W1, b1, W2, b2, W3, b3 = unpack(P)
    r = bf16 if rounding else (lambda a: np.asarray(a, np.float64))
    W2r, W3r = r(W2), r(W3)
    out, (xn, z1, h1, z2, h2) = forward(P, mean, inv_std, X, rounding)
    nb = X.shape[0]
    g = 2.0 * (out - y) / nb
    dW3 = h2.T @ g
    db3 = g.sum()
    gz2 = (g[:, None] * W3r[None, :]) * (z2 > 0)
    dW2 = gz2.T @ h1
    db2 = gz2.sum(axis=0)
    gz1 = (gz2 @ W2r) * (z1 > 0)
    dW1 = gz1.T @ xn
    db1 = gz1.sum(axis=0)
    G = np.concatenate([dW1.reshape(-1), db1, dW2.reshape(-1), db2, dW3, [db3]])
    return G, float(np.mean((out - y) ** 2))
