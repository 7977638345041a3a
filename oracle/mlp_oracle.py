"""CPU oracle of the surrogate MLP's forward and backward pass -- TEST INFRASTRUCTURE ONLY.

Restates, in numpy f64, the network the B200 library trains
(gpumetropolis_b200/csrc/mlp.cu): standardised inputs, two SiLU layers, a
linear head, mean squared error.  The BF16 roundings of the GPU path are
emulated at the same points (round-to-nearest-even of the f32 values that
feed the tensor cores), so the oracle's gradients differ from the GPU's only
by f32 accumulation order and f32 elementwise rounding.  Used by tests only.
"""
from __future__ import annotations

import numpy as np


def bf16(x):
    """Round to bfloat16 (nearest even), returned as float64."""
    f = np.asarray(x, dtype=np.float32)
    b = f.view(np.uint32).astype(np.uint64)
    b = (b + 0x7FFF + ((b >> 16) & 1)) & 0xFFFF0000
    return b.astype(np.uint32).view(np.float32).astype(np.float64)


def f32(x):
    return np.asarray(x, dtype=np.float32).astype(np.float64)


def silu(z):
    return z / (1.0 + np.exp(-z))


def dsilu(z):
    s = 1.0 / (1.0 + np.exp(-z))
    return s * (1.0 + z * (1.0 - s))


def unpack(params, d, H):
    dp = (d + 63) // 64 * 64
    sizes = [H * dp, H, H * H, H, H, 1]
    out, off = [], 0
    for s in sizes:
        out.append(np.asarray(params[off:off + s], dtype=np.float64))
        off += s
    W1, b1, W2, b2, w3, b3 = out
    return W1.reshape(H, dp), b1, W2.reshape(H, H), b2, w3, b3, dp


def forward_backward(params, d, H, X, t):
    """Loss and gradients for standardised inputs X (n x d) and targets t.
    Returns (loss, [dW1, db1, dW2, db2, dw3, db3]) in the GPU's layout."""
    W1, b1, W2, b2, w3, b3, dp = unpack(params, d, H)
    n = X.shape[0]
    Xp = np.zeros((n, dp))
    Xp[:, :d] = X
    Xh = bf16(Xp)
    Z1 = f32(Xh @ bf16(W1).T + b1)
    A1h = bf16(silu(Z1))
    Z2 = f32(A1h @ bf16(W2).T + b2)
    yhat = silu(Z2) @ w3 + b3[0]
    r = yhat - t
    loss = np.mean(r * r)
    dy = 2.0 * r / n
    dw3 = silu(Z2).T @ dy
    db3 = np.array([dy.sum()])
    dZ2 = f32(dy[:, None] * w3[None, :] * dsilu(Z2))
    db2 = dZ2.sum(axis=0)
    dZ2h = bf16(dZ2)
    dW2 = dZ2h.T @ A1h
    dA1 = f32(dZ2h @ bf16(W2))
    dZ1 = f32(dA1 * dsilu(Z1))
    db1 = dZ1.sum(axis=0)
    dW1 = bf16(dZ1).T @ Xh
    return loss, [dW1, db1, dW2, db2, dw3, db3]


def predict(params, d, H, X):
    W1, b1, W2, b2, w3, b3, dp = unpack(params, d, H)
    Xp = np.zeros((X.shape[0], dp))
    Xp[:, :d] = X
    Z1 = f32(bf16(Xp) @ bf16(W1).T + b1)
    Z2 = f32(bf16(silu(Z1)) @ bf16(W2).T + b2)
    return silu(Z2) @ w3 + b3[0]


def input_grad(params, d, H, X):
    """Gradient of the network output with respect to its (standardised or
    whitened) input X (n x d), through the same BF16 roundings as the GPU's
    backward pass: dZ2 = w3 silu'(Z2), dZ1 = bf16(dZ2) bf16(W2) * silu'(Z1),
    dX = bf16(dZ1) bf16(W1).  Returns (y (n,), dX (n x d))."""
    W1, b1, W2, b2, w3, b3, dp = unpack(params, d, H)
    Xp = np.zeros((X.shape[0], dp))
    Xp[:, :d] = X
    Z1 = f32(bf16(Xp) @ bf16(W1).T + b1)
    Z2 = f32(bf16(silu(Z1)) @ bf16(W2).T + b2)
    y = silu(Z2) @ w3 + b3[0]
    dZ2 = f32(w3[None, :] * dsilu(Z2))
    dZ1 = f32(f32(bf16(dZ2) @ bf16(W2)) * dsilu(Z1))
    dX = bf16(dZ1) @ bf16(W1)
    return y, dX[:, :d]

