"""TEST INFRASTRUCTURE ONLY: an FP64 numpy restatement of the surrogate MLP's forward and
backward passes (indicatrix_b200/surrogate.py on the kernels of include/ix_surrogate.h),
used to check the device gradients.  The inputs of every GEMM are rounded to bfloat16 as
the device rounds them, so the comparison measures the device's FP32 accumulation and
elementwise steps, not bf16 quantisation.  Nothing in ``indicatrix_b200`` imports it."""
from __future__ import annotations

import numpy as np


def bf16(x: np.ndarray) -> np.ndarray:
    """Round float32 values to bfloat16 (round to nearest even), returned as float64."""
    u = np.asarray(x, np.float32).view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return r.astype(np.uint32).view(np.float32).astype(np.float64)


def _logistic(z):
    return 1.0 / (1.0 + np.exp(-z))


def silu(z):
    return z * _logistic(z)


def silu_grad(z):
    s = _logistic(z)
    return s * (1.0 + z * (1.0 - s))


def forward(ws, bs, x):
    """ws, bs: per layer weights [out, in] and biases; SiLU between layers, none after the
    last.  Returns (per layer (bf16 input, pre-activation), output)."""
    acts = []
    h = bf16(x)
    for i, (w, b) in enumerate(zip(ws, bs)):
        z = h @ bf16(w).T + np.asarray(b, np.float64)
        acts.append((h, z))
        if i < len(ws) - 1:
            h = bf16(silu(z))
    return acts, z


def gradients(ws, bs, x, t):
    """MSE loss and [(dW, db)] per layer (dW [out, in])."""
    acts, y = forward(ws, bs, x)
    m, n = y.shape
    d = y - np.asarray(t, np.float64)
    loss = float(np.mean(d * d))
    dz = 2.0 * d / (m * n)
    grads = [None] * len(ws)
    for i in range(len(ws) - 1, -1, -1):
        h_in, _ = acts[i]
        dzb = bf16(dz)
        grads[i] = (dzb.T @ h_in, dz.sum(axis=0))
        if i > 0:
            dh = dzb @ bf16(ws[i])
            dz = dh * silu_grad(acts[i - 1][1])
    return loss, grads
