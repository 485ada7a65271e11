"""CPU oracle of the warm-start network's forward and backward passes (test
infrastructure only).

Mirrors fiber3d_b200.warmstart.FiberMLP: every product rounds both operands
to BF16 (round to nearest even) and accumulates in float64 here (FP32 in
the tensor cores), ReLU hidden layers, linear output, mean-squared-error
loss.  Used to check the GPU gradients.
"""
from __future__ import annotations

import numpy as np


def bf16(x: np.ndarray) -> np.ndarray:
    """Round float32 values to the nearest BF16 (ties to even), as float32."""
    u = np.ascontiguousarray(x, dtype=np.float32).view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32)


def _mm(a, b):
    return (bf16(a).astype(np.float64) @ bf16(b).astype(np.float64)).astype(np.float32)


def forward(W, b, X):
    acts, pres = [X.astype(np.float32)], []
    h = acts[0]
    for k in range(len(W)):
        z = _mm(h, W[k].T) + b[k]
        pres.append(z)
        h = z if k == len(W) - 1 else np.maximum(z, 0.0)
        acts.append(h)
    return h, acts, pres


def grads(W, b, X, T):
    Y, acts, pres = forward(W, b, X)
    B, N = Y.shape
    D = (2.0 / (B * N) * (Y - T)).astype(np.float32)
    loss = float(np.mean((Y - T) ** 2))
    gW, gb = [None] * len(W), [None] * len(W)
    for k in range(len(W) - 1, -1, -1):
        gW[k] = _mm(D.T, acts[k])
        gb[k] = D.sum(axis=0)
        if k > 0:
            D = _mm(D, W[k]) * (pres[k - 1] > 0)
    return loss, gW, gb
