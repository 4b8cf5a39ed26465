"""Oracle (test infrastructure, not the product): the regrid forecaster's network in numpy, FP64.

The forecaster has no counterpart in the reference; this restatement is the CPU check of the GPU
kernels in dacti_b200/csrc/forecast.cu: the same layout (W1[64][n_in], b1[64], W2[64][64], b2[64],
W3[64], b3), ReLU hidden layers, logistic output, and the positive-weighted binary cross-entropy on the
logit z, l = pw y softplus(-z) + (1 - y) softplus(z). Gradients come from explicit backpropagation and
are themselves checked against central differences in the tests.
"""
from __future__ import annotations

import numpy as np

H = 64


def unpack(params: np.ndarray, n_in: int):
    p = np.asarray(params, np.float64)
    o = 0
    W1 = p[o:o + H * n_in].reshape(H, n_in); o += H * n_in
    b1 = p[o:o + H]; o += H
    W2 = p[o:o + H * H].reshape(H, H); o += H * H
    b2 = p[o:o + H]; o += H
    W3 = p[o:o + H]; o += H
    b3 = p[o]; o += 1
    assert o == p.size
    return W1, b1, W2, b2, W3, b3


def n_params(n_in: int) -> int:
    return H * n_in + H + H * H + H + H + 1


def logits(params: np.ndarray, x: np.ndarray) -> np.ndarray:
    W1, b1, W2, b2, W3, b3 = unpack(params, x.shape[1])
    a1 = np.maximum(x @ W1.T + b1, 0.0)
    a2 = np.maximum(a1 @ W2.T + b2, 0.0)
    return a2 @ W3 + b3


def predict(params: np.ndarray, x: np.ndarray) -> np.ndarray:
    return 1.0 / (1.0 + np.exp(-logits(params, np.asarray(x, np.float64))))


def _softplus(z):
    return np.where(z > 0, z + np.log1p(np.exp(-np.abs(z))), np.log1p(np.exp(-np.abs(z))))


def loss_grad(params: np.ndarray, x: np.ndarray, y: np.ndarray, pw: float):
    """(sum of the loss over samples, gradient of that sum) in FP64."""
    x = np.asarray(x, np.float64)
    y = np.asarray(y, np.float64)
    W1, b1, W2, b2, W3, b3 = unpack(params, x.shape[1])
    z1 = x @ W1.T + b1
    a1 = np.maximum(z1, 0.0)
    z2 = a1 @ W2.T + b2
    a2 = np.maximum(z2, 0.0)
    z = a2 @ W3 + b3
    loss = float((pw * y * _softplus(-z) + (1 - y) * _softplus(z)).sum())
    s = 1.0 / (1.0 + np.exp(-z))
    dz = s * (pw * y + 1 - y) - pw * y
    gW3 = dz @ a2
    gb3 = dz.sum()
    dz2 = np.outer(dz, W3) * (z2 > 0)
    gW2 = dz2.T @ a1
    gb2 = dz2.sum(axis=0)
    dz1 = (dz2 @ W2) * (z1 > 0)
    gW1 = dz1.T @ x
    gb1 = dz1.sum(axis=0)
    return loss, np.concatenate([gW1.ravel(), gb1, gW2.ravel(), gb2, gW3, [gb3]])


def bf16(params: np.ndarray) -> np.ndarray:
    """FP32 values rounded to BF16 (round to nearest, ties to even), returned as FP64."""
    u = np.asarray(params, np.float32).view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return r.astype(np.uint32).view(np.float32).astype(np.float64)
