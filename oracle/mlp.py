"""CPU restatement of the scan surrogate's perceptron: the checker of the device kernels.

Test infrastructure only (imported by ``tests/`` and the benchmark's CPU leg): the product
path is ``solprop_b200/surrogate.py`` over the CUDA kernels of ``csrc/mlp_kernels.cu``.

The perceptron has no counterpart in the reference; this module states its arithmetic
the way the kernels perform it: every matrix product rounds both operands to BF16 (round
to nearest even) and accumulates in float64 here (FP32 on the device), the hidden layers
apply the exact GELU ``x Phi(x)``, the output layer is linear, and the loss is the mean
squared error.  The gradients follow by the chain rule; ``numeric_gradient`` checks them
by central differences without the BF16 rounding.
"""

from __future__ import annotations

import numpy as np
from scipy.special import erf


def bf16(x: np.ndarray) -> np.ndarray:
    """Round float32 values to bfloat16 (nearest even), returned as float64."""
    bits = np.asarray(x, dtype=np.float32).view(np.uint32).astype(np.uint64)
    rounded = (bits + 0x7FFF + ((bits >> 16) & 1)) & 0xFFFF0000
    return rounded.astype(np.uint32).view(np.float32).astype(np.float64)


def gelu(x):
    return 0.5 * x * (1.0 + erf(x / np.sqrt(2.0)))


def gelu_grad(x):
    return 0.5 * (1.0 + erf(x / np.sqrt(2.0))) + x * np.exp(-0.5 * x * x) / np.sqrt(2.0 * np.pi)


def _matmul(a, b, rounded: bool):
    return (bf16(a) @ bf16(b)) if rounded else (np.asarray(a, np.float64) @ np.asarray(b, np.float64))


def forward(weights, biases, x, *, rounded: bool = True):
    """Outputs and the per-layer (input, pre-activation) pairs of a forward pass."""
    a = np.asarray(x, np.float64)
    cache = []
    last = len(weights) - 1
    for i, (w, b) in enumerate(zip(weights, biases)):
        z = _matmul(a, np.asarray(w).T, rounded) + b
        cache.append((a, z))
        a = z if i == last else gelu(z)
    return a, cache


def mse(y, t):
    d = np.asarray(y, np.float64) - t
    return float(np.mean(d * d)), 2.0 * d / d.size


def backward(weights, cache, dy, *, rounded: bool = True):
    """Gradients (dW, db) of every layer from dL/dy."""
    grads = []
    g = np.asarray(dy, np.float64)
    for i in range(len(weights) - 1, -1, -1):
        a, z = cache[i]
        if i != len(weights) - 1:
            g = g * gelu_grad(z)
        dw = _matmul(g.T, a, rounded)
        db = g.sum(axis=0)
        grads.append((dw, db))
        if i:
            g = _matmul(g, np.asarray(weights[i]), rounded)
    return grads[::-1]


def loss_of(weights, biases, x, t):
    y, _ = forward(weights, biases, x, rounded=False)
    return mse(y, t)[0]


def numeric_gradient(weights, biases, x, t, layer: int, index: tuple, eps: float = 1e-6) -> float:
    """Central difference of the unrounded loss in one weight."""
    w = [np.array(v, np.float64) for v in weights]
    w[layer][index] += eps
    up = loss_of(w, biases, x, t)
    w[layer][index] -= 2 * eps
    down = loss_of(w, biases, x, t)
    return (up - down) / (2 * eps)
