"""CPU oracle of the trace surrogate's forward and backward passes.

Test infrastructure only: it restates, in float64 NumPy, what the surrogate
kernels compute (ionosphere_fdtd_b200/surrogate.py), with the same bfloat16
roundings at the same points (weights, layer inputs and the error signal fed
to the products are bf16; products accumulate in float64 here, float32 on the
GPU).  With ``bf16=False`` every rounding is skipped, which the finite-
difference test uses to pin the backward formulas.
"""

from __future__ import annotations

import numpy as np


def bf16(x, enabled: bool = True) -> np.ndarray:
    """Round to bfloat16 (nearest, ties to even) and return float64."""

    a = np.asarray(x, dtype=np.float64)
    if not enabled:
        return a
    b = a.astype(np.float32).view(np.uint32)
    r = (b + np.uint32(0x7FFF) + ((b >> np.uint32(16)) & np.uint32(1))) & np.uint32(0xFFFF0000)
    return r.view(np.float32).astype(np.float64)


def silu(z):
    return z / (1.0 + np.exp(-z))


def silu_grad(z):
    s = 1.0 / (1.0 + np.exp(-z))
    return s * (1.0 + z * (1.0 - s))


def forward(layers, weights, biases, x, use_bf16: bool = True):
    """layers: (fan_in, fan_out, act, expand) tuples; returns predictions and
    the per-layer (input, pre-activation) pairs."""

    rows = x.shape[0]
    inp = bf16(x, use_bf16)
    acts = []
    z = None
    for i, (fi, fo, act, expand) in enumerate(layers):
        z = inp @ bf16(weights[i], use_bf16).T + biases[i]
        acts.append((inp, z))
        if i < len(layers) - 1:
            y = bf16(silu(z) if act else z, use_bf16)
            rows *= expand
            inp = y.reshape(rows, fo // expand)
    return z.reshape(x.shape[0], -1), acts


def backward(layers, weights, acts, grad, use_bf16: bool = True):
    gw, gb = [None] * len(layers), [None] * len(layers)
    dy = grad.reshape(acts[-1][1].shape)
    for i in range(len(layers) - 1, -1, -1):
        fi, fo, act, expand = layers[i]
        x, z = acts[i]
        dz = dy * silu_grad(z) if act else dy
        dz16 = bf16(dz, use_bf16)
        gw[i] = dz16.T @ x
        gb[i] = dz.sum(axis=0)
        if i > 0:
            dx = dz16 @ bf16(weights[i], use_bf16)
            prev = layers[i - 1]
            dy = dx.reshape(dx.shape[0] // prev[3], prev[1])
    return gw, gb


def mse(pred, target):
    d = pred - target
    return float(np.mean(d * d)), 2.0 * d / d.size
