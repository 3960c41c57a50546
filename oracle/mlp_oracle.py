"""CPU restatement of the surrogate network (include/negf_mlp.h) in NumPy FP64.

TEST INFRASTRUCTURE ONLY: imported by ``tests/`` as the checker of the
network's forward pass and gradients; nothing in the product path imports it.
It has no counterpart in the reference (NEGFtrans samples energies on a
uniform grid, main.f90:369-375), so it is pinned by finite differences of its
own FP64 loss (tests/test_oracle.py) rather than by reference outputs.

``bf16=True`` rounds every product operand to BF16 (round to nearest even)
the way the GPU stages them, accumulating exactly in FP64; ``bf16=False`` is
the exact FP64 network.
"""
from __future__ import annotations

import numpy as np
from scipy.special import erf


def bf16(a):
    """Round to the nearest BF16 value (ties to even), returned as float64."""
    u = np.array(a, dtype=np.float32).view(np.uint32)
    r = ((u + np.uint32(0x7FFF) + ((u >> np.uint32(16)) & np.uint32(1))) & np.uint32(0xFFFF0000))
    return r.view(np.float32).astype(np.float64)


def gelu(z):
    return 0.5 * z * (1.0 + erf(z / np.sqrt(2.0)))


def gelu_grad(z):
    return 0.5 * (1.0 + erf(z / np.sqrt(2.0))) + z * np.exp(-0.5 * z * z) / np.sqrt(2.0 * np.pi)


def unpack(params, widths):
    """Packed order W_0 (out x in, row-major), b_0, W_1, b_1, ..."""
    out, o = [], 0
    for a, b in zip(widths[:-1], widths[1:]):
        W = np.asarray(params[o:o + a * b], np.float64).reshape(b, a)
        o += a * b
        bb = np.asarray(params[o:o + b], np.float64)
        o += b
        out.append((W, bb))
    assert o == len(params)
    return out


def forward(params, widths, x, bf16_ops=True):
    """Returns (y, cache) for x (batch x widths[0])."""
    q = bf16 if bf16_ops else (lambda a: np.asarray(a, np.float64))
    layers = unpack(params, widths)
    h = np.asarray(x, np.float64)
    cache = []
    for l, (W, b) in enumerate(layers):
        z = q(h) @ q(W).T + b
        cache.append((h, z))
        h = z if l == len(layers) - 1 else gelu(z)
    return h, cache


def loss_and_grad(params, widths, x, t, w, bf16_ops=True):
    """Weighted MSE sum w (y - t)^2 / sum w and its gradient (packed)."""
    q = bf16 if bf16_ops else (lambda a: np.asarray(a, np.float64))
    layers = unpack(params, widths)
    y, cache = forward(params, widths, x, bf16_ops)
    t = np.asarray(t, np.float64)
    w = np.asarray(w, np.float64)
    den = w.sum() if w.sum() > 0 else 1.0
    loss = float(np.sum(w * (y - t) ** 2) / den)
    dz = 2.0 * w * (y - t) / den
    grads = [None] * len(layers)
    for l in range(len(layers) - 1, -1, -1):
        h, _ = cache[l]
        W, _ = layers[l]
        gW = q(dz).T @ q(h)
        gb = q(dz).sum(axis=0)
        grads[l] = (gW, gb)
        if l:
            dz = (q(dz) @ q(W)) * gelu_grad(cache[l - 1][1])
    flat = np.concatenate([np.concatenate([gW.ravel(), gb]) for gW, gb in grads])
    return loss, flat
