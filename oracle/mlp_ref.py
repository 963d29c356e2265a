"""CPU reference of the surrogate MLP -- TEST INFRASTRUCTURE ONLY.

Float64 restatement of the network the library trains (12 -> 4 x 128 GELU ->
10, inputs padded to 16, outputs to 16) with the same points of BF16 rounding
as the GPU kernels: weights and layer inputs are rounded to BF16, sums are
exact, GELU uses the tanh form.  The backward pass treats rounding as the
identity (straight-through), which is what the GPU backward computes up to
its own BF16 rounding of the upstream gradients.
"""
from __future__ import annotations

import numpy as np

SHAPES = [(128, 16), (128, 128), (128, 128), (128, 128), (16, 128)]
C = 0.7978845608028654


def bf16(x):
    """Round-to-nearest-even to bfloat16, returned as float64."""
    a = np.ascontiguousarray(x, dtype=np.float32)
    u = a.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return r.astype(np.uint32).view(np.float32).astype(np.float64)


def gelu(x):
    return 0.5 * x * (1.0 + np.tanh(C * (x + 0.044715 * x ** 3)))


def gelu_grad(x):
    t = np.tanh(C * (x + 0.044715 * x ** 3))
    return 0.5 * (1.0 + t) + 0.5 * x * (1.0 - t * t) * C * (1.0 + 3 * 0.044715 * x * x)


def unflatten(p):
    out, off = [], 0
    for o, i in SHAPES:
        W = np.asarray(p[off:off + o * i], np.float64).reshape(o, i)
        off += o * i
        b = np.asarray(p[off:off + o], np.float64)
        off += o
        out.append((W, b))
    return out


def forward(p, x):
    """x: (B, 16) bf16-representable features.  Returns outputs and caches."""
    layers = unflatten(p)
    h = bf16(x)
    cache = []
    for l, (W, b) in enumerate(layers):
        z = h @ bf16(W).T + b
        cache.append((h, z))
        if l < len(layers) - 1:
            h = bf16(gelu(z))
    return z, cache


def loss_and_grad(p, x, y):
    """Mean squared error over the first 10 outputs and its gradient."""
    out, cache = forward(p, x)
    B = x.shape[0]
    e = out[:, :10] - y
    loss = float(np.mean(e * e))
    d = np.zeros_like(out)
    d[:, :10] = 2.0 * e / (B * 10)
    layers = unflatten(p)
    grads = []
    for l in range(len(layers) - 1, -1, -1):
        h, z = cache[l]
        W, _ = layers[l]
        gW = d.T @ h
        gb = d.sum(0)
        grads.append((gW, gb))
        if l == 0:
            break
        dh = d @ bf16(W)
        d = dh * gelu_grad(cache[l - 1][1])
    grads.reverse()
    flat = np.concatenate([np.concatenate([gW.ravel(), gb]) for gW, gb in grads])
    return loss, flat
