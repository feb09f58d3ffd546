"""CPU oracle of the warm-start network (test infrastructure only).

FP64 numpy restatement of the forward pass, the mean-squared-error loss and
its backward pass for the 4 -> 256 -> 256 -> 256 -> 512 SiLU network, with
optional emulation of the GPU's BF16 roundings (inputs, weights, hidden
activations, output and hidden deltas rounded to BF16 where the GPU stores
them in BF16; products accumulated exactly).  The reference code has no
learned part, so there is nothing to pin against except calculus: the
gradients of the unrounded form are checked against central finite
differences.
"""
from __future__ import annotations

import numpy as np

DIMS_IN = (16, 256, 256, 256)
DIMS_OUT = (256, 256, 256, 512)


def bf16(a):
    """Round to the nearest BF16 value (ties to even), returned as float64."""
    x = np.ascontiguousarray(a, dtype=np.float32).view(np.uint32).astype(np.uint64)
    r = ((x + 0x7FFF + ((x >> 16) & 1)) >> 16) << 16
    return r.astype(np.uint32).view(np.float32).astype(np.float64)


def unflatten(flat):
    out, off = [], 0
    for i, o in zip(DIMS_IN, DIMS_OUT):
        w = np.asarray(flat[off:off + o * i], dtype=np.float64).reshape(o, i)
        off += o * i
        b = np.asarray(flat[off:off + o], dtype=np.float64)
        off += o
        out.append((w, b))
    return out


def flatten(layers):
    return np.concatenate([np.concatenate([w.ravel(), b]) for w, b in layers])


def _silu(z):
    return z / (1.0 + np.exp(-z))


def _silu_grad(z):
    s = 1.0 / (1.0 + np.exp(-z))
    return s * (1.0 + z * (1.0 - s))


def forward(flat, x, rounding=True):
    """y (B x 512) and the cache of the backward pass; x is B x 4."""
    r = bf16 if rounding else (lambda a: np.asarray(a, dtype=np.float64))
    layers = unflatten(flat)
    h = np.zeros((len(x), 16))
    h[:, :4] = x
    h = r(h)
    cache = {"h": [h], "z": []}
    for l, (w, b) in enumerate(layers):
        z = h @ r(w).T + b
        if l < 3:
            cache["z"].append(z)
            h = r(_silu(z))
            cache["h"].append(h)
        else:
            y = z
    return y, cache


def loss_and_gradients(flat, x, t, rounding=True):
    r = bf16 if rounding else (lambda a: np.asarray(a, dtype=np.float64))
    layers = unflatten(flat)
    y, cache = forward(flat, x, rounding)
    B = len(x)
    d = y - t
    loss = float((d * d).sum() / (B * 512))
    delta = r(2.0 * d / (B * 512))
    grads = [None] * 4
    for l in range(3, -1, -1):
        hin = cache["h"][l]
        grads[l] = (delta.T @ hin, delta.sum(axis=0))
        if l > 0:
            w = r(layers[l][0])
            delta = r((delta @ w) * _silu_grad(cache["z"][l - 1]))
    return loss, flatten(grads)
