"""The warm-start network over the C ABI (ek_mlp_*): a 4 -> 256 -> 256 ->
256 -> 512 MLP with SiLU, trained and evaluated on the GPU by the library's
own tensor-core kernels (BF16 operands, FP32 accumulation, FP32 master
weights, Adam)."""
from __future__ import annotations

import ctypes

import numpy as np

from ._lib import check, lib

N_IN, N_IN_PAD, N_HID, N_OUT = 4, 16, 256, 512
DIMS_IN = (N_IN_PAD, N_HID, N_HID, N_HID)
DIMS_OUT = (N_HID, N_HID, N_HID, N_OUT)

_fp = ctypes.POINTER(ctypes.c_float)
_dp = ctypes.POINTER(ctypes.c_double)


def _f32(a, shape):
    a = np.ascontiguousarray(a, dtype=np.float32)
    if a.shape != shape:
        raise ValueError(f"expected shape {shape}, got {a.shape}")
    return a


def layer_slices():
    """[(W slice, W shape, b slice)] of the flat parameter array."""
    out, off = [], 0
    for i, o in zip(DIMS_IN, DIMS_OUT):
        w = slice(off, off + o * i)
        off += o * i
        b = slice(off, off + o)
        off += o
        out.append((w, (o, i), b))
    return out


def unflatten(flat):
    return [(flat[w].reshape(shape), flat[b]) for w, shape, b in layer_slices()]


class Mlp:
    def __init__(self, batch=256, seed=0):
        h = ctypes.c_void_p()
        check(lib().ek_mlp_create(int(batch), int(seed), ctypes.byref(h)))
        self._h = h
        self.batch = int(batch)
        n = ctypes.c_int64(0)
        check(lib().ek_mlp_param_count(self._h, ctypes.byref(n)))
        self.n_params = int(n.value)

    def close(self):
        if getattr(self, "_h", None):
            check(lib().ek_mlp_destroy(self._h))
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    @property
    def params(self):
        out = np.empty(self.n_params, dtype=np.float32)
        check(lib().ek_mlp_get_params(self._h, out.ctypes.data_as(_fp)))
        return out

    @params.setter
    def params(self, flat):
        flat = _f32(flat, (self.n_params,))
        check(lib().ek_mlp_set_params(self._h, flat.ctypes.data_as(_fp)))

    def set_data(self, x, t):
        x = _f32(x, (len(x), N_IN))
        t = _f32(t, (len(x), N_OUT))
        check(lib().ek_mlp_set_data(self._h, x.ctypes.data_as(_fp), t.ctypes.data_as(_fp), len(x)))

    def train(self, iters, lr):
        loss = np.zeros(int(iters))
        check(lib().ek_mlp_train(self._h, int(iters), float(lr), loss.ctypes.data_as(_dp)))
        return loss

    def gradients(self, x, t):
        x = _f32(x, (self.batch, N_IN))
        t = _f32(t, (self.batch, N_OUT))
        g = np.empty(self.n_params, dtype=np.float32)
        loss = ctypes.c_double(0.0)
        check(lib().ek_mlp_gradients(self._h, x.ctypes.data_as(_fp), t.ctypes.data_as(_fp), g.ctypes.data_as(_fp),
                                     ctypes.byref(loss)))
        return g, float(loss.value)

    def forward(self, x):
        x = _f32(x, (len(x), N_IN))
        y = np.empty((len(x), N_OUT), dtype=np.float32)
        check(lib().ek_mlp_forward(self._h, x.ctypes.data_as(_fp), len(x), y.ctypes.data_as(_fp)))
        return y

    @property
    def launches(self):
        v = ctypes.c_int64(0)
        check(lib().ek_mlp_launch_count(self._h, ctypes.byref(v)))
        return int(v.value)


def gemm_bf16(a, b, c, stream=0):
    """c = a @ b.T on the tensor cores; torch CUDA tensors (a, b bfloat16, c float32)."""
    m, k = a.shape
    n = b.shape[0]
    check(lib().ek_gemm_bf16(ctypes.c_void_p(a.data_ptr()), a.stride(0), ctypes.c_void_p(b.data_ptr()), b.stride(0),
                             ctypes.c_void_p(c.data_ptr()), c.stride(0), m, n, k, ctypes.c_void_p(stream)))
    return c
