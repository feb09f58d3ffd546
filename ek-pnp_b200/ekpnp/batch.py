"""Batches of independent channels stepped in lockstep (ek_batch_* of the C ABI).

The reference runs one channel per process (main.cu); a Batch runs hundreds
of channels of different sizes and parameters with four kernel launches per
step for all of them (five with the FP32 Poisson form).  Each channel is a Channel view (fields in and out,
wall profiles, Poisson-Boltzmann start, residual) that is stepped only
through the batch.
"""
from __future__ import annotations

import ctypes

import numpy as np

from ._lib import EkParams, check, lib
from .channel import Channel


class Batch:
    def __init__(self, params_list):
        self.params = [dict(p) for p in params_list]
        if not self.params:
            raise ValueError("a batch needs at least one channel")
        arr = (EkParams * len(self.params))(*[EkParams.from_dict(p) for p in self.params])
        h = ctypes.c_void_p()
        check(lib().ek_batch_create(arr, len(self.params), ctypes.byref(h)))
        self._h = h
        self.channels = []
        for i, p in enumerate(self.params):
            ch = ctypes.c_void_p()
            check(lib().ek_batch_channel(self._h, i, ctypes.byref(ch)))
            self.channels.append(Channel._borrowed(ch, p, self))
        n = ctypes.c_int64(0)
        check(lib().ek_batch_count(self._h, None, ctypes.byref(n)))
        self.nodes = int(n.value)

    # -- lifetime ---------------------------------------------------------
    def close(self):
        if getattr(self, "_h", None):
            for ch in self.channels:
                ch._h = None
            check(lib().ek_batch_destroy(self._h))
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

    def __len__(self):
        return len(self.channels)

    def __getitem__(self, i):
        return self.channels[i]

    # -- stepping ---------------------------------------------------------
    def set_cycle(self, steps=200, rebase=True, graph=True):
        check(lib().ek_batch_set_cycle(self._h, int(steps), 1 if rebase else 0, 1 if graph else 0))

    def init_equilibrium(self):
        check(lib().ek_batch_init_equilibrium(self._h))

    def step(self, n=1):
        check(lib().ek_batch_step(self._h, int(n)))

    def sync(self):
        check(lib().ek_batch_sync(self._h))

    @property
    def steps(self):
        v = ctypes.c_int64(0)
        check(lib().ek_batch_step_count(self._h, ctypes.byref(v)))
        return int(v.value)

    @property
    def launches(self):
        v = ctypes.c_int64(0)
        check(lib().ek_batch_launch_count(self._h, ctypes.byref(v)))
        return int(v.value)

    @property
    def stream(self):
        v = ctypes.c_void_p()
        check(lib().ek_batch_stream(self._h, ctypes.byref(v)))
        return int(v.value or 0)

    @staticmethod
    def shapes():
        """Block shapes of the batched LBM kernel: (threads, widest tile, blocks per SM)."""
        out = []
        n = 0
        while True:
            t, w, m = ctypes.c_int32(0), ctypes.c_int32(0), ctypes.c_int32(0)
            if lib().ek_batch_shape_info(n, ctypes.byref(t), ctypes.byref(w), ctypes.byref(m)) != 0:
                return out
            out.append((int(t.value), int(w.value), int(m.value)))
            n += 1

    @property
    def shape(self):
        v = ctypes.c_int32(0)
        check(lib().ek_batch_shape(self._h, ctypes.byref(v)))
        return int(v.value)

    @shape.setter
    def shape(self, index):
        check(lib().ek_batch_set_shape(self._h, int(index)))

    def autotune(self, steps=20):
        """Time each block shape (advances the state); returns (chosen index, [ms/step per shape])."""
        chosen = ctypes.c_int32(0)
        ms = np.zeros(len(self.shapes()))
        check(lib().ek_batch_autotune(self._h, int(steps), ctypes.byref(chosen),
                                      ms.ctypes.data_as(ctypes.POINTER(ctypes.c_double))))
        return int(chosen.value), ms.tolist()

    def resync(self):
        """Adopt the channels' current states (after Channel.tile_x)."""
        check(lib().ek_batch_resync(self._h))

    def restart(self, mask):
        """Restart the masked channels in place from the fields loaded through
        their own handles (Channel.set_fields); the others step on untouched."""
        m = np.ascontiguousarray(np.asarray(mask, dtype=bool).astype(np.uint8))
        if m.shape != (len(self.channels),):
            raise ValueError("one flag per channel")
        check(lib().ek_batch_restart(self._h, ctypes.c_void_p(m.ctypes.data)))

    def set_active(self, mask):
        """Freeze (False) or step (True) each channel."""
        m = np.ascontiguousarray(np.asarray(mask, dtype=bool).astype(np.uint8))
        if m.shape != (len(self.channels),):
            raise ValueError("one flag per channel")
        check(lib().ek_batch_set_active(self._h, ctypes.c_void_p(m.ctypes.data)))

    @property
    def active(self):
        m = np.zeros(len(self.channels), dtype=np.uint8)
        n = ctypes.c_int64(0)
        check(lib().ek_batch_active(self._h, ctypes.c_void_p(m.ctypes.data), ctypes.byref(n)))
        return m.astype(bool), int(n.value)

    def residual(self, interval):
        """Per-channel residuals (n, 5): u_x, c+, c-, psi, max (inf before the first snapshot)."""
        out = np.zeros((len(self.channels), 5))
        worst = np.zeros(5)
        dp = ctypes.POINTER(ctypes.c_double)
        check(lib().ek_batch_residual(self._h, int(interval), out.ctypes.data_as(dp), worst.ctypes.data_as(dp)))
        return out
