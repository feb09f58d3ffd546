"""Host-side channel object over the C ABI.

Mirrors the reference's host entry points (LBM.h:149-169) for one channel:
    read_data          -> Channel.set_fields            (LBM.cu:1350-1391)
    init_equilibrium   -> Channel.init_equilibrium      (LBM.cu:183-193)
    stream_collide_save + fast_Poisson (one loop body of main.cu:190-233)
                       -> Channel.step(1)
    fast_Poisson       -> Channel.poisson               (poisson.cu:180-208)
Errors raise EkError with the library's status instead of exiting.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib
from ._lib import EkParams, check, lib

FIELD_NAMES = ("rho", "ux", "uy", "cp", "cn", "psi", "ex", "ey")


def set_device(device: int):
    check(lib().ek_set_device(int(device)))


def device_count() -> int:
    n = ctypes.c_int32(0)
    rc = lib().ek_get_device_count(ctypes.byref(n))
    return int(n.value) if rc == _lib.EK_OK else 0


def _ptr(a):
    return None if a is None else a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


class Channel:
    def __init__(self, params):
        self.params = dict(params) if not isinstance(params, EkParams) else params.to_dict()
        self._p = EkParams.from_dict(self.params)
        self.nx, self.ny = int(self._p.nx), int(self._p.ny)
        h = ctypes.c_void_p()
        check(lib().ek_create(ctypes.byref(self._p), ctypes.byref(h)))
        self._h = h
        self._owner = None

    @classmethod
    def _borrowed(cls, handle, params, owner):
        """A view of a context owned by `owner` (a Batch): never destroyed here."""
        ch = cls.__new__(cls)
        ch.params = dict(params)
        ch._p = EkParams.from_dict(ch.params)
        ch.nx, ch.ny = int(ch._p.nx), int(ch._p.ny)
        ch._h = handle
        ch._owner = owner
        return ch

    # -- lifetime ---------------------------------------------------------
    def close(self):
        if getattr(self, "_owner", None) is not None:
            self._h = None
            return
        if getattr(self, "_h", None):
            check(lib().ek_destroy(self._h))
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

    # -- state ------------------------------------------------------------
    def _arr(self, a):
        if a is None:
            return None
        a = np.ascontiguousarray(a, dtype=np.float64)
        if a.shape != (self.ny, self.nx):
            raise ValueError(f"field shape {a.shape} != {(self.ny, self.nx)}")
        return a

    def set_fields(self, rho=None, ux=None, uy=None, cp=None, cn=None, psi=None, ex=None, ey=None):
        arrs = [self._arr(a) for a in (rho, ux, uy, cp, cn, psi, ex, ey)]
        check(lib().ek_set_fields(self._h, *[_ptr(a) for a in arrs]))

    read_data = set_fields

    def set_wall_profile(self, zeta_lo=None, zeta_hi=None, cp_lo=None, cp_hi=None, cn_lo=None, cn_hi=None):
        arrs = []
        for a in (zeta_lo, zeta_hi, cp_lo, cp_hi, cn_lo, cn_hi):
            if a is not None:
                a = np.ascontiguousarray(a, dtype=np.float64)
                if a.shape != (self.nx,):
                    raise ValueError("wall profiles have nx entries")
            arrs.append(a)
        check(lib().ek_set_wall_profile(self._h, *[_ptr(a) for a in arrs]))

    def init_poisson_boltzmann(self, method="newton", iterations=501, omega=0.05, e_kt=1.0):
        """Poisson-Boltzmann fields (u = 0).  method "reference" is the
        reference's own under-relaxed iteration (LBM.cu:95-145); "newton" a
        damped Newton solve per x-column."""
        m = {"reference": 0, "newton": 1}[method]
        check(lib().ek_init_poisson_boltzmann(self._h, m, int(iterations), float(omega), float(e_kt)))

    def init_equilibrium(self):
        check(lib().ek_init_equilibrium(self._h))

    def tile_x(self, src):
        """This channel's state := src's repeated along x (ek_tile_x): same ny
        and storage, this nx a multiple of src's.  A channel inside a batch
        is followed by Batch.resync()."""
        check(lib().ek_tile_x(self._h, src._h))

    def step(self, n=1):
        check(lib().ek_step(self._h, int(n)))

    def set_lbm_kernel(self, form):
        """'auto', 'plain' or 'tma' (shifted storage; both forms are bit-identical)."""
        check(lib().ek_set_option(self._h, 1, {"auto": 0, "plain": 1, "tma": 2}[form]))

    def save_restart(self, path, time=0.0):
        """The channel's fields as the reference's data_end.dat (save_data_end)."""
        import os
        check(lib().ek_save_restart(self._h, os.fsencode(path), float(time)))

    def load_restart(self, path):
        """Fields from a data_end.dat file (read_data); returns its time."""
        import os
        t = ctypes.c_double(0.0)
        check(lib().ek_load_restart(self._h, os.fsencode(path), ctypes.byref(t)))
        return float(t.value)

    def set_poisson(self, form):
        """Arithmetic of the Poisson solve: "auto", "f64" or "f32" (row FFTs and
        column solves of the x-modes >= 1 in FP32, the zero mode in FP64)."""
        check(lib().ek_set_option(self._h, 2, {"auto": 0, "f64": 1, "f32": 2}[form]))

    def rebase(self):
        check(lib().ek_rebase(self._h))

    def set_rebase_interval(self, steps):
        check(lib().ek_set_rebase_interval(self._h, int(steps)))

    def poisson(self):
        check(lib().ek_poisson(self._h))

    fast_Poisson = poisson

    def poisson_jacobi(self, max_sweeps=1_000_000, tol=1e-9, omega=1.0, check_every=100):
        """Grid relaxation of the Poisson equation from the current psi (the
        reference's poisson_phi, made schedule-independent); returns (sweeps,
        last measured largest change)."""
        n, ch = ctypes.c_int32(0), ctypes.c_double(0.0)
        check(lib().ek_poisson_jacobi(self._h, int(max_sweeps), float(tol), float(omega), int(check_every),
                                      ctypes.byref(n), ctypes.byref(ch)))
        return int(n.value), float(ch.value)

    poisson_phi = poisson_jacobi

    def sync(self):
        check(lib().ek_sync(self._h))

    def get_fields(self, names=FIELD_NAMES):
        out = {n: np.empty((self.ny, self.nx)) for n in names}
        check(lib().ek_get_fields(self._h, *[_ptr(out.get(n)) for n in FIELD_NAMES]))
        return out

    def residual(self, interval):
        out = np.empty(5)
        check(lib().ek_residual(self._h, int(interval), _ptr(out)))
        return out

    @property
    def steps(self):
        v = ctypes.c_int64()
        check(lib().ek_step_count(self._h, ctypes.byref(v)))
        return int(v.value)

    # -- profiling ----------------------------------------------------------
    PHASES = ("lbm", "poisson_rows_fwd", "poisson_tridiag", "poisson_rows_inv")

    def profile(self, on=True):
        check(lib().ek_profile_enable(self._h, 1 if on else 0))

    def profile_read(self):
        ms = (ctypes.c_double * 4)()
        n = (ctypes.c_int64 * 4)()
        check(lib().ek_profile_read(self._h, ms, n))
        return {ph: (float(ms[i]), int(n[i])) for i, ph in enumerate(self.PHASES)}

    def mark(self, slot):
        check(lib().ek_mark(self._h, int(slot)))

    def elapsed_ms(self, a, b):
        v = ctypes.c_double()
        check(lib().ek_elapsed(self._h, int(a), int(b), ctypes.byref(v)))
        return float(v.value)

    @property
    def launches(self):
        v = ctypes.c_int64()
        check(lib().ek_launch_count(self._h, ctypes.byref(v)))
        return int(v.value)

    def set_fields_from_pointers(self, ptrs):
        """set_fields from raw host addresses (e.g. pinned buffers); ptrs is a
        sequence of 8 integers (0 = leave the field unchanged)."""
        dp = ctypes.POINTER(ctypes.c_double)
        args = [ctypes.cast(ctypes.c_void_p(p), dp) if p else None for p in ptrs]
        check(lib().ek_set_fields(self._h, *args))

    def get_fields_to_pointers(self, ptrs):
        dp = ctypes.POINTER(ctypes.c_double)
        args = [ctypes.cast(ctypes.c_void_p(p), dp) if p else None for p in ptrs]
        check(lib().ek_get_fields(self._h, *args))

    def set_stream(self, stream_handle: int):
        check(lib().ek_set_stream(self._h, ctypes.c_void_p(stream_handle)))
