"""The reference's file formats and diagnostics (host side, ek_write_* /
ek_read_restart / ek_diag_* of the C ABI): the data_end.dat restart file,
Tecplot zones with the reference's derived fields, DMD snapshots, the
electric current through the top wall and the reference's umax."""
from __future__ import annotations

import ctypes
import os

import numpy as np

from ._lib import check, lib

_dp = ctypes.POINTER(ctypes.c_double)
ORDER = ("ux", "uy", "rho", "cp", "psi", "ex", "ey", "cn")  # column order of the restart file after time


def _arr(a, shape):
    a = np.ascontiguousarray(a, dtype=np.float64)
    if a.shape != shape:
        raise ValueError(f"expected shape {shape}, got {a.shape}")
    return a


def _path(p):
    return os.fsencode(p)


def write_restart(path, time, fields):
    ny, nx = np.shape(fields["ux"])
    arrs = [_arr(fields[k], (ny, nx)) for k in ORDER]
    check(lib().ek_write_restart(_path(path), nx, ny, float(time), *[a.ctypes.data_as(_dp) for a in arrs]))


def read_restart(path, nx, ny):
    """(time, fields) from a data_end.dat file."""
    out = {k: np.empty((ny, nx)) for k in ORDER}
    t = ctypes.c_double(0.0)
    check(lib().ek_read_restart(_path(path), nx, ny, ctypes.byref(t), *[out[k].ctypes.data_as(_dp) for k in ORDER]))
    return float(t.value), out


def write_tecplot(path, time, fields, dx=1.0, dy=1.0, first=True):
    ny, nx = np.shape(fields["ux"])
    arrs = [_arr(fields[k], (ny, nx)) for k in ORDER]
    check(lib().ek_write_tecplot(_path(path), 1 if first else 0, float(time), nx, ny, float(dx), float(dy),
                                 *[a.ctypes.data_as(_dp) for a in arrs]))


def write_dmd(path, cp, append=False):
    ny, nx = np.shape(cp)
    a = _arr(cp, (ny, nx))
    check(lib().ek_write_dmd(_path(path), 1 if append else 0, nx, ny, a.ctypes.data_as(_dp)))


def current(cp, ey, mob_p, dy=1.0):
    ny, nx = np.shape(cp)
    a, b = _arr(cp, (ny, nx)), _arr(ey, (ny, nx))
    v = ctypes.c_double(0.0)
    check(lib().ek_diag_current(nx, ny, a.ctypes.data_as(_dp), b.ctypes.data_as(_dp), float(mob_p), float(dy),
                                ctypes.byref(v)))
    return float(v.value)


def umax(uy):
    ny, nx = np.shape(uy)
    a = _arr(uy, (ny, nx))
    v = ctypes.c_double(0.0)
    check(lib().ek_diag_umax(nx, ny, a.ctypes.data_as(_dp), ctypes.byref(v)))
    return float(v.value)
