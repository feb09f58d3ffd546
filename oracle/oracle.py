"""Python handle on the CPU oracle (oracle/ek_oracle.cpp).  TEST INFRASTRUCTURE:
imported only by tests/, __graft_entry__.smoke() and bench.py's CPU-baseline
leg, always as the checker or the reported CPU baseline, never as the product.

build() compiles oracle/libekoracle.so with g++ -O3 -fopenmp -ffp-contract=off
(no FMA contraction, no fast-math).  OracleChannel has the same methods as the
product's ekpnp.Channel so tests can drive both the same way.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(HERE, "ek_oracle.cpp")
LIB = os.path.join(HERE, "libekoracle.so")
HDR = os.path.join(os.path.dirname(HERE), "include", "ekpnp.h")
FIELDS = ("rho", "ux", "uy", "cp", "cn", "psi", "ex", "ey")
_DOUBLES = ("dx", "dy", "dt", "cfl", "cs2", "lx", "rho0", "c0", "nu", "magic_f", "diff_p", "magic_p",
            "mob_p", "diff_n", "magic_n", "mob_n", "eps", "f_charge", "zeta_lo", "zeta_hi", "cp_lo",
            "cp_hi", "cn_lo", "cn_hi", "ext_x", "exf", "uw")


class _Params(ctypes.Structure):
    _fields_ = [("nx", ctypes.c_int32), ("ny", ctypes.c_int32), ("storage", ctypes.c_int32),
                ("flags", ctypes.c_int32)] + [(n, ctypes.c_double) for n in _DOUBLES]


def build(force=False):
    if not force and os.path.exists(LIB) and os.path.getmtime(LIB) >= max(os.path.getmtime(SRC),
                                                                          os.path.getmtime(HDR)):
        return LIB
    cmd = ["g++", "-O3", "-std=c++17", "-fopenmp", "-ffp-contract=off", "-fPIC", "-shared", "-o", LIB, SRC]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("oracle build failed:\n" + r.stderr)
    return LIB


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            build()
        h = ctypes.CDLL(LIB)
        dp = ctypes.POINTER(ctypes.c_double)
        vp = ctypes.c_void_p
        h.ekor_create.argtypes = [ctypes.POINTER(_Params), ctypes.POINTER(vp)]
        h.ekor_destroy.argtypes = [vp]
        h.ekor_destroy.restype = None
        h.ekor_set_threads.argtypes = [ctypes.c_int]
        h.ekor_set_fields.argtypes = [vp] + [dp] * 8
        h.ekor_set_wall_profile.argtypes = [vp] + [dp] * 6
        h.ekor_init_equilibrium.argtypes = [vp]
        h.ekor_step.argtypes = [vp, ctypes.c_int]
        h.ekor_poisson.argtypes = [vp]
        h.ekor_get_fields.argtypes = [vp] + [dp] * 8
        h.ekor_get_populations.argtypes = [vp, dp, dp, dp]
        h.ekor_init_pb.argtypes = [vp, ctypes.c_int, ctypes.c_double, ctypes.c_double]
        _lib = h
    return _lib


def set_threads(n=0):
    return lib().ekor_set_threads(int(n))


def _ptr(a):
    return None if a is None else a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


class OracleChannel:
    def __init__(self, params):
        p = _Params()
        for name, _ in _Params._fields_:
            setattr(p, name, params[name])
        self.nx, self.ny = int(params["nx"]), int(params["ny"])
        h = ctypes.c_void_p()
        rc = lib().ekor_create(ctypes.byref(p), ctypes.byref(h))
        if rc != 0:
            raise ValueError(f"oracle rejected the parameters (status {rc})")
        self._h = h

    def close(self):
        if getattr(self, "_h", None):
            lib().ekor_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()

    def _arr(self, a):
        return None if a is None else np.ascontiguousarray(a, dtype=np.float64).reshape(self.ny, self.nx)

    def set_fields(self, rho=None, ux=None, uy=None, cp=None, cn=None, psi=None, ex=None, ey=None):
        arrs = [self._arr(a) for a in (rho, ux, uy, cp, cn, psi, ex, ey)]
        lib().ekor_set_fields(self._h, *[_ptr(a) for a in arrs])

    def set_wall_profile(self, *profiles):
        arrs = [None if a is None else np.ascontiguousarray(a, dtype=np.float64) for a in profiles]
        arrs += [None] * (6 - len(arrs))
        lib().ekor_set_wall_profile(self._h, *[_ptr(a) for a in arrs])

    def init_equilibrium(self):
        lib().ekor_init_equilibrium(self._h)

    def init_poisson_boltzmann(self, iterations=501, omega=0.05, e_kt=1.0):
        lib().ekor_init_pb(self._h, int(iterations), float(omega), float(e_kt))

    def step(self, n=1):
        lib().ekor_step(self._h, int(n))

    def poisson(self):
        lib().ekor_poisson(self._h)

    def get_fields(self, names=FIELDS):
        out = {n: np.empty((self.ny, self.nx)) for n in names}
        lib().ekor_get_fields(self._h, *[_ptr(out.get(n)) for n in FIELDS])
        return out

    def get_populations(self):
        n = self.nx * self.ny
        f, h, t = (np.empty(9 * n) for _ in range(3))
        lib().ekor_get_populations(self._h, _ptr(f), _ptr(h), _ptr(t))
        return [a.reshape(9, self.ny, self.nx) for a in (f, h, t)]


def jacobi_poisson(params, cp, cn, psi0, zlo, zhi, sweeps, omega=1.0):
    """Grid relaxation of the channel's Poisson equation, numpy FP64:
    gpu_poisson's five-point update (poisson.cu:75-130) written for dx != dy
    and made deterministic (each sweep reads the previous iterate only):
        psi = ((L + R)/dx^2 + (U + D)/dy^2 - rhs) / (2/dx^2 + 2/dy^2),
        rhs = -f_charge (c+ - c-) / eps,
    relaxed by omega, periodic in x, rows 0 and ny-1 held at zlo(x), zhi(x)
    (voltage / voltage2 in the reference, poisson.cu:99-106).  Returns the
    iterate after `sweeps` sweeps and the largest change of the last one."""
    p = params
    idx2, idy2 = 1.0 / (p["dx"] * p["dx"]), 1.0 / (p["dy"] * p["dy"])
    rhs = -p["f_charge"] * (np.asarray(cp) - np.asarray(cn)) / p["eps"]
    a = np.array(psi0, dtype=np.float64, copy=True)
    a[0], a[-1] = zlo, zhi
    change = 0.0
    for _ in range(int(sweeps)):
        c = a[1:-1]
        fit = ((np.roll(c, 1, axis=1) + np.roll(c, -1, axis=1)) * idx2 + (a[:-2] + a[2:]) * idy2
               - rhs[1:-1]) / (2.0 * idx2 + 2.0 * idy2)
        new = c + omega * (fit - c)
        change = float(np.abs(new - c).max())
        a = a.copy()
        a[1:-1] = new
    return a, change


def five_point_poisson(params, cp, cn, zlo, zhi):
    """Direct solve of the five-point system whose fixed point jacobi_poisson
    relaxes to: per x-mode m the three-point x-symbol (4/dx^2) sin^2(pi m/nx)
    (where the spectral solve has kx^2), then the tridiagonal y-system with the
    walls lifted into the first and last interior rows.  numpy FP64."""
    from scipy.linalg import solve_banded
    p = params
    ny, nx = np.asarray(cp).shape
    idy2 = 1.0 / (p["dy"] * p["dy"])
    rhs = -p["f_charge"] * (np.asarray(cp) - np.asarray(cn))[1:-1] / p["eps"]
    rhs = rhs.astype(np.complex128)
    zlo, zhi = np.broadcast_to(zlo, (nx,)), np.broadcast_to(zhi, (nx,))
    rhs[0] -= zlo * idy2
    rhs[-1] -= zhi * idy2
    s = np.fft.fft(rhs, axis=1)
    lam = 4.0 / (p["dx"] * p["dx"]) * np.sin(np.pi * np.arange(nx) / nx) ** 2
    n = ny - 2
    out = np.empty_like(s)
    for m in range(nx):
        ab = np.zeros((3, n))
        ab[0, 1:] = idy2
        ab[1] = -2.0 * idy2 - lam[m]
        ab[2, :-1] = idy2
        out[:, m] = solve_banded((1, 1), ab, s[:, m])
    psi = np.empty((ny, nx))
    psi[1:-1] = np.fft.ifft(out, axis=1).real
    psi[0], psi[-1] = zlo, zhi
    return psi
