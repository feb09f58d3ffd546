"""Parity cases and the lattice-unit parameter mapping.  TEST INFRASTRUCTURE.

A case is a channel (nx, ny), physics in lattice units, a seeded initial state
and a step count.  The same dictionary drives three things:
  * the patched reference build (oracle/ref_build.py writes these constants
    into a copy of LBM.h, whose symbols are named per field below),
  * the CPU oracle (oracle/ek_oracle.cpp, through tests/ and bench.py),
  * the GPU product (through its C ABI), in the parity tests.

Lattice-unit mapping of the reference's SI constants (LBM.h:39-112):
  dx = dy = dt = CFL = 1, cs_square = 1/3, Lx = nx*dx, Ly = (ny-1)*dy
  nu = cs2*(tau_s - 1/2)*dt (tau_s = 1 gives 1/6); V = VC = VT = Lambda
  diffu = D = diffusivity of both ions; K = +D, Kn = -D (Einstein relation
  with the potential in thermal volts, e/kT = 1)
  eps = 1; convertCtoCharge = eps*kappa^2/(2*c0) with kappa = kappaH/H and
  H = ny-1, the wall-to-wall distance between the Dirichlet rows of the
  Poisson solve (linearised Poisson-Boltzmann: lap(psi) = kappa^2 psi)
  voltage = voltage2 = zeta; charge0/1 = c0*exp(-zeta), charge0n/1n =
  c0*exp(+zeta) (Boltzmann wall concentrations); Ext = E_x; exf = uw = 0
  rho0 = 1, chargeinf = c0.
"""
from __future__ import annotations

import math

import numpy as np

FLAG_FORCE = 1
FLAG_REST_QUIRK = 2
FLAG_MOMENTS_EVERY_STEP = 4
FLAG_EXPLICIT_E = 8


def lattice_params(nx, ny, *, kappa_h=8.0, zeta=-2.0, ex=1e-4, diff=0.05, tau_s=1.0,
                   magic=0.25, c0=1.0, rho0=1.0, eps=1.0, force=True, rest_quirk=True,
                   zeta_hi=None, uw=0.0, cfl=1.0, dx=1.0):
    """ek_params fields (as a dict) for a channel in lattice-like units.

    cfl/dx other than 1 keep the reference's dimensional form: dt = cfl*dx,
    cs2 = 1/(3 cfl^2) (LBM.h:50-52), nu = cs2*(tau_s-1/2)*dt."""
    zeta_hi = zeta if zeta_hi is None else zeta_hi
    dt = cfl * dx
    cs2 = 1.0 / 3.0 / (cfl * cfl)
    h = (ny - 1) * dx
    kappa = kappa_h / h
    flags = (FLAG_FORCE if force else 0) | (FLAG_REST_QUIRK if rest_quirk else 0)
    return dict(
        nx=int(nx), ny=int(ny), storage=0, flags=flags,
        dx=dx, dy=dx, dt=dt, cfl=cfl, cs2=cs2, lx=nx * dx,
        rho0=rho0, c0=c0,
        nu=cs2 * (tau_s - 0.5) * dt, magic_f=magic,
        diff_p=diff, magic_p=magic, mob_p=diff,
        diff_n=diff, magic_n=magic, mob_n=-diff,
        eps=eps, f_charge=eps * kappa * kappa / (2.0 * c0),
        zeta_lo=zeta, zeta_hi=zeta_hi,
        cp_lo=c0 * math.exp(-zeta), cp_hi=c0 * math.exp(-zeta_hi),
        cn_lo=c0 * math.exp(zeta), cn_hi=c0 * math.exp(zeta_hi),
        ext_x=ex, exf=0.0, uw=uw,
    )


def initial_state(nx, ny, seed, c0=1.0, rho0=1.0, noise=1e-3):
    """u = 0, psi = 0, E = 0, rho = rho0, c+- = c0*(1 + noise*N(0,1)).

    numpy default_rng(seed); a standard normal of shape (ny, nx) is drawn first
    for c+ and then for c-."""
    rng = np.random.default_rng(seed)
    cp = c0 * (1.0 + noise * rng.standard_normal((ny, nx)))
    cn = c0 * (1.0 + noise * rng.standard_normal((ny, nx)))
    z = np.zeros((ny, nx))
    return dict(rho=np.full((ny, nx), rho0), ux=z.copy(), uy=z.copy(), cp=cp, cn=cn,
                psi=z.copy(), ex=z.copy(), ey=z.copy())


# name -> (params, seed, steps).  Small cases pin the oracle (fixtures under
# tests/golden/); "config1" is the 256x128 channel run for 20,000 steps.
def _cases():
    c = {}
    c["g16x12"] = (lattice_params(16, 12, kappa_h=4.0, zeta=-2.0, ex=1e-3), 10, 200)
    c["g32x33"] = (lattice_params(32, 33, kappa_h=8.0, zeta=-2.0, ex=1e-4), 11, 300)
    # the reference's default shape (NX = 10 is not a power of two)
    c["g10x101"] = (lattice_params(10, 101, kappa_h=6.0, zeta=-1.0, ex=5e-4), 12, 100)
    # asymmetric walls and a moving top wall
    c["g24x17w"] = (lattice_params(24, 17, kappa_h=3.0, zeta=-1.5, zeta_hi=-0.5, ex=2e-3,
                                   uw=1e-3, diff=0.08), 13, 150)
    # dimensional form: CFL and dx other than one
    c["g16x12d"] = (lattice_params(16, 12, kappa_h=4.0, zeta=-2.0, ex=1e-3, cfl=0.5, dx=0.5),
                    14, 100)
    # force off: the reference as shipped
    c["g16x12f"] = (lattice_params(16, 12, kappa_h=4.0, zeta=-2.0, ex=1e-3, force=False), 15, 100)
    c["config1"] = (lattice_params(256, 128, kappa_h=8.0, zeta=-2.0, ex=1e-4, diff=0.05), 0, 20000)
    # speed only: the 4096x1024 channel's physics in FP64, 1000 steps of the
    # reference's own loop (its "speed:" line) against the drop-in build
    c["speed2"] = (lattice_params(4096, 1024, kappa_h=32.0, zeta=-4.0, ex=5e-5, diff=0.05), 1, 1000)
    return c


CASES = _cases()
FIELDS = ("rho", "ux", "uy", "cp", "cn", "psi", "ex", "ey")
