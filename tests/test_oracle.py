"""CPU oracle checks (no GPU): pinned against the reference build's own output
(fixtures under tests/golden/, produced by tests/golden/make_golden.py from the
patched reference binary), and against independent numpy restatements of the
Poisson step.

Tolerance against the reference: 1e-12 of the field's max-abs plus 1e-15
absolute.  Bitwise agreement is not expected: the reference uses cuFFT and FMA
contraction, the oracle its own FFT and no contraction.  The absolute term is
the rounding level of the populations (~1e-17 per operation on values ~0.1)
accumulated over the few hundred steps of a fixture run; it matters only for
velocities that are still small (u ~ 2e-5 after 100 steps of the 10x101 case).
"""
import glob
import json
import os

import numpy as np
import pytest

from conftest import GOLDEN, rel_err

RTOL, ATOL = 1e-12, 1e-15
PARITY_FIELDS = ("rho", "ux", "uy", "cp", "cn", "psi", "ey")


def golden_files():
    return sorted(glob.glob(os.path.join(GOLDEN, "g*.npz")))


def load_golden(path):
    z = np.load(path)
    p = json.loads(str(z["params"]))
    return p, int(z["seed"]), int(z["steps"]), bool(z["deterministic"]), {k: z[k] for k in z.files}


def close(a, b, rtol=RTOL, atol=ATOL):
    return float(np.abs(a - b).max()) <= rtol * float(np.abs(b).max()) + atol


def test_golden_fixtures_present():
    names = {os.path.basename(f)[:-4] for f in golden_files()}
    assert {"g16x12", "g32x33", "g10x101", "g24x17w", "g16x12d", "g16x12f"} <= names


@pytest.mark.parametrize("path", golden_files(), ids=lambda p: os.path.basename(p)[:-4])
def test_oracle_matches_reference_build(path, oracle_mod):
    from cases import initial_state
    p, seed, steps, _, ref = load_golden(path)
    o = oracle_mod.OracleChannel(p)
    o.set_fields(**initial_state(p["nx"], p["ny"], seed, c0=p["c0"], rho0=p["rho0"]))
    o.init_equilibrium()
    o.step(steps)
    got = o.get_fields()
    bad = {k: rel_err(got[k], ref[k]) for k in PARITY_FIELDS if not close(got[k], ref[k])}
    assert not bad, bad


def _numpy_poisson(p, cp, cn, zlo, zhi):
    """Independent numpy restatement of fast_Poisson + efield (poisson.cu:132-306,
    wavenumbers main.cu:119-137) on the odd-extended array with numpy's FFT."""
    ny, nx = cp.shape
    ne = 2 * (ny - 1)
    ext = np.zeros((ne, nx))
    s = -p["f_charge"] * (cp - cn) / p["eps"]
    ext[1:ny - 1] = s[1:ny - 1]
    ext[1] -= zlo / p["dy"] / p["dy"]
    ext[ny - 2] -= zhi / p["dy"] / p["dy"]
    for y in range(ny, ne):
        ext[y] = -ext[ne - y]
    kx = np.array([(i if i <= nx // 2 else i - nx) * 2.0 * np.pi / p["lx"] for i in range(nx)])
    ky = np.array([(i if i <= ne // 2 else i - ne) * 2.0 * np.pi / (ne * p["dy"]) for i in range(ne)])
    mu = (4.0 / p["dy"] ** 2) * np.sin(ky[:, None] * p["dy"] * 0.5) ** 2 + kx[None, :] ** 2
    mu[0, 0] = 1.0
    phi = np.real(np.fft.ifft2(-np.fft.fft2(ext) / mu))[:ny]
    phi[0], phi[-1] = zlo, zhi
    ex = 0.5 * (np.roll(phi, 1, axis=1) - np.roll(phi, -1, axis=1)) / p["dx"]
    ey = 0.5 * (np.roll(phi, 1, axis=0) - np.roll(phi, -1, axis=0)) / p["dy"]
    ey[0], ey[-1] = ey[1], ey[-2]
    return phi, ex, ey


@pytest.mark.parametrize("shape", [(16, 12), (10, 101), (24, 17), (64, 33)])
def test_oracle_poisson_matches_numpy(shape, oracle_mod):
    from cases import lattice_params
    nx, ny = shape
    p = lattice_params(nx, ny, kappa_h=5.0, zeta=-1.5, zeta_hi=-0.7)
    rng = np.random.default_rng(7)
    cp = 1.0 + 0.3 * rng.standard_normal((ny, nx))
    cn = 1.0 + 0.3 * rng.standard_normal((ny, nx))
    o = oracle_mod.OracleChannel(p)
    o.set_fields(cp=cp, cn=cn)
    o.poisson()
    got = o.get_fields(("psi", "ex", "ey"))
    phi, ex, ey = _numpy_poisson(p, cp, cn, p["zeta_lo"], p["zeta_hi"])
    assert rel_err(got["psi"], phi) < 1e-13
    assert np.abs(got["ex"] - ex).max() < 1e-13 * np.abs(phi).max()
    assert np.abs(got["ey"] - ey).max() < 1e-13 * np.abs(phi).max()


def test_oracle_poisson_manufactured_solution(oracle_mod):
    """phi = linear wall interpolation + A sin(pi n y/H) cos(2 pi m x/Lx) is an
    exact discrete solution: the x-derivative is spectral and the sine is an
    eigenvector of the three-point y-Laplacian with eigenvalue
    -(4/dy^2) sin^2(pi n/(2H)), H = ny-1."""
    from cases import lattice_params
    nx, ny, n, m, A = 32, 21, 3, 2, 0.7
    p = lattice_params(nx, ny, zeta=-1.0, zeta_hi=-0.25)
    H = ny - 1
    y = np.arange(ny)[:, None]
    x = np.arange(nx)[None, :]
    lam = (4.0 / p["dy"] ** 2) * np.sin(np.pi * n / (2 * H)) ** 2
    kx = 2 * np.pi * m / p["lx"]
    mode = A * np.sin(np.pi * n * y / H) * np.cos(kx * x)
    phi = p["zeta_lo"] + (p["zeta_hi"] - p["zeta_lo"]) * y / H + mode
    lap = -(kx ** 2 + lam) * mode                 # discrete Laplacian of phi
    charge = -lap * p["eps"] / p["f_charge"]      # lap(phi) = -f_charge (c+ - c-)/eps
    o = oracle_mod.OracleChannel(p)
    o.set_fields(cp=1.0 + 0.5 * charge, cn=1.0 - 0.5 * charge)
    o.poisson()
    assert rel_err(o.get_fields(("psi",))["psi"], phi) < 1e-13


def test_initial_state_is_seeded():
    from cases import initial_state
    a = initial_state(8, 6, 3)
    b = initial_state(8, 6, 3)
    assert all(np.array_equal(a[k], b[k]) for k in a)
    assert abs(a["cp"].std() - 1e-3) < 5e-4 and np.all(a["ux"] == 0)
