"""CPU checks of the grid-relaxation restatement (oracle.jacobi_poisson, the
reference's poisson_phi / gpu_poisson, poisson.cu:35-130) and of the direct
five-point solve it converges to (oracle.five_point_poisson)."""
import numpy as np

from conftest import rel_err


def _case(nx=24, ny=13, seed=5):
    from cases import lattice_params
    p = lattice_params(nx, ny, kappa_h=4.0, zeta=-1.2, zeta_hi=-0.6)
    rng = np.random.default_rng(seed)
    cp = 1.0 + 0.2 * rng.standard_normal((ny, nx))
    cn = 1.0 + 0.2 * rng.standard_normal((ny, nx))
    return p, cp, cn


def test_five_point_manufactured_solution(oracle_mod):
    """phi = linear wall interpolation + A sin(pi n y/H) cos(2 pi m x/nx) is an
    exact solution of the five-point system: the cosine is an eigenvector of
    the three-point x-Laplacian, eigenvalue -(4/dx^2) sin^2(pi m/nx), the
    sine one of the three-point y-Laplacian."""
    from cases import lattice_params
    nx, ny, n, m, A = 32, 21, 3, 2, 0.7
    p = lattice_params(nx, ny, zeta=-1.0, zeta_hi=-0.25)
    H = ny - 1
    y = np.arange(ny)[:, None]
    x = np.arange(nx)[None, :]
    lx = (4.0 / p["dx"] ** 2) * np.sin(np.pi * m / nx) ** 2
    ly = (4.0 / p["dy"] ** 2) * np.sin(np.pi * n / (2 * H)) ** 2
    mode = A * np.sin(np.pi * n * y / H) * np.cos(2 * np.pi * m * x / nx)
    phi = p["zeta_lo"] + (p["zeta_hi"] - p["zeta_lo"]) * y / H + mode
    charge = (lx + ly) * mode * p["eps"] / p["f_charge"]   # lap5(phi) = -f_charge (c+ - c-)/eps
    got = oracle_mod.five_point_poisson(p, 1.0 + 0.5 * charge, 1.0 - 0.5 * charge, p["zeta_lo"], p["zeta_hi"])
    assert rel_err(got, phi) < 1e-13


def test_jacobi_converges_to_the_five_point_solution(oracle_mod):
    p, cp, cn = _case()
    direct = oracle_mod.five_point_poisson(p, cp, cn, p["zeta_lo"], p["zeta_hi"])
    psi, change = oracle_mod.jacobi_poisson(p, cp, cn, np.zeros_like(cp), p["zeta_lo"], p["zeta_hi"], 4000)
    assert change < 1e-12
    assert rel_err(psi, direct) < 1e-10


def test_five_point_and_spectral_solves_differ_by_the_x_discretisation(oracle_mod):
    """The spectral solve (fast_Poisson: exact kx^2) and the five-point system
    agree for smooth fields and part for the shortest x-waves."""
    p, cp, cn = _case(nx=64, ny=17)
    o = oracle_mod.OracleChannel(p)
    o.set_fields(cp=cp, cn=cn)
    o.poisson()
    spectral = o.get_fields(("psi",))["psi"]
    o.close()
    direct = oracle_mod.five_point_poisson(p, cp, cn, p["zeta_lo"], p["zeta_hi"])
    e = rel_err(direct, spectral)
    assert 1e-6 < e < 0.5, e
