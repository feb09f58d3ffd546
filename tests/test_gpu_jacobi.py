"""ek_poisson_jacobi (the reference's grid relaxation, poisson.cu:35-130) on
the GPU against the numpy restatement in the oracle: the same iterate after a
fixed number of sweeps, and convergence to the direct five-point solve."""
import numpy as np
import pytest

from conftest import rel_err

pytestmark = pytest.mark.gpu


def _channel(storage, nx=48, ny=19, seed=3, walls=False):
    import ekpnp
    p = ekpnp.channel_params(nx, ny, kappa_h=4.0, zeta=-1.2, zeta_hi=-0.6, storage=storage)
    rng = np.random.default_rng(seed)
    cp = 1.0 + 0.2 * rng.standard_normal((ny, nx))
    cn = 1.0 + 0.2 * rng.standard_normal((ny, nx))
    zlo = np.full(nx, p["zeta_lo"])
    zhi = np.full(nx, p["zeta_hi"])
    if walls:
        x = np.arange(nx)
        zlo = -1.2 + 0.4 * np.sin(2 * np.pi * x / nx)
        zhi = -0.6 + 0.2 * np.cos(2 * np.pi * x / nx)
    return p, dict(cp=cp, cn=cn, psi=np.zeros((ny, nx))), zlo, zhi


@pytest.mark.parametrize("storage", [0, 1], ids=["f64", "f32"])
@pytest.mark.parametrize("omega", [1.0, 1.6])
def test_fixed_sweeps_match_numpy(storage, omega, oracle_mod):
    import ekpnp
    p, f, zlo, zhi = _channel(storage, walls=True)
    with ekpnp.Channel(p) as ch:
        ch.set_wall_profile(zeta_lo=zlo, zeta_hi=zhi)
        ch.set_fields(**f)
        n, change = ch.poisson_jacobi(max_sweeps=300, tol=0.0, omega=omega, check_every=1000)
        got = ch.get_fields(("psi", "ex", "ey"))
    assert n == 300
    ref, ref_change = oracle_mod.jacobi_poisson(p, f["cp"], f["cn"], f["psi"], zlo, zhi, 300, omega=omega)
    assert rel_err(got["psi"], ref) < 1e-13
    assert abs(change - ref_change) <= 1e-12 * max(ref_change, 1e-300) + 1e-16
    # E follows psi (central differences, gpu_efield)
    ex = (np.roll(ref, 1, axis=1) - np.roll(ref, -1, axis=1)) / (2 * p["dx"])
    assert np.abs(got["ex"] - ex).max() <= 1e-12 * np.abs(ref).max()


def test_converges_to_the_direct_five_point_solve(oracle_mod):
    import ekpnp
    p, f, zlo, zhi = _channel(0, nx=32, ny=15)
    with ekpnp.Channel(p) as ch:
        ch.set_fields(**f)
        n, change = ch.poisson_jacobi(max_sweeps=100_000, tol=1e-13, omega=1.0, check_every=50)
        got = ch.get_fields(("psi",))["psi"]
    assert change < 1e-13 and n < 100_000 and n % 50 == 0
    direct = oracle_mod.five_point_poisson(p, f["cp"], f["cn"], p["zeta_lo"], p["zeta_hi"])
    assert rel_err(got, direct) < 1e-10


def test_bad_arguments_are_rejected():
    import ekpnp
    p, f, _, _ = _channel(0, nx=16, ny=9)
    with ekpnp.Channel(p) as ch:
        ch.set_fields(**f)
        for kw in (dict(max_sweeps=0), dict(tol=-1.0), dict(omega=0.0), dict(omega=2.0), dict(check_every=0)):
            with pytest.raises(ekpnp.EkError):
                ch.poisson_jacobi(**kw)
