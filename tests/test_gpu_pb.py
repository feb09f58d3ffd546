"""Poisson-Boltzmann start (ek_init_poisson_boltzmann).

* The reference form (under-relaxed Picard iteration of LBM.cu:95-145) on the
  GPU matches the CPU oracle's restatement of it where it converges.
* The Newton form solves the discrete PB equation to rounding (residual
  checked in numpy) at the strong coupling of the 4096x1024 workload
  (kappa*H = 32, zeta = -4), where the reference form diverges.
* From that start the coupled step stays finite at zeta = -4 (from the
  uniform start it diverges within 100 steps in the reference's own scheme).
"""
import numpy as np
import pytest

from conftest import rel_err

pytestmark = pytest.mark.gpu


def pb_residual(p, psi):
    """Discrete PB residual of the interior rows, relative to the largest term."""
    col = psi[:, 0]
    lap = (col[:-2] - 2 * col[1:-1] + col[2:]) / p["dy"] ** 2
    src = p["f_charge"] * p["c0"] * (np.exp(-col[1:-1]) - np.exp(col[1:-1])) / p["eps"]
    return float(np.abs(lap + src).max() / max(np.abs(lap).max(), np.abs(src).max()))


def test_reference_pb_matches_oracle(oracle_mod):
    import ekpnp
    p = ekpnp.channel_params(16, 128, kappa_h=8.0, zeta=-2.0)
    with ekpnp.Channel(p) as ch:
        ch.init_poisson_boltzmann("reference", iterations=501, omega=0.05)
        got = ch.get_fields()
    o = oracle_mod.OracleChannel(p)
    o.init_poisson_boltzmann(501, 0.05)
    ref = o.get_fields()
    for k in ("psi", "cp", "cn"):
        assert rel_err(got[k], ref[k]) < 1e-12, k


def test_newton_pb_matches_converged_reference_pb(oracle_mod):
    import ekpnp
    p = ekpnp.channel_params(16, 128, kappa_h=8.0, zeta=-2.0)
    with ekpnp.Channel(p) as ch:
        ch.init_poisson_boltzmann("newton")
        got = ch.get_fields()
    o = oracle_mod.OracleChannel(p)
    o.init_poisson_boltzmann(3001, 0.05)
    ref = o.get_fields()
    assert rel_err(got["psi"], ref["psi"]) < 1e-11
    assert pb_residual(p, got["psi"]) < 1e-12


def test_newton_pb_strong_coupling_and_stable_start():
    import ekpnp
    p = ekpnp.channel_params(64, 1024, kappa_h=32.0, zeta=-4.0, ex=5e-5)
    with ekpnp.Channel(dict(p, storage=ekpnp.STORE_F32)) as ch:
        ch.init_poisson_boltzmann("newton")
        f = ch.get_fields()
        assert pb_residual(p, f["psi"]) < 1e-12
        assert abs(f["psi"][0, 0] + 4.0) < 1e-15 and abs(f["psi"][512, 0]) < 1e-3
        assert np.allclose(f["cp"] * f["cn"], 1.0, rtol=1e-12)
        ch.init_equilibrium()
        ch.step(500)
        g = ch.get_fields()
        assert all(np.all(np.isfinite(g[k])) for k in g)
        assert np.abs(g["ux"]).max() < 0.05
