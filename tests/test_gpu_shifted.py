"""Shifted-storage forms (FP32 and FP16 populations, FP32 arithmetic) against
the FP64 path, which itself matches the reference build (test_gpu_parity.py).

Bar for FP32: 1e-5 of the field's max-abs on u_x, c+, c-, psi and the plug
velocity (mean u_x over the centre half of the rows).  FP16 storage is held
to 2e-2 and its errors are reported, not optimised for.
"""
import numpy as np
import pytest

from conftest import rel_err

pytestmark = pytest.mark.gpu


def run(p, init, steps, storage):
    import ekpnp
    with ekpnp.Channel(dict(p, storage=storage)) as ch:
        ch.set_fields(**init)
        ch.init_equilibrium()
        ch.step(steps)
        return ch.get_fields()


def plug(u):
    ny = u.shape[0]
    return float(u[ny // 4: ny - ny // 4].mean())


def errors(a, b):
    e = {k: rel_err(a[k], b[k]) for k in ("ux", "cp", "cn", "psi")}
    e["u_plug"] = abs(plug(a["ux"]) - plug(b["ux"])) / abs(plug(b["ux"]))
    return e


@pytest.fixture(scope="module")
def medium():
    """128x64, kappa*H = 16, zeta = -2 from the noisy uniform start.  (At
    zeta = -4 that start diverges within 100 steps in the reference's own
    scheme -- the CPU oracle shows it -- so the stronger wall potential is
    tested from the Poisson-Boltzmann start instead.)"""
    import ekpnp
    p = ekpnp.channel_params(128, 64, kappa_h=16.0, zeta=-2.0, ex=5e-5, diff=0.05)
    init = ekpnp.noisy_uniform_state(128, 64, seed=1)
    ref = run(p, init, 3000, ekpnp.STORE_F64)
    return p, init, ref


def test_fp32_within_1e5_of_fp64(medium):
    import ekpnp
    p, init, ref = medium
    e = errors(run(p, init, 3000, ekpnp.STORE_F32), ref)
    assert max(e.values()) <= 1e-5, e


def test_fp16_storage_bounded(medium):
    import ekpnp
    p, init, ref = medium
    e = errors(run(p, init, 3000, ekpnp.STORE_F16), ref)
    assert max(e.values()) <= 2e-2, e


@pytest.mark.parametrize("name", ["g24x17w", "g16x12d", "g16x12f"])
def test_fp32_wall_and_unit_variants(name):
    """Moving top wall, asymmetric walls, CFL != 1 and force off in FP32."""
    import ekpnp
    from cases import CASES, initial_state
    p, seed, steps = CASES[name]
    init = initial_state(p["nx"], p["ny"], seed)
    a = run(p, init, steps, ekpnp.STORE_F32)
    b = run(p, init, steps, ekpnp.STORE_F64)
    e = {k: rel_err(a[k], b[k]) for k in ("cp", "cn", "psi")}
    assert max(e.values()) <= 1e-5, e
    # u is still at the 1e-6 level after a few hundred steps: absolute bound
    assert np.abs(a["ux"] - b["ux"]).max() <= 1e-5 * np.abs(b["ux"]).max() + 1e-9
