"""Behaviour of the C ABI on a GPU: status codes, field round trips, the
residual reduction and its NaN detection, launch accounting."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def small():
    import ekpnp
    p = ekpnp.channel_params(32, 17, kappa_h=4.0, zeta=-1.0, ex=1e-3)
    return p, ekpnp.noisy_uniform_state(32, 17, seed=3)


def test_step_before_init_is_rejected():
    import ekpnp
    p, _ = small()
    with ekpnp.Channel(p) as ch:
        with pytest.raises(ekpnp.EkError) as ei:
            ch.step(1)
        assert ei.value.status == 1


def test_set_get_round_trip():
    import ekpnp
    p, init = small()
    with ekpnp.Channel(p) as ch:
        ch.set_fields(**init)
        got = ch.get_fields()
        for k in ("rho", "ux", "uy", "cp", "cn", "psi", "ex", "ey"):
            assert np.array_equal(got[k], init[k]), k


def test_residual_decreases_and_detects_nan():
    import ekpnp
    p, init = small()
    with ekpnp.Channel(p) as ch:
        ch.set_fields(**init)
        ch.init_equilibrium()
        ch.step(100)
        r0 = ch.residual(100)
        assert np.isinf(r0[4])
        ch.step(100)
        r1 = ch.residual(100)
        ch.step(2000)
        ch.residual(2000)
        ch.step(100)
        r2 = ch.residual(100)
        assert np.all(np.isfinite(r1)) and r2[4] < r1[4]
    bad = dict(init)
    bad["cp"] = init["cp"].copy()
    bad["cp"][5, 7] = np.nan
    with ekpnp.Channel(p) as ch:
        ch.set_fields(**bad)
        ch.init_equilibrium()
        ch.step(10)
        with pytest.raises(ekpnp.EkError) as ei:
            ch.residual(10)
        assert ei.value.status == 4


def test_launch_accounting_and_profile():
    import ekpnp
    p, init = small()
    for storage in (ekpnp.STORE_F64, ekpnp.STORE_F32, ekpnp.STORE_F16):
        with ekpnp.Channel(dict(p, storage=storage)) as ch:
            ch.set_fields(**init)
            ch.init_equilibrium()
            n0 = ch.launches
            ch.profile(True)
            ch.step(25)
            prof = ch.profile_read()
            # one LBM kernel and three Poisson passes, in every storage form
            per_step = 4
            assert ch.launches - n0 == per_step * 25
            assert all(prof[ph][1] == 25 for ph in ch.PHASES)
            assert all(prof[ph][0] > 0 for ph in ch.PHASES)


def test_wall_profile_uniform_equals_default():
    """A wall profile equal to the uniform constants changes nothing."""
    import ekpnp
    p, init = small()
    outs = []
    for use_profile in (False, True):
        with ekpnp.Channel(p) as ch:
            if use_profile:
                nx = p["nx"]
                ch.set_wall_profile(*(np.full(nx, p[k]) for k in ("zeta_lo", "zeta_hi", "cp_lo", "cp_hi", "cn_lo", "cn_hi")))
            ch.set_fields(**init)
            ch.init_equilibrium()
            ch.step(50)
            outs.append(ch.get_fields())
    for k in outs[0]:
        assert np.array_equal(outs[0][k], outs[1][k]), k


def test_restart_file_round_trip(tmp_path):
    """ek_save_restart / ek_load_restart: a context's fields through the
    reference's data_end.dat (six decimals), and the run continued from it
    matches the run continued from the same rounded fields set directly."""
    import ekpnp
    from ekpnp import io
    p = ekpnp.channel_params(32, 20, kappa_h=4.0, zeta=-1.0)
    init = ekpnp.noisy_uniform_state(32, 20, seed=3)
    path = tmp_path / "data_end.dat"
    with ekpnp.Channel(p) as ch:
        ch.set_fields(**init)
        ch.init_equilibrium()
        ch.step(50)
        ch.save_restart(path, 50.0)
        before = ch.get_fields()
    t, f = io.read_restart(path, 32, 20)
    assert t == 50.0
    for k in ("ux", "uy", "rho", "cp", "cn", "psi", "ex", "ey"):
        assert np.abs(f[k] - before[k]).max() <= 5e-7 + 1e-15, k
    outs = []
    for how in ("file", "direct"):
        with ekpnp.Channel(p) as ch:
            if how == "file":
                assert ch.load_restart(path) == 50.0
            else:
                ch.set_fields(**{k: f[k] for k in ("rho", "ux", "uy", "cp", "cn", "psi", "ex", "ey")})
            ch.init_equilibrium()
            ch.step(20)
            outs.append(ch.get_fields())
    for k in ("ux", "cp", "cn", "psi"):
        assert np.array_equal(outs[0][k], outs[1][k]), k
