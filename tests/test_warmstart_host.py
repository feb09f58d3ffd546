"""Host side of the learned warm start (no GPU): descriptor features, the
profile encoding and its decoding back to fields, and the fallback rule."""
import numpy as np


def test_features_span_the_workload_ranges():
    import ekpnp
    from ekpnp import warmstart as ws
    f = ws.features(ekpnp.batch_specs(512, seed=2))
    assert f.dtype == np.float32 and f.shape == (512, 4)
    assert f.min() >= -1.0 - 1e-6 and f.max() <= 1.0 + 1e-6
    assert np.all(f.max(axis=0) - f.min(axis=0) > 1.5)   # every descriptor varies


def pb_like(spec):
    """Debye-Hueckel-shaped profiles of a channel (for the round trip)."""
    ny, z = spec["ny"], spec["zeta"]
    y = np.arange(ny, dtype=float)
    k = spec["kappa_h"] / (ny - 1)
    h = (ny - 1) / 2
    psi = z * np.cosh(k * (y - h)) / np.cosh(k * h)
    from ekpnp import warmstart as ws, spec_params
    p = spec_params(spec, 0)
    return dict(psi=psi, cp=np.exp(-psi), cn=np.exp(psi), ux=ws.u_hs(p) * (1 - psi / z))


def test_encode_decode_round_trip():
    from ekpnp import warmstart as ws
    for spec in (dict(nx=32, ny=40, kappa_h=4.0, zeta=-1.0, ex=1e-4, diff=0.05, eps=0.01),
                 dict(nx=16, ny=511, kappa_h=50.0, zeta=-4.0, ex=1e-3, diff=0.05, eps=0.01),
                 dict(nx=64, ny=97, kappa_h=12.0, zeta=-2.5, ex=3e-5, diff=0.05, eps=0.01)):
        prof = pb_like(spec)
        vec = ws.encode(spec, prof)
        assert vec.shape == (512,) and np.all(np.isfinite(vec))
        f = ws.decode(spec, vec)
        assert f["psi"].shape == (spec["ny"], spec["nx"])
        for k in ("psi", "cp", "cn", "ux"):
            err = np.abs(f[k][:, 0] - prof[k]).max() / np.abs(prof[k]).max()
            assert err < 3e-2, (spec["ny"], k, err)
        assert f["psi"][0, 0] == spec["zeta"] and f["psi"][-1, 0] == spec["zeta"]
        assert np.all(f["ux"][0] == 0) and np.all(f["ux"][-1] == 0)


def test_fallback_rule():
    from ekpnp import warmstart as ws
    hist = np.array([[1e-3, 1e-3, 1e-3, 1e-3],
                     [5e-4, 2e-3, 1e-3, np.nan],
                     [2e-4, 4e-3, 9e-4, np.nan],
                     [1e-4, 8e-3, 1.1e-3, np.nan]])
    bad = ws.rising_channels(hist, 1, 3)
    assert bad.tolist() == [False, True, True, True]
    assert ws.rising_channels(hist[:2], 1, 3).tolist() == [False, False, False, True]


def test_pb_column_solves_the_discrete_equation():
    import ekpnp
    from ekpnp import spec_params, warmstart as ws
    for s in ekpnp.batch_specs(16, seed=7):
        psi = ws.pb_column(s)
        p = spec_params(s, 0)
        g = p["f_charge"] * p["c0"] / p["eps"]
        lap = psi[:-2] - 2 * psi[1:-1] + psi[2:]
        src = g * (np.exp(-psi[1:-1]) - np.exp(psi[1:-1]))
        # rounding of the second difference of O(|zeta|) values bounds the residual
        assert np.abs(lap + src).max() <= 1e-14 * max(abs(s["zeta"]), 1.0) * 8
        assert psi[0] == psi[-1] == s["zeta"] and np.all(np.diff(psi[: len(psi) // 2]) >= 0)


def test_xreduced_start_needs_widths_that_tile():
    """The x-reduced run tiles 16-column states: every nx must be a multiple
    of the narrow width (checked before any device work)."""
    import pytest
    from ekpnp import warmstart as ws
    specs = [dict(nx=64, ny=32, kappa_h=4.0, zeta=-1.0, ex=1e-4, diff=0.05),
             dict(nx=40, ny=32, kappa_h=4.0, zeta=-1.0, ex=1e-4, diff=0.05)]
    with pytest.raises(ValueError):
        ws.xreduced_start_run(specs, start="cold")
    with pytest.raises(ValueError):
        ws.xreduced_start_run(specs[:1], start="nowhere")
