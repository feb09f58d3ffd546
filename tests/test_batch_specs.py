"""Host side of the batched workload (no GPU): the channel draws are
deterministic, inside their ranges, and map to valid batch channels."""
import numpy as np


def test_batch_specs_deterministic_and_in_range():
    import ekpnp
    a, b = ekpnp.batch_specs(512, seed=2), ekpnp.batch_specs(512, seed=2)
    assert a == b and len(a) == 512
    assert a != ekpnp.batch_specs(512, seed=3)
    assert {s["nx"] for s in a} == set(ekpnp.BATCH_NX)
    ny = np.array([s["ny"] for s in a])
    assert ny.min() >= 32 and ny.max() <= 512
    kh = np.array([s["kappa_h"] for s in a])
    assert kh.min() >= 1.0 and kh.max() <= 50.0
    z = np.array([s["zeta"] for s in a])
    assert z.min() >= -4.0 and z.max() <= -0.5
    ex = np.array([s["ex"] for s in a])
    assert ex.min() >= 1e-5 and ex.max() <= 1e-3
    d = np.array([s["diff"] for s in a])
    assert d.min() >= 0.02 and d.max() <= 0.1


def test_spec_params_are_batchable():
    import ekpnp
    for s in ekpnp.batch_specs(64, seed=2):
        p = ekpnp.spec_params(s, ekpnp.STORE_F32)
        assert p["nx"] & (p["nx"] - 1) == 0 and 16 <= p["nx"] <= 4096
        assert p["storage"] == ekpnp.STORE_F32 and not p["flags"] & ekpnp.FLAG_EXPLICIT_E
        assert not p["flags"] & ekpnp.FLAG_REST_QUIRK and p["flags"] & ekpnp.FLAG_FORCE
        assert p["eps"] == s["eps"] == ekpnp.params.BATCH_EPS
        assert abs(p["f_charge"] - p["eps"] * (s["kappa_h"] / (s["ny"] - 1)) ** 2 / 2) < 1e-15
        assert p["mob_p"] == s["diff"] and p["mob_n"] == -s["diff"]


def test_batch_entry_points_exported():
    import ekpnp
    from ekpnp import _lib
    names = [n for n in _lib.exported_symbols() if n.startswith("ek_batch_")]
    assert len(names) >= 14
    for n in names:
        assert hasattr(ekpnp.lib(), n)
