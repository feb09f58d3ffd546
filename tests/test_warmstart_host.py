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


class ScriptedBatch:
    """Stands in for ekpnp.Batch in run_to_steady: channel i's residual at its
    k-th check since its (re)start is script[i](k, restarted)."""

    def __init__(self, scripts):
        self.scripts = scripts
        self.steps = 0
        self.mask = np.ones(len(scripts), bool)
        self.since = np.zeros(len(scripts), int)      # checks since the channel's start
        self.restarts = []
        self.was_restarted = np.zeros(len(scripts), bool)

    def __len__(self):
        return len(self.scripts)

    def sync(self):
        pass

    def step(self, k):
        self.steps += k

    @property
    def active(self):
        return self.mask.copy(), int(self.mask.sum())

    def set_active(self, mask):
        self.mask = np.asarray(mask, bool).copy()

    def residual(self, check):
        out = np.zeros((len(self.scripts), 5))
        for i, f in enumerate(self.scripts):
            out[i, 4] = f(self.since[i], self.was_restarted[i])
            if self.mask[i]:
                self.since[i] += 1
        return out

    def restart(self, idx):
        self.restarts.append(list(idx))
        for i in idx:
            self.was_restarted[i] = True
            self.since[i] = 0
            self.mask[i] = True


def test_run_to_steady_restarts_judged_channels_in_place():
    """Channels whose residual rises between the judged checks, or that go
    non-finite, are restarted once, in place, and reach steady state in the
    same run; the check right after a restart is not judged; the others are
    untouched."""
    from ekpnp import warmstart as ws
    decay = lambda k, r: 10.0 ** (-2 - k)                       # converges at its 7th check
    rise = lambda k, r: 10.0 ** (-2 - k) if r else 1e-3 * (k + 1)   # rises until restarted
    nan = lambda k, r: 10.0 ** (-2 - k) if r else float("nan")      # diverges until restarted
    b = ScriptedBatch([decay, rise, nan])
    info = ws.run_to_steady(b, tol=1e-8, check=2, max_steps=200, judge=(1, 3),
                            restart=b.restart)
    assert b.restarts == [[2], [1]]                # the non-finite one at once, the rising one at check 3
    assert info["restarted"].tolist() == [False, True, True]
    assert np.all(info["steps"] > 0) and not info["diverged"].any()
    assert info["steps"][0] < info["steps"][2] < info["steps"][1]
    # without restart the judged channels are frozen and reported as rising
    b2 = ScriptedBatch([decay, rise, nan])
    info2 = ws.run_to_steady(b2, tol=1e-8, check=2, max_steps=200, judge=(1, 3))
    assert b2.restarts == [] and info2["rising"].tolist() == [False, True, True]
    assert info2["steps"][0] > 0 and info2["steps"][1] < 0 and info2["steps"][2] < 0
