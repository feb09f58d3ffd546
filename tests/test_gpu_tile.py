"""ek_tile_x / ek_batch_resync: a narrow channel's state repeated along x
into a wider channel of the same height, and a batch adopting the tiled
states of its channels.

With walls uniform along x the coupled step is translation invariant, so a
wide channel holding k copies of a narrow channel's state evolves as the
narrow one does.  The copy itself is exact; after stepping, the two differ
only through the row sums of the Poisson zero mode (a sum of 16 equal
values against one of 16 k), i.e. by rounding.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

NAMES = ("rho", "ux", "uy", "cp", "cn", "psi")
# relative to each field's max-abs, after 41 steps from the tiled state
TOL = {0: 1e-12, 1: 1e-6, 2: 1e-3}


def params(nx, ny, storage, **kw):
    import ekpnp
    return ekpnp.channel_params(nx, ny, kappa_h=6.0, zeta=-1.5, ex=2e-4, storage=storage, **kw)


def relaxed_narrow(storage, ny=33, steps=60):
    import ekpnp
    ch = ekpnp.Channel(params(16, ny, storage))
    ch.init_poisson_boltzmann("newton")
    ch.init_equilibrium()
    ch.step(steps)
    return ch


@pytest.mark.parametrize("storage", [0, 1, 2], ids=["f64", "f32", "f16"])
def test_tiled_state_is_an_exact_copy_and_evolves_as_the_narrow_one(storage):
    import ekpnp
    with relaxed_narrow(storage) as narrow, ekpnp.Channel(params(64, 33, storage)) as wide:
        wide.tile_x(narrow)
        a, b = narrow.get_fields(NAMES), wide.get_fields(NAMES)
        for k in NAMES:
            assert np.array_equal(b[k], np.tile(a[k], (1, 4))), k
        narrow.step(41)
        wide.step(41)
        a, b = narrow.get_fields(NAMES), wide.get_fields(NAMES)
        for k in NAMES:
            scale = max(np.abs(a[k]).max(), 1e-300)
            err = np.abs(b[k] - np.tile(a[k], (1, 4))).max() / scale
            assert err <= TOL[storage], (k, err)


def test_tile_x_refuses_mismatched_channels():
    import ekpnp
    with relaxed_narrow(1) as narrow:
        for bad in (params(40, 33, 1), params(64, 34, 1), params(64, 33, 0)):
            with ekpnp.Channel(bad) as wide:
                with pytest.raises(ekpnp.EkError):
                    wide.tile_x(narrow)
        with ekpnp.Channel(params(16, 33, 1)) as fresh, ekpnp.Channel(params(32, 33, 1)) as wide:
            with pytest.raises(ekpnp.EkError):  # the source holds no populations yet
                wide.tile_x(fresh)


def test_batch_steps_on_from_tiled_states():
    """A batch of wide channels tiled from a batch of 16-column channels and
    resynchronised steps as the narrow batch does (graph-captured cycles)."""
    import ekpnp
    from ekpnp.warmstart import physics_start
    specs = [dict(nx=64, ny=40, kappa_h=4.0, zeta=-1.0, ex=1e-4, diff=0.05),
             dict(nx=128, ny=57, kappa_h=12.0, zeta=-2.5, ex=3e-4, diff=0.03),
             dict(nx=32, ny=33, kappa_h=2.0, zeta=-0.7, ex=5e-5, diff=0.08)]
    narrow_specs = [dict(s, nx=16) for s in specs]
    with ekpnp.Batch([ekpnp.spec_params(s, ekpnp.STORE_F32) for s in narrow_specs]) as nb, \
            ekpnp.Batch([ekpnp.spec_params(s, ekpnp.STORE_F32) for s in specs]) as wb:
        physics_start(nb, narrow_specs)
        nb.set_cycle(10)
        nb.init_equilibrium()
        nb.step(70)
        nb.sync()
        wb.set_cycle(10)
        wb.init_equilibrium()
        for w, n in zip(wb, nb):
            w.tile_x(n)
        wb.resync()
        nb.step(40)
        wb.step(40)
        for s, w, n in zip(specs, wb, nb):
            a, b = n.get_fields(NAMES), w.get_fields(NAMES)
            for k in NAMES:
                scale = max(np.abs(a[k]).max(), 1e-300)
                err = np.abs(b[k] - np.tile(a[k], (1, s["nx"] // 16))).max() / scale
                assert err <= TOL[1], (s, k, err)


def test_resync_refuses_channels_at_different_parities():
    import ekpnp
    ps = [ekpnp.spec_params(dict(nx=32, ny=20, kappa_h=4.0, zeta=-1.0, ex=1e-4, diff=0.05), ekpnp.STORE_F32)] * 2
    with ekpnp.Batch(ps) as b:
        b.init_equilibrium()
        b.step(2)
        b[1].step(1)
        with pytest.raises(ekpnp.EkError):
            b.resync()


def test_xreduced_start_passes_the_full_width_check_at_once():
    """Relaxed on 16 columns and tiled, each channel meets the residual test
    at the first full-width check."""
    from ekpnp import warmstart as ws
    from ekpnp.params import BATCH_EPS, BATCH_REST_QUIRK
    specs = [dict(nx=64, ny=24, kappa_h=3.0, zeta=-1.0, ex=1e-4, diff=0.08),
             dict(nx=32, ny=30, kappa_h=6.0, zeta=-2.0, ex=3e-4, diff=0.06),
             dict(nx=128, ny=20, kappa_h=2.0, zeta=-0.8, ex=5e-5, diff=0.1)]
    specs = [dict(s, eps=BATCH_EPS, rest_quirk=BATCH_REST_QUIRK) for s in specs]
    r = ws.xreduced_start_run(specs, start="cold", tol=1e-7, check=500, max_steps=60_000, cycle=100)
    assert np.all(r["narrow_steps"] > 0), r["narrow_steps"]
    assert np.all(r["full_steps"] == 500), r["full_steps"]
    assert np.array_equal(r["steps"], r["narrow_steps"] + 500)
    assert not np.any(r["diverged"])
