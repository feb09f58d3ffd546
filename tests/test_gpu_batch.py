"""Batched channels (ek_batch_*): many channels of uneven size and physics in
lockstep, one persistent LBM kernel over a tile work-list plus three batched
Poisson passes per step, cycles replayed from a CUDA graph.

Per channel a batch must give exactly the bits of ek_step with the same
re-base interval: the node update, Poisson bodies and re-basing formula are
shared, so any difference is a scheduling or indexing bug (a tile that
missed rows, a channel's constants staged from the wrong entry, a graph
replayed at the wrong parity).
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

NAMES = ("rho", "ux", "uy", "cp", "cn", "psi")

# uneven sizes: narrow channels share tiles across rows, odd ny leaves a
# partial last tile, and the physics differs per channel
SPECS = [
    dict(nx=16, ny=33, kappa_h=4.0, zeta=-1.0, ex=1e-4, diff=0.05),
    dict(nx=64, ny=47, kappa_h=8.0, zeta=-2.0, ex=3e-4, diff=0.03),
    dict(nx=128, ny=64, kappa_h=16.0, zeta=-1.5, ex=5e-5, diff=0.08),
    dict(nx=256, ny=37, kappa_h=2.0, zeta=-0.5, ex=1e-3, diff=0.1),
    dict(nx=512, ny=130, kappa_h=24.0, zeta=-3.0, ex=2e-5, diff=0.02),
    dict(nx=32, ny=9, kappa_h=1.0, zeta=-2.5, ex=1e-5, diff=0.06),
]


def params(storage):
    import ekpnp
    return [ekpnp.spec_params(s, storage) for s in SPECS]


def inits():
    import ekpnp
    return [ekpnp.noisy_uniform_state(s["nx"], s["ny"], seed=10 + i) for i, s in enumerate(SPECS)]


def single(p, init, steps, cycle):
    import ekpnp
    with ekpnp.Channel(p) as ch:
        ch.set_fields(**init)
        ch.init_equilibrium()
        ch.set_rebase_interval(cycle)
        ch.step(steps)
        return ch.get_fields(NAMES)


@pytest.fixture(scope="module", params=["f32", "f16"])
def storage(request):
    import ekpnp
    return {"f32": ekpnp.STORE_F32, "f16": ekpnp.STORE_F16}[request.param]


@pytest.fixture(scope="module")
def singles(storage):
    ps, ins = params(storage), inits()
    return {steps: [single(p, i, steps, 10) for p, i in zip(ps, ins)] for steps in (37,)}


@pytest.mark.parametrize("shape", range(6))
@pytest.mark.parametrize("graph", [True, False])
def test_batch_bitwise_equals_single_channels(storage, singles, shape, graph):
    import ekpnp
    with ekpnp.Batch(params(storage)) as b:
        for ch, init in zip(b, inits()):
            ch.set_fields(**init)
        b.set_cycle(10, rebase=True, graph=graph)
        b.shape = shape
        b.init_equilibrium()
        b.step(5)       # first step + partial cycle
        b.step(30)      # cycle-aligned run: graphs of 10 steps where allowed
        b.step(2)
        b.sync()
        assert b.steps == 37
        for i, ch in enumerate(b):
            got = ch.get_fields(NAMES)
            ref = singles[37][i]
            for k in NAMES:
                assert np.array_equal(got[k], ref[k]), (i, k, float(np.abs(got[k] - ref[k]).max()))


def test_autotune_keeps_the_bits():
    import ekpnp
    steps = len(ekpnp.Batch.shapes()) * (4 + 2) + 11  # the autotuner runs steps + 2 per shape
    ref = [single(p, i, steps, 10) for p, i in zip(params(ekpnp.STORE_F32), inits())]
    with ekpnp.Batch(params(ekpnp.STORE_F32)) as b:
        for ch, init in zip(b, inits()):
            ch.set_fields(**init)
        b.set_cycle(10)
        b.init_equilibrium()
        w, ms = b.autotune(4)
        assert w in range(len(ekpnp.Batch.shapes())) and b.shape == w
        assert len(ms) == len(ekpnp.Batch.shapes()) and all(v > 0 for v in ms)
        b.step(11)
        for i, ch in enumerate(b):
            got = ch.get_fields(NAMES)
            for k in NAMES:
                assert np.array_equal(got[k], ref[i][k]), (i, k)


def test_batch_residual_equals_channel_residual():
    import ekpnp
    ps, ins = params(ekpnp.STORE_F32), inits()
    with ekpnp.Batch(ps) as b:
        for ch, init in zip(b, inits()):
            ch.set_fields(**init)
        b.set_cycle(10)
        b.init_equilibrium()
        b.step(20)
        first = b.residual(10)
        assert np.all(np.isinf(first))
        b.step(20)
        r = b.residual(20)
    for i, (p, init) in enumerate(zip(ps, ins)):
        with ekpnp.Channel(p) as ch:
            ch.set_fields(**init)
            ch.init_equilibrium()
            ch.set_rebase_interval(10)
            ch.step(20)
            ch.residual(10)
            ch.step(20)
            want = ch.residual(20)
        assert np.array_equal(r[i], want), (i, r[i], want)


def test_launch_count_is_independent_of_channel_count():
    import ekpnp
    counts = []
    for n in (1, len(SPECS)):
        with ekpnp.Batch(params(ekpnp.STORE_F32)[:n]) as b:
            b.set_cycle(10)
            b.init_equilibrium()
            before = b.launches
            b.step(40)
            b.sync()
            counts.append(b.launches - before)
    # 4 launches per step (the column pass carries the FP64 zero modes in its
    # own blocks) + 3 re-basing launches per cycle, whatever the batch size
    assert counts[0] == counts[1] == 40 * 4 + 4 * 3


def test_stepping_a_channel_alone_is_refused():
    import ekpnp
    with ekpnp.Batch(params(ekpnp.STORE_F32)[:2]) as b:
        b.init_equilibrium()
        b.step(2)
        b[1].step(1)
        with pytest.raises(ekpnp.EkError):
            b.step(1)
        b.init_equilibrium()  # re-synchronises
        b.step(2)


def test_mixed_explicit_e_start_runs():
    """One channel carries E from the reference Poisson-Boltzmann start, the
    others get E of their psi written before the first step."""
    import ekpnp
    ps = params(ekpnp.STORE_F32)[:3]
    with ekpnp.Batch(ps) as b:
        b[0].init_poisson_boltzmann("reference", iterations=50, omega=0.05)
        b[1].init_poisson_boltzmann("newton")
        b[2].set_fields(**inits()[2])
        b.init_equilibrium()
        b.step(50)
        for ch in b:
            f = ch.get_fields(NAMES)
            assert all(np.all(np.isfinite(f[k])) for k in NAMES)


def test_unsupported_channels_are_rejected():
    import ekpnp
    p = ekpnp.spec_params(SPECS[0], ekpnp.STORE_F32)
    for bad in (dict(nx=48), dict(nx=8192), dict(storage=ekpnp.STORE_F64)):
        with pytest.raises(ekpnp.EkError):
            ekpnp.Batch([dict(p, **bad)])
    with pytest.raises(ekpnp.EkError):
        ekpnp.Batch([p, dict(p, storage=ekpnp.STORE_F16)])


def test_frozen_channels_keep_their_state_and_others_keep_the_bits():
    import ekpnp
    ps, ins = params(ekpnp.STORE_F32), inits()
    with ekpnp.Batch(ps) as b:
        for ch, init in zip(b, ins):
            ch.set_fields(**init)
        b.set_cycle(10)
        b.init_equilibrium()
        b.step(10)
        mask = np.ones(len(ps), bool)
        mask[[1, 4]] = False
        b.set_active(mask)
        active, nodes = b.active
        assert active.tolist() == mask.tolist()
        assert nodes == sum(s["nx"] * s["ny"] for s, m in zip(SPECS, mask) if m)
        frozen = {i: b[i].get_fields(NAMES) for i in (1, 4)}
        b.step(27)
        with pytest.raises(ekpnp.EkError):   # 27 steps later the parity differs
            b.set_active(np.ones(len(ps), bool))
        for i in range(len(ps)):
            got = b[i].get_fields(NAMES)
            ref = frozen[i] if i in frozen else single(ps[i], ins[i], 37, 10)
            for k in NAMES:
                assert np.array_equal(got[k], ref[k]), (i, k)
        b.step(1)
        b.set_active(np.ones(len(ps), bool))  # even now: rejoin allowed
        b.step(2)
        assert all(np.all(np.isfinite(ch.get_fields(("ux",))["ux"])) for ch in b)


@pytest.mark.parametrize("storage", ["f32", "f16"])
def test_restart_in_place_keeps_the_other_channels_bits(storage):
    """ek_batch_restart gives the masked channels a new start in place: the
    other channels keep exactly the bits of a batch without the restart, the
    restarted one holds its new fields right after it, steps on finite with
    its step count started over, and can be restarted again."""
    import ekpnp
    st = {"f32": ekpnp.STORE_F32, "f16": ekpnp.STORE_F16}[storage]
    ps, ins = params(st), inits()
    j = 2
    new = ekpnp.noisy_uniform_state(SPECS[j]["nx"], SPECS[j]["ny"], seed=99)

    def run(restart):
        with ekpnp.Batch(ps) as b:
            for ch, init in zip(b, ins):
                ch.set_fields(**init)
            b.set_cycle(10)
            b.init_equilibrium()
            b.step(20)
            if restart:
                b[j].set_fields(**new)
                mask = np.zeros(len(b), bool)
                mask[j] = True
                b.restart(mask)
                assert np.array_equal(b[j].get_fields(("cp",))["cp"], new["cp"])
            b.step(24)
            out = [ch.get_fields(NAMES) for ch in b]
            if restart:
                assert b[j].steps == 24 and b[0].steps == 44
                b[j].set_fields(**new)
                b.restart(mask)
                b.step(4)
                assert all(np.isfinite(v).all() for v in b[j].get_fields(NAMES).values())
            return out

    plain, restarted = run(False), run(True)
    for i in range(len(ps)):
        for k in NAMES:
            if i == j:
                assert np.isfinite(restarted[i][k]).all(), k
            else:
                assert np.array_equal(plain[i][k], restarted[i][k]), (i, k)
