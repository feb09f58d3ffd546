"""Bounded device waits run out, report, and leave the GPU usable.

Every spin-wait of this project's kernels (the tensor-core GEMMs' waits for
their MMAs, the TMA-fed LBM kernel's mbarrier ring) gives up after a bound of
SM clock cycles and reports EK_ERR_TIMEOUT to the host instead of hanging.
These tests make such waits run out without faulting anything:

  * ek_wait_selftest waits on a barrier that nothing completes, with a bound
    of a few thousand cycles: it must return EK_ERR_TIMEOUT, promptly, and
    with the arrival present EK_OK;
  * the GEMM and the TMA ring run with a bound of one cycle: each call either
    finishes (EK_OK) or reports EK_ERR_TIMEOUT, never hangs;
  * afterwards, at the default bound, the same work gives the right answer
    on the same device (the context is still usable).
"""
import time

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

EK_OK, EK_ERR_TIMEOUT = 0, 5


def test_selftest_wait_runs_out_and_reports():
    import ekpnp
    from ekpnp import lib
    ekpnp.set_device(0)
    t0 = time.time()
    assert lib().ek_wait_selftest(4000, 0) == EK_ERR_TIMEOUT
    assert time.time() - t0 < 5.0
    assert lib().ek_wait_selftest(4000, 1) == EK_OK
    assert lib().ek_wait_selftest(1, 0) == EK_ERR_TIMEOUT
    # the device still runs real work correctly
    _check_forward_usable()


def _forward(net, x):
    import ctypes
    from ekpnp import lib
    from ekpnp.mlp import N_OUT
    y = np.empty((len(x), N_OUT), dtype=np.float32)
    fp = ctypes.POINTER(ctypes.c_float)
    rc = lib().ek_mlp_forward(net._h, np.ascontiguousarray(x, dtype=np.float32).ctypes.data_as(fp), len(x),
                              y.ctypes.data_as(fp))
    return rc, y


def _check_forward_usable():
    from ekpnp.mlp import Mlp, N_IN
    x = np.random.default_rng(5).uniform(-1, 1, (256, N_IN)).astype(np.float32)
    with Mlp(batch=128, seed=3) as a, Mlp(batch=128, seed=3) as b:
        ya = a.forward(x)
        yb = b.forward(x)
    assert np.all(np.isfinite(ya)) and np.array_equal(ya, yb)


def test_gemm_wait_bound_of_one_cycle_then_default():
    from ekpnp import lib
    from ekpnp.mlp import Mlp, N_IN
    x = np.random.default_rng(6).uniform(-1, 1, (512, N_IN)).astype(np.float32)
    with Mlp(batch=128, seed=4) as ref:
        want = ref.forward(x)
    with Mlp(batch=128, seed=4) as net:
        assert lib().ek_mlp_set_wait_cycles(net._h, 1) == EK_OK
        codes = set()
        for _ in range(5):
            rc, _ = _forward(net, x)
            codes.add(rc)
        assert codes <= {EK_OK, EK_ERR_TIMEOUT}, codes
        assert lib().ek_mlp_set_wait_cycles(net._h, 1 << 31) == EK_OK
        rc, got = _forward(net, x)
        assert rc == EK_OK
        assert np.array_equal(got, want)


def test_tma_ring_wait_bound_of_one_cycle_then_default():
    import ctypes
    import ekpnp
    from ekpnp import lib
    from cases import initial_state
    p = ekpnp.channel_params(256, 40, kappa_h=4.0, zeta=-1.0, storage=ekpnp.STORE_F32)
    init = initial_state(256, 40, 21)
    steps = 40
    with ekpnp.Channel(p) as plain:
        plain.set_lbm_kernel("plain")
        plain.set_fields(**init)
        plain.init_equilibrium()
        plain.step(steps)
        want = plain.get_fields()
    with ekpnp.Channel(p) as ch:
        ch.set_lbm_kernel("tma")
        assert lib().ek_set_option(ch._h, 4, 1) == EK_OK  # EK_OPT_WAIT_CYCLES = 1
        ch.set_fields(**init)
        ch.init_equilibrium()
        assert lib().ek_step(ch._h, 5) == EK_OK  # launches are asynchronous
        assert lib().ek_sync(ch._h) in (EK_OK, EK_ERR_TIMEOUT)
        assert lib().ek_sync(ch._h) == EK_OK  # the error word was cleared
        # default bound, same context: a fresh start gives the plain kernel's bits
        assert lib().ek_set_option(ch._h, 4, ctypes.c_int64(1 << 31)) == EK_OK
        ch.set_fields(**init)
        ch.init_equilibrium()
        ch.step(steps)
        got = ch.get_fields()
    for k in ("ux", "cp", "cn", "psi"):
        assert np.array_equal(got[k], want[k]), k
