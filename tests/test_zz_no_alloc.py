"""ek_poisson_noalloc against the allocating Poisson solve (ek_poisson).

ek_poisson_noalloc exists for callers that cannot allocate device memory in
their time loop -- the reference allocates four buffers in every Poisson call;
a host program that owns all device memory through its own pool cannot.  Its
scratch lives in device arrays built into the library.  This test calls it
through the C ABI twice in a row, with different channels and charges, and
checks psi, Ex and Ey against the allocating entry point at the tolerance of
the other parity tests (1e-12 of the field's max-abs).  The second call
checks that what the first call left in the shared scratch does not leak into
the next result.
"""
import ctypes

import numpy as np
import pytest

from conftest import rel_err

pytestmark = pytest.mark.gpu


def allocating_solve(p, cp, cn):
    import ekpnp
    with ekpnp.Channel(p) as ch:
        ch.set_fields(cp=cp, cn=cn)
        ch.poisson()
        return ch.get_fields(("psi", "ex", "ey"))


def noalloc_solve(p, cp, cn):
    import torch
    import ekpnp
    from ekpnp import EkParams, lib
    dev = torch.device("cuda", 0)
    tcp = torch.from_numpy(cp).to(dev)
    tcn = torch.from_numpy(cn).to(dev)
    out = {k: torch.full_like(tcp, float("nan")) for k in ("psi", "ex", "ey")}
    torch.cuda.synchronize()
    params = EkParams.from_dict(p)
    rc = lib().ek_poisson_noalloc(ctypes.byref(params), ctypes.c_void_p(tcp.data_ptr()),
                                  ctypes.c_void_p(tcn.data_ptr()), ctypes.c_void_p(out["psi"].data_ptr()),
                                  ctypes.c_void_p(out["ex"].data_ptr()), ctypes.c_void_p(out["ey"].data_ptr()),
                                  None)
    ekpnp._lib.check(rc)
    torch.cuda.synchronize()
    return {k: v.cpu().numpy() for k, v in out.items()}


def charges(nx, ny, seed, amp):
    rng = np.random.default_rng(seed)
    x = np.arange(nx)[None, :]
    y = np.arange(ny)[:, None]
    base = amp * np.sin(np.pi * y / (ny - 1)) * (1.0 + 0.3 * np.cos(2 * np.pi * x / nx))
    cp = 1.0 + base + 1e-3 * rng.standard_normal((ny, nx))
    cn = 1.0 - base + 1e-3 * rng.standard_normal((ny, nx))
    return cp, cn


def test_noalloc_matches_allocating_solve_twice():
    import ekpnp
    ekpnp.set_device(0)
    calls = [
        (ekpnp.channel_params(256, 128, kappa_h=8.0, zeta=-2.0), charges(256, 128, 1, 0.4)),
        (ekpnp.channel_params(96, 61, kappa_h=3.0, zeta=-1.0, zeta_hi=-0.5), charges(96, 61, 2, 0.1)),
    ]
    _check_calls(calls)


@pytest.mark.parametrize("nx,ny", [(8, 20), (1024, 512), (8192, 64)])
def test_noalloc_scratch_layout_edges(nx, ny):
    """The shapes where the no-allocation scratch differs most from the
    allocating path's padded layout: a power-of-two row shorter than 16 (the
    small-row transform), a channel exactly at the 524,288-node limit, and
    8192-long rows (the widest row transform).  Two calls each."""
    import ekpnp
    ekpnp.set_device(0)
    calls = [(ekpnp.channel_params(nx, ny, kappa_h=4.0, zeta=-1.5), charges(nx, ny, 3, 0.2)),
             (ekpnp.channel_params(nx, ny, kappa_h=2.0, zeta=-0.5, zeta_hi=-1.0), charges(nx, ny, 4, 0.05))]
    _check_calls(calls)


def _check_calls(calls):
    """psi within 1e-12 of its max-abs.  E is a central difference of psi
    over one spacing, so its rounding is bounded by psi's, not by E's own
    size (a channel whose charge barely varies along x has an Ex far below
    psi): Ex and Ey within 1e-12 of max |psi| / spacing."""
    for p, (cp, cn) in calls:
        want = allocating_solve(p, cp, cn)
        got = noalloc_solve(p, cp, cn)
        for k in ("psi", "ex", "ey"):
            assert np.all(np.isfinite(got[k])), k
        assert rel_err(got["psi"], want["psi"]) <= 1e-12, rel_err(got["psi"], want["psi"])
        scale = np.abs(want["psi"]).max()
        for k, h in (("ex", p["dx"]), ("ey", p["dy"])):
            err = np.abs(got[k] - want[k]).max()
            assert err <= 1e-12 * scale / h, (k, err, scale)


def test_noalloc_rejects_oversized_channel():
    """2048 x 512 nodes is above the 524,288-node limit.  The buffers are real
    and full-size, so the call is safe whatever it does; it must return
    EK_ERR_TOO_LARGE and leave psi untouched."""
    import torch
    import ekpnp
    from ekpnp import EkParams, lib
    p = EkParams.from_dict(ekpnp.channel_params(2048, 512))
    buf = [torch.zeros((512, 2048), dtype=torch.float64, device="cuda:0") for _ in range(3)]
    torch.cuda.synchronize()
    rc = lib().ek_poisson_noalloc(ctypes.byref(p), *[ctypes.c_void_p(b.data_ptr()) for b in buf],
                                  None, None, None)
    torch.cuda.synchronize()
    assert rc == 7  # EK_ERR_TOO_LARGE
    assert float(buf[2].abs().max()) == 0.0


def test_noalloc_rejects_tall_narrow_channel():
    """4 x 70000 has fewer nodes than the limit, but more rows than a launch
    grid can index: the call must refuse it before queueing any work."""
    import torch
    import ekpnp
    from ekpnp import EkParams, lib
    p = EkParams.from_dict(ekpnp.channel_params(4, 70000))
    buf = [torch.zeros((70000, 4), dtype=torch.float64, device="cuda:0") for _ in range(3)]
    torch.cuda.synchronize()
    rc = lib().ek_poisson_noalloc(ctypes.byref(p), *[ctypes.c_void_p(b.data_ptr()) for b in buf],
                                  None, None, None)
    torch.cuda.synchronize()
    assert rc == 7  # EK_ERR_TOO_LARGE
    assert float(buf[2].abs().max()) == 0.0
