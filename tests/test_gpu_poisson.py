"""The GPU Poisson solve (ek_poisson) against the numpy restatement of the
reference's fast_Poisson (test_oracle._numpy_poisson), over the shapes that
select each code path: radix-16 row FFTs with 1-4 register passes
(nx = 16 ... 8192), the direct DFT (nx not a power of two or below 16), and
the partitioned shared-memory column solve at 8, 4, 2 and 1 modes per block
plus the one-thread-per-mode fallback for very tall channels.
Bar: 1e-12 of max |psi| (FP64 throughout).  For columns taller than any
workload (ny > 2048) the bar is 2e-19 n^2: the tridiagonal route and the FFT
route are both FP64 but the y-operator's conditioning grows like n^2 (numpy
alone shows 4e-12 between them at n = 6000 and 1.7e-11 at n = 13000)."""
import numpy as np
import pytest

from conftest import rel_err
from test_oracle import _numpy_poisson

pytestmark = pytest.mark.gpu

SHAPES = [(16, 12), (32, 40), (64, 33), (128, 20), (512, 17), (1024, 9), (2048, 6), (4096, 6), (8192, 5),
          (10, 101), (24, 17), (8, 30), (96, 61),
          (16, 1500), (16, 3000), (16, 6000), (16, 12000), (16, 13000)]


@pytest.mark.parametrize("shape", SHAPES, ids=lambda s: f"{s[0]}x{s[1]}")
def test_gpu_poisson_matches_numpy(shape):
    import ekpnp
    nx, ny = shape
    p = ekpnp.channel_params(nx, ny, kappa_h=5.0, zeta=-1.5, zeta_hi=-0.7)
    rng = np.random.default_rng(nx * 7 + ny)
    x = np.arange(nx)[None, :]
    y = np.arange(ny)[:, None]
    smooth = 0.3 * np.sin(np.pi * y / (ny - 1)) * np.cos(2 * np.pi * 3 * x / nx)
    cp = 1.0 + smooth + 0.1 * rng.standard_normal((ny, nx))
    cn = 1.0 - smooth + 0.1 * rng.standard_normal((ny, nx))
    with ekpnp.Channel(p) as ch:
        ch.set_fields(cp=cp, cn=cn)
        ch.poisson()
        got = ch.get_fields(("psi", "ex", "ey"))
    phi, ex, ey = _numpy_poisson(p, cp, cn, p["zeta_lo"], p["zeta_hi"])
    tol = max(1e-12, 2e-19 * (ny - 2) ** 2)
    assert rel_err(got["psi"], phi) < tol
    assert np.abs(got["ex"] - ex).max() < tol * np.abs(phi).max()
    assert np.abs(got["ey"] - ey).max() < tol * np.abs(phi).max()


# every transform length 16 ... 8192: log2 nx = 4 ... 13 covers the radix-2,
# -4 and -8 closing passes of the row transforms
F32_SHAPES = [(16, 12), (32, 20), (64, 33), (128, 9), (256, 1500), (512, 17), (1024, 129), (2048, 35),
              (4096, 66), (8192, 18)]


@pytest.mark.parametrize("shape", F32_SHAPES, ids=lambda s: f"{s[0]}x{s[1]}")
@pytest.mark.parametrize("wall", ["uniform", "varying"])
def test_fp32_poisson_form_against_fp64(shape, wall):
    """The FP32 form (x-modes >= 1 in FP32 about a row offset, zero mode in
    FP64) against the FP64 solve of the same charges, on the second solve of
    a context (whose offsets are the first solve's row means): psi within
    1e-6 of max |psi|, E within 1e-6 of max |psi| (per lattice spacing)."""
    import ekpnp
    nx, ny = shape
    p = ekpnp.channel_params(nx, ny, kappa_h=5.0, zeta=-1.5, zeta_hi=-0.7, storage=ekpnp.STORE_F32)
    rng = np.random.default_rng(nx + 3 * ny)
    x = np.arange(nx)[None, :]
    y = np.arange(ny)[:, None]
    smooth = 0.3 * np.sin(np.pi * y / (ny - 1)) * np.cos(2 * np.pi * 3 * x / nx)
    cp = 1.0 + smooth + 0.1 * rng.standard_normal((ny, nx))
    cn = 1.0 - smooth + 0.1 * rng.standard_normal((ny, nx))
    zlo = -2.0 + 1.5 * np.sin(2 * np.pi * np.arange(nx) / max(nx // 4, 1)) if wall == "varying" else None
    out = {}
    for form in ("f64", "f32"):
        with ekpnp.Channel(p) as ch:
            if zlo is not None:
                ch.set_wall_profile(zeta_lo=zlo)
            ch.set_poisson(form)
            # a first solve of other charges: the second solve then transforms
            # about that solve's row means, not its own
            ch.set_fields(cp=cn, cn=cp)
            ch.poisson()
            ch.set_fields(cp=cp, cn=cn)
            ch.poisson()
            out[form] = ch.get_fields(("psi", "ex", "ey"))
    ref, got = out["f64"], out["f32"]
    scale = np.abs(ref["psi"]).max()
    assert np.abs(got["psi"] - ref["psi"]).max() < 1e-6 * scale
    assert np.abs(got["ex"] - ref["ex"]).max() < 1e-6 * scale
    assert np.abs(got["ey"] - ref["ey"]).max() < 1e-6 * scale
    # the wall rows are the Dirichlet values exactly
    assert np.array_equal(got["psi"][0], ref["psi"][0]) and np.array_equal(got["psi"][-1], ref["psi"][-1])


def test_fp32_poisson_form_is_refused_where_it_does_not_apply():
    import ekpnp
    for nx, ny, storage in ((24, 17, ekpnp.STORE_F32), (64, 33, ekpnp.STORE_F64), (8, 30, ekpnp.STORE_F32)):
        with ekpnp.Channel(ekpnp.channel_params(nx, ny, storage=storage)) as ch:
            with pytest.raises(ekpnp.EkError):
                ch.set_poisson("f32")
            ch.set_poisson("auto")
