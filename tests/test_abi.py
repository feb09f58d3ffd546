"""C ABI checks that need no GPU: the library loads, exports every entry point
declared in include/ekpnp.h, its parameter struct matches the header's
layout, and invalid parameters are rejected on the host."""
import ctypes
import os
import re
import subprocess
import tempfile

import pytest

from conftest import ROOT

HEADER = os.path.join(ROOT, "include", "ekpnp.h")


def declared_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(ek_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    import ekpnp
    h = ekpnp.lib()
    names = declared_functions()
    assert len(names) >= 20
    missing = [n for n in names if not hasattr(h, n)]
    assert not missing, missing


def test_binding_declares_every_header_function():
    from ekpnp import _lib
    assert set(declared_functions()) == set(_lib.exported_symbols())


def test_params_layout_matches_header():
    """sizeof/offsetof of ek_params from a C compile of the header == ctypes."""
    from ekpnp import EkParams
    fields = [n for n, _ in EkParams._fields_]
    prog = "#include <stdio.h>\n#include <stddef.h>\n#include \"ekpnp.h\"\nint main(void){\n"
    prog += 'printf("%zu\\n", sizeof(ek_params));\n'
    for f in fields:
        prog += f'printf("%zu\\n", offsetof(ek_params, {f}));\n'
    prog += "return 0;}\n"
    with tempfile.TemporaryDirectory() as d:
        src = os.path.join(d, "t.c")
        exe = os.path.join(d, "t")
        open(src, "w").write(prog)
        subprocess.check_call(["gcc", "-I", os.path.join(ROOT, "include"), src, "-o", exe])
        out = [int(v) for v in subprocess.check_output([exe]).split()]
    assert out[0] == ctypes.sizeof(EkParams)
    assert out[1:] == [getattr(EkParams, f).offset for f in fields]


def _create_status(**over):
    import ekpnp
    p = ekpnp.channel_params(16, 12)
    p.update(over)
    h = ctypes.c_void_p()
    params = ekpnp.EkParams.from_dict(p)
    return ekpnp.lib().ek_create(ctypes.byref(params), ctypes.byref(h))


@pytest.mark.parametrize("over", [
    dict(nx=1), dict(ny=3), dict(nu=-1.0), dict(nu=float("nan")), dict(cs2=0.0), dict(eps=0.0),
    dict(flags=1 << 10), dict(storage=7), dict(zeta_lo=float("inf")), dict(diff_p=0.0),
])
def test_invalid_parameters_rejected_on_host(over):
    assert _create_status(**over) == 1  # EK_ERR_INVALID, before any CUDA call


def test_oversized_channel_unsupported():
    assert _create_status(nx=16384) == 6
    assert _create_status(nx=3000) == 6


def test_status_strings():
    import ekpnp
    for code in range(8):
        assert ekpnp.lib().ek_status_string(code)
    assert ekpnp.lib().ek_version() >= 100


def test_params_mapping_matches_oracle_cases():
    """The product's lattice-unit mapping equals the one the parity cases use."""
    import ekpnp
    from cases import lattice_params
    a = ekpnp.channel_params(256, 128, kappa_h=8.0, zeta=-2.0, ex=1e-4, diff=0.05)
    b = lattice_params(256, 128, kappa_h=8.0, zeta=-2.0, ex=1e-4, diff=0.05)
    assert a == b


def test_state_copy_entry_points_reject_null_handles_on_host():
    """ek_tile_x and ek_batch_resync check their handles before any CUDA call."""
    import ekpnp
    lib = ekpnp.lib()
    assert lib.ek_tile_x(None, None) == 1  # EK_ERR_INVALID
    assert lib.ek_batch_resync(None) == 1
