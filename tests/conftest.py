import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for sub in ("ek-pnp_b200", "oracle"):
    p = os.path.join(ROOT, sub)
    if p not in sys.path:
        sys.path.insert(0, p)
GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); parity and kernel tests")


def rel_err(a, b):
    """max |a - b| / max |b| (max-norm relative to the reference's max-abs)."""
    scale = float(np.abs(b).max())
    return float(np.abs(np.asarray(a) - np.asarray(b)).max() / (scale if scale > 0 else 1.0))


@pytest.fixture(scope="session")
def oracle_mod():
    import oracle
    oracle.build()
    return oracle
