"""Run a patched reference binary (built by oracle/ref_build.py).  TEST
INFRASTRUCTURE; needs a GPU.

The initial state goes in through the reference's own restart reader: a
data_end.dat with the columns that read_data parses (LBM.cu:1350-1391):
    time ux uy rho c+ phi Ex Ey c-
one line per node in y-major order, written with %.17g so fscanf("%lf") gives
the exact doubles back.  After the loop the patched main.cu dumps every field
as raw doubles through save_scalar (LBM.cu:1062-1098).
"""
from __future__ import annotations

import glob
import os
import re
import subprocess
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
from cases import CASES, FIELDS  # noqa: E402


def write_restart(path, f):
    ny, nx = f["cp"].shape
    cols = np.stack([np.zeros(ny * nx), f["ux"].ravel(), f["uy"].ravel(), f["rho"].ravel(),
                     f["cp"].ravel(), f["psi"].ravel(), f["ex"].ravel(), f["ey"].ravel(),
                     f["cn"].ravel()], axis=1)
    np.savetxt(path, cols, fmt="%.17g")


def run_case(name, init, workdir, timeout=900, binary="ekref"):
    """Run case `name` from the fields `init`; return (fields, info).
    binary "ekref" is the patched reference build, "ekshim" the reference's
    main.cu over this project's drop-in LBM.cu/poisson.cu and libekpnp."""
    p, _, _ = CASES[name]
    exe = os.path.join(HERE, "_ref", name, binary)
    if not os.path.exists(exe):
        raise FileNotFoundError(exe + " (build it with oracle/ref_build.py)")
    os.makedirs(workdir, exist_ok=True)
    for old in glob.glob(os.path.join(workdir, "*.bin")):
        os.remove(old)
    write_restart(os.path.join(workdir, "data_end.dat"), init)
    r = subprocess.run([exe], cwd=workdir, capture_output=True, text=True, timeout=timeout,
                       stdin=subprocess.DEVNULL)
    if r.returncode != 0:
        raise RuntimeError(f"reference run failed ({r.returncode}):\n{r.stdout[-2000:]}{r.stderr[-2000:]}")
    out = {}
    for n in FIELDS:
        hits = sorted(glob.glob(os.path.join(workdir, n + "[0-9]*.bin")))
        if len(hits) != 1:
            raise RuntimeError(f"expected one dump for {n}, found {hits}")
        out[n] = np.fromfile(hits[0], dtype=np.float64).reshape(p["ny"], p["nx"])
    info = {}
    for key, pat in (("gpu_runtime_s", r"gpu runtime:\s*([0-9.eE+-]+)"),
                     ("clock_runtime_s", r"clock runtime:\s*([0-9.eE+-]+)"),
                     ("mlups", r"speed:\s*([0-9.eE+-]+)")):
        m = re.search(pat, r.stdout)
        if m:
            info[key] = float(m.group(1))
    return out, info
