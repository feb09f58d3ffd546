"""Speed of the reference's own CUDA build against the drop-in build on one
GPU.  TEST INFRASTRUCTURE: both binaries are the reference's main.cu loop
(main.cu:190-233) with its own timing and "speed:" line (main.cu:236-261);
ekref runs the reference's kernels (LBM.cu, poisson.cu, cuFFT), ekshim runs
this project's library through the drop-in LBM.cu/poisson.cu.  Both start
from the same seeded state through read_data.

Usage (on a GPU, after oracle/ref_build.py built both binaries):
    python oracle/ref_speed.py [--pb] [case ...] > speed.json
Prints one JSON object per case: MLUPS, GPU and clock runtimes of each
binary.  The reference's MLUPS counts NSTEPS = steps - 1 steps (main.cu:244).
--pb starts from the Poisson-Boltzmann state (the library's Newton form,
the steady double layers a long run spends its time near) instead of the
case's noisy uniform state.
"""
from __future__ import annotations

import json
import os
import sys
import tempfile
import time

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
from cases import CASES, initial_state  # noqa: E402
from ref_run import run_case  # noqa: E402


def pb_state(p):
    sys.path.insert(0, os.path.join(os.path.dirname(HERE), "ek-pnp_b200"))
    import ekpnp
    with ekpnp.Channel(p) as ch:
        ch.init_poisson_boltzmann("newton")
        f = ch.get_fields()
    return f


def main(names, pb=False):
    for name in names:
        p, seed, steps = CASES[name]
        init = pb_state(p) if pb else initial_state(p["nx"], p["ny"], seed, c0=p["c0"], rho0=p["rho0"])
        out = {"case": name, "nx": p["nx"], "ny": p["ny"], "steps": steps, "arithmetic": "f64",
               "start": "poisson-boltzmann" if pb else f"noisy uniform, seed {seed}"}
        for binary in ("ekref", "ekshim"):
            with tempfile.TemporaryDirectory(prefix="ekspeed_") as tmp:
                t0 = time.perf_counter()
                _, info = run_case(name, init, tmp, timeout=1800, binary=binary)
                info["process_s"] = time.perf_counter() - t0
            out[binary] = info
        if out["ekref"].get("mlups") and out["ekshim"].get("mlups"):
            out["dropin_over_reference"] = out["ekshim"]["mlups"] / out["ekref"]["mlups"]
        print(json.dumps(out), flush=True)


if __name__ == "__main__":
    args = sys.argv[1:]
    pb = "--pb" in args
    args = [a for a in args if a != "--pb"]
    main(args or ["config1", "speed2"], pb=pb)
