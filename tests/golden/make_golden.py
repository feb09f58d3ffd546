"""Generate the golden fixtures of tests/golden/ by running the patched
reference build (oracle/ref_build.py) on a GPU.

    python tests/golden/make_golden.py [--out DIR] [case ...]

For each small case of oracle/cases.py it writes <case>.npz holding the case's
parameters, seed and step count, and the reference's output fields after the
run (rho, ux, uy, c+, c-, psi, Ex, Ey as raw doubles from save_scalar).  Each
case is run twice; the fixture records whether the two runs were bitwise
equal (the reference reads row 1's rest populations while another block may
be rewriting them, LBM.cu:403-405 vs 775-777).
"""
from __future__ import annotations

import argparse
import json
import os
import sys
import tempfile

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
from cases import CASES, FIELDS, initial_state  # noqa: E402
from ref_run import run_case  # noqa: E402

SMALL = [n for n in CASES if n.startswith("g")]


def make(name, out_dir):
    p, seed, steps = CASES[name]
    init = initial_state(p["nx"], p["ny"], seed, c0=p["c0"], rho0=p["rho0"])
    with tempfile.TemporaryDirectory(prefix="ekgold_") as tmp:
        a, info = run_case(name, init, os.path.join(tmp, "a"))
        b, _ = run_case(name, init, os.path.join(tmp, "b"))
    same = all(np.array_equal(a[k], b[k], equal_nan=True) for k in FIELDS)
    path = os.path.join(out_dir, name + ".npz")
    np.savez_compressed(path, params=json.dumps(p), seed=seed, steps=steps, deterministic=same,
                        **{k: a[k] for k in FIELDS})
    return path, same, info


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=os.path.dirname(os.path.abspath(__file__)))
    ap.add_argument("cases", nargs="*", default=SMALL)
    args = ap.parse_args()
    os.makedirs(args.out, exist_ok=True)
    for name in args.cases:
        path, same, info = make(name, args.out)
        print(f"{name}: {path} deterministic={same} {info}")


if __name__ == "__main__":
    main()
