"""Regenerate ref_solves.npz: solves of the cases in solve_cases.py by the
reference's own fem_solve, built with GCC from the reference sources
(oracle/Makefile, target ``refsolver``; oracle/ref_solver/ref_run.py calls it).

Per case and build ("shipped", "fp64") the file holds the iteration count, the
residual history (L-inf before each iteration), the digest of the input blob,
and the displacements: the whole field [blocks][64][3] for the small cases,
otherwise a seeded sample of node slots with per-component sums and maxima of
the whole field.

The FP64 build sums with OpenMP reductions, so its outputs depend on the
host's thread count at round-off (1e-16 relative); the tests compare them with
tolerances.  Given case names, only those cases are solved and their entries
replaced or added in the existing file.

Run from the repository root:  python tests/golden/make_solve_golden.py [case ...]
"""
from __future__ import annotations

import os
import subprocess
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, HERE)

from solve_cases import CASES, SAMPLES, digest, inputs  # noqa: E402


def main() -> None:
    subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle"), "refsolver"], check=True)
    from oracle.ref_solver import ref_run
    names = sys.argv[1:] or list(CASES)
    path = os.path.join(HERE, "ref_solves.npz")
    out = {}
    if sys.argv[1:] and os.path.exists(path):  # keep the other cases' entries
        old = np.load(path)
        out = {k: old[k] for k in old.files if k.split("/")[0] not in names}
    for name in names:
        _, tol_shipped, tol_fp64, whole = CASES[name]
        for flavour, tol in (("shipped", tol_shipped), ("fp64", tol_fp64)):
            inp = inputs(name, tol)
            res, iterations, history = ref_run.solve(inp, flavour)
            assert res.success, (name, flavour, res.info)
            u = np.asarray(res.displacements.data)[..., :3]
            key = f"{name}/{flavour}"
            out[key + "/digest"] = np.array(digest(inp))
            out[key + "/iterations"] = np.array(iterations)
            out[key + "/history"] = np.array(history)
            if whole:
                out[key + "/u"] = u
            else:
                rng = np.random.default_rng(1234)
                flat = u.reshape(-1, 3)
                slots = np.sort(rng.choice(len(flat), size=min(SAMPLES, len(flat)), replace=False))
                out[key + "/slots"] = slots
                out[key + "/u_sample"] = flat[slots]
                out[key + "/u_sum"] = flat.sum(0)
                out[key + "/u_absmax"] = np.abs(flat).max(0)
            print(f"{key}: {iterations} iterations, |u|max {np.abs(u).max():.6g}")
    np.savez_compressed(path, **out)
    print("written", path)


if __name__ == "__main__":
    main()
