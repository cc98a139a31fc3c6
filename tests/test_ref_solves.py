"""The oracle against the reference's own solver (CPU, no GPU needed).

tests/golden/ref_solves.npz holds solves of the cases in
tests/golden/solve_cases.py by the reference's fem_solve, compiled here from
the reference sources (tests/golden/make_solve_golden.py).  The oracle's FP64
mode must reproduce the reference's FP64 build to round-off -- iteration count,
residual history and displacements -- and its reference-rounding mode the
shipped build's iteration count and displacements; that pins the oracle (and,
through the GPU parity tests, the CUDA path) to the reference's arithmetic:
K u, the coloured Gauss-Seidel smoother with its boundary band, the transfers,
the Galerkin operators, the bottom solve and the PCG.
"""
import os
import sys

import numpy as np
import pytest

from oracle.oracle import MODE_FP64, MODE_REF, Oracle

GOLD = os.path.join(os.path.dirname(__file__), "golden")
sys.path.insert(0, GOLD)
from solve_cases import CASES, digest, inputs  # noqa: E402

REF = np.load(os.path.join(GOLD, "ref_solves.npz"))
# the oracle restatement is slow at 64^3; the CUDA path is checked there by the GPU tests
ORACLE_CASES = ["cantilever16", "shell24", "config0_box32"]


def reference_u(key):
    """(slots, u) of a stored case: all node slots or the sample."""
    if key + "/u" in REF:
        u = REF[key + "/u"].reshape(-1, 3)
        return np.arange(len(u)), u
    return REF[key + "/slots"], REF[key + "/u_sample"]


def rel_u(u_full, key):
    slots, ref = reference_u(key)
    flat = np.asarray(u_full)[..., :3].reshape(-1, 3)
    scale = float(REF[key + "/u_absmax"].max()) if key + "/u_absmax" in REF else float(np.abs(ref).max())
    return float(np.abs(flat[slots] - ref).max() / scale)


@pytest.mark.parametrize("name", list(CASES))
def test_generators_reproduce_the_stored_inputs(name):
    for flavour, tol in (("shipped", CASES[name][1]), ("fp64", CASES[name][2])):
        assert digest(inputs(name, tol)) == str(REF[f"{name}/{flavour}/digest"]), (name, flavour)


@pytest.mark.parametrize("name", ORACLE_CASES)
def test_oracle_fp64_matches_reference_fp64_build(name):
    key = f"{name}/fp64"
    inp = inputs(name, CASES[name][2])
    r = Oracle(inp, mode=MODE_FP64, tolerance=CASES[name][2]).solve()
    assert r["iterations"] == int(REF[key + "/iterations"])
    h, hr = np.asarray(r["history"]), REF[key + "/history"]
    assert np.abs(h - hr).max() / hr[0] < 1e-12 and np.max(np.abs(h - hr) / hr) < 1e-8
    assert rel_u(r["displacements"], key) < 1e-12


@pytest.mark.parametrize("name", ORACLE_CASES)
def test_oracle_reference_rounding_matches_shipped_build(name):
    key = f"{name}/shipped"
    inp = inputs(name, CASES[name][1])
    r = Oracle(inp, mode=MODE_REF, tolerance=CASES[name][1]).solve()
    assert r["iterations"] == int(REF[key + "/iterations"])
    assert rel_u(r["displacements"], key) < 1e-6
