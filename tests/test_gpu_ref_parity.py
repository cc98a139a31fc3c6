"""The CUDA path against the reference's own solver, at the benchmark configs'
sizes (config 0: the 64^3 cantilever, density 0.1, mg_bottom_size 16,
tolerance 1e-4; a 64^3 sphere shell for config 1's generator).

tests/golden/ref_solves.npz holds the reference's fem_solve outputs (compiled
from the reference sources, tests/golden/make_solve_golden.py) in its shipped
build and in the same code with the float rounding switched off.  Through the
drop-in fem_solve:

* reference-rounding mode (the default) against the shipped build: the same
  iteration count, displacements to 1e-6 relative (L-inf, over the stored
  nodes, scaled by the field's largest displacement);
* FP64 mode against the FP64 build: the same iteration count, the residual
  history to 1e-8 (1e-11 of the initial residual for entries at round-off) and
  the displacements to 1e-9;
* mixed precision (FP32 V-cycle) against the FP64 build: displacements to
  1e-8 when both solve to 1e-10, and to 1e-5 at the benchmark's 1e-6.
"""
import os
import sys

import numpy as np
import pytest

from spgrid_topo_opt_b200 import native

GOLD = os.path.join(os.path.dirname(__file__), "golden")
sys.path.insert(0, GOLD)
from solve_cases import CASES, inputs  # noqa: E402
from test_ref_solves import REF, rel_u  # noqa: E402

pytestmark = pytest.mark.gpu


def solve(name, tol, precision):
    inp = inputs(name, tol)
    inp.extra_ints["sgs_precision"] = precision
    out = native.fem_solve(inp)
    assert out.success, out.info
    return out


@pytest.mark.parametrize("name", list(CASES))
def test_reference_rounding_matches_shipped_reference(native_lib, name):
    key = f"{name}/shipped"
    out = solve(name, CASES[name][1], native.PRECISION_REFERENCE)
    assert out.extra_ints["iterations"] == int(REF[key + "/iterations"])
    assert rel_u(out.displacements.data, key) < 1e-6


@pytest.mark.parametrize("name", list(CASES))
def test_fp64_matches_fp64_reference(native_lib, name):
    key = f"{name}/fp64"
    out = solve(name, CASES[name][2], native.PRECISION_FP64)
    assert out.extra_ints["iterations"] == int(REF[key + "/iterations"])
    h, hr = np.asarray(out.residuals), REF[key + "/history"]
    # entries at round-off (an exact bottom solve converges in one step) are held
    # to 1e-11 of the initial residual instead
    assert len(h) == len(hr) and np.all(np.abs(h - hr) <= 1e-8 * hr + 1e-11 * hr[0])
    assert rel_u(out.displacements.data, key) < 1e-9


@pytest.mark.parametrize("name", ["config0_box64", "shell64", "cantilever16", "spheres_band96"])
def test_mixed_precision_matches_fp64_reference(native_lib, name):
    key = f"{name}/fp64"
    tight = solve(name, 1e-10, native.PRECISION_MIXED)
    assert rel_u(tight.displacements.data, key) < 1e-8
    bench_tol = solve(name, 1e-6, native.PRECISION_MIXED)
    assert rel_u(bench_tol.displacements.data, key) < 1e-5
