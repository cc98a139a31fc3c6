"""Bottom levels beyond the dense inverse, as the reference driver's default
mg_bottom_size 64 produces them (spgrid_topo_opt.cpp:1022-1030): a box of 64
cells or less gets mg_level 1, the whole problem being the bottom that the
reference factors with PARDISO (Elasticity_Matrix.cpp:169-269); a 128^3 box
gets mg_level 3 with a ~10^5-unknown bottom.  Such bottoms are solved by CG
with V-cycles over further levels to round-off.

Checked: against the reference's own solver (tests/golden/ref_solves.npz) on a
one-level 16^3 cantilever, with the dense inverse and with the inner solve
forced (extra_ints sgs_dense_bottom_max); on the 64^3 config-0 box and a 128^3
cantilever with mg_bottom_size 64, against solves of the same equations with
the hierarchy of mg_bottom_size 16 (a different preconditioner, the same
solution).
"""
import os
import sys

import numpy as np
import pytest

from spgrid_topo_opt_b200 import configs, native

GOLD = os.path.join(os.path.dirname(__file__), "golden")
sys.path.insert(0, GOLD)
from solve_cases import CASES, inputs  # noqa: E402
from test_ref_solves import REF, rel_u  # noqa: E402

pytestmark = pytest.mark.gpu


def solve(inp, precision, dense_max=None):
    inp.extra_ints["sgs_precision"] = precision
    if dense_max is not None:
        inp.extra_ints["sgs_dense_bottom_max"] = dense_max
    out = native.fem_solve(inp)
    assert out.success and out.extra_ints.get("converged", 1) == 1, out.info
    return out


@pytest.mark.parametrize("dense_max", [None, 1000])
def test_one_level_cantilever_matches_reference(native_lib, dense_max):
    name = "cantilever16_bottom64"
    assert inputs(name, 1e-10).mg_level == 1
    fp64 = solve(inputs(name, CASES[name][2]), native.PRECISION_FP64, dense_max)
    assert fp64.extra_ints["iterations"] <= int(REF[f"{name}/fp64/iterations"]) + 1
    assert rel_u(fp64.displacements.data, f"{name}/fp64") < 1e-9
    ref = solve(inputs(name, CASES[name][1]), native.PRECISION_REFERENCE, dense_max)
    assert abs(ref.extra_ints["iterations"] - int(REF[f"{name}/shipped/iterations"])) <= 1
    assert rel_u(ref.displacements.data, f"{name}/shipped") < 1e-6
    mixed = solve(inputs(name, CASES[name][2]), native.PRECISION_MIXED, dense_max)
    assert rel_u(mixed.displacements.data, f"{name}/fp64") < 1e-8


def test_config0_box_with_the_driver_default_bottom(native_lib):
    """64^3 box, density 0.1, mg_bottom_size 64: one level with 8.2e5 unknowns."""
    inp = configs.to_inputs(configs.cantilever_box(64, density=0.1, bottom_size=64), tolerance=1e-10)
    assert inp.mg_level == 1
    with native.Session(inp, precision=native.PRECISION_FP64) as s:
        st = s.solve(tolerance=1e-10)
        assert st["levels"] > 1 and st["bottom_unknowns"] <= 24576
        u = s.displacements()
    assert rel_u(u, "config0_box64/fp64") < 1e-8
    out = solve(configs.to_inputs(configs.cantilever_box(64, density=0.1, bottom_size=64), tolerance=1e-4),
                native.PRECISION_REFERENCE)
    assert rel_u(out.displacements.data, "config0_box64/fp64") < 1e-5


@pytest.mark.parametrize("precision", [native.PRECISION_FP64, native.PRECISION_MIXED])
def test_cantilever128_with_the_driver_default_bottom(native_lib, precision):
    big = configs.to_inputs(configs.cantilever_box(128, density=(0.05, 1.0), bottom_size=64), tolerance=1e-10)
    small = configs.to_inputs(configs.cantilever_box(128, density=(0.05, 1.0), bottom_size=16), tolerance=1e-10)
    assert big.mg_level == 3 and small.mg_level == 4
    with native.Session(big, precision=precision) as s:
        st = s.solve(tolerance=1e-10)
        assert st["levels"] > 3
        u_big = s.displacements()[..., :3]
    with native.Session(small, precision=native.PRECISION_FP64) as s:
        s.solve(tolerance=1e-10)
        u_small = s.displacements()[..., :3]
    assert np.abs(u_big - u_small).max() / np.abs(u_small).max() < 1e-8
