"""GPU parity: every operator of the CUDA library against the oracle on the same
seeded inputs, then whole solves through the session API and the drop-in
fem_solve entry.

Tolerances: FP64 operators agree with the oracle to round-off (relative 1e-11
of the field's magnitude; the summation order differs).  Whole FP64 solves run
to a relative L-inf residual of 1e-10 and agree to 1e-7.  The reference-rounding
mode reproduces the oracle's iteration count and agrees to 1e-5.  The mixed
FP32 V-cycle solve is compared with the FP64 oracle after both converge to
1e-9 and agrees to 1e-6.
"""
import numpy as np
import pytest

from oracle import oracle as orc
from spgrid_topo_opt_b200 import configs, native
from spgrid_topo_opt_b200 import fem_interface as fi

pytestmark = pytest.mark.gpu


def _rel(a, b):
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


@pytest.fixture(scope="module")
def small(native_lib):
    prob = configs.cantilever_box(16, density=(0.2, 1.0), bottom_size=4)
    inp = configs.to_inputs(prob)
    ref = orc.Oracle(inp, mode=orc.MODE_FP64)
    ses = native.Session(inp, precision=native.PRECISION_FP64)
    return inp, ref, ses


def _field(ses, level, seed, masked=True, dirichlet_zero=False):
    n = ses.blocks(level).shape[0] * 128
    x = np.random.default_rng(seed).standard_normal((3, n))
    fl = ses.flags(level)
    if masked:
        x *= (fl & 0x10) != 0
    if dirichlet_zero:  # the V-cycle keeps u zero on Dirichlet components
        for v, bit in enumerate((0x20, 0x40, 0x80)):
            x[v][(fl & bit) != 0] = 0
    return x


def test_levels_match(small):
    _, ref, ses = small
    assert ses.levels == ref.levels >= 3
    for lev in range(ref.levels):
        assert np.array_equal(ses.blocks(lev), ref.blocks(lev))


def test_level0_matvec_and_residual(small):
    _, ref, ses = small
    u, b = _field(ses, 0, 1), _field(ses, 0, 2)
    assert _rel(ses.apply(native.OP_KU, 0, u), ref.apply(orc.OP_KU, 0, u)) < 1e-11
    assert _rel(ses.apply(native.OP_RESIDUAL, 0, u, b), ref.apply(orc.OP_RESIDUAL, 0, u, b)) < 1e-11


@pytest.mark.parametrize("tensor_cores", [1, 0])
def test_packed_fp32_residual_matches_fp64_oracle(small, tensor_cores):
    """The mixed V-cycle's level-0 residual in FP32: on the tensor cores (TF32
    split into high and low parts, FP32 accumulation) and on the CUDA cores,
    both within FP32 rounding (1e-5 of the field's magnitude) of the FP64
    oracle."""
    inp, ref, _ = small
    i2 = fi.deserialize_inputs(fi.serialize_inputs(inp))
    i2.extra_ints["sgs_tensor_cores"] = tensor_cores
    with native.Session(i2, precision=native.PRECISION_MIXED) as s:
        u, b = _field(s, 0, 21), _field(s, 0, 22)
        got = s.apply(native.OP_PACKED_RESIDUAL, 0, u, b)
    want = ref.apply(orc.OP_RESIDUAL, 0, u, b)
    assert _rel(got, want) < 1e-5


@pytest.mark.parametrize("arg", [0, 1, 2, 3])
def test_level0_smoother(small, arg):
    _, ref, ses = small
    u, b = _field(ses, 0, 3), _field(ses, 0, 4)
    assert _rel(ses.apply(native.OP_SMOOTH, 0, u, b, arg=arg), ref.apply(orc.OP_SMOOTH, 0, u, b, arg=arg)) < 1e-11


def test_transfers(small):
    _, ref, ses = small
    for lev in range(ses.levels - 1):
        f = _field(ses, lev, 5 + lev, masked=False)
        assert _rel(ses.apply(native.OP_RESTRICT, lev, f, out_level=lev + 1),
                    ref.apply(orc.OP_RESTRICT, lev, f, out_level=lev + 1)) < 1e-12
        c = _field(ses, lev + 1, 9 + lev, masked=False)
        base = _field(ses, lev, 13 + lev, masked=False)
        assert _rel(ses.apply(native.OP_PROLONG, lev, c, base), ref.apply(orc.OP_PROLONG, lev, c, base)) < 1e-12


def test_galerkin_operators(small):
    _, ref, ses = small
    for lev in range(2, ses.levels):
        a, sa = ses.stencils(lev)
        b, sb = ref.stencils(lev)
        assert _rel(a, b) < 1e-11, lev
        assert np.array_equal(sa & 0x07FFFFFF, sb & 0x07FFFFFF), lev
        u = _field(ses, lev, 17 + lev, dirichlet_zero=True)
        assert _rel(ses.apply(native.OP_STENCIL, lev, u), ref.apply(orc.OP_STENCIL, lev, u)) < 1e-11
        ub = _field(ses, lev, 21 + lev)
        for arg in (1, 0, 3):
            assert _rel(ses.apply(native.OP_SMOOTH, lev, u, ub, arg=arg), ref.apply(orc.OP_SMOOTH, lev, u, ub, arg=arg)) < 1e-11


@pytest.fixture(scope="module")
def deep(native_lib):
    """Six levels: in the FP64 and mixed modes the operators of levels 3-5 come
    from the cell matrices of the level above them, while the oracle sums every
    level from the finest cells (the reference's construction)."""
    inp = configs.to_inputs(configs.cantilever_box(48, density=(0.2, 1.0), bottom_size=2))
    ref = orc.Oracle(inp, mode=orc.MODE_FP64)
    ses = native.Session(inp, precision=native.PRECISION_FP64)
    assert ses.levels == 6
    return inp, ref, ses


def test_galerkin_operators_of_a_deep_hierarchy(deep):
    _, ref, ses = deep
    for lev in range(2, ses.levels):
        a, sa = ses.stencils(lev)
        b, sb = ref.stencils(lev)
        assert _rel(a, b) < 1e-11, lev
        assert np.array_equal(sa & 0x07FFFFFF, sb & 0x07FFFFFF), lev


def test_coarse_smoothers_of_a_deep_hierarchy(deep):
    """Full and boundary-band sweeps, both directions, on every level with
    stencils: each colour pass runs over the level's list of the active (or
    active band) nodes of that colour, down to levels of a few blocks."""
    _, ref, ses = deep
    for lev in range(2, ses.levels - 1):
        u = _field(ses, lev, 41 + lev, dirichlet_zero=True)
        b = _field(ses, lev, 47 + lev)
        for arg in (0, 1, 2, 3):
            assert _rel(ses.apply(native.OP_SMOOTH, lev, u, b, arg=arg),
                        ref.apply(orc.OP_SMOOTH, lev, u, b, arg=arg)) < 1e-11, (lev, arg)


def test_bottom_solve_and_vcycle(small):
    _, ref, ses = small
    top = ses.levels - 1
    b = _field(ses, top, 31)
    assert _rel(ses.apply(native.OP_BOTTOM, top, b), ref.apply(orc.OP_BOTTOM, top, b)) < 1e-10
    r = _field(ses, 0, 33)
    assert _rel(ses.apply(native.OP_VCYCLE, 0, r), ref.apply(orc.OP_VCYCLE, 0, r)) < 1e-10


def _solve_pair(inp, mode, precision, tol):
    r = orc.Oracle(inp, mode=mode, tolerance=tol).solve()
    assert r["status"] == 0
    with native.Session(inp, precision=precision) as s:
        st = s.solve(tolerance=tol)
        d = s.displacements()
        h = s.history()
    return r, st, d, h


@pytest.mark.parametrize("n,bottom", [(16, 4), (32, 16)])
def test_fp64_solve_matches_oracle(native_lib, n, bottom):
    inp = configs.to_inputs(configs.cantilever_box(n, bottom_size=bottom))
    r, st, d, _ = _solve_pair(inp, orc.MODE_FP64, native.PRECISION_FP64, 1e-10)
    assert abs(st["iterations"] - r["iterations"]) <= 1
    assert _rel(d[..., :3], r["displacements"][..., :3]) < 1e-7


def test_reference_rounding_solve_matches_oracle(native_lib):
    inp = configs.to_inputs(configs.cantilever_box(32, bottom_size=16))
    r, st, d, h = _solve_pair(inp, orc.MODE_REF, native.PRECISION_REFERENCE, inp.krylov.tolerance)
    assert st["iterations"] == r["iterations"]
    assert _rel(d[..., :3], r["displacements"][..., :3]) < 1e-5
    assert np.allclose(h[:len(r["history"])], r["history"], rtol=1e-4, atol=1e-12 * r["history"][0])


def test_mixed_precision_solve_matches_fp64_oracle(native_lib):
    inp = configs.to_inputs(configs.sphere_shell(32, bottom_size=8))
    r, st, d, _ = _solve_pair(inp, orc.MODE_FP64, native.PRECISION_MIXED, 1e-9)
    assert st["iterations"] <= r["iterations"] + 3
    assert _rel(d[..., :3], r["displacements"][..., :3]) < 1e-6


def test_drop_in_fem_solve(native_lib):
    inp = configs.to_inputs(configs.cantilever_box(16, bottom_size=4))
    out = native.fem_solve(inp)
    assert out.success and out.error_code == 0
    assert np.array_equal(out.displacements.base, inp.density.base)
    r = orc.Oracle(inp, mode=orc.MODE_REF).solve()
    assert out.extra_ints["iterations"] == r["iterations"]
    assert _rel(out.displacements.data[..., :3], r["displacements"][..., :3]) < 1e-5
    assert len(out.residuals) == r["iterations"] + 1


def test_sensitivity_matches_oracle(native_lib):
    prob = configs.cantilever_box(16, density=(0.05, 1.0), bottom_size=4)
    inp = configs.to_inputs(prob)
    o = orc.Oracle(inp, mode=orc.MODE_FP64, tolerance=1e-11)
    o.solve()
    obj_r, dc_r, se_r = o.sensitivity()
    with native.Session(inp, precision=native.PRECISION_FP64) as s:
        s.solve(tolerance=1e-11)
        obj, dc, se = s.sensitivity()
    assert _rel(dc, dc_r) < 1e-6 and _rel(se, se_r) < 1e-6
    assert obj == pytest.approx(obj_r, rel=1e-7)
