"""Edge cases of the drop-in solve, against the oracle where it has an answer:
no load, prescribed (non-zero) Dirichlet values, input blocks in any order
and repeated, a single level (the exact bottom solve on level 0), and the
iteration cap.
"""
import copy

import numpy as np
import pytest

from oracle import oracle as orc
from spgrid_topo_opt_b200 import configs, native
from spgrid_topo_opt_b200.fem_interface import BlockedGrid

pytestmark = pytest.mark.gpu


def _rel(a, b):
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


def test_zero_load_converges_at_once(native_lib):
    inp = configs.to_inputs(configs.cantilever_box(16, bottom_size=4))
    inp.forces = inp.forces[:0]
    out = native.fem_solve(inp)
    r = orc.Oracle(inp, mode=orc.MODE_REF).solve()
    assert out.success and r["status"] == 0
    assert out.extra_ints["iterations"] == r["iterations"] == 0
    assert np.all(out.displacements.data[..., :3] == 0)
    assert list(out.residuals) == [0.0]


def test_prescribed_displacement(native_lib):
    """Non-zero Dirichlet values go through the lift (SPGrid_CPU_Solver.cpp:281-341):
    without forces the body translates rigidly by the prescribed value."""
    inp = configs.to_inputs(configs.cantilever_box(16, bottom_size=4))
    inp.forces = inp.forces[:0]
    d = inp.dirichlet_nodes
    d["value"][d["axis"] == 0] = 1e-3
    r = orc.Oracle(inp, mode=orc.MODE_FP64, tolerance=1e-10).solve()
    with native.Session(inp, precision=native.PRECISION_FP64) as s:
        s.solve(tolerance=1e-10)
        u = s.displacements()
    assert _rel(u[..., :3], r["displacements"][..., :3]) < 1e-7
    solid = np.asarray(inp.density.data) > 0
    ux = u[..., 0][solid]
    assert np.abs(ux - 1e-3).max() < 1e-9
    assert np.abs(u[..., 1:3][solid]).max() < 1e-9


def test_block_order_and_repeated_blocks(native_lib):
    inp = configs.to_inputs(configs.cantilever_box(16, density=(0.2, 1.0), bottom_size=4))
    base, data = np.asarray(inp.density.base), np.asarray(inp.density.data)
    out0 = native.fem_solve(inp)
    perm = np.random.default_rng(3).permutation(len(base))
    shuffled = copy.copy(inp)
    shuffled.density = BlockedGrid(resolution=list(inp.density.resolution), base=base[perm].copy(),
                                   data=data[perm].copy())
    out1 = native.fem_solve(shuffled)
    assert out1.success and out1.extra_ints["iterations"] == out0.extra_ints["iterations"]
    assert np.array_equal(out1.displacements.base, base[perm])
    assert np.array_equal(out1.displacements.data, out0.displacements.data[perm])
    # a repeated block (the later copy wins, here with the same values) changes nothing
    rep = copy.copy(inp)
    rep.density = BlockedGrid(resolution=list(inp.density.resolution), base=np.concatenate([base, base[:1]]),
                              data=np.concatenate([data, data[:1]]))
    rep.preserve_output(len(base) + 1)
    out2 = native.fem_solve(rep)
    assert out2.success
    assert np.array_equal(out2.displacements.data[:-1], out0.displacements.data)
    assert np.array_equal(out2.displacements.data[-1], out0.displacements.data[0])


def test_single_level_is_an_exact_solve(native_lib):
    prob = configs.cantilever_box(8, density=(0.2, 1.0), bottom_size=64)
    inp = configs.to_inputs(prob, mg_level=1)
    r = orc.Oracle(inp, mode=orc.MODE_FP64, tolerance=1e-12).solve()
    with native.Session(inp, precision=native.PRECISION_FP64) as s:
        st = s.solve(tolerance=1e-12)
        u = s.displacements()
    assert st["levels"] == 1
    assert st["iterations"] <= 2 and r["iterations"] <= 2
    assert _rel(u[..., :3], r["displacements"][..., :3]) < 1e-9


def test_iteration_cap(native_lib):
    inp = configs.to_inputs(configs.cantilever_box(16, bottom_size=4))
    inp.krylov.max_iterations = 3
    inp.extra_ints["sgs_honor_max_iterations"] = 1
    out = native.fem_solve(inp)
    assert out.extra_ints["iterations"] == 3
    assert len(out.residuals) == 4


def _with_state(inp, out, keep=1, forced=1):
    nxt = copy.deepcopy(inp)
    nxt.extra_ints["keep_state"] = keep
    nxt.extra_ints["forced_reuse"] = forced
    nxt.extra_ints["state_ptr_lower"] = out.extra_ints["state_ptr_lower"]
    nxt.extra_ints["state_ptr_higher"] = out.extra_ints["state_ptr_higher"]
    return nxt


def test_keep_state_warm_start(native_lib):
    """keep_state returns a solver state through extra_ints (fem_interface.h:200-214);
    passed back, it warm-starts the next solve from the last solution, with the
    stopping rule still relative to the first call's zero-guess residual
    (SPGrid_CPU_Solver.cpp:240-321, 389-408)."""
    inp = configs.to_inputs(configs.cantilever_box(16, density=(0.2, 1.0), bottom_size=4))
    inp.extra_ints["keep_state"] = 1
    out1 = native.fem_solve(inp)
    assert out1.success and "state_ptr_lower" in out1.extra_ints and out1.extra_ints["iterations"] > 0
    # the same problem again: the converged solution is reused, no iteration is needed
    out2 = native.fem_solve(_with_state(inp, out1))
    assert out2.success and out2.extra_ints["warm_start_reused"] == 1
    assert out2.extra_ints["iterations"] == 0
    assert np.array_equal(out2.displacements.data[..., :3], out1.displacements.data[..., :3])
    assert out2.extra_doubles["initial_residual"] == out1.extra_doubles["initial_residual"]
    # a slightly stiffer design: the warm start needs fewer iterations than a cold solve
    stiffer = _with_state(inp, out2)
    stiffer.density = BlockedGrid(resolution=list(inp.density.resolution), base=np.asarray(inp.density.base),
                                  data=np.minimum(np.asarray(inp.density.data) * 1.05, 1.0))
    out3 = native.fem_solve(stiffer)
    cold = copy.deepcopy(stiffer)
    for k in ("keep_state", "state_ptr_lower", "state_ptr_higher"):
        cold.extra_ints.pop(k)
    out_cold = native.fem_solve(cold)
    assert out3.success and out3.extra_ints["iterations"] < out_cold.extra_ints["iterations"]
    assert _rel(out3.displacements.data[..., :3], out_cold.displacements.data[..., :3]) < 1e-3
    # without keep_state the state passed in is released and none is returned
    out4 = native.fem_solve(_with_state(inp, out3, keep=0))
    assert out4.success and "state_ptr_lower" not in out4.extra_ints


def test_foreign_state_pointer_is_rejected(native_lib):
    inp = configs.to_inputs(configs.cantilever_box(16, bottom_size=4))
    junk = np.zeros(8, np.uint64)
    addr = junk.ctypes.data
    inp.extra_ints["state_ptr_lower"] = int(np.uint32(addr & 0xFFFFFFFF).view(np.int32))
    inp.extra_ints["state_ptr_higher"] = int(np.uint32(addr >> 32).view(np.int32))
    out = native.fem_solve(inp)
    assert not out.success and out.error_code == 1


def _two_bodies(gap_cells: int = 4):
    """A 24x16x16 cantilever fixed at x = 0 and, beyond a gap of empty cells, a
    loose 8x8x8 box carrying a load: the second body has no support."""
    n = (24 + gap_cells + 8, 16, 16)
    rho = np.zeros(n)
    rho[:24] = 0.5
    rho[24 + gap_cells:, 4:12, 4:12] = 0.5
    cells = np.argwhere(np.ones((1, 16, 16), bool)).astype(np.int32)
    f = np.zeros(2, configs.FORCE_DTYPE)
    f["coord"][0] = (24, 8, 8)
    f["f"][0] = (0.0, -1.0, 0.0)
    f["coord"][1] = (n[0], 8, 8)
    f["f"][1] = (0.0, -1.0, 0.0)
    return configs.Problem("two_bodies", n, rho, cells, f, 1.0 / n[0], configs.mg_level_for(n[0], 8))


def test_indefinite_operator_reports_breakdown(native_lib):
    """Material whose SIMP stiffness is negative (a negative minimum_stiffness:
    E = (1 - Emin) rho^p + Emin < 0 for rho^p < -Emin / (1 - Emin)) makes the
    operator indefinite.  The reference's CG throws on s.q <= 0
    (CONJUGATE_GRADIENT.cpp:49-52) and its PARDISO factorization fails on the
    bottom; here the call returns success = 0 with SGS_ERR_BREAKDOWN, whichever
    check sees it first, and the context stays usable."""
    prob = _two_bodies()
    prob.density[:24] = np.where(np.arange(24)[:, None, None] >= 12, 0.2, 0.9)
    inp = configs.to_inputs(prob, minimum_stiffness=-0.5)
    out = native.fem_solve(inp)
    assert not out.success and out.error_code == 8, (out.error_code, out.info)
    # the device is still usable afterwards
    ok = native.fem_solve(configs.to_inputs(configs.cantilever_box(16, bottom_size=4)))
    assert ok.success


def test_unsupported_island_is_reported_as_not_converged(native_lib):
    """A loaded body with no Dirichlet support makes the operator singular (its
    rigid motions cost no energy) and the equations inconsistent.  The reference
    perturbs tiny pivots in its factorization (iparm[9] = 13,
    Elasticity_Matrix.cpp:186) and runs its CG to the cap of 500 iterations
    (SPGrid_CPU_Solver.cpp:326), then returns success.  Here every precision
    mode ends the same way without a hang or a fault -- either the bottom
    inverse or the CG checks report SGS_ERR_BREAKDOWN, or the solve stops at the
    cap with success set, extra_ints["converged"] = 0 and a message that says so."""
    inp = configs.to_inputs(_two_bodies())
    inp.extra_ints["sgs_honor_max_iterations"] = 1
    inp.krylov.max_iterations = 60
    for prec in (native.PRECISION_REFERENCE, native.PRECISION_FP64, native.PRECISION_MIXED):
        inp.extra_ints["sgs_precision"] = prec
        out = native.fem_solve(inp)
        if out.success:
            assert out.extra_ints["converged"] == 0 and out.extra_ints["iterations"] == 60, (prec, out.extra_ints)
            assert "without converging" in out.info, out.info
        else:
            assert out.error_code == 8, (prec, out.error_code, out.info)
    # a supported body converges, and says so
    ok = native.fem_solve(configs.to_inputs(configs.cantilever_box(16, bottom_size=4)))
    assert ok.success and ok.extra_ints["converged"] == 1 and "converged in" in ok.info
