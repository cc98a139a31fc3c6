"""Behaviour of the oracle itself (the CPU restatement used as the checker)."""
import numpy as np
import pytest

from oracle.oracle import Oracle, OracleError, MODE_REF, MODE_FP64, OP_KU
from spgrid_topo_opt_b200 import configs


def test_single_level_is_an_exact_solve():
    inp = configs.to_inputs(configs.cantilever_box(8, bottom_size=8))
    r = Oracle(inp, mode=MODE_FP64, tolerance=1e-12).solve()
    assert r["status"] == 0 and r["iterations"] == 1


def test_mgpcg_converges_and_reference_rounding_stays_close():
    inp = configs.to_inputs(configs.cantilever_box(16, bottom_size=4))
    a = Oracle(inp, mode=MODE_FP64, tolerance=1e-10).solve()
    b = Oracle(inp, mode=MODE_REF).solve()
    assert a["status"] == 0 and b["status"] == 0
    assert a["iterations"] < 40 and b["iterations"] < 15
    ua, ub = a["displacements"][..., :3], b["displacements"][..., :3]
    assert np.abs(ua - ub).max() <= 2e-3 * np.abs(ua).max()


def test_operator_is_symmetric_and_rigid_motions_are_in_its_null_space():
    inp = configs.to_inputs(configs.cantilever_box(8, bottom_size=8))
    o = Oracle(inp, mode=MODE_FP64)
    n = o.blocks(0).shape[0] * 128
    rng = np.random.default_rng(0)
    x, y = rng.standard_normal((3, n)), rng.standard_normal((3, n))
    assert abs((o.apply(OP_KU, 0, x) * y).sum() - (x * o.apply(OP_KU, 0, y)).sum()) < 1e-9 * abs((o.apply(OP_KU, 0, x) * y).sum())
    # a translation produces no force at nodes whose cells are all present
    t = np.zeros((3, n)); t[1] = 1.0
    f = o.apply(OP_KU, 0, t)
    interior = (o.flags(0) & 0x10) != 0
    assert np.abs(f[:, interior]).max() < 1e-6 * np.abs(o.apply(OP_KU, 0, x)).max()


def test_sensitivity_matches_finite_differences():
    prob = configs.cantilever_box(8, density=(0.3, 1.0), bottom_size=8)
    inp = configs.to_inputs(prob)
    base = Oracle(inp, mode=MODE_FP64, tolerance=1e-13)
    r = base.solve()
    _, dc, _ = base.sensitivity()
    # compliance C = f.u = dx * sum_e E_e s_e ; dC/drho_e = -dx * dc_e
    f = inp.forces
    def compliance(rho_blocks):
        inp2 = configs.to_inputs(prob)
        inp2.density.data = rho_blocks
        o = Oracle(inp2, mode=MODE_FP64, tolerance=1e-13)
        d = o.solve()["displacements"]
        node = f["coord"][0]
        for b, base_c in enumerate(inp2.density.base):
            off = node - base_c
            if np.all(off >= 0) and np.all(off < 4):
                return float(np.dot(d[b, off[0] * 16 + off[1] * 4 + off[2], :3], f["f"][0]))
    rng = np.random.default_rng(3)
    cells = np.argwhere(inp.density.data > 0)
    for b, e in cells[rng.choice(len(cells), 4, replace=False)]:
        h = 1e-4
        rp, rm = inp.density.data.copy(), inp.density.data.copy()
        rp[b, e] += h
        rm[b, e] -= h
        fd = (compliance(rp) - compliance(rm)) / (2 * h)
        assert fd == pytest.approx(-inp.dx * dc[b, e], rel=1e-4, abs=1e-12)


def test_setup_errors():
    with pytest.raises(OracleError):
        Oracle(configs.to_inputs(configs.cantilever_box(8), mg_level=2))


def test_topo_oracle_uniform_cases():
    """Hand-checked cases of the optimizer-step restatement: a uniform field
    filters to dc0 rho/(rho + 1e-3) away from the container's edge, and a uniform
    gradient leaves a density at the volume fraction unchanged."""
    from oracle import topo_oracle as torc
    base = np.array([[x, y, z] for x in (0, 4, 8) for y in (0, 4, 8) for z in (0, 4, 8)], np.int32)
    rho = np.full((len(base), 64), 0.4)
    dc0 = np.full((len(base), 64), -2.0)
    out = torc.filter_dc(base, [12, 12, 12], rho, dc0, 1.5)
    centre = 13 * 64 + 1 * 16 + 1 * 4 + 1  # block (4,4,4), cell (1,1,1): all neighbours inside
    assert out.reshape(-1)[centre] == pytest.approx(-2.0 * 0.4 / 0.401, rel=1e-14)
    new, mid, change = torc.oc_update(rho, dc0, 0.4, step_limit=0.2)
    assert np.allclose(new, 0.4, rtol=1e-6) and change < 1e-6
    assert mid == pytest.approx(2.0, rel=1e-6)
