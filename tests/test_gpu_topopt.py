"""The optimizer step after a solve on the GPU: the driver's density-weighted
sensitivity filter (topo_opt/spgrid_topo_opt.cpp:527-579) and the
optimality-criteria update (topo_opt/optimizer/optimality_criterion.cpp:19-145),
against the oracle's restatement, and three SIMP iterations end to end.
"""
import copy

import numpy as np
import pytest

from oracle import oracle as orc
from oracle import topo_oracle as torc
from spgrid_topo_opt_b200 import configs, native
from spgrid_topo_opt_b200.topopt import SIMP

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def case(native_lib):
    inp = configs.to_inputs(configs.cantilever_box(24, density=(0.05, 1.0), bottom_size=6))
    ses = native.Session(inp, precision=native.PRECISION_FP64)
    yield inp, ses
    ses.close()


@pytest.mark.parametrize("filter_size", [1.5, 2.2])
def test_filter_matches_oracle(case, filter_size):
    inp, ses = case
    rng = np.random.default_rng(11)
    rho = inp.density.data
    dc0 = -rng.uniform(0.0, 2.0, rho.shape)
    got = ses.filter_sensitivity(rho, dc0, filter_size)
    ref = torc.filter_dc(inp.density.base, inp.resolution, rho, dc0, filter_size)
    assert np.all(got[rho <= 0] == 0)
    assert np.abs(got - ref).max() <= 1e-12 * np.abs(ref).max()


@pytest.mark.parametrize("smart", [False, True])
def test_oc_update_matches_oracle(case, smart):
    inp, ses = case
    rng = np.random.default_rng(12)
    rho = inp.density.data
    dc0 = -rng.uniform(0.0, 1.0, rho.shape) + (0.05 if smart else 0.0)
    fixed = (rng.uniform(size=rho.shape) < 0.03).astype(np.uint8)
    got, lag, chg = ses.oc_update(rho, dc0, 0.3, step_limit=0.2, minimum_density=1e-3, fixed=fixed,
                                  fixed_density=1.0, smart_oc=smart)
    ref, rlag, rchg = torc.oc_update(rho, dc0, 0.3, step_limit=0.2, minimum_density=1e-3, fixed=fixed,
                                     fixed_density=1.0, smart_oc=smart)
    # the bisection may part ways on one comparison at round-off: one interval, 1e-7 relative
    assert lag == pytest.approx(rlag, rel=1e-6)
    assert np.abs(got - ref).max() <= 1e-6
    assert chg == pytest.approx(rchg, abs=1e-6)
    inside = rho > 0
    assert np.all(got[~inside] == rho[~inside])
    assert np.all(got[inside & (fixed != 0)] == 1.0)
    assert np.all(np.abs(got - rho)[inside & (fixed == 0)] <= 0.2 + 1e-12)


def test_simp_iterations_match_oracle(native_lib):
    inp = configs.to_inputs(configs.cantilever_box(16, density=0.5, bottom_size=4), tolerance=1e-12)
    # the session mirrors its densities into the inputs it was given: keep the oracle's apart
    opt = SIMP(copy.deepcopy(inp), precision=native.PRECISION_FP64, tolerance=1e-12, volume_fraction=0.4,
               minimum_density=1e-3, device=False)
    rho = inp.density.data.copy()
    inside = rho > 0
    for it in range(3):
        r = opt.iterate()
        o = orc.Oracle(inp, mode=orc.MODE_FP64, tolerance=1e-12)
        o.solve()
        obj, dc, _ = o.sensitivity()
        dc1 = torc.filter_dc(inp.density.base, inp.resolution, rho, -dc, 1.5)
        rho, _, _ = torc.oc_update(rho, dc1, 0.4, step_limit=0.2, minimum_density=1e-3)
        rho = np.where(inside, np.maximum(rho, np.finfo(np.float64).tiny), 0.0)
        inp.density.data = rho.copy()
        assert r["objective"] == pytest.approx(obj, rel=1e-8), it
        assert np.abs(opt.density - rho).max() <= 1e-6, it
    opt.close()


def test_device_loop_matches_host_loop(native_lib):
    """sgs_design_step (densities kept on the GPU) against the same iterations
    through the host-array entry points."""
    inp = configs.to_inputs(configs.cantilever_box(16, density=0.5, bottom_size=4), tolerance=1e-12)
    kw = dict(precision=native.PRECISION_FP64, tolerance=1e-12, volume_fraction=0.4, minimum_density=1e-3)
    host = SIMP(copy.deepcopy(inp), device=False, **kw)
    dev = SIMP(copy.deepcopy(inp), device=True, **kw)
    for it in range(3):
        a, b = host.iterate(), dev.iterate()
        assert b["objective"] == pytest.approx(a["objective"], rel=1e-10), it
        assert b["lagrange"] == pytest.approx(a["lagrange"], rel=1e-9), it
        assert np.abs(dev.density - host.density).max() <= 1e-9, it
    host.close()
    dev.close()
