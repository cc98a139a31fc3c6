"""The PCG loop on the device (one graph whose WHILE node a convergence-test
kernel drives) against the same loop tested on the host after every iteration
("sgs_device_loop" = 0).  Both run the same kernels in the same order, so the
residual histories, iteration counts and displacements must agree bit for bit,
also when the loop pauses at the end of its history buffer (the host takes the
history out and relaunches) and when it ends in a breakdown.
"""
import numpy as np
import pytest

from spgrid_topo_opt_b200 import configs, native

pytestmark = pytest.mark.gpu


def _pair(inp):
    dev = native.fem_solve(inp)
    inp.extra_ints["sgs_device_loop"] = 0
    host = native.fem_solve(inp)
    del inp.extra_ints["sgs_device_loop"]
    return dev, host


@pytest.mark.parametrize("prec", [native.PRECISION_REFERENCE, native.PRECISION_FP64, native.PRECISION_MIXED])
def test_device_loop_matches_host_loop(native_lib, prec):
    inp = configs.to_inputs(configs.cantilever_box(16, density=(0.05, 1.0), bottom_size=4))
    inp.extra_ints["sgs_precision"] = prec
    dev, host = _pair(inp)
    assert dev.success and host.success, (dev.info, host.info)
    assert dev.extra_ints["device_loop"] == 1 and host.extra_ints["device_loop"] == 0
    assert dev.extra_ints["iterations"] == host.extra_ints["iterations"] > 3
    assert np.array_equal(np.asarray(dev.residuals), np.asarray(host.residuals))
    assert np.array_equal(dev.displacements.data, host.displacements.data)


@pytest.mark.parametrize("prec", [native.PRECISION_FP64, native.PRECISION_MIXED])
def test_device_loop_pauses_and_resumes(native_lib, prec):
    # four residuals per launch: the loop pauses every three iterations, the
    # host takes the history out and relaunches from the iteration it stopped at
    inp = configs.to_inputs(configs.cantilever_box(16, density=(0.05, 1.0), bottom_size=4))
    inp.extra_ints["sgs_precision"] = prec
    inp.extra_ints["sgs_loop_history"] = 4
    dev, host = _pair(inp)
    assert dev.success and host.success, (dev.info, host.info)
    assert dev.extra_ints["device_loop"] == 1
    assert dev.extra_ints["iterations"] == host.extra_ints["iterations"] > 6
    assert len(dev.residuals) == dev.extra_ints["iterations"] + 1
    assert np.array_equal(np.asarray(dev.residuals), np.asarray(host.residuals))
    assert np.array_equal(dev.displacements.data, host.displacements.data)


def test_device_loop_reports_breakdown_like_the_host_loop(native_lib):
    # one level (an exact bottom solve) and a tolerance no residual reaches: the
    # recursively updated residual falls until s.q underflows to zero, which
    # both loops must report as a breakdown at the same iteration
    inp = configs.to_inputs(configs.cantilever_box(8, bottom_size=8))
    inp.extra_ints["sgs_precision"] = native.PRECISION_FP64
    inp.extra_ints["sgs_honor_max_iterations"] = 1
    inp.krylov.max_iterations = 1100
    inp.krylov.tolerance = 1e-300
    dev, host = _pair(inp)
    assert dev.extra_ints["device_loop"] == 1
    assert (dev.success, dev.error_code) == (host.success, host.error_code)
    assert dev.extra_ints["iterations"] == host.extra_ints["iterations"]
    assert np.array_equal(np.asarray(dev.residuals), np.asarray(host.residuals))


def test_device_loop_zero_iteration_cap(native_lib):
    # the test before the first iteration stops the loop: no iteration runs
    inp = configs.to_inputs(configs.cantilever_box(8, bottom_size=8))
    inp.extra_ints["sgs_honor_max_iterations"] = 1
    inp.krylov.max_iterations = 0
    dev, host = _pair(inp)
    assert dev.extra_ints["iterations"] == host.extra_ints["iterations"] == 0
    assert len(dev.residuals) == len(host.residuals) == 1
    assert np.array_equal(np.asarray(dev.residuals), np.asarray(host.residuals))
