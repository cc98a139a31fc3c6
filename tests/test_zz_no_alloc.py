"""The allocation-free sensitivity entry point, sgs_sensitivity_static.

It serves callers that cannot allocate device memory while they run: they own
every buffer, and the entry point's only scratch is a static device array.  The
test drives it through the C ABI with device buffers it allocated itself and
checks two calls in a row against sgs_sensitivity, the entry point that
allocates its own buffers, within the 1e-12 relative tolerance the parity tests
use for the same quantity computed twice on the GPU, and that further calls
take no device memory.  It also checks that a problem larger than the static
array is refused, and a call made with another device current.  Collected last so a
stop-at-first-failure run has already run every other test when it gets here.
"""
import ctypes as C

import numpy as np
import pytest

from spgrid_topo_opt_b200 import configs, native

pytestmark = pytest.mark.gpu


def _rel(a, b):
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


def test_static_sensitivity_matches_allocating_entry_point(native_lib):
    import torch

    torch.cuda.set_device(0)
    inp = configs.to_inputs(configs.cantilever_box(16, density=(0.05, 1.0), bottom_size=4))
    lib = native.load()
    with native.Session(inp, precision=native.PRECISION_FP64) as s:
        s.solve(tolerance=1e-10)
        obj_ref, dc_ref, se_ref = s.sensitivity()
        rho = torch.tensor(np.ascontiguousarray(inp.density.data), dtype=torch.float64, device="cuda")
        dc = torch.full_like(rho, np.nan)
        se = torch.full_like(rho, np.nan)
        obj = torch.full((1,), np.nan, dtype=torch.float64, device="cuda")
        torch.cuda.synchronize()

        def call_static():
            return lib.sgs_sensitivity_static(s.h, C.c_void_p(rho.data_ptr()), C.c_void_p(dc.data_ptr()),
                                              C.c_void_p(se.data_ptr()), C.c_void_p(obj.data_ptr()))

        for call in range(2):
            rc = call_static()
            assert rc == 0, lib.sgs_last_error(s.h)
            assert _rel(dc.cpu().numpy(), dc_ref) < 1e-12, call
            assert _rel(se.cpu().numpy(), se_ref) < 1e-12, call
            assert float(obj.item()) == pytest.approx(obj_ref, rel=1e-12), call
            dc.fill_(np.nan)
            se.fill_(np.nan)
            obj.fill_(np.nan)
        # the point of the entry point: further calls take no device memory, neither
        # from the driver (free memory unchanged) nor from torch's caching pool
        torch.cuda.synchronize()
        free_before, _ = torch.cuda.mem_get_info()
        reserved_before = torch.cuda.memory_reserved()
        for _ in range(3):
            assert call_static() == 0, lib.sgs_last_error(s.h)
        torch.cuda.synchronize()
        free_after, _ = torch.cuda.mem_get_info()
        assert free_after == free_before
        assert torch.cuda.memory_reserved() == reserved_before


@pytest.mark.skipif("__import__('torch').cuda.device_count() < 2", reason="needs two visible GPUs")
def test_static_sensitivity_rejects_another_current_device(native_lib):
    import torch

    torch.cuda.set_device(0)
    inp = configs.to_inputs(configs.cantilever_box(8, bottom_size=8))
    lib = native.load()
    with native.Session(inp, precision=native.PRECISION_FP64) as s:
        s.solve(tolerance=1e-8)
        n = inp.density.data.size
        with torch.cuda.device(1):
            bufs = [torch.zeros(n, dtype=torch.float64, device="cuda:1") for _ in range(3)]
            obj = torch.zeros(1, dtype=torch.float64, device="cuda:1")
            rc = lib.sgs_sensitivity_static(s.h, *[C.c_void_p(b.data_ptr()) for b in bufs],
                                            C.c_void_p(obj.data_ptr()))
        assert rc == 1 and b"device 1 current" in lib.sgs_last_error(s.h)


def test_static_sensitivity_rejects_problems_above_the_limit(native_lib):
    import torch

    torch.cuda.set_device(0)
    limit = 16384 * 256 // 64  # input blocks that fit the static partial-sum array
    inp = configs.to_inputs(configs.cantilever_box(8, bottom_size=8))
    nb = inp.density.base.shape[0]
    reps = limit // nb + 1
    # more input blocks than the static array can reduce (duplicates of the same blocks)
    inp.density.base = np.tile(inp.density.base, (reps, 1))
    inp.density.data = np.tile(inp.density.data, (reps, 1))
    lib = native.load()
    with native.Session(inp, precision=native.PRECISION_FP64) as s:
        n = inp.density.data.size
        buf = torch.zeros(n, dtype=torch.float64, device="cuda")
        out = torch.zeros(n, dtype=torch.float64, device="cuda")
        out2 = torch.zeros(n, dtype=torch.float64, device="cuda")
        obj = torch.zeros(1, dtype=torch.float64, device="cuda")
        rc = lib.sgs_sensitivity_static(s.h, C.c_void_p(buf.data_ptr()), C.c_void_p(out.data_ptr()),
                                        C.c_void_p(out2.data_ptr()), C.c_void_p(obj.data_ptr()))
        assert rc == 1 and b"at most" in lib.sgs_last_error(s.h)
