"""The driver's loop with its narrow band on the GPU (BandSIMP: page-map update,
repacking of the solver input from the fatter blocks, sgs_band_step) against
the oracle: its page maps, the FP64 MGPCG solve and sensitivity of the packed
input, the band filter (stale sensitivities outside the fat map included) and
the band OC update (volume target against the whole container).
"""
import copy

import numpy as np
import pytest

from oracle import oracle as orc
from oracle import topo_oracle as torc
from spgrid_topo_opt_b200 import configs, native
from spgrid_topo_opt_b200.fem_interface import BlockedGrid
from spgrid_topo_opt_b200.topopt import BandSIMP

pytestmark = pytest.mark.gpu
DBL_MIN = np.finfo(np.float64).tiny


def void_cantilever():
    prob = configs.cantilever_box(24, density=0.5, bottom_size=6)
    prob.density[4:20, 12:24, :] = 1e-3     # a void at the minimum density: its blocks leave the thin map
    return configs.to_inputs(prob, tolerance=1e-12)


def test_band_loop_matches_oracle(native_lib):
    inp = void_cantilever()
    kw = dict(tolerance=1e-12, volume_fraction=0.4, minimum_density=1e-3, step_limit=0.2)
    opt = BandSIMP(copy.deepcopy(inp), precision=native.PRECISION_FP64, grid_update_start=0, **kw)
    base = np.asarray(inp.density.base)
    flags = opt.band.flags
    inside = (flags & torc.CELL_INSIDE) != 0
    rho = np.array(inp.density.data, copy=True)
    dc0 = np.zeros_like(rho)
    fat = np.ones(len(base), bool)
    fatter = fat.copy()
    repacked, smallest = 0, len(base)
    for it in range(3):
        r = opt.iterate()
        thin, fat, fatter, st = torc.update_page_maps(base, rho, flags, fat, minimum_density=1e-3)
        g_thin, g_fat, g_fatter = opt.band.maps()
        assert np.array_equal(g_thin, thin) and np.array_equal(g_fat, fat) and np.array_equal(g_fatter, fatter)
        assert r["fatter"] == st["fatter_blocks"]
        repacked += r["repacked"]
        smallest = min(smallest, int(fatter.sum()))
        idx = np.nonzero(fatter)[0]
        packed = copy.copy(inp)
        packed.density = BlockedGrid(resolution=list(inp.density.resolution), base=base[idx].copy(),
                                     data=np.where(fat[idx, None] & inside[idx], np.maximum(rho[idx], DBL_MIN), 0.0))
        o = orc.Oracle(packed, mode=orc.MODE_FP64, tolerance=1e-12)
        o.solve()
        obj, dc, _ = o.sensitivity()
        dc0[fat] = 0.0
        mat = packed.density.data > 0
        d = dc0[idx]
        d[mat] += -dc[mat]
        dc0[idx] = d
        dc0 = torc.band_filter(base, inp.resolution, flags, fat, rho, dc0, 1.5)
        rho, lag, chg = torc.band_oc(flags, fat, rho, dc0, int(inside.sum()), 0.4, step_limit=0.2,
                                     minimum_density=1e-3)
        assert r["session_blocks"] == len(idx), it
        assert r["objective"] == pytest.approx(obj, rel=1e-8), it
        assert r["lagrange"] == pytest.approx(lag, rel=1e-6), it
        assert np.abs(opt.density - rho).max() <= 1e-6, it
    assert repacked >= 1            # the void blocks were pruned and the input repacked
    assert smallest < len(base)
    opt.close()


def test_band_loop_without_updates_matches_device_loop(native_lib):
    """Before grid_update_start every map is the whole container: the band step
    is the plain device loop (sgs_design_step) on the same blocks."""
    from spgrid_topo_opt_b200.topopt import SIMP
    inp = configs.to_inputs(configs.cantilever_box(16, density=0.5, bottom_size=4), tolerance=1e-12)
    kw = dict(precision=native.PRECISION_FP64, tolerance=1e-12, volume_fraction=0.4, minimum_density=1e-3)
    band = BandSIMP(copy.deepcopy(inp), grid_update_start=100, **kw)
    dev = SIMP(copy.deepcopy(inp), device=True, **kw)
    for it in range(2):
        a, b = dev.iterate(), band.iterate()
        assert b["objective"] == pytest.approx(a["objective"], rel=1e-10), it
        assert np.abs(band.density - dev.density).max() <= 1e-9, it
    band.close()
    dev.close()


def test_threshold_and_compute_objective(native_lib):
    """The driver's threshold_and_compute_objective (spgrid_topo_opt.cpp:839-864)
    after two band iterations: the design thresholded by the bisection, the
    packed input solved, and the compliance against the oracle's FP64 solve of
    the same packed input."""
    inp = void_cantilever()
    opt = BandSIMP(copy.deepcopy(inp), precision=native.PRECISION_FP64, grid_update_start=0, tolerance=1e-12,
                   volume_fraction=0.4, minimum_density=1e-3)
    for _ in range(2):
        opt.iterate()
    opt.session.close()
    opt.session = None
    band = opt.band
    flags = band.flags
    base = np.asarray(inp.density.base)
    _, fat, fatter = band.maps()
    rho = band.density()
    total = int(np.count_nonzero(flags & torc.CELL_INSIDE))
    ref, t, solid = torc.threshold_density(flags, fat, rho, total, 0.4)
    r = band.threshold_and_compute_objective(opt._template_blob, volume_fraction=0.4,
                                             precision=native.PRECISION_FP64, tolerance=1e-12)
    assert r["threshold"] == t and r["solid_voxels"] == solid and r["volume"] == 0.4 * total
    assert np.array_equal(band.density(), ref)
    idx = np.nonzero(fatter)[0]
    inside = (flags & torc.CELL_INSIDE) != 0
    packed = copy.copy(inp)
    packed.density = BlockedGrid(resolution=list(inp.density.resolution), base=base[idx].copy(),
                                 data=np.where(fat[idx, None] & inside[idx], np.maximum(ref[idx], DBL_MIN), 0.0))
    assert np.array_equal(band.packed_density(), packed.density.data)
    o = orc.Oracle(packed, mode=orc.MODE_FP64, tolerance=1e-12)
    o.solve()
    obj, _, _ = o.sensitivity()
    assert r["objective"] == pytest.approx(obj, rel=1e-6)
    opt.close()
