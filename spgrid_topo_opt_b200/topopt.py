"""SIMP topology optimization on the GPU solver.

``SIMP``: one iteration follows the reference driver's Opt::iterate
(topo_opt/spgrid_topo_opt.cpp:1289-1331) on a fixed block set:
solve (MGPCG), compliance sensitivity (minimal_compliance.cpp:86-146, gradient
dc0 = -dc), density-weighted filter (Opt::smooth_dc, :527-579), optimality-
criteria update (optimality_criterion.cpp:19-145), and the new densities fed
back into the resident session (material pattern kept: densities stay
positive, clamped at DBL_MIN like the driver, :1122).

With ``device=True`` (the default) the whole iteration runs in the library
(sgs_design_step): densities and sensitivities stay on the GPU and the new
stiffness scales are computed there; ``device=False`` goes through the host
arrays of the individual entry points (the same arithmetic).

``BandSIMP``: the same iteration with the driver's narrow band (page maps,
repacking of the solver input; see the class).

Command line: ``python -m spgrid_topo_opt_b200.topopt --bridge 512 128 256 --iterations 20
[--narrow-band]`` prints one JSON line per iteration.
"""
from __future__ import annotations

import argparse
import copy
import json
import sys
import time
from typing import Optional

import numpy as np

from . import native

DBL_MIN = np.finfo(np.float64).tiny


class SIMP:
    def __init__(self, inputs, *, precision: int = native.PRECISION_MIXED, tolerance: float = 1e-6,
                 volume_fraction: float = 0.1, step_limit: float = 0.2, filter_size: float = 1.5,
                 minimum_density: float = 0.0, fixed: Optional[np.ndarray] = None, fixed_density: float = 1.0,
                 smart_oc: bool = False, exclude_fixed: bool = True, device: bool = True):
        self.session = native.Session(inputs, precision=precision)
        self.device = device
        self._density = np.array(inputs.density.data, np.float64, copy=True)
        self.inside = self._density > 0
        self.tolerance = tolerance
        self.volume_fraction = volume_fraction
        self.step_limit = step_limit
        self.filter_size = filter_size
        self.minimum_density = minimum_density
        self.fixed = fixed
        self.fixed_density = fixed_density
        self.smart_oc = smart_oc
        self.exclude_fixed = exclude_fixed
        if device:
            self.session.design_set(self._density, fixed)

    @property
    def density(self) -> np.ndarray:
        if self.device:
            self._density = self.session.design_get()
        return self._density

    def iterate(self) -> dict:
        if self.device:
            r = self.session.design_step(self.tolerance, self.volume_fraction, self.step_limit, self.filter_size,
                                         self.minimum_density, self.fixed_density, self.smart_oc, self.exclude_fixed)
            return {"objective": r["objective"], "change": r["change"], "lagrange": r["lagrange"],
                    "cg_iterations": r["cg_iterations"], "solve_device_s": round(r["solve_device_seconds"], 4),
                    "solve_s": round(r["solve_seconds"], 4), "update_s": round(r["step_seconds"], 4)}
        t0 = time.perf_counter()
        st = self.session.solve(tolerance=self.tolerance)
        t1 = time.perf_counter()
        objective, dc, _ = self.session.sensitivity(self._density)
        dc1 = self.session.filter_sensitivity(self._density, -dc, self.filter_size)
        rho, lagrange, change = self.session.oc_update(
            self._density, dc1, self.volume_fraction, self.step_limit, self.minimum_density, self.fixed,
            self.fixed_density, self.smart_oc, self.exclude_fixed)
        rho = np.where(self.inside, np.maximum(rho, DBL_MIN), 0.0)
        t2 = time.perf_counter()
        self._density = rho
        self.session.set_density(rho)
        t3 = time.perf_counter()
        return {"objective": objective, "change": change, "lagrange": lagrange, "cg_iterations": st["iterations"],
                "solve_device_s": round(st["solve_device_seconds"], 4), "solve_s": round(t1 - t0, 4),
                "sensitivity_filter_oc_s": round(t2 - t1, 4), "set_density_s": round(t3 - t2, 4)}

    def close(self):
        self.session.close()


class BandSIMP:
    """The driver's loop with its narrow band (Opt::iterate,
    topo_opt/spgrid_topo_opt.cpp:1289-1331, page maps included): the design
    lives on the container (the blocks of ``inputs.density``) in a GPU band;
    from iteration ``grid_update_start`` on, every iteration first updates the
    thin / fat / fatter maps (sgs_band_update) and, when the fat map changed,
    repacks the solver input from the fatter blocks as the driver does
    (spgrid_topo_opt.cpp:1068-1160) and builds a new session; then one
    sgs_band_step runs solve, sensitivity, filter and OC on the GPU.

    Container cells are those with positive density in ``inputs``; the cells
    around each force node carry has_force (add_force, spgrid_topo_opt.h:577-592);
    ``fixed`` marks fixed-density cells."""

    def __init__(self, inputs, *, precision: int = native.PRECISION_MIXED, tolerance: float = 1e-6,
                 volume_fraction: float = 0.1, step_limit: float = 0.2, filter_size: float = 1.5,
                 minimum_density: float = 0.0, fixed: Optional[np.ndarray] = None, fixed_density: float = 1.0,
                 smart_oc: bool = False, exclude_fixed: bool = True, grid_update_start: int = 5,
                 active_threshold: float = 1e-6, fraction_to_keep: float = 1.0, fat_margin: int = 1,
                 connectivity_filtering: bool = True):
        self.template = inputs
        self.precision = precision
        base = np.asarray(inputs.density.base, np.int32)
        dens = np.array(inputs.density.data, np.float64, copy=True)
        self.inside = dens > 0
        flags = np.where(self.inside, native.CELL_INSIDE, 0).astype(np.uint8)
        # has_force on the container cells around every force node
        gdim = (np.asarray(inputs.resolution) + 3) // 4 + 1
        lut = np.full(tuple(gdim), -1, np.int64)
        lut[base[:, 0] // 4, base[:, 1] // 4, base[:, 2] // 4] = np.arange(len(base))
        fc = np.asarray(inputs.forces["coord"], np.int64).reshape(-1, 3)
        if len(fc):
            corners = np.array([[a, b, c] for a in (-1, 0) for b in (-1, 0) for c in (-1, 0)])
            cells = (fc[:, None, :] + corners[None]).reshape(-1, 3)
            cells = cells[((cells >= 0) & (cells // 4 < gdim)).all(axis=1)]
            blk = lut[cells[:, 0] // 4, cells[:, 1] // 4, cells[:, 2] // 4]
            cells, blk = cells[blk >= 0], blk[blk >= 0]
            e = (cells[:, 0] % 4) * 16 + (cells[:, 1] % 4) * 4 + cells[:, 2] % 4
            hit = (flags[blk, e] & native.CELL_INSIDE) != 0
            flags[blk[hit], e[hit]] |= native.CELL_FORCE
        if fixed is not None:
            flags |= np.where(np.asarray(fixed).reshape(flags.shape) != 0, native.CELL_FIXED, 0).astype(np.uint8)
        self.band = native.Band(base, inputs.resolution, flags, dens)
        self.base = base
        # settings and boundary conditions for every repack; the density grid comes from the band
        from .fem_interface import BlockedGrid, serialize_inputs
        tmpl = copy.copy(inputs)
        tmpl.density = BlockedGrid(resolution=list(inputs.density.resolution), base=np.zeros((0, 3), np.int32),
                                   data=np.zeros((0, 64)))
        self._template_blob = serialize_inputs(tmpl)
        self.step_params = dict(tolerance=tolerance, volume_fraction=volume_fraction, step_limit=step_limit,
                                filter_size=filter_size, minimum_density=minimum_density,
                                fixed_density=fixed_density, smart_oc=smart_oc, exclude_fixed=exclude_fixed)
        self.map_params = dict(minimum_density=minimum_density, active_threshold=active_threshold,
                               fraction_to_keep=fraction_to_keep, fat_margin=fat_margin,
                               connectivity_filtering=connectivity_filtering)
        self.grid_update_start = grid_update_start
        self.iteration = 0
        self.session = None
        self._pack()

    def _pack(self):
        """New solver input from the fatter blocks (spgrid_topo_opt.cpp:1068-1160),
        packed and set up by the library (sgs_band_session)."""
        _, _, fatter = self.band.maps()
        if self.session is not None:
            self.session.close()
        self.session = self.band.session(self._template_blob, self.precision)
        self.session_blocks = int(fatter.sum())

    @property
    def density(self) -> np.ndarray:
        return self.band.density()

    def iterate(self) -> dict:
        out = {}
        if self.iteration >= self.grid_update_start:
            t = time.perf_counter()
            st = self.band.update(**self.map_params)
            repacked = st["fat_changed"] != 0
            if repacked:
                self._pack()
            out.update(thin=st["thin_blocks"], fat=st["fat_blocks"], fatter=st["fatter_blocks"],
                       maps_device_s=round(st["device_seconds"], 5), repacked=repacked,
                       maps_s=round(time.perf_counter() - t, 4))
        r = self.band.step(self.session, **self.step_params)
        self.iteration += 1
        out.update(objective=r["objective"], change=r["change"], lagrange=r["lagrange"],
                   cg_iterations=r["cg_iterations"], solve_device_s=round(r["solve_device_seconds"], 4),
                   solve_s=round(r["solve_seconds"], 4), update_s=round(r["step_seconds"], 4),
                   session_blocks=self.session_blocks)
        return out

    def close(self):
        if self.session is not None:
            self.session.close()
            self.session = None
        self.band.close()


def main(argv=None) -> int:
    from . import configs
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("--bridge", type=int, nargs=3, default=[512, 128, 256], metavar=("NX", "NY", "NZ"))
    ap.add_argument("--iterations", type=int, default=20)
    ap.add_argument("--volume-fraction", type=float, default=0.1)
    ap.add_argument("--step-limit", type=float, default=0.2)
    ap.add_argument("--precision", choices=["mixed", "fp64"], default="mixed")
    ap.add_argument("--host-loop", action="store_true", help="run the step through the host-array entry points")
    ap.add_argument("--narrow-band", action="store_true",
                    help="keep the driver's page maps: prune, repack and re-solve on the fatter blocks")
    ap.add_argument("--grid-update-start", type=int, default=5)
    ap.add_argument("--render", metavar="PPM", help="render the final design (surface mode) into a PPM image")
    ap.add_argument("--render-size", type=int, nargs=2, default=[640, 360], metavar=("W", "H"))
    args = ap.parse_args(argv)
    t = time.perf_counter()
    prob = configs.bridge(*args.bridge)
    inp = configs.to_inputs(prob)
    prec = native.PRECISION_MIXED if args.precision == "mixed" else native.PRECISION_FP64
    if args.narrow_band:
        opt = BandSIMP(inp, precision=prec, volume_fraction=args.volume_fraction, step_limit=args.step_limit,
                       grid_update_start=args.grid_update_start)
    else:
        opt = SIMP(inp, precision=prec, volume_fraction=args.volume_fraction, step_limit=args.step_limit,
                   device=not args.host_loop)
    print(json.dumps({"workload": prob.name, "container_cells": int(np.count_nonzero(opt.inside)),
                      "narrow_band": bool(args.narrow_band), "setup_s": round(time.perf_counter() - t, 2)}),
          flush=True)
    total = time.perf_counter()
    for it in range(args.iterations):
        r = opt.iterate()
        r["iter"] = it
        print(json.dumps(r), flush=True)
    rho = opt.density
    print(json.dumps({"iterations": args.iterations, "total_s": round(time.perf_counter() - total, 2),
                      "volume": float(rho[opt.inside].mean())}), flush=True)
    if args.render:
        t = time.perf_counter()
        cam = native.view_matrix(20, -35, 0, 0, 0, -3.0)
        kw = dict(mode=0, frames=16, threshold=0.5)
        w, h = args.render_size
        if isinstance(opt, BandSIMP):
            img, res = opt.band.render(w, h, cam, **kw)
        else:
            img, res = native.render(inp.density.base, rho, w, h, cam, **kw)
        native.write_ppm(args.render, img)
        print(json.dumps({"render": args.render, "volume_res": res.tolist(),
                          "render_s": round(time.perf_counter() - t, 3)}), flush=True)
    opt.close()
    return 0


if __name__ == "__main__":
    sys.exit(main())
