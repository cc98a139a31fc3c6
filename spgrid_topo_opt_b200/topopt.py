"""SIMP topology optimization on the GPU solver.

One iteration follows the reference driver's Opt::iterate
(topo_opt/spgrid_topo_opt.cpp:1289-1331) without its page-map maintenance:
solve (MGPCG), compliance sensitivity (minimal_compliance.cpp:86-146, gradient
dc0 = -dc), density-weighted filter (Opt::smooth_dc, :527-579), optimality-
criteria update (optimality_criterion.cpp:19-145), and the new densities fed
back into the resident session (material pattern kept: densities stay
positive, clamped at DBL_MIN like the driver, :1122).

With ``device=True`` (the default) the whole iteration runs in the library
(sgs_design_step): densities and sensitivities stay on the GPU and the new
stiffness scales are computed there; ``device=False`` goes through the host
arrays of the individual entry points (the same arithmetic).

Command line: ``python -m spgrid_topo_opt_b200.topopt --bridge 512 128 256 --iterations 20``
prints one JSON line per iteration.
"""
from __future__ import annotations

import argparse
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


def main(argv=None) -> int:
    from . import configs
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("--bridge", type=int, nargs=3, default=[512, 128, 256], metavar=("NX", "NY", "NZ"))
    ap.add_argument("--iterations", type=int, default=20)
    ap.add_argument("--volume-fraction", type=float, default=0.1)
    ap.add_argument("--step-limit", type=float, default=0.2)
    ap.add_argument("--precision", choices=["mixed", "fp64"], default="mixed")
    ap.add_argument("--host-loop", action="store_true", help="run the step through the host-array entry points")
    args = ap.parse_args(argv)
    t = time.perf_counter()
    prob = configs.bridge(*args.bridge)
    inp = configs.to_inputs(prob)
    prec = native.PRECISION_MIXED if args.precision == "mixed" else native.PRECISION_FP64
    opt = SIMP(inp, precision=prec, volume_fraction=args.volume_fraction, step_limit=args.step_limit,
               device=not args.host_loop)
    print(json.dumps({"workload": prob.name, "container_cells": int(np.count_nonzero(opt.inside)),
                      "setup_s": round(time.perf_counter() - t, 2)}), flush=True)
    total = time.perf_counter()
    for it in range(args.iterations):
        r = opt.iterate()
        r["iter"] = it
        print(json.dumps(r), flush=True)
    rho = opt.density
    print(json.dumps({"iterations": args.iterations, "total_s": round(time.perf_counter() - total, 2),
                      "volume": float(rho[opt.inside].mean())}), flush=True)
    opt.close()
    return 0


if __name__ == "__main__":
    sys.exit(main())
