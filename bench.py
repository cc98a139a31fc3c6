#!/usr/bin/env python
"""Benchmark: MGPCG time-to-solution and MDOF/s to a relative L-inf residual of
1e-6 on one B200, mixed precision (FP32 V-cycle, FP64 outer PCG) against the
same GPU's plain FP64 MGPCG.  Default workload: the 1024^3 narrow band (a
12-voxel shell around the union of 8 seeded random spheres, seeded uniform
density in [1e-3, 1], Dirichlet on the lowest band cell layer, 16 seeded unit
point loads).  ``--workload shell`` runs the 256^3 sphere shell instead.

One step = one complete PCG solve (first residual to convergence) of the
resident problem; set-up (flags, Galerkin operators, bottom inverse) is done
once before the timed region and reported separately.  MDOF/s = 3 * nodes of
the active level-0 blocks / solve time / 1e6.  After the timed solves the FP64
session solves again to a relative residual of 1e-12; the displacements and
the compliance f.u of both arms are reported with their relative errors
against that FP64 solution.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Multi-GPU runs (torchrun, one process per GPU) solve an independent replica per
rank: the solve does not shard ("replicas only"), so per-GPU work is fixed.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "MGPCG time & MDOF/s to rel.res 1e-6: mixed-prec vs FP64, same B200"
ACTIVE_NODE = 0x10  # node flag of an active node (solver/Flags.h); DOF = 3 x active nodes
TOL = 1e-6
TIGHT_TOL = 1e-12  # the FP64 solution the errors are measured against
# DRAM bytes (dram__bytes_read.sum + dram__bytes_write.sum) of one level-0 FP32
# sweep (its 8 colour launches) per workload, from ncu captures of this kernel
SWEEP_DRAM_BYTES = {"sphere_shell256": 1.125e9,
                    # captured at 512^3 (1.747 GB for 6.04 M active nodes), scaled to 24.15 M
                    "spheres_band1024": 1.747e9 * 24.15 / 6.04}
L2_BYTES = 126 * 1024 * 1024


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", choices=["shell", "band"], default="band",
                    help="band: 1024^3 narrow band around 8 spheres; shell: 256^3 sphere shell")
    ap.add_argument("--n", type=int, default=None, help="grid size (default 1024 band, 256 shell)")
    ap.add_argument("--bottom-size", type=int, default=None)
    ap.add_argument("--cpu-sample-n", type=int, default=None,
                    help="grid size of the CPU-baseline sample (default 128 band, 64 shell)")
    ap.add_argument("--no-tight", action="store_true", help="skip the tight FP64 solve the errors are measured against")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--profile-iterations", type=int, default=0,
                    help="profiling mode: set up, warm up, then one solve of this many PCG iterations "
                         "between cudaProfilerStart/Stop (for ncu --profile-from-start off); prints stats only")
    ap.add_argument("--profile-setup", action="store_true",
                    help="profiling mode: after one warm-up set-up, one more session set-up (levels, "
                         "operators, bottom solve) between cudaProfilerStart/Stop; prints its wall time only")
    ap.add_argument("--precision", choices=["mixed", "fp64", "reference"], default="mixed",
                    help="precision of the profiled solve or set-up")
    args = ap.parse_args()
    if args.n is None:
        args.n = 256 if args.workload == "shell" else 1024
    if args.cpu_sample_n is None:
        args.cpu_sample_n = 64 if args.workload == "shell" else 128
    if args.bottom_size is None:
        # mg_bottom_size 16, the value of the reference's dense-box configuration
        args.bottom_size = 16
    return args


def workload(n: int, bottom: int, kind: str = "shell"):
    from spgrid_topo_opt_b200 import configs
    if kind == "band":
        return None, configs.spheres_band_inputs(n, bottom_size=bottom, tolerance=TOL)
    prob = configs.sphere_shell(n, bottom_size=bottom)
    inp = configs.to_inputs(prob, tolerance=TOL)
    return prob, inp


def config_dict(args, inp, extra=None, n=None):
    """The workload's description; n names a smaller grid of the same generator
    (the CPU samples)."""
    n = args.n if n is None else n
    common = {"mg_level": int(inp.mg_level), "mg_bottom_size": int(args.bottom_size),
              "smoothing": [int(inp.pre_and_post_smoothing_iter), int(inp.extra_ints["boundary_smoothing"])],
              "tolerance": TOL, "stopping_rule": "L-inf residual <= tol * zero-guess L-inf residual",
              "input_blocks_4x4x4": int(inp.density.base.shape[0]),
              "l2": "flushed (256 MiB write) before every timed solve"}
    if args.workload == "band":
        d = {"workload": f"spheres_band{n}", "grid": [n] * 3,
             "band": "12-voxel shell around the union of 8 seeded spheres (radii 0.1-0.3), seed 7",
             "density": "uniform [1e-3, 1], seeded", **common}
    else:
        d = {"workload": f"sphere_shell{n}", "grid": [n] * 3, "shell_radii": [0.4, 0.5],
             "density": "clamp(0.5+0.3*smoothed uniform noise, 1e-3, 1), seed 1234", **common}
    if extra:
        d.update(extra)
    return d


class ClockSampler:
    """nvidia-smi samples during the timed region (SM clock, throttle reasons)."""

    FIELDS = "index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown," \
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap"

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            threading.Thread(target=self._read, daemon=True).start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.lines:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx.append(float(parts[2]))
            except ValueError:
                continue
            for nm, val in zip(names, parts[5:9]):
                if val.lower() == "active":
                    reasons.add(nm)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx), "reasons": sorted(reasons), "samples": len(sm)}


def measured_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            j = json.load(f)
        return float(j["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def cpu_sample(args):
    """A bounded CPU sample of the workload: the same generator at the smaller
    grid args.cpu_sample_n, with the same mg_bottom_size, solved completely."""
    return workload(args.cpu_sample_n, args.bottom_size, args.workload)[1]


def reference_solver_sample(args, steps, warmup):
    """Time the bounded CPU sample: the reference's own fem_solve (built with GCC
    from the reference sources, oracle/_ref) when it is there, else its CPU
    restatement (the oracle, reference-rounding mode); all host threads.
    Returns (seconds per solve, DOF, iterations, kind, description)."""
    from oracle.oracle import Oracle, MODE_REF
    from oracle.ref_solver import ref_run
    inp = cpu_sample(args)
    cores = os.cpu_count() or 1
    o = Oracle(inp, mode=MODE_REF, tolerance=TOL, threads=cores)
    dof = 3 * int(np.count_nonzero(o.flags(0) & ACTIVE_NODE))
    if ref_run.available("shipped"):
        kind = "reference"
        what = ("the reference's own fem_solve (solver/SPGrid_CPU_Solver.cpp, its AVX2 double configuration, "
                "built with GCC from the reference sources; PARDISO replaced by an exact band Cholesky)")

        def one():
            out, it, _ = ref_run.solve(inp, "shipped")
            if not out.success:
                raise RuntimeError("reference solve failed")
            return it
    else:
        kind = "port"
        what = "the oracle (oracle/spgrid_oracle.cpp, a CPU restatement of the reference solver)"

        def one():
            return o.solve()["iterations"]
    for _ in range(warmup):
        one()
    times, iters = [], []
    for _ in range(steps):
        t0 = time.perf_counter()
        iters.append(one())
        times.append(time.perf_counter() - t0)
    return float(np.mean(times)), dof, int(np.median(iters)), kind, what, cores


def cpu_baseline(args):
    """One complete solve of the bounded sample on the host cores."""
    t, dof, it, kind, what, cores = reference_solver_sample(args, 1, 0)
    name = config_dict(args, cpu_sample(args), n=args.cpu_sample_n)["workload"]
    return {"value": dof / t / 1e6, "unit": "MDOF/s", "cores": cores, "kind": kind,
            "sample": f"one complete solve of {name} ({dof} DOF, {it} iterations, {t:.2f} s, tol {TOL}, "
                      f"mg_bottom_size {args.bottom_size}) by {what}, OMP threads = {cores}"}


def flush_l2(buf):
    if buf is not None:
        buf.fill_(1.0)


def aggregate_replicas(per_step: float, dof: int, world: int, dist=None, device: str = "cuda"):
    """Whole-job throughput of `world` independent replicas: the slowest rank's
    seconds per step (max over ranks) and world x DOF / that time in MDOF/s."""
    if dist is not None and world > 1:
        import torch
        tt = torch.tensor([per_step], dtype=torch.float64, device=device)
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        per_step = float(tt.item())
    return per_step, world * dof / per_step / 1e6


def run_ours(args, rank, world):
    import torch
    from spgrid_topo_opt_b200 import fem_interface as fi
    from spgrid_topo_opt_b200 import native
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=600))
    native.load(build_if_missing=(rank == 0))
    prob, inp = workload(args.n, args.bottom_size, args.workload)
    prec = {"mixed": native.PRECISION_MIXED, "fp64": native.PRECISION_FP64,
            "reference": native.PRECISION_REFERENCE}[args.precision]
    if args.profile_setup:
        with native.Session(inp, precision=prec):  # the process-wide scratch and staging are made here
            pass
        torch.cuda.synchronize()
        torch.cuda.cudart().cudaProfilerStart()
        t0 = time.perf_counter()
        with native.Session(inp, precision=prec):
            torch.cuda.synchronize()
            setup_seconds = time.perf_counter() - t0
            torch.cuda.cudart().cudaProfilerStop()
        return {"profile": True, "setup_seconds": round(setup_seconds, 4)} if rank == 0 else None
    if args.profile_iterations > 0:
        # the per-iteration graph (same kernels as the device-side loop, whose
        # WHILE node the profiler is not asked to walk)
        inp.extra_ints["sgs_device_loop"] = 0
        with native.Session(inp, precision=prec) as ses:
            ses.solve(tolerance=TOL, max_iterations=args.profile_iterations)
            torch.cuda.synchronize()
            torch.cuda.cudart().cudaProfilerStart()
            st = ses.solve(tolerance=TOL, max_iterations=args.profile_iterations)
            torch.cuda.synchronize()
            torch.cuda.cudart().cudaProfilerStop()
        return {"profile": True, "stats": st} if rank == 0 else None
    flush = torch.empty(2 * L2_BYTES // 4, dtype=torch.float32, device="cuda")

    def timed_solves(ses, steps, warmup):
        for _ in range(warmup):
            ses.solve(tolerance=TOL)
        times, iters, launches = [], [], 0
        for _ in range(steps):
            flush_l2(flush)
            torch.cuda.synchronize()
            st = ses.solve(tolerance=TOL)
            times.append(st["solve_device_seconds"])
            iters.append(st["iterations"])
            launches += st["kernel_launches"]
        return times, iters, launches, st

    # mixed precision (the headline) and the FP64 reference arm on the same GPU
    mixed = native.Session(inp, precision=native.PRECISION_MIXED)
    fp64 = native.Session(inp, precision=native.PRECISION_FP64)
    gpu_index = torch.cuda.current_device()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    with ClockSampler(gpu_index) as clocks:
        t_mix, it_mix, launches, st_mix = timed_solves(mixed, args.steps, args.warmup)
        if dist:
            dist.barrier()
    t_64, it_64, _, st_64 = timed_solves(fp64, max(2, args.steps // 2), 1)
    dof = st_mix["dof"]
    per_step, value = aggregate_replicas(float(np.mean(t_mix)), dof, world, dist, "cuda")

    # accuracy of both arms against a tight FP64 solve of the same problem on the
    # same GPU: displacements (L-inf relative) and the compliance f.u
    u_mix, u_64 = mixed.displacements()[..., :3], fp64.displacements()[..., :3]
    accuracy = None
    if not args.no_tight:
        st_t = fp64.solve(tolerance=TIGHT_TOL)
        u_ref = fp64.displacements()[..., :3]
        f_at, f_val = force_layout(inp)
        c_ref, c_mix, c_64 = (compliance(u, f_at, f_val) for u in (u_ref, u_mix, u_64))
        nrm = float(np.abs(u_ref).max())
        accuracy = {"against": f"FP64 MGPCG on the same GPU to relative L-inf residual {TIGHT_TOL:g} "
                               f"({st_t['iterations']} iterations)",
                    "rel_err_u_mixed": float(np.abs(u_mix - u_ref).max() / nrm),
                    "rel_err_u_fp64": float(np.abs(u_64 - u_ref).max() / nrm),
                    "rel_err_u_mixed_vs_fp64": float(np.abs(u_mix - u_64).max() / float(np.abs(u_64).max())),
                    "compliance": c_ref,
                    "rel_err_compliance_mixed": abs(c_mix - c_ref) / abs(c_ref),
                    "rel_err_compliance_fp64": abs(c_64 - c_ref) / abs(c_ref)}

    # dominant kernel: the level-0 smoothing sweep (8 colour launches); its
    # algorithmic bytes per node are u read+write (6w) + b (3w) + E (w) + flags (4 B)
    sweep_ms = mixed.time_op(2, reps=20)
    ku32_ms = mixed.time_op(4, reps=20)
    res32_ms = mixed.time_op(1, reps=20)
    res32tc_ms = mixed.time_op(5, reps=20)
    ku64_ms = mixed.time_op(0, reps=20)
    vcyc_ms = mixed.time_op(3, reps=5)
    nodes = dof // 3
    peak, peak_kind = measured_peaks()
    sweep_bytes = nodes * (10 * 4 + 4)
    achieved = sweep_bytes / (sweep_ms * 1e-3) / 1e9
    # K u: u read and f written (3w each) + the cell's stiffness scale E (w)
    ku32_bytes, ku64_bytes, res32_bytes = nodes * 7 * 4, nodes * 7 * 8, nodes * 10 * 4
    gbs = lambda b, ms: b / (ms * 1e-3) / 1e9
    traffic = SWEEP_DRAM_BYTES.get(config_dict(args, inp)["workload"])
    roofline = {"bound": "hbm", "kernel": "level0 Gauss-Seidel sweep (8 colour launches of gs0_list4_kernel, FP32)",
                "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s", "frac": round(achieved / peak, 4),
                "peak_kind": peak_kind, "traffic": traffic,
                "algorithmic_bytes_per_launch_set": sweep_bytes, "sweep_ms": round(sweep_ms, 4),
                "vcycle_ms": round(vcyc_ms, 4),
                "ku_fp32": {"kernel": "level0_op_kernel<float, K u> (planar fields, CUDA cores)",
                            "ms": round(ku32_ms, 4),
                            "algorithmic_bytes": ku32_bytes, "achieved": round(gbs(ku32_bytes, ku32_ms), 1),
                            "frac": round(gbs(ku32_bytes, ku32_ms) / peak, 4)},
                "residual_fp32": {"kernel": "level0_res4_kernel<float> (the V-cycle's residual, CUDA cores)",
                                  "ms": round(res32_ms, 4),
                                  "algorithmic_bytes": res32_bytes, "achieved": round(gbs(res32_bytes, res32_ms), 1),
                                  "frac": round(gbs(res32_bytes, res32_ms) / peak, 4)},
                "residual_fp32_tensor_cores": {"kernel": "level0_tc_kernel<b - K u> (tcgen05 TF32 hi/lo split, "
                                                         "FP32 result; not the default)",
                                               "ms": round(res32tc_ms, 4), "algorithmic_bytes": res32_bytes,
                                               "achieved": round(gbs(res32_bytes, res32tc_ms), 1),
                                               "frac": round(gbs(res32_bytes, res32tc_ms) / peak, 4)},
                "ku_fp64": {"kernel": "level0_op_kernel<double, PCG matvec>", "ms": round(ku64_ms, 4),
                            "algorithmic_bytes": ku64_bytes, "achieved": round(gbs(ku64_bytes, ku64_ms), 1),
                            "frac": round(gbs(ku64_bytes, ku64_ms) / peak, 4)}}

    # end to end through the drop-in C ABI: serialize on the host, fem_solve (set-up,
    # H2D, solve, D2H), deserialize; mixed precision selected through extra_ints
    e2e_inp = fi.deserialize_inputs(fi.serialize_inputs(inp))
    e2e_inp.extra_ints["sgs_precision"] = native.PRECISION_MIXED
    blob = fi.serialize_inputs(e2e_inp)
    e2e_times, h2d, d2h, phases = [], 0.0, 0.0, {}
    for i in range(0 if args.no_e2e else 2 + max(1, args.steps // 2)):
        t0 = time.perf_counter()
        out = native.fem_solve_outputs(blob)
        dt = time.perf_counter() - t0
        if not out.success:
            raise RuntimeError(out.info)
        if i >= 2:
            e2e_times.append(dt)
            h2d, d2h = out.extra_doubles.get("h2d_bytes", 0), out.extra_doubles.get("d2h_bytes", 0)
            for k in ("decode_seconds", "host_setup_seconds", "host_level0_seconds", "host_coarsen_seconds",
                      "host_flags_seconds", "host_rest_seconds", "device_levels_seconds", "device_operators_seconds",
                      "device_bottom_seconds", "device_vectors_seconds", "solve_seconds", "output_seconds",
                      "teardown_seconds"):
                phases.setdefault(k, []).append(out.extra_doubles.get(k, 0.0))
    e2e_s = float(np.mean(e2e_times)) if e2e_times else float("nan")

    result = None
    if rank == 0:
        cpu = None if (args.no_cpu_baseline or world > 1) else cpu_baseline(args)
        result = {
            "metric": METRIC, "value": round(value, 3), "unit": "MDOF/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(per_step * 1e3, 3), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32 V-cycle / f64 PCG", "data": "synthetic (seeded)",
            "config": config_dict(args, inp, {"dof": int(dof), "iterations_mixed": int(np.median(it_mix)),
                                              "iterations_fp64": int(np.median(it_64)),
                                              "parallelism": "replicas" if world > 1 else "single GPU"}),
            "fp64": {"ms_per_step": round(float(np.mean(t_64)) * 1e3, 3),
                     "value": round(dof / float(np.mean(t_64)) / 1e6, 3), "unit": "MDOF/s",
                     "iterations": int(np.median(it_64))},
            "mixed_over_fp64_speedup": round(float(np.mean(t_64)) / per_step, 3),
            "accuracy": accuracy,
            "setup_seconds": round(st_mix["setup_seconds"], 3),
            "roofline": roofline,
            "cpu_baseline": cpu,
            "e2e": None if args.no_e2e else {"value": round(world * dof / e2e_s / 1e6, 3), "unit": "MDOF/s",
                    "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h),
                    "seconds_per_step": round(e2e_s, 4),
                    "phases_seconds": {k: round(float(np.mean(v)), 4) for k, v in phases.items()},
                    "path": "fem_solve C ABI: decode, set-up, H2D, solve, pack, D2H, encode"},
            "gpu_launches": int(launches),
            "clocks": clocks.summary(),
        }
    mixed.close()
    fp64.close()
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    return result


def force_layout(inp):
    """For each force of the input: the (input block, node) slot of its node in
    the displacement output [nblocks][64] (in-block index i*16 + j*4 + k), or -1
    when no input block holds it; and the force vectors."""
    base = np.asarray(inp.density.base)
    index = {tuple(b): i for i, b in enumerate(base.tolist())}
    slots = []
    for c in np.asarray(inp.forces["coord"]).tolist():
        b = index.get((c[0] & ~3, c[1] & ~3, c[2] & ~3), -1)
        slots.append(-1 if b < 0 else b * 64 + (c[0] & 3) * 16 + (c[1] & 3) * 4 + (c[2] & 3))
    return np.array(slots), np.asarray(inp.forces["f"], dtype=np.float64)


def compliance(u, slots, f):
    """f.u over the forces whose node lies in an input block."""
    flat = u.reshape(-1, 3)
    ok = slots >= 0
    return float((flat[slots[ok]] * f[ok]).sum())


def run_reference(args, rank, world):
    """The reference arm: the reference's own CPU solver (built with GCC from the
    reference sources; its CPU restatement when that build is absent) on the
    host cores, each step one complete solve of a bounded sample of the
    workload (the same generator on a smaller grid)."""
    if rank != 0:
        return None
    inp = cpu_sample(args)
    t, dof, it, kind, what, cores = reference_solver_sample(args, args.steps, args.warmup)
    value = dof / t / 1e6
    cfg = config_dict(args, inp, n=args.cpu_sample_n)
    cfg["sample_of"] = f"spheres_band{args.n}" if args.workload == "band" else f"sphere_shell{args.n}"
    sample = (f"one complete solve of {cfg['workload']} ({dof} DOF, {it} iterations) per step, a bounded sample of "
              f"{cfg['sample_of']}, by {what}, OMP threads = {cores}")
    return {"metric": METRIC, "value": round(value, 4), "unit": "MDOF/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(t * 1e3, 3), "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64 (float-rounded CG updates, as the reference)", "data": "synthetic (seeded)",
            "config": cfg, "impl": "reference",
            "cpu_baseline": {"value": round(value, 4), "unit": "MDOF/s", "cores": cores, "kind": kind,
                             "sample": sample},
            "e2e": {"value": round(value, 4), "unit": "MDOF/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}


def main():
    args = parse()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    if args.impl == "reference":
        res = run_reference(args, rank, world)
    else:
        res = run_ours(args, rank, world)
    if rank == 0 and res is not None:
        print(json.dumps(res))


if __name__ == "__main__":
    main()
