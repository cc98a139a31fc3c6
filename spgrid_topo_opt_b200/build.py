"""Build the CUDA extension libspgrid_gpu_solver.so in-tree for sm_100a.

nvcc compiles the kernels and the host code (C++17) into one shared library that
exports the C ABI of include/spgrid_fem.h.  The library is built next to this
file so it travels with the repository; nothing is installed into site-packages.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libspgrid_gpu_solver.so")
SOURCES = ["solver.cu", "band.cu", "render.cu", "setup.cpp", "wire.cpp"]
# the renderer's ray arithmetic is kept free of fused multiply-adds so that it
# rounds like its float32 restatement in the oracle
FILE_FLAGS = {"render.cu": ["-fmad=false"]}
HEADERS = ["common.cuh", "band.hpp", "kernels.cuh", "setup_kernels.cuh", "tc_kernels.cuh", "topo_kernels.cuh", "setup.hpp", "wire.hpp"]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def host_compiler() -> str:
    # the system g++ (the toolchain wrapper in $CXX lacks OpenMP specs)
    return "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else (shutil.which("g++") or "g++")


def needs_build() -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = [os.path.join(CSRC, f) for f in SOURCES + HEADERS] + [os.path.join(ROOT, "include", "spgrid_fem.h")]
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def build(force: bool = False, verbose: bool = False, extra=()) -> str:
    """Compile every source to an object (in parallel, per-file flags from
    FILE_FLAGS), then link the shared library."""
    if not force and not needs_build():
        return LIB
    import concurrent.futures
    import tempfile
    base = [nvcc(), "-ccbin", host_compiler(), "-std=c++17", "-O3", "-lineinfo",
            "-gencode", "arch=compute_100a,code=sm_100a",
            "-Xcompiler", "-fPIC,-fvisibility=hidden,-fopenmp", "-Xptxas", "-O3",
            "--expt-relaxed-constexpr", *extra]
    with tempfile.TemporaryDirectory() as tmp:
        def compile_one(f):
            obj = os.path.join(tmp, f + ".o")
            cmd = base + FILE_FLAGS.get(f, []) + ["-c", os.path.join(CSRC, f), "-o", obj]
            if verbose:
                print(" ".join(cmd))
            return obj, subprocess.run(cmd, capture_output=True, text=True)
        with concurrent.futures.ThreadPoolExecutor(max_workers=len(SOURCES)) as ex:
            results = list(ex.map(compile_one, SOURCES))
        for _, res in results:
            if res.returncode != 0:
                sys.stderr.write(res.stdout + res.stderr)
                raise RuntimeError("nvcc failed to build libspgrid_gpu_solver.so")
        link = [nvcc(), "-ccbin", host_compiler(), "-shared", "-gencode", "arch=compute_100a,code=sm_100a",
                "-Xcompiler", "-fopenmp", "-o", LIB + ".tmp", *[o for o, _ in results], "-lgomp"]
        if verbose:
            print(" ".join(link))
        res = subprocess.run(link, capture_output=True, text=True)
        if res.returncode != 0:
            sys.stderr.write(res.stdout + res.stderr)
            raise RuntimeError("linking libspgrid_gpu_solver.so failed")
    os.replace(LIB + ".tmp", LIB)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True, extra=[a for a in sys.argv[1:] if a != "--force"]))
