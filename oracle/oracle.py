"""ctypes wrapper of the oracle (test infrastructure only).

The oracle is a CPU restatement of the reference solver path (see
spgrid_oracle.cpp).  tests/, ``__graft_entry__.smoke()`` and the CPU-baseline
leg of bench.py use it as the checker; the product never imports it.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from typing import Optional

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")

MODE_REF, MODE_FP64 = 0, 1

OP_KU, OP_RESIDUAL, OP_SMOOTH, OP_RESTRICT, OP_PROLONG, OP_STENCIL, OP_BOTTOM, OP_VCYCLE = range(8)


class OracleParams(C.Structure):
    _fields_ = [("resolution", C.c_int32 * 3), ("mg_level", C.c_int32), ("dx", C.c_double),
                ("global_mu", C.c_double), ("global_lambda", C.c_double), ("penalty", C.c_double),
                ("minimum_stiffness", C.c_double), ("minimum_density", C.c_double), ("tolerance", C.c_double),
                ("smoothing_iter", C.c_int32), ("boundary_smoothing", C.c_int32), ("max_iterations", C.c_int32),
                ("mode", C.c_int32), ("explicit_level", C.c_int32), ("num_threads", C.c_int32)]


_lib = None


def build() -> str:
    subprocess.run(["make", "-s", "-C", HERE, "oracle"], check=True)
    return LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = C.CDLL(LIB_PATH)
        P = C.c_void_p
        L.oracle_create.restype = P
        L.oracle_create.argtypes = [C.POINTER(OracleParams), C.c_int, P, P, C.c_int, P, P, C.c_int, P, P, P,
                                    C.POINTER(C.c_int), C.c_char_p, C.c_int]
        L.oracle_destroy.argtypes = [P]
        L.oracle_levels.argtypes = [P]
        L.oracle_level_blocks.argtypes = [P, C.c_int, P]
        L.oracle_level_size.argtypes = [P, C.c_int, P]
        L.oracle_boundary_blocks.argtypes = [P, C.c_int, P]
        L.oracle_get_flags.argtypes = [P, C.c_int, P]
        L.oracle_get_material.argtypes = [P, P, P]
        L.oracle_apply.argtypes = [P, C.c_int, C.c_int, C.c_int, P, P, P]
        L.oracle_get_stencils.argtypes = [P, C.c_int, P, P]
        L.oracle_solve.argtypes = [P, P, P, P, C.c_int, C.c_char_p, C.c_int]
        L.oracle_tables.argtypes = [P, P]
        L.oracle_page_keys.argtypes = [C.c_int, P, P]
        L.oracle_sensitivity.restype = C.c_double
        L.oracle_sensitivity.argtypes = [P, P, P, P]
        _lib = L
    return _lib


def _ptr(a: Optional[np.ndarray]):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


class OracleError(RuntimeError):
    pass


class Oracle:
    """One FEM problem set up the way the reference solver sets it up."""

    def __init__(self, inputs, mode: int = MODE_REF, max_iterations: int = 500,
                 tolerance: Optional[float] = None, threads: int = 0):
        L = lib()
        self.inputs = inputs
        p = OracleParams()
        p.resolution[:] = [int(v) for v in inputs.resolution]
        p.mg_level = int(inputs.mg_level)
        p.dx = inputs.dx
        p.global_mu, p.global_lambda = inputs.global_mu, inputs.global_lambda
        p.penalty = inputs.extra_doubles.get("penalty", 0.0)
        p.minimum_stiffness = inputs.extra_doubles.get("minimum_stiffness", 0.0)
        p.minimum_density = inputs.extra_doubles.get("minimum_density", 0.0)
        p.tolerance = inputs.krylov.tolerance if tolerance is None else tolerance
        p.smoothing_iter = inputs.pre_and_post_smoothing_iter
        p.boundary_smoothing = inputs.extra_ints.get("boundary_smoothing", 5)
        p.max_iterations = max_iterations
        p.mode = mode
        p.explicit_level = 2
        p.num_threads = threads
        self.params = p
        base = np.ascontiguousarray(inputs.density.base, np.int32)
        dens = np.ascontiguousarray(inputs.density.data, np.float64)
        fc = np.ascontiguousarray(inputs.forces["coord"], np.int32)
        fv = np.ascontiguousarray(inputs.forces["f"], np.float64)
        dc = np.ascontiguousarray(inputs.dirichlet_nodes["coord"], np.int32)
        da = np.ascontiguousarray(inputs.dirichlet_nodes["axis"], np.int32)
        dv = np.ascontiguousarray(inputs.dirichlet_nodes["value"], np.float64)
        st = C.c_int(0)
        err = C.create_string_buffer(256)
        self.h = L.oracle_create(C.byref(p), base.shape[0], _ptr(base), _ptr(dens), len(fc), _ptr(fc), _ptr(fv),
                                 len(dc), _ptr(dc), _ptr(da), _ptr(dv), C.byref(st), err, 256)
        self.status = st.value
        self.error = err.value.decode()
        if self.status != 0:
            raise OracleError(f"oracle setup failed ({self.status}): {self.error}")

    def __del__(self):
        if getattr(self, "h", None):
            lib().oracle_destroy(self.h)
            self.h = None

    @property
    def levels(self) -> int:
        return lib().oracle_levels(self.h)

    def blocks(self, level: int) -> np.ndarray:
        n = lib().oracle_level_blocks(self.h, level, None)
        out = np.zeros((n, 3), np.int32)
        lib().oracle_level_blocks(self.h, level, _ptr(out))
        return out

    def level_size(self, level: int):
        out = np.zeros(3, np.int32)
        lib().oracle_level_size(self.h, level, _ptr(out))
        return out

    def boundary_blocks(self, level: int) -> np.ndarray:
        n = lib().oracle_boundary_blocks(self.h, level, None)
        out = np.zeros(n, np.int32)
        lib().oracle_boundary_blocks(self.h, level, _ptr(out))
        return out

    def flags(self, level: int) -> np.ndarray:
        n = self.blocks(level).shape[0]
        out = np.zeros(n * 128, np.uint32)
        lib().oracle_get_flags(self.h, level, _ptr(out))
        return out

    def material(self):
        n = self.blocks(0).shape[0]
        mu = np.zeros(n * 128)
        la = np.zeros(n * 128)
        lib().oracle_get_material(self.h, _ptr(mu), _ptr(la))
        return mu, la

    def apply(self, op: int, level: int, x: np.ndarray, x2: Optional[np.ndarray] = None, arg: int = 0,
              out_level: Optional[int] = None) -> np.ndarray:
        ol = level if out_level is None else out_level
        n = self.blocks(ol).shape[0] * 128
        out = np.zeros((3, n))
        x = np.ascontiguousarray(x, np.float64)
        x2 = None if x2 is None else np.ascontiguousarray(x2, np.float64)
        rc = lib().oracle_apply(self.h, op, level, arg, _ptr(x), _ptr(x2), _ptr(out))
        if rc != 0:
            raise OracleError(f"oracle_apply({op}) failed: {rc}")
        return out

    def stencils(self, level: int):
        n = self.blocks(level).shape[0] * 128
        out = np.zeros((n, 243))
        fl = np.zeros(n, np.uint32)
        if lib().oracle_get_stencils(self.h, level, _ptr(out), _ptr(fl)) != 0:
            raise OracleError("no stencils on this level")
        return out, fl

    def solve(self):
        nb = self.inputs.density.base.shape[0]
        disp = np.zeros((nb, 64, 4))
        stats = np.zeros(3)
        hist = np.zeros(600)
        err = C.create_string_buffer(256)
        rc = lib().oracle_solve(self.h, _ptr(disp), _ptr(stats), _ptr(hist), 600, err, 256)
        it = int(stats[0])
        return {"status": rc, "error": err.value.decode(), "displacements": disp, "iterations": it,
                "initial_residual": stats[1], "final_residual": stats[2], "history": hist[:it + 1].copy()}

    def sensitivity(self):
        nb = self.inputs.density.base.shape[0]
        dens = np.ascontiguousarray(self.inputs.density.data, np.float64)
        dc = np.zeros((nb, 64))
        s = np.zeros((nb, 64))
        obj = lib().oracle_sensitivity(self.h, _ptr(dens), _ptr(dc), _ptr(s))
        return obj, dc, s


def tables():
    mu = np.zeros((8, 8, 3, 3))
    la = np.zeros((8, 8, 3, 3))
    lib().oracle_tables(_ptr(mu), _ptr(la))
    return mu, la


def page_keys(block_ijk: np.ndarray) -> np.ndarray:
    b = np.ascontiguousarray(block_ijk, np.int32)
    out = np.zeros(b.shape[0], np.uint64)
    lib().oracle_page_keys(b.shape[0], _ptr(b), _ptr(out))
    return out
