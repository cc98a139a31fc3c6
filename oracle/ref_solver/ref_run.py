"""Run the reference CPU solver's own ``fem_solve`` (test infrastructure).

``oracle/Makefile`` (target ``refsolver``) builds the reference solver library
with GCC into ``oracle/_ref``: ``libspgrid_ref_solver.so`` as shipped (float-
rounded CG updates and V-cycle casts) and ``libspgrid_ref_solver_fp64.so`` with
that rounding switched off.  This module calls its C ABI entry (the same
``fem_solve(void *input, void *output)`` the product replaces,
solver/SPGrid_CPU_Solver.cpp:26) on a serialized ``FEMInputs`` blob, decodes the
output blob, and reads the iteration count and the residual history from the
solver's prints (solver/CG/CONJUGATE_GRADIENT.cpp:34-37, printed with all digits
in this build).  Only the tests, the fixture generator and the benchmark's CPU
legs use it, as the checker and the CPU baseline.
"""
from __future__ import annotations

import ctypes as C
import os
import re
import sys
import tempfile
import threading

HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(os.path.dirname(HERE), "_ref")
LIBS = {"shipped": "libspgrid_ref_solver.so", "fp64": "libspgrid_ref_solver_fp64.so"}
_libs = {}
_lock = threading.Lock()


def available(flavour: str = "shipped") -> bool:
    return os.path.exists(os.path.join(REF_DIR, LIBS[flavour]))


def _load(flavour: str):
    if flavour not in _libs:
        lib = C.CDLL(os.path.join(REF_DIR, LIBS[flavour]))
        lib.fem_solve.argtypes = [C.c_void_p, C.c_void_p]
        lib.fem_solve.restype = None
        lib.ref_free.argtypes = [C.c_void_p]
        _libs[flavour] = lib
    return _libs[flavour]


def solve(inputs, flavour: str = "shipped"):
    """Solve with the reference.  Returns (FEMOutputs, iterations, residual
    history): the history is the L-inf norm before each iteration, the first
    entry the initial residual, as the product's ``residuals`` field."""
    from spgrid_topo_opt_b200 import fem_interface as fi
    lib = _load(flavour)
    inp = fi.deserialize_inputs(fi.serialize_inputs(inputs))
    inp.krylov = fi.KrylovSolverParameters(inp.krylov.tolerance, inp.krylov.max_iterations,
                                           inp.krylov.restart_iterations, True)
    blob = fi.serialize_inputs(inp)
    buf = C.create_string_buffer(blob, len(blob))
    out = C.c_void_p(0)
    with _lock:
        sys.stdout.flush()
        with tempfile.TemporaryFile() as tmp:
            saved = os.dup(1)
            os.dup2(tmp.fileno(), 1)
            try:
                lib.fem_solve(buf, C.byref(out))
                C.CDLL(None).fflush(None)
            finally:
                os.dup2(saved, 1)
                os.close(saved)
            tmp.seek(0)
            text = tmp.read().decode(errors="replace")
    try:
        n = C.c_uint64.from_address(out.value).value
        outputs = fi.deserialize_outputs(C.string_at(out.value, n))
    finally:
        lib.ref_free(out)
    m = re.search(r"initial residual L_inf\s*:\s*\S+\n(.*?)cg (?:iterations: (\d+)|not converged)", text, re.S)
    if not m:
        raise RuntimeError("reference output without a CG log:\n" + text[-2000:])
    history = [float(x) for x in m.group(1).split()]
    iterations = int(m.group(2)) if m.group(2) else len(history) - 1
    return outputs, iterations, history
