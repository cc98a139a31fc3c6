"""Prepare the reference CPU solver for GCC (test infrastructure).

The reference's solver library (solver/ + external/SPGrid/ + the interface
headers of topo_opt/) is written for the Intel compiler and MKL: GCC rejects its
explicit specialisations without ``template<>``, its dependent member templates
without the ``template`` disambiguator, a local variable that shadows a
template parameter, and a never-instantiated function that names an undeclared
``omega``.  This script copies those sources, unchanged apart from the
mechanical patch below (plus a compile-time switch for the float rounding and
full-precision residual prints, both for the tests), into a build folder that is not committed
(``oracle/_ref/src``); ``oracle/Makefile`` then compiles them with
``oracle/ref_solver/ref_support.cpp`` (an exact SPD solve behind the
``pardiso_64`` calling convention, replacing MKL PARDISO) into
``oracle/_ref/libspgrid_ref_solver.so``.  Nothing of the copy is shipped or
committed; it exists to produce reference outputs for the parity tests.

    python prepare.py <reference tree> <output folder>

Every patch line states the file glob, the regular expression, the replacement
and the smallest number of matches expected, so a change in the reference tree
shows up as an error instead of a silently different build.
"""
from __future__ import annotations

import glob
import os
import re
import shutil
import sys

# the source folders the solver library needs
TREES = ["solver", "external/SPGrid"]
FILES = ["topo_opt/fem_interface.h", "topo_opt/serialization.h"]

PATCH = [
    # ICC accepts explicit specialisations written without template<>
    ("external/SPGrid/Tools/SPGrid_SIMD_Utilities.h", r"^(struct|class)(\s+\w+\s*<)", r"template<> \1\2", 16),
    ("solver/MG/Linear_Elasticity_SIMD_Cell_Multiply.h", r"^(struct|class)(\s+\w+\s*<)", r"template<> \1\2", 4),
    ("solver/MG/Trilinear_Cell_Transfer_Operators_SIMD.h", r"^(struct|class)(\s+\w+\s*<)", r"template<> \1\2", 4),
    # member templates of dependent types need the template disambiguator
    ("**/*.[hc]*", r"::(?<!template )(Packed_Offset\w*)<", r"::template \1<", 0),
    ("**/*.[hc]*", r"(?<!template )\b(\w+)\.operator\(\)<", r"\1.template operator()<", 0),
    # a local named d shadows the template parameter d
    ("solver/CG/CG_VECTOR.cpp", r"\bauto d = ", "auto d_arr = ", 2),
    ("solver/CG/CG_VECTOR.cpp", r"\bd\(offset\)", "d_arr(offset)", 4),
    # Correction::Run (never instantiated) uses an omega it does not declare
    ("solver/CPU_Kernels/Correction.h", r"(const T Struct_Type::\* const d_fields\[6\])\)", r"\1, T omega = T(1))", 1),
    # test toggle: SGS_REF_FLOAT_ROUNDING (compiler definition, true as shipped)
    # switches the float rounding of the CG updates (SPGrid_CPU_Solver.cpp:164-168)
    # and of the V-cycle's Cast_To_Float (Multigrid_Hierarchy.h:439-451), so that
    # a plain FP64 build of the same code exists for tight parity checks
    ("solver/SPGrid_CPU_Solver.cpp", r"\b(\w)\.using_float = true;", r"\1.using_float = SGS_REF_FLOAT_ROUNDING;", 5),
    ("solver/MG/Multigrid_Hierarchy.h", r"float tmp = d\(offset\);\s*d\(offset\) = tmp;",
     "if (SGS_REF_FLOAT_ROUNDING) { float tmp = d(offset); d(offset) = tmp; }", 1),
    # residual prints with all digits (the harness reads the residual history from them)
    ("solver/SPGrid_CPU_Solver.cpp", r'extern "C" void fem_solve\(void \*input, void \*output\) \{',
     r"\g<0> std::cout.precision(17);", 1),
]


def main(ref: str, out: str) -> None:
    if os.path.isdir(out):
        shutil.rmtree(out)
    for t in TREES:
        shutil.copytree(os.path.join(ref, t), os.path.join(out, t))
    for f in FILES:
        os.makedirs(os.path.dirname(os.path.join(out, f)), exist_ok=True)
        shutil.copy(os.path.join(ref, f), os.path.join(out, f))
    for pattern, regex, repl, at_least in PATCH:
        total = 0
        for path in glob.glob(os.path.join(out, pattern), recursive=True):
            if not os.path.isfile(path):
                continue
            with open(path, encoding="latin-1") as fh:
                text = fh.read()
            new, n = re.subn(regex, repl, text, flags=re.M)
            if n:
                with open(path, "w", encoding="latin-1") as fh:
                    fh.write(new)
            total += n
        if total < at_least:
            raise SystemExit(f"patch {regex!r} on {pattern} matched {total} times, expected at least {at_least}")


if __name__ == "__main__":
    main(sys.argv[1], sys.argv[2])
