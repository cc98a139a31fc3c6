"""The solve cases whose reference outputs are committed in ref_solves.npz.

Each case is a seeded synthetic input built by spgrid_topo_opt_b200.configs
(the tests rebuild it and check its serialized bytes against the stored
digest), solved by the reference's own fem_solve in two builds: as shipped
("shipped": float-rounded CG updates and V-cycle casts) and with that rounding
switched off ("fp64").  Config 0 of the benchmark suite is the 64^3 cantilever
with density 0.1, mg_bottom_size 16 and tolerance 1e-4; spheres_band96 is a
96^3 instance of the narrow-band generator of config 4 (1024^3) at its
tolerance 1e-6.
"""
from __future__ import annotations

import hashlib

from spgrid_topo_opt_b200 import configs, fem_interface as fi

# name: (builder, tolerance of the shipped solve, tolerance of the fp64 solve, full field stored)
CASES = {
    "cantilever16": (lambda: configs.cantilever_box(16, density=(0.2, 1.0), bottom_size=4), 1e-10, 1e-10, True),
    "shell24": (lambda: configs.sphere_shell(24, bottom_size=4), 1e-10, 1e-10, True),
    "config0_box32": (lambda: configs.cantilever_box(32, density=0.1, bottom_size=16), 1e-4, 1e-10, False),
    "config0_box64": (lambda: configs.cantilever_box(64, density=0.1, bottom_size=16), 1e-4, 1e-10, False),
    "shell64": (lambda: configs.sphere_shell(64, bottom_size=16), 1e-6, 1e-10, False),
    # the driver's default mg_bottom_size 64 (spgrid_topo_opt.cpp:1022-1030): one
    # level, the whole problem is the bottom (factored by PARDISO in the reference)
    "cantilever16_bottom64": (lambda: configs.cantilever_box(16, density=(0.2, 1.0), bottom_size=64), 1e-10, 1e-10,
                              True),
    # a narrow band: sparse pages, ghost blocks on every level, partly filled blocks
    "spheres_band96": (lambda: configs.spheres_band_inputs(96, bottom_size=16), 1e-6, 1e-10, False),
}
SAMPLES = 4096  # nodes sampled (seeded) from the displacement field where it is not stored whole


def inputs(name: str, tolerance: float):
    built = CASES[name][0]()
    if isinstance(built, fi.FEMInputs):  # a generator that packs its own inputs
        built.krylov.tolerance = tolerance
        return built
    return configs.to_inputs(built, tolerance=tolerance)


def digest(inp) -> str:
    return hashlib.sha256(fi.serialize_inputs(inp)).hexdigest()
