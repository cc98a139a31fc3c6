"""Host-side pieces of the CUDA library, checked without a GPU: the exported C ABI,
the C++ codec against the reference's golden blobs, the error paths of fem_solve
that fail before any device work, and the host-built hierarchy (page order,
flags, boundary band) against the oracle."""
import gzip
import os
import re

import numpy as np
import pytest

from oracle.oracle import Oracle, MODE_FP64
from spgrid_topo_opt_b200 import configs, native
from spgrid_topo_opt_b200 import fem_interface as fi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLD = os.path.join(ROOT, "tests", "golden")


def test_library_exports_every_declared_symbol(native_lib):
    header = open(os.path.join(ROOT, "include", "spgrid_fem.h")).read()
    declared = set(re.findall(r"SGS_API\s+[\w\s\*]+?\b(\w+)\s*\(", header))
    assert {"fem_solve", "fem_solve_free", "sgs_create", "sgs_apply"} <= declared
    for name in declared:
        assert hasattr(native_lib, name), name
    assert set(native.EXPORTED_SYMBOLS) == declared


@pytest.mark.parametrize("name,which", [("kat_inputs.bin.gz", 0), ("kat_outputs.bin.gz", 1)])
def test_cpp_codec_is_byte_compatible(native_lib, name, which):
    blob = gzip.open(os.path.join(GOLD, name)).read()
    assert native.codec_roundtrip(blob, which) == blob


def _fem_outputs(blob):
    out = fi.deserialize_outputs(native.fem_solve_blob(blob))
    # the in-place decoder must read the same record as the byte-copy path
    direct = native.fem_solve_outputs(blob)
    assert (direct.success, direct.error_code, direct.info) == (out.success, out.error_code, out.info)
    return out


def test_fem_solve_reports_malformed_blob(native_lib):
    blob = bytearray(gzip.open(os.path.join(GOLD, "kat_inputs.bin.gz")).read())
    blob[8] = 9  # version_major
    out = _fem_outputs(bytes(blob))
    assert not out.success and out.error_code == 9 and "malformed" in out.info


def test_fem_solve_rejects_mg_level_two(native_lib):
    inp = configs.to_inputs(configs.cantilever_box(8), mg_level=2)
    out = _fem_outputs(fi.serialize_inputs(inp))
    assert not out.success and out.error_code == 3


def test_fem_solve_rejects_padding_violation(native_lib):
    inp = configs.to_inputs(configs.cantilever_box(8))
    inp.resolution = [24, 24, 24]  # blocks now sit on the upper padding
    out = _fem_outputs(fi.serialize_inputs(inp))
    assert not out.success and out.error_code in (4, 6)


def test_fem_solve_rejects_missing_neighbour_blocks(native_lib):
    inp = configs.to_inputs(configs.cantilever_box(8))
    keep = ~np.all(inp.density.base == inp.density.base.max(axis=0), axis=1)
    inp.density.base = inp.density.base[keep]
    inp.density.data = inp.density.data[keep]
    inp.density.data[:] = np.where(inp.density.data > 0, inp.density.data, 0.1)  # material up to the edge
    out = _fem_outputs(fi.serialize_inputs(inp))
    assert not out.success and out.error_code == 5


def _shuffled_repeated_cantilever():
    """A cantilever whose input blocks come in a seeded random order, a third of
    them twice (the later copy with scaled densities: the last one wins)."""
    inp = configs.to_inputs(configs.cantilever_box(24, density=(0.05, 1.0), bottom_size=4))
    n = inp.density.base.shape[0]
    rng = np.random.default_rng(3)
    perm = rng.permutation(n)
    idx = np.concatenate([perm, perm[: n // 3]])
    inp.density.base = inp.density.base[idx].copy()
    inp.density.data = inp.density.data[idx].copy()
    inp.density.data[n:] *= rng.uniform(0.5, 1.0, size=inp.density.data[n:].shape)
    return inp


@pytest.mark.parametrize("problem", ["cantilever", "shell", "band", "shuffled"])
def test_host_hierarchy_matches_oracle(native_lib, problem):
    """Page order, ghost blocks, flags and band lists of every level, bit for bit:
    the blocks are numbered by parallel passes that must reproduce the serial
    construction's order, which sparse bands (many ghost blocks on every level)
    and shuffled, repeated input blocks exercise."""
    if problem == "band":
        inp = configs.spheres_band_inputs(96, bottom_size=4)
    elif problem == "shuffled":
        inp = _shuffled_repeated_cantilever()
    else:
        prob = configs.cantilever_box(16, bottom_size=4) if problem == "cantilever" else configs.sphere_shell(24, bottom_size=4)
        inp = configs.to_inputs(prob)
    ref = Oracle(inp, mode=MODE_FP64)
    ses = native.Session(inp, precision=native.HOST_SETUP_ONLY)
    assert ses.levels == ref.levels
    for lev in range(ref.levels):
        assert np.array_equal(ses.blocks(lev), ref.blocks(lev)), lev
        assert np.array_equal(ses.flags(lev), ref.flags(lev)), lev
        assert np.array_equal(ses.boundary_blocks(lev), ref.boundary_blocks(lev)), lev


def test_small_band_keeps_material_inside_the_box(native_lib):
    """At 64^3 the 12-voxel band reaches the box's faces, so the generator adds
    node blocks one past the last block index; none may carry material (a
    material cell there would need pages beyond the grid)."""
    inp = configs.spheres_band_inputs(64, bottom_size=4)
    blk = (inp.density.base - configs.PADDING) // 4
    outside = (blk >= 64 // 4).any(axis=1)
    assert outside.any()
    assert not (inp.density.data.reshape(len(blk), -1)[outside] > 0).any()
    ses = native.Session(inp, precision=native.HOST_SETUP_ONLY)
    assert ses.levels >= 2
    ses.close()


def test_host_hierarchy_on_recycled_buffers(native_lib):
    """Host buffers of 8 MiB and more go back to a process-wide cache when
    released and come out of it with their old contents.  A 256^3 band
    (21354 level-0 blocks: its density records, stiffness scales and level-0
    flags are above 8 MiB) is set up, then a decoy with the same blocks and
    other densities (a tenth of the cells empty) is set up and released, and
    the band is set up again on the decoy's buffers: every level must come out
    as the first time."""
    inp = configs.spheres_band_inputs(256, bottom_size=8)

    def hierarchy(inputs):
        ses = native.Session(inputs, precision=native.HOST_SETUP_ONLY)
        try:
            return [(ses.blocks(lev), ses.flags(lev), ses.boundary_blocks(lev)) for lev in range(ses.levels)]
        finally:
            ses.close()

    first = hierarchy(inp)
    decoy = fi.deserialize_inputs(fi.serialize_inputs(inp))
    rng = np.random.default_rng(11)
    decoy.density.data = decoy.density.data * rng.uniform(0.3, 0.9, size=decoy.density.data.shape)
    decoy.density.data[rng.random(decoy.density.data.shape) < 0.1] = 0.0
    decoyed = hierarchy(decoy)
    assert any(not np.array_equal(a[1], b[1]) for a, b in zip(first, decoyed))  # the decoy's flags differ
    again = hierarchy(inp)
    assert len(again) == len(first)
    for lev, (a, b) in enumerate(zip(first, again)):
        for x, y in zip(a, b):
            assert np.array_equal(x, y), lev


# ---- host-injected failures (the reference's abort/throw sites,
# solver/CG/CG_SYSTEM.cpp:59-74 and solver/CG/CONJUGATE_GRADIENT.cpp:49-52): each one is caught on
# the host before any device work and comes back as success = 0 with a code
@pytest.mark.parametrize("bad", [np.nan, np.inf])
def test_fem_solve_rejects_non_finite_force(native_lib, bad):
    inp = configs.to_inputs(configs.cantilever_box(8))
    inp.forces["f"][0, 1] = bad
    out = _fem_outputs(fi.serialize_inputs(inp))
    assert not out.success and out.error_code == 4 and "non-finite force" in out.info


def test_fem_solve_rejects_non_finite_dirichlet_value(native_lib):
    inp = configs.to_inputs(configs.cantilever_box(8))
    inp.dirichlet_nodes["value"][3] = np.nan
    out = _fem_outputs(fi.serialize_inputs(inp))
    assert not out.success and out.error_code == 4 and "non-finite Dirichlet" in out.info


def test_negative_and_nan_density_cells_are_empty(native_lib):
    """The reference stores material only where density > 0
    (SPGrid_CPU_Solver.cpp:123-129): a negative or NaN density leaves the cell
    empty, exactly as 0 does, so the hierarchy and its flags are those of the
    zero-density input."""
    prob = configs.cantilever_box(16, density=(0.2, 1.0), bottom_size=4)
    zero = prob.density.copy()
    zero[10:14, 4:9, 2:6] = 0.0
    ref = native.Session(configs.to_inputs(configs.Problem(**{**prob.__dict__, "density": zero})),
                         precision=native.HOST_SETUP_ONLY)
    for fill in (-0.5, np.nan):
        rho = prob.density.copy()
        rho[10:14, 4:9, 2:6] = fill
        ses = native.Session(configs.to_inputs(configs.Problem(**{**prob.__dict__, "density": rho})),
                             precision=native.HOST_SETUP_ONLY)
        assert ses.levels == ref.levels
        for lev in range(ref.levels):
            assert np.array_equal(ses.blocks(lev), ref.blocks(lev)), (fill, lev)
            assert np.array_equal(ses.flags(lev), ref.flags(lev)), (fill, lev)


def test_levels_below_a_large_bottom_leave_the_v_cycle_levels_unchanged(native_lib):
    """A bottom above the dense limit gets further levels for its inner solve;
    the V-cycle's own levels (mg_level of them) stay as the reference builds
    them."""
    prob = configs.cantilever_box(16, density=(0.2, 1.0), bottom_size=64)
    inp = configs.to_inputs(prob)
    assert inp.mg_level == 1
    plain = native.Session(inp, precision=native.HOST_SETUP_ONLY)
    inp.extra_ints["sgs_dense_bottom_max"] = 1000
    deep = native.Session(inp, precision=native.HOST_SETUP_ONLY)
    assert plain.levels == 1 and deep.levels > 1
    assert np.array_equal(plain.blocks(0), deep.blocks(0))
    assert np.array_equal(plain.flags(0), deep.flags(0))
    ref = Oracle(configs.to_inputs(configs.cantilever_box(16, density=(0.2, 1.0), bottom_size=4)), mode=MODE_FP64)
    for lev in range(1, deep.levels):  # the same coarsening rule as the reference's levels
        assert np.array_equal(deep.blocks(lev), ref.blocks(lev)), lev
        assert np.array_equal(deep.flags(lev), ref.flags(lev)), lev
