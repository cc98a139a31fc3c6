"""The oracle and the codecs checked against fixtures produced by the reference's
own code (tests/golden/make_golden.py builds the harnesses in oracle/ref_harness
from the reference sources)."""
import gzip
import os

import numpy as np
import pytest

from oracle import oracle as orc
from spgrid_topo_opt_b200 import fem_interface as fi

GOLD = os.path.join(os.path.dirname(__file__), "golden")


def _blob(name):
    with gzip.open(os.path.join(GOLD, name), "rb") as f:
        return f.read()


def test_stiffness_tables_match_reference():
    ref = np.load(os.path.join(GOLD, "stiffness_tables.npy"))
    mu, la = orc.tables()
    assert np.array_equal(ref[0], mu.ravel())
    assert np.array_equal(ref[1], la.ravel())
    # Km_cell[v][w][i][j] == K_mu[i][j][v][w] (Linear_Elasticity_Stiffness_Matrix.h)
    assert np.array_equal(ref[2].reshape(3, 3, 8, 8), mu.transpose(2, 3, 0, 1))
    assert np.array_equal(ref[3].reshape(3, 3, 8, 8), la.transpose(2, 3, 0, 1))


@pytest.mark.parametrize("case", [0, 1, 2])
def test_page_order_matches_reference(case):
    z = np.load(os.path.join(GOLD, "spgrid_order.npz"))
    b, ordered = z[f"bases{case}"], z[f"ordered{case}"]
    keys = orc.page_keys(np.stack([b[:, 0] // 4, b[:, 1] // 4, b[:, 2] // 8], 1))
    assert np.array_equal(b[np.argsort(keys, kind="stable")], ordered)


def test_level_maps_match_reference():
    z = np.load(os.path.join(GOLD, "spgrid_offsets.npz"))
    c = z["coords"]
    # DownsampleOffset<4,4,8>: c = (f + B) >> 1 ; UpsampleOffset<4,4,8>: f = 2c - B
    B = np.array([4, 4, 8])
    assert np.array_equal((c + B) >> 1, z["down"])
    assert np.array_equal(2 * c - B, z["up"])
    # the node offset's page index is the block's page key
    keys = orc.page_keys(np.stack([c[:, 0] // 4, c[:, 1] // 4, c[:, 2] // 8], 1))
    assert np.array_equal(keys, z["offset"] >> np.uint64(14))


def test_python_codec_roundtrips_reference_inputs():
    blob = _blob("kat_inputs.bin.gz")
    p = fi.deserialize_inputs(blob)
    assert fi.serialize_inputs(p) == blob
    # values of the reference's interface test (topo_opt/interface_test.cpp:45-95)
    assert p.resolution == [16, 32, 64] and p.use_density_only
    assert p.dx == np.float32(0.01)
    assert len(p.forces) == 17
    for i, f in enumerate(p.forces):
        assert list(f["coord"]) == [i * 2 + 1, i * i + 14, i // 3 + 1]
        assert list(f["f"]) == [np.sqrt(1.0 * i), i * i, i * i * i / 10000.0]
    assert [list(d["coord"]) + [d["axis"], d["value"]] for d in p.dirichlet_nodes] == [
        [95, 6, 3, 2, 0.1234], [94, 11, 16, 1, 0.5432]]
    assert (p.krylov.tolerance, p.krylov.max_iterations, p.krylov.restart_iterations, p.krylov.print_residuals) == (
        1e-5, 10000, 1000, True)
    assert p.caller_method == "topology_optimization"
    assert p.extra_ints["multigrid_num_pre_smoothing"] == 2
    assert p.extra_strings["log_file_path"] == "/tmp/fem_solver.log"
    assert p.extra_doubles["smoother_jacobi_damping"] == np.float32(0.66667)
    assert p.get_solver_state_ptr() == 0x1234567890543200
    # the reference reader's dump of the same blob
    dump = open(os.path.join(GOLD, "kat_inputs.txt")).read()
    assert f"density res 16 32 64 blocks {p.density.num_blocks}" in dump
    basesum = int((p.density.base[:, 0].astype(np.int64) * 1000003 + p.density.base[:, 1] * 1009 +
                   p.density.base[:, 2]).sum())
    assert f"density basesum {basesum} " in dump


def test_python_codec_roundtrips_reference_outputs():
    blob = _blob("kat_outputs.bin.gz")
    o = fi.deserialize_outputs(blob)
    assert fi.serialize_outputs(o) == blob
    assert list(o.residuals) == [1.0, 0.25, 1e-5] and o.error_code == 7 and o.success
    assert o.displacements.data.shape[1:] == (64, 4)
    dump = open(os.path.join(GOLD, "kat_outputs.txt")).read()
    w = 1 + (np.arange(64)[:, None] + np.arange(4)[None, :]) % 5
    assert "displacements checksum %.17g" % float((o.displacements.data * w).sum()) in dump or \
        abs(float(dump.split("displacements checksum ")[1].split()[0]) - float((o.displacements.data * w).sum())) < 1e-6


def test_codec_rejects_truncated_blob():
    blob = _blob("kat_inputs.bin.gz")
    with pytest.raises(fi.WireFormatError):
        fi.deserialize_inputs(blob[:-10])
