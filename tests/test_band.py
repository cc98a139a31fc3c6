"""Narrow-band page maps of the optimizer driver (thin / fat / fatter,
fraction_to_keep, isolated-block filter; topo_opt/spgrid_topo_opt.cpp:92-241,
1404-1510): the oracle against the reference's block order and hand-made cases
on the CPU, the GPU band against the oracle.
"""
import os

import numpy as np
import pytest

from oracle import topo_oracle as torc

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
PAD = 8


def container(shape=(60, 40, 48), seed=0, islands=True, pruned=0.3, force=True):
    """An ellipsoidal container (cells) in a padded grid, plus a small island.
    Densities are uniform in (0, 1]; a fraction ``pruned`` of the blocks is set
    to 1e-9 so that the thin map drops them.  Returns base, resolution, flags,
    density in the FEMInputs block layout."""
    rng = np.random.default_rng(seed)
    nx, ny, nz = shape
    x, y, z = np.meshgrid(np.arange(nx) + 0.5, np.arange(ny) + 0.5, np.arange(nz) + 0.5, indexing="ij")
    inside = ((x - nx / 2) / (nx / 2)) ** 2 + ((y - ny / 2) / (ny / 2)) ** 2 + ((z - nz / 2) / (nz / 2)) ** 2 <= 1
    if islands:
        inside[1:4, 1:4, 1:4] = True   # a few cells in a corner: an island of one block
    bx, by, bz = (nx + 3) // 4 + 1, (ny + 3) // 4 + 1, (nz + 3) // 4 + 1
    pad = np.zeros((bx * 4, by * 4, bz * 4), bool)
    pad[:nx, :ny, :nz] = inside
    occ = pad.reshape(bx, 4, by, 4, bz, 4).any(axis=(1, 3, 5))
    bidx = np.argwhere(occ)
    bidx = bidx[rng.permutation(len(bidx))]          # any caller order
    base = (bidx * 4 + PAD).astype(np.int32)
    cells = pad.reshape(bx, 4, by, 4, bz, 4).transpose(0, 2, 4, 1, 3, 5)[bidx[:, 0], bidx[:, 1], bidx[:, 2]]
    cells = cells.reshape(-1, 64)
    flags = np.where(cells, torc.CELL_INSIDE, 0).astype(np.uint8)
    dens = np.where(cells, rng.uniform(1e-3, 1.0, cells.shape), 0.0)
    low = rng.random(len(base)) < pruned
    dens[low] = np.where(cells[low], 1e-9, 0.0)
    if force:
        top = np.argmax(base[:, 1])
        flags[top, :] |= torc.CELL_FORCE
        dens[top] = np.where(cells[top], 1e-9, 0.0)   # kept thin by its force alone
    res = np.array([PAD + nx + 6 * PAD, PAD + ny + 6 * PAD, PAD + nz + 6 * PAD], np.int32)
    return base, res, flags, dens


# ---------------------------------------------------------------- CPU (oracle)
def test_driver_block_order_matches_reference():
    d = np.load(os.path.join(GOLDEN, "driver_order.npz"))
    for c in range(2):
        b = d[f"bases{c}"]
        got = b[np.argsort(torc.driver_page_keys(b // 4), kind="stable")]
        assert np.array_equal(got, d[f"ordered{c}"])


def test_oracle_island_and_fat_closure():
    base, res, flags, dens = container(pruned=0.0, force=False)
    thin, fat, fatter, st = torc.update_page_maps(base, dens, flags, np.ones(len(base), bool))
    corner = np.nonzero((base == PAD).all(axis=1))[0]
    assert len(corner) == 1 and not thin[corner[0]]          # the island is filtered out
    assert st["components"] == 2 and st["thin_blocks"] == st["thin_before_pruning"] - 1
    assert np.all(fat[thin]) and np.all(fatter[fat])           # thin <= fat <= fatter here
    # fatter = fat plus every +1 neighbour (in the container) of a fat block
    where = {tuple(b): i for i, b in enumerate(base)}
    exp = fat.copy()
    for i in np.nonzero(fat)[0]:
        for o in np.array([[a, b, c] for a in (0, 4) for b in (0, 4) for c in (0, 4)]):
            j = where.get(tuple(base[i] + o))
            if j is not None:
                exp[j] = True
    assert np.array_equal(exp, fatter)


def test_oracle_force_keeps_a_block_and_threshold_is_inclusive():
    base = np.array([[8, 8, 8], [12, 8, 8], [16, 8, 8]], np.int32)
    flags = np.full((3, 64), torc.CELL_INSIDE, np.uint8)
    dens = np.full((3, 64), 0.5)
    dens[1] = 0.0
    dens[1, 0] = 0.25                      # density_max == minimum_density + active_threshold: kept
    dens[2] = 0.0
    flags[2, 5] |= torc.CELL_FORCE         # kept by the force
    thin, fat, fatter, st = torc.update_page_maps(base, dens, flags, np.ones(3, bool), minimum_density=0.25 - 1e-6,
                                                  connectivity_filtering=False)
    assert thin.tolist() == [True, True, True]
    thin, *_ = torc.update_page_maps(base, dens, flags, np.ones(3, bool), minimum_density=0.25,
                                     connectivity_filtering=False)
    assert thin.tolist() == [True, False, True]
    # a block outside the previous fat map never becomes thin
    thin, *_ = torc.update_page_maps(base, dens, flags, np.array([True, True, False]), connectivity_filtering=False)
    assert thin.tolist() == [True, True, False]


def test_oracle_stops_where_the_reference_stops():
    base, res, flags, dens = container(islands=False, pruned=0.0, force=False)
    # two halves of equal size: two components above 30%
    cut = base[:, 0] == np.median(np.unique(base[:, 0]))
    dens2 = dens.copy()
    dens2[cut] = np.where(dens[cut] > 0, 1e-9, 0.0)
    with pytest.raises(torc.PageMapError):
        torc.update_page_maps(base, dens2, flags, np.ones(len(base), bool))
    with pytest.raises(torc.PageMapError):
        torc.update_page_maps(base, np.zeros_like(dens), flags, np.ones(len(base), bool))


# ---------------------------------------------------------------- GPU
def _compare(band, ref, st):
    thin, fat, fatter = band.maps()
    t, f, ff, rst = ref
    assert np.array_equal(thin, t)
    assert np.array_equal(fat, f)
    assert np.array_equal(fatter, ff)
    for k in ("thin_before_pruning", "thin_blocks", "fat_blocks", "fatter_blocks", "components", "active_voxels"):
        assert st[k] == rst[k], k


@pytest.mark.gpu
def test_band_updates_match_oracle(native_lib):
    from spgrid_topo_opt_b200 import native
    base, res, flags, dens = container(seed=1)
    band = native.Band(base, res, flags, dens)
    fat_prev = np.ones(len(base), bool)
    rng = np.random.default_rng(5)
    for step in range(3):
        st = band.update()
        ref = torc.update_page_maps(base, dens, flags, fat_prev)
        _compare(band, ref, st)
        assert st["fat_changed"] == int(np.count_nonzero(ref[1] != fat_prev))
        fat_prev = ref[1]
        # the design moves: some blocks fade, others regain material
        fade = rng.random(len(base)) < 0.1
        dens = np.where(flags & torc.CELL_INSIDE, dens, 0.0)
        dens[fade] = np.where(dens[fade] > 0, 1e-9, 0.0)
        band.set_density(dens)
    assert np.array_equal(band.density(), dens)
    band.close()


@pytest.mark.gpu
@pytest.mark.parametrize("margin", [0, 2, 4])
def test_band_fat_margin(native_lib, margin):
    from spgrid_topo_opt_b200 import native
    base, res, flags, dens = container(seed=2)
    band = native.Band(base, res, flags, dens)
    st = band.update(fat_margin=margin, active_threshold=0.5)
    _compare(band, torc.update_page_maps(base, dens, flags, np.ones(len(base), bool), fat_margin=margin,
                                         active_threshold=0.5), st)
    band.close()


@pytest.mark.gpu
def test_band_fraction_to_keep(native_lib):
    from spgrid_topo_opt_b200 import native
    base, res, flags, dens = container(seed=3, pruned=0.5)
    n = len(base)
    fat_prev = np.random.default_rng(4).random(n) < 0.9
    thin0, *_ = torc.update_page_maps(base, dens, flags, fat_prev, connectivity_filtering=False)
    frac = (thin0.sum() + 0.25 * (fat_prev.sum() - thin0.sum())) / n   # between the thin and fat counts
    band = native.Band(base, res, flags, dens)
    band.set_fat(fat_prev)
    st = band.update(fraction_to_keep=frac, connectivity_filtering=False)
    ref = torc.update_page_maps(base, dens, flags, fat_prev, fraction_to_keep=frac, connectivity_filtering=False)
    _compare(band, ref, st)
    assert st["thin_blocks"] != st["thin_before_pruning"]
    band.close()


@pytest.mark.gpu
def test_band_errors_leave_maps_unchanged(native_lib):
    from spgrid_topo_opt_b200 import native
    base, res, flags, dens = container(seed=6, islands=False, pruned=0.0, force=False)
    band = native.Band(base, res, flags, dens)
    band.update()
    before = band.maps()
    cut = base[:, 0] == np.median(np.unique(base[:, 0]))
    dens2 = dens.copy()
    dens2[cut] = np.where(dens[cut] > 0, 1e-9, 0.0)
    band.set_density(dens2)
    with pytest.raises(native.SolverError) as e:
        band.update()
    assert e.value.code == 1
    after = band.maps()
    assert all(np.array_equal(a, b) for a, b in zip(before, after))
    with pytest.raises(native.SolverError):
        band.update(fat_margin=5)
    band.set_density(np.zeros_like(dens))
    with pytest.raises(native.SolverError):
        band.update()
    band.close()
    with pytest.raises(native.SolverError):
        native.Band(base + 1, res, flags, dens)


# ---------------------------------------------------------------- voxel filter (CPU, oracle)
def _row(cells_per_block):
    """Three blocks in a row along x; cells_per_block[b] lists the inside cells of block b."""
    base = np.array([[8, 8, 8], [12, 8, 8], [16, 8, 8]], np.int32)
    flags = np.zeros((3, 64), np.uint8)
    for b, cells in enumerate(cells_per_block):
        flags[b, cells] = torc.CELL_INSIDE
    dens = np.where(flags != 0, 0.5, 0.0)
    return base, flags, dens


def test_oracle_voxel_filter_removes_a_small_island():
    # block 0 full; block 2 holds one cell that touches nothing
    base, flags, dens = _row([list(range(64)), [], [21]])
    f, d, st = torc.filter_isolated_voxels(base, dens, flags, np.ones(3, bool))
    assert st == {"voxels": 65, "components": 2, "kept": 64, "removed": 1}
    assert f[2, 21] == 0 and d[2, 21] == 0.0
    assert np.array_equal(f[:2], flags[:2]) and np.array_equal(d[:2], dens[:2])


def test_oracle_voxel_filter_crosses_block_faces_but_not_edges():
    # cell (3, 1, 1) of block 0 and (0, 1, 1) of block 1 share a face: one component
    e_hi, e_lo = 3 * 16 + 1 * 4 + 1, 0 * 16 + 1 * 4 + 1
    base, flags, dens = _row([list(range(64)), [e_lo], []])
    _, _, st = torc.filter_isolated_voxels(base, dens, flags, np.ones(3, bool))
    assert st["components"] == 1 and st["removed"] == 0
    # (0, 2, 2) touches (3, 1, 1) only along an edge: a second component, removed
    base, flags, dens = _row([list(range(64)), [0 * 16 + 2 * 4 + 2], []])
    flags[0, 3 * 16 + 2 * 4 + 2] = 0
    flags[0, 3 * 16 + 1 * 4 + 2] = 0
    flags[0, 3 * 16 + 2 * 4 + 1] = 0
    f, _, st = torc.filter_isolated_voxels(base, dens, flags, np.ones(3, bool))
    assert st["components"] == 2 and st["removed"] == 1 and f[1].sum() == 0


def test_oracle_voxel_filter_only_searches_thin_blocks():
    base, flags, dens = _row([list(range(64)), [], [21]])
    f, d, st = torc.filter_isolated_voxels(base, dens, flags, np.array([True, True, False]))
    assert st["components"] == 1 and st["voxels"] == 64
    assert np.array_equal(f, flags) and np.array_equal(d, dens)


def test_oracle_voxel_filter_stops_where_the_reference_stops():
    base, flags, dens = _row([list(range(32)), [], list(range(32))])     # two halves of 50%
    with pytest.raises(torc.PageMapError):
        torc.filter_isolated_voxels(base, dens, flags, np.ones(3, bool))
    # four pieces of 25%: none above 30%
    base, flags, dens = _row([[0, 63], [], [0, 63]])
    with pytest.raises(torc.PageMapError):
        torc.filter_isolated_voxels(base, dens, flags, np.ones(3, bool))
    base, flags, dens = _row([[], [], []])
    with pytest.raises(torc.PageMapError):
        torc.filter_isolated_voxels(base, dens, flags, np.ones(3, bool))


def test_oracle_kill_below_keeps_density_and_nan():
    flags = np.full((1, 64), torc.CELL_INSIDE | torc.CELL_FORCE, np.uint8)
    flags[0, 7] = 0
    dens = np.full((1, 64), 0.9)
    dens[0, :4] = 0.1
    dens[0, 4] = np.nan
    dens[0, 7] = 0.0
    f, k = torc.kill_below(dens, flags, 0.5)
    assert k == 4
    assert f[0, :4].tolist() == [torc.CELL_FORCE] * 4 and f[0, 4] == flags[0, 4] and f[0, 7] == 0


# ---------------------------------------------------------------- voxel filter (GPU)
def _voxel_islands(flags, base):
    """Clear the 26 neighbours of one inside cell per chosen block so that it is
    an island (cells of other blocks are not touched, so some may stay connected
    across a face)."""
    out = flags.copy()
    rng = np.random.default_rng(11)
    for b in rng.choice(len(base), size=max(1, len(base) // 20), replace=False):
        e = 1 * 16 + 1 * 4 + 1 + 21 * int(rng.integers(0, 2))      # (1,1,1) or (2,2,2): interior cells
        i, j, k = e >> 4, (e >> 2) & 3, e & 3
        for di in (-1, 0, 1):
            for dj in (-1, 0, 1):
                for dk in (-1, 0, 1):
                    out[b, (i + di) * 16 + (j + dj) * 4 + (k + dk)] &= np.uint8(~torc.CELL_INSIDE & 0xFF)
        out[b, e] |= torc.CELL_INSIDE
    return out


@pytest.mark.gpu
@pytest.mark.parametrize("after_update", [False, True])
def test_band_voxel_filter_matches_oracle(native_lib, after_update):
    from spgrid_topo_opt_b200 import native
    base, res, flags, dens = container(seed=7)
    flags = _voxel_islands(flags, base)
    band = native.Band(base, res, flags, dens)
    thin = np.ones(len(base), bool)
    if after_update:
        band.update()
        thin = band.maps()[0]
    st = band.filter_voxels()
    f, d, rst = torc.filter_isolated_voxels(base, dens, flags, thin)
    assert {k: st[k] for k in rst} == rst
    assert rst["removed"] > 0 and rst["components"] > 2
    assert np.array_equal(band.cell_flags(), f) and np.array_equal(band.flags, f)
    assert np.array_equal(band.density(), d)
    # a second pass finds a single component and changes nothing
    st2 = band.filter_voxels()
    assert st2["components"] == 1 and st2["removed"] == 0 and st2["voxels"] == rst["kept"]
    band.close()


@pytest.mark.gpu
def test_band_voxel_filter_errors_change_nothing(native_lib):
    from spgrid_topo_opt_b200 import native
    base, flags, dens = _row([list(range(32)), [], list(range(32))])
    band = native.Band(base, np.array([40, 24, 24], np.int32), flags, dens)
    with pytest.raises(native.SolverError) as e:
        band.filter_voxels()
    assert e.value.code == 1
    assert np.array_equal(band.cell_flags(), flags) and np.array_equal(band.density(), dens)
    band.close()


@pytest.mark.gpu
def test_band_threshold_and_kill_matches_oracle(native_lib):
    from spgrid_topo_opt_b200 import native
    base, res, flags, dens = container(seed=8, pruned=0.1)
    band = native.Band(base, res, flags, dens)
    band.update()
    _, fat0, *_ = torc.update_page_maps(base, dens, flags, np.ones(len(base), bool))
    thin0 = band.maps()[0]
    out = band.threshold_and_kill(0.3)
    f1, killed = torc.kill_below(dens, flags, 0.3)
    f2, d2, vst = torc.filter_isolated_voxels(base, dens, f1, thin0)
    ref = torc.update_page_maps(base, d2, f2, fat0, connectivity_filtering=False)
    assert out["killed"] == killed > 0
    assert {k: out["voxels"][k] for k in vst} == vst and vst["removed"] > 0
    assert np.array_equal(band.cell_flags(), f2) and np.array_equal(band.density(), d2)
    _compare(band, ref, out["maps"])
    band.close()


# ---------------------------------------------------------------- threshold_density
def test_oracle_threshold_bisection_meets_the_target():
    rng = np.random.default_rng(2)
    rho = rng.random((40, 64))
    flags = np.full((40, 64), torc.CELL_INSIDE, np.uint8)
    flags[0, :8] |= torc.CELL_FIXED
    rho[0, :8] = 0.0                                   # fixed cells count as solid whatever their density
    rho[1, 0] = np.nan                                 # NaN is never >= t: void
    fat = np.ones(40, bool)
    fat[39] = False                                    # outside the fat map: untouched
    out, t, solid = torc.threshold_density(flags, fat, rho, 40 * 64, 0.25)
    target = 0.25 * 40 * 64
    d = rho[fat]
    fx = (flags[fat] & torc.CELL_FIXED) != 0
    assert np.count_nonzero((d >= t) | fx) == solid > target >= np.count_nonzero((d >= t + 1e-8) | fx)
    assert np.all(out[fat][fx] == 1.0) and out[1, 0] == 0.0 and np.array_equal(out[39], rho[39])
    assert set(np.unique(out[fat])) <= {0.0, 1.0}
    out2, t2, solid2 = torc.threshold_density(flags, fat, rho, 40 * 64, 0.25, threshold=0.5)
    assert t2 == 0.5 and solid2 == np.count_nonzero((d >= 0.5) | fx)


@pytest.mark.gpu
@pytest.mark.parametrize("threshold", [None, 0.4])
def test_band_threshold_density_matches_oracle(native_lib, threshold):
    from spgrid_topo_opt_b200 import native
    base, res, flags, dens = container(seed=9)
    flags[:5, :3] |= torc.CELL_FIXED
    band = native.Band(base, res, flags, dens)
    band.update()
    fat = band.maps()[1]
    t, solid = band.threshold_density(0.3, threshold)
    total = int(np.count_nonzero(flags & torc.CELL_INSIDE))
    ref, rt, rsolid = torc.threshold_density(flags, fat, dens, total, 0.3, threshold)
    assert t == rt and solid == rsolid
    assert np.array_equal(band.density(), ref)
    band.close()
