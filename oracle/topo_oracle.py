"""CPU restatement of the optimizer step that follows a solve in the
reference's driver -- test infrastructure (the oracle), not part of the product.

* filter_dc: the density-weighted sensitivity filter Opt::smooth_dc
  (topo_opt/spgrid_topo_opt.cpp:527-579).
* oc_update: the optimality-criteria update OptimalityCriterion::optimize
  (topo_opt/optimizer/optimality_criterion.cpp:19-145).
* update_page_maps / filter_isolated_voxels / kill_below: the driver's
  narrow-band page maps and its voxel-level clean-up
  (topo_opt/spgrid_topo_opt.cpp:92-241, 1333-1344, 1404-1633).

Both act on the FEMInputs density layout: input 4x4x4 blocks (base coordinates
``base[nblocks][3]``), cell e = i*16 + j*4 + k.  A cell is inside the container
when its density is positive.

Parity unpinned: the reference's driver needs Taichi, which is absent, so no
reference output exists for these steps; they are restated from the source
lines cited above and checked in tests/ against the GPU kernels and against
hand-made cases.  Everything is float64, like the driver's ``real`` (Taichi
compiled in double precision, static_assert at spgrid_topo_opt.h:28-29).
"""
from __future__ import annotations

import math

import numpy as np


def _dense(base: np.ndarray, resolution, values: np.ndarray) -> np.ndarray:
    """Scatter [nblocks][64] cell values into a dense [X][Y][Z] array (zeros elsewhere)."""
    res = [int(r) + 4 for r in resolution]
    out = np.zeros(res)
    v = values.reshape(-1, 4, 4, 4)
    for b, (x, y, z) in enumerate(base):
        out[x:x + 4, y:y + 4, z:z + 4] = v[b]
    return out


def _gather(base: np.ndarray, dense: np.ndarray) -> np.ndarray:
    out = np.empty((base.shape[0], 64))
    for b, (x, y, z) in enumerate(base):
        out[b] = dense[x:x + 4, y:y + 4, z:z + 4].reshape(64)
    return out


def filter_dc(base, resolution, rho, dc0, filter_size: float = 1.5) -> np.ndarray:
    """spgrid_topo_opt.cpp:527-579: dc1(c) = sum_n w dc0(n) rho(n) / (sum_n w (rho(c) + 1e-3)),
    n over the container cells with |n - c|_inf <= floor(filter_size), w = max(0, filter_size - |n - c|).
    Cells outside the container get 0."""
    base = np.asarray(base, np.int64)
    R = _dense(base, resolution, np.asarray(rho, np.float64))
    D = _dense(base, resolution, np.asarray(dc0, np.float64))
    half = int(math.floor(filter_size))
    pad = half + 1
    Rp = np.pad(R, pad)
    Dp = np.pad(D, pad)
    Ip = (Rp > 0).astype(np.float64)
    s = np.zeros_like(R)
    ws = np.zeros_like(R)
    X, Y, Z = R.shape
    for dx in range(-half, half + 1):
        for dy in range(-half, half + 1):
            for dz in range(-half, half + 1):
                w = max(0.0, filter_size - math.sqrt(dx * dx + dy * dy + dz * dz))
                sl = (slice(pad + dx, pad + dx + X), slice(pad + dy, pad + dy + Y), slice(pad + dz, pad + dz + Z))
                s += (w * Dp[sl]) * Rp[sl] * Ip[sl]   # (weight * dc0) * density, the reference's order
                ws += w * Ip[sl]
    with np.errstate(divide="ignore", invalid="ignore"):
        out = np.where(R > 0, s / (ws * (R + 1e-3)), 0.0)
    return _gather(base, out)


def oc_update(rho, dc0, volume_fraction: float, step_limit: float = 0.2, minimum_density: float = 0.0,
              fixed=None, fixed_density: float = 1.0, smart_oc: bool = False, exclude_fixed: bool = True):
    """optimality_criterion.cpp:19-145.  Returns (new density, multiplier, largest change)."""
    rho = np.asarray(rho, np.float64)
    dc0 = np.asarray(dc0, np.float64)
    inside = rho > 0
    fx = np.zeros(rho.shape, bool) if fixed is None else (np.asarray(fixed) != 0)
    neg_dc_min = float(np.min(-dc0[inside])) if (smart_oc and inside.any()) else 1e30
    shift = min(0.0, neg_dc_min)
    nfix = int(np.count_nonzero(fx & inside)) if exclude_fixed else 0
    # the driver's real is float64 (static_assert, spgrid_topo_opt.h:28-29)
    target = float(volume_fraction) * float(int(np.count_nonzero(inside)) - nfix)

    def trial(mid):
        old = rho[inside]
        nd = old * np.sqrt(np.maximum(0.0, -dc0[inside] - shift) / mid)
        nd = np.minimum(np.maximum(nd, old - step_limit), old + step_limit)
        nd = np.minimum(np.maximum(nd, minimum_density), 1.0)
        f = fx[inside]
        nd = np.where(f, fixed_density, nd)
        counted = ~f if exclude_fixed else np.ones_like(f)
        return nd, float(np.sum(nd[counted]))

    lower, upper, mid = 1e-20, 1e20, 0.0
    factor = 1 + 1e-7
    while lower * factor < upper:
        mid = 0.5 * (lower + upper)
        _, s = trial(mid)
        if s > target:
            lower = mid
        else:
            upper = mid
    nd, _ = trial(mid)
    out = rho.copy()
    out[inside] = nd
    change = float(np.max(np.abs(nd - rho[inside]))) if nd.size else 0.0
    return out, mid, change


# ---------------------------------------------------------------------------
# Narrow-band page maps of the driver (thin / fat / fatter)
# ---------------------------------------------------------------------------
CELL_INSIDE, CELL_FORCE, CELL_FIXED = 1, 2, 4   # TopOptFlags bits 0-2 (spgrid_topo_opt.h:30-42)


class PageMapError(RuntimeError):
    """A state the reference stops on (TC_ASSERT / TC_ERROR in the driver)."""


def driver_page_keys(block_ijk) -> np.ndarray:
    """Page index of the driver's 4x4x4 grid (64-byte nodes, 4 KiB pages): from the
    SPGrid page masks (external/SPGrid/Core/SPGrid_Mask.h:38-47) with
    block_bits = 6, bit 3m holds bit m of the block's z, 3m+1 of y, 3m+2 of x.
    Sorting by it gives the order of the driver's page-map block lists."""
    b = np.asarray(block_ijk, np.int64).reshape(-1, 3)
    k = np.zeros(len(b), np.uint64)
    for m in range(21):
        k |= ((b[:, 2] >> m) & 1).astype(np.uint64) << np.uint64(3 * m)
        k |= ((b[:, 1] >> m) & 1).astype(np.uint64) << np.uint64(3 * m + 1)
        k |= ((b[:, 0] >> m) & 1).astype(np.uint64) << np.uint64(3 * m + 2)
    return k


def update_page_maps(base, density, flags, fat_prev, *, minimum_density: float = 0.0,
                     active_threshold: float = 1e-6, fraction_to_keep: float = 1.0, fat_margin: int = 1,
                     connectivity_filtering: bool = True):
    """One page-map update of the driver: Opt::update_thin_page_map
    (spgrid_topo_opt.cpp:92-152), Opt::filter_isolated_blocks (:1404-1510, when
    ``connectivity_filtering``) and Opt::update_fat_page_map (:154-241).

    base[n][3]: the container's 4x4x4 blocks (any order); density, flags[n][64]
    per cell (i*16 + j*4 + k); fat_prev[n]: the fat map the thin map is pruned
    from (the container itself before the first update, :391-394).  Returns
    (thin, fat, fatter, stats) with the maps as bool[n] in the caller's order."""
    base = np.asarray(base, np.int64).reshape(-1, 3)
    n = len(base)
    dens = np.asarray(density, np.float64).reshape(n, 64)
    flg = np.asarray(flags, np.uint8).reshape(n, 64)
    order = np.argsort(driver_page_keys(base // 4), kind="stable")   # list position -> block
    where = {tuple(base[b]): b for b in range(n)}
    fat_prev = np.asarray(fat_prev, bool)

    # thin: blocks of the fat map whose largest density reaches the threshold or
    # that carry a force (:100-116); BlockMeta starts at max 0, min 1, sum 0
    fat_list = [b for b in order if fat_prev[b]]
    sums = np.zeros(len(fat_list))
    thin = np.zeros(n, bool)
    for p, b in enumerate(fat_list):
        dmax = max(0.0, float(dens[b].max()))
        sums[p] = float(np.cumsum(dens[b])[-1])           # sequential, in region order
        has_force = bool((flg[b] & CELL_FORCE).any())
        thin[b] = dmax >= minimum_density + active_threshold or has_force
    stats = {"thin_before_pruning": int(thin.sum())}

    # fraction_to_keep (:121-151): note the reference reads block_meta (indexed by
    # the fat list) at the position of each block in the thin list
    if fraction_to_keep != 1.0:
        keep = int(fraction_to_keep * n)
        thin_list = [b for b in order if thin[b]]
        if keep >= len(thin_list):
            if keep < 1 or keep > len(fat_list):
                raise PageMapError("fraction_to_keep selects outside the fat block list")
            threshold = np.partition(sums, keep - 1)[keep - 1]
            thin[:] = False
            for p, b in enumerate(thin_list):
                if sums[p] > threshold:
                    thin[b] = True

    # isolated-block filter: 6-connected components of the thin blocks (:1404-1510)
    components = 0
    if connectivity_filtering:
        color = {}
        sizes = []
        for b in order:
            if not thin[b] or b in color:
                continue
            queue = [b]
            color[b] = len(sizes)
            count = 1
            head = 0
            while head < len(queue):
                u = queue[head]
                head += 1
                for d in ((4, 0, 0), (-4, 0, 0), (0, 4, 0), (0, -4, 0), (0, 0, 4), (0, 0, -4)):
                    v = where.get((base[u][0] + d[0], base[u][1] + d[1], base[u][2] + d[2]))
                    if v is not None and thin[v] and v not in color:
                        color[v] = len(sizes)
                        queue.append(v)
                        count += 1
            sizes.append(count)
        components = len(sizes)
        if components == 0:
            raise PageMapError("no thin blocks left for the connectivity filter")
        if components > 1:
            total = sum(sizes)
            big = [i for i, s in enumerate(sizes) if 1.0 * s / total > 0.3]
            if len(big) != 1:
                raise PageMapError(f"{len(big)} block components hold more than 30% of the thin blocks")
            for b in range(n):
                if thin[b] and color[b] != big[0]:
                    thin[b] = False
    stats["components"] = components

    # fat: the pages of the diagonal neighbours at fat_margin of every cell above
    # the threshold in a thin block, within the container (:166-186)
    fat = np.zeros(n, bool)
    offs = np.array([[a, b, c] for a in (-1, 1) for b in (-1, 1) for c in (-1, 1)]) * fat_margin
    ijk = np.array([[e >> 4, (e >> 2) & 3, e & 3] for e in range(64)])
    for b in np.nonzero(thin)[0]:
        cells = ijk[dens[b] > active_threshold] + base[b]
        pages = np.unique((((cells[:, None, :] + offs[None]) // 4) * 4).reshape(-1, 3), axis=0)
        for pg in pages:
            v = where.get(tuple(pg))
            if v is not None:
                fat[v] = True
    # fatter: the fat blocks and their +1 neighbours in every combination (:188-200)
    fatter = np.zeros(n, bool)
    for b in np.nonzero(fat)[0]:
        for a in (0, 4):
            for bb in (0, 4):
                for c in (0, 4):
                    v = where.get((base[b][0] + a, base[b][1] + bb, base[b][2] + c))
                    if v is not None:
                        fatter[v] = True
    inside = (flg & CELL_INSIDE) != 0
    stats.update(container_blocks=n, thin_blocks=int(thin.sum()), fat_blocks=int(fat.sum()),
                 fatter_blocks=int(fatter.sum()),
                 active_voxels=int(np.count_nonzero((inside & (dens > active_threshold))[fatter])))
    return thin, fat, fatter, stats


# ---------------------------------------------------------------------------
# The optimizer step on a band (container state + fat map)
# ---------------------------------------------------------------------------
def band_filter(base, resolution, flags, fat, rho, dc0, filter_size: float = 1.5) -> np.ndarray:
    """Opt::smooth_dc over the fat blocks (spgrid_topo_opt.cpp:527-579): every
    neighbour inside the container counts with its stored dc0 and density, also
    outside the fat map.  Returns dc0 after the swap: filtered on the container
    cells of fat blocks, unchanged elsewhere (other cells of fat blocks get 0;
    nothing reads them)."""
    base = np.asarray(base, np.int64)
    flg = np.asarray(flags, np.uint8).reshape(-1, 64)
    inside = (flg & CELL_INSIDE) != 0
    R = _dense(base, resolution, np.asarray(rho, np.float64))
    D = _dense(base, resolution, np.asarray(dc0, np.float64))
    INS = _dense(base, resolution, inside.astype(np.float64))
    half = int(math.floor(filter_size))
    pad = half + 1
    Rp, Dp, Ip = np.pad(R, pad), np.pad(D, pad), np.pad(INS, pad)
    s = np.zeros_like(R)
    ws = np.zeros_like(R)
    X, Y, Z = R.shape
    for dx in range(-half, half + 1):
        for dy in range(-half, half + 1):
            for dz in range(-half, half + 1):
                w = max(0.0, filter_size - math.sqrt(dx * dx + dy * dy + dz * dz))
                sl = (slice(pad + dx, pad + dx + X), slice(pad + dy, pad + dy + Y), slice(pad + dz, pad + dz + Z))
                s += (w * Dp[sl]) * Rp[sl] * Ip[sl]
                ws += w * Ip[sl]
    with np.errstate(divide="ignore", invalid="ignore"):
        out = _gather(base, s / (ws * (R + 1e-3)))
    res = np.array(dc0, np.float64, copy=True).reshape(-1, 64)
    fat = np.asarray(fat, bool)
    res[fat] = np.where(inside[fat], out[fat], 0.0)
    return res


def band_oc(flags, fat, rho, dc0, total_inside: int, volume_fraction: float, step_limit: float = 0.2,
            minimum_density: float = 0.0, fixed_density: float = 1.0, smart_oc: bool = False,
            exclude_fixed: bool = True):
    """OptimalityCriterion::optimize over the container cells of the fat blocks
    with the volume target against all container cells
    (optimality_criterion.cpp:19-145).  Returns (new density, multiplier, change)."""
    flg = np.asarray(flags, np.uint8).reshape(-1, 64)
    rho = np.asarray(rho, np.float64).reshape(-1, 64)
    dc0 = np.asarray(dc0, np.float64).reshape(-1, 64)
    sel = np.asarray(fat, bool)[:, None] & ((flg & CELL_INSIDE) != 0)
    fx = ((flg & CELL_FIXED) != 0)[sel]
    neg_dc_min = float(np.min(-dc0[sel])) if (smart_oc and sel.any()) else 1e30
    shift = min(0.0, neg_dc_min)
    nfix = int(np.count_nonzero(fx)) if exclude_fixed else 0
    target = float(volume_fraction) * float(total_inside - nfix)
    old = rho[sel]

    def trial(mid):
        nd = old * np.sqrt(np.maximum(0.0, -dc0[sel] - shift) / mid)
        nd = np.minimum(np.maximum(nd, old - step_limit), old + step_limit)
        nd = np.minimum(np.maximum(nd, minimum_density), 1.0)
        nd = np.where(fx, fixed_density, nd)
        return nd, float(np.sum(nd[~fx] if exclude_fixed else nd))

    lower, upper, mid = 1e-20, 1e20, 0.0
    while lower * (1 + 1e-7) < upper:
        mid = 0.5 * (lower + upper)
        if trial(mid)[1] > target:
            lower = mid
        else:
            upper = mid
    nd, _ = trial(mid)
    out = rho.copy()
    out[sel] = nd
    change = float(np.max(np.abs(nd - old))) if nd.size else 0.0
    return out, mid, change


# ---------------------------------------------------------------------------
# Voxel-level connectivity filter and threshold-and-kill
# ---------------------------------------------------------------------------
def filter_isolated_voxels(base, density, flags, thin):
    """Opt::filter_isolated_voxels (spgrid_topo_opt.cpp:1512-1633): breadth-first
    search over the container cells of the thin blocks with 6-connectivity, in
    the order of the thin list and of the cells in a block.  With one component
    nothing changes; otherwise exactly one component must hold more than 30% of
    those cells, and every other cell loses its container flag and its density.
    The container voxel count the optimizer's volume target uses is not changed.
    Returns (flags, density, stats) as new arrays."""
    base = np.asarray(base, np.int64).reshape(-1, 3)
    n = len(base)
    dens = np.array(density, np.float64, copy=True).reshape(n, 64)
    flg = np.array(flags, np.uint8, copy=True).reshape(n, 64)
    thin = np.asarray(thin, bool)
    part = thin[:, None] & ((flg & CELL_INSIDE) != 0)          # the cells the search can reach
    ijk = np.array([[e >> 4, (e >> 2) & 3, e & 3] for e in range(64)])
    lo = base.min(axis=0) - 1
    ext = base.max(axis=0) - lo + 5
    index = np.full(tuple(ext), -1, np.int64)                   # cell coordinate -> b * 64 + e
    for b in range(n):
        x, y, z = base[b] - lo
        index[x:x + 4, y:y + 4, z:z + 4] = np.where(part[b], b * 64 + np.arange(64), -1).reshape(4, 4, 4)
    color = np.full(n * 64, -1, np.int64)
    sizes = []
    order = np.argsort(driver_page_keys(base // 4), kind="stable")
    steps = ((1, 0, 0), (-1, 0, 0), (0, 1, 0), (0, -1, 0), (0, 0, 1), (0, 0, -1))
    for b in order:
        if not thin[b]:
            continue
        for e in range(64):
            c0 = b * 64 + e
            if not part[b, e] or color[c0] >= 0:
                continue
            color[c0] = len(sizes)
            queue, head = [c0], 0
            while head < len(queue):
                u = queue[head]
                head += 1
                p = base[u // 64] - lo + ijk[u % 64]
                for d in steps:
                    v = index[p[0] + d[0], p[1] + d[1], p[2] + d[2]]
                    if v >= 0 and color[v] < 0:
                        color[v] = len(sizes)
                        queue.append(v)
            sizes.append(len(queue))
    total = int(sum(sizes))
    stats = {"voxels": total, "components": len(sizes), "kept": total, "removed": 0}
    if not sizes:
        raise PageMapError("no container voxels in the thin blocks")
    if len(sizes) == 1:
        return flg, dens, stats
    big = [i for i, s in enumerate(sizes) if 1.0 * s / total > 0.3]
    if len(big) != 1:
        raise PageMapError(f"{len(big)} voxel components hold more than 30% of the voxels")
    drop = (part.reshape(-1) & (color != big[0])).reshape(n, 64)
    flg[drop] &= np.uint8(~CELL_INSIDE & 0xFF)
    dens[drop] = 0.0
    stats.update(kept=int(sizes[big[0]]), removed=int(np.count_nonzero(drop)))
    return flg, dens, stats


def kill_below(density, flags, threshold: float):
    """The first loop of Opt::threshold_and_kill (spgrid_topo_opt.cpp:1333-1344):
    every container cell whose density is below the threshold leaves the
    container (its density stays).  Returns (flags, cells killed)."""
    flg = np.array(flags, np.uint8, copy=True)
    kill = ((flg & CELL_INSIDE) != 0) & (np.asarray(density, np.float64).reshape(flg.shape) < threshold)
    flg[kill] &= np.uint8(~CELL_INSIDE & 0xFF)
    return flg, int(np.count_nonzero(kill))


def threshold_density(flags, fat, rho, total_inside: int, volume_fraction: float, threshold=None):
    """Opt::threshold_density (spgrid_topo_opt.cpp:1780-1797) over
    threshold_density_trail (:1756-1778): all 64 cells of every fat block count
    as solid when their density is >= t or they have a fixed density; the
    bisection on [0, 1] runs until lo + 1e-8 >= hi, keeping lo while the solid
    count exceeds volume_fraction x total_inside, and the design is thresholded
    at lo (1 solid, 0 otherwise; cells outside fat blocks keep their density).
    A given threshold is applied directly.  Returns (density, threshold, solid count)."""
    flg = np.asarray(flags, np.uint8).reshape(-1, 64)
    rho = np.asarray(rho, np.float64).reshape(-1, 64)
    fat = np.asarray(fat, bool)
    fixed = (flg[fat] & CELL_FIXED) != 0
    d = rho[fat]

    def count(t):
        return int(np.count_nonzero((d >= t) | fixed))

    if threshold is None:
        target = volume_fraction * float(total_inside)
        lo, hi = 0.0, 1.0
        while lo + 1e-8 < hi:
            mid = (lo + hi) * 0.5
            if float(count(mid)) > target:
                lo = mid
            else:
                hi = mid
        threshold = lo
    out = rho.copy()
    out[fat] = np.where((d >= threshold) | fixed, 1.0, 0.0)
    return out, threshold, count(threshold)
