"""CPU restatement of the optimizer step that follows a solve in the
reference's driver -- test infrastructure (the oracle), not part of the product.

* filter_dc: the density-weighted sensitivity filter Opt::smooth_dc
  (topo_opt/spgrid_topo_opt.cpp:527-579).
* oc_update: the optimality-criteria update OptimalityCriterion::optimize
  (topo_opt/optimizer/optimality_criterion.cpp:19-145).

Both act on the FEMInputs density layout: input 4x4x4 blocks (base coordinates
``base[nblocks][3]``), cell e = i*16 + j*4 + k.  A cell is inside the container
when its density is positive.

Parity unpinned: the reference's driver needs Taichi, which is absent, so no
reference output exists for these steps; they are restated from the source
lines cited above and checked in tests/ against the GPU kernels and against
hand-made cases.  Sums are accumulated in float64 here (the reference uses
Taichi's ``real``).
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
    DRp = np.pad(D * R, pad)
    Ip = (Rp > 0).astype(np.float64)
    s = np.zeros_like(R)
    ws = np.zeros_like(R)
    X, Y, Z = R.shape
    for dx in range(-half, half + 1):
        for dy in range(-half, half + 1):
            for dz in range(-half, half + 1):
                w = max(0.0, filter_size - math.sqrt(dx * dx + dy * dy + dz * dz))
                sl = (slice(pad + dx, pad + dx + X), slice(pad + dy, pad + dy + Y), slice(pad + dz, pad + dz + Z))
                s += w * DRp[sl] * Ip[sl]
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
    # volume_fraction is a float in the reference, multiplied by the cell count
    target = float(np.float32(volume_fraction) * np.float32(int(np.count_nonzero(inside)) - nfix))

    def trial(mid):
        old = rho[inside]
        nd = old * np.sqrt(np.maximum(0.0, -dc0[inside] - shift) / mid)
        nd = np.minimum(np.maximum(nd, old - step_limit), old + step_limit)
        nd = np.minimum(np.maximum(nd, minimum_density), 1.0)
        f = fx[inside]
        nd = np.where(f, fixed_density, nd)
        counted = ~f if exclude_fixed else np.ones_like(f)
        return nd, float(np.sum(nd[counted]))

    lower, upper, mid = float(np.float32(1e-20)), 1e20, 0.0
    factor = float(np.float32(1.0) + np.float32(1e-7))
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
