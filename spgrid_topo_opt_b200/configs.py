"""Seeded synthetic problem generators that stand in for the caller side.

The reference's SIMP driver packs a density field, Dirichlet nodes and nodal
forces into ``FEMInputs`` before every solve (topo_opt/spgrid_topo_opt.cpp:977-1228).
These generators build the same kind of input for the benchmark workloads:

* the container's cells start at the grid padding of 8 and the solver
  resolution is the container's upper bound plus 48 (spgrid_topo_opt.cpp:992,
  spgrid_topo_opt.h:93);
* the density blocks are the 4x4x4 blocks touching any node of a material cell,
  so every material cell's +1 neighbours are present (spgrid_topo_opt.cpp:1123-1145);
* Dirichlet conditions are emitted as whole cells, all 8 corner nodes on each
  fixed axis, because the solver keeps a Dirichlet node only when it completes
  a cell (add_cell_boundary, spgrid_topo_opt.h:627-654; node->cell rule,
  SPGrid_CPU_Solver.cpp:169-192); duplicates are removed (spgrid_topo_opt.cpp:1176-1193);
* ``mg_level`` follows the driver's rule (spgrid_topo_opt.cpp:1022-1037).
"""
from __future__ import annotations

from dataclasses import dataclass
from typing import Optional, Tuple

import numpy as np

from .fem_interface import DIRICHLET_DTYPE, FORCE_DTYPE, BlockedGrid, FEMInputs, KrylovSolverParameters

PADDING = 8


def lame(E: float = 1e6, nu: float = 0.3) -> Tuple[float, float]:
    """(mu, lambda) of an isotropic material (topo_opt/hex_fem.h:20-23)."""
    return E / (2 * (1 + nu)), E * nu / ((1 + nu) * (1 - 2 * nu))


def mg_level_for(container_size: int, bottom_size: int = 64) -> int:
    """Driver's level-count rule (spgrid_topo_opt.cpp:1022-1037)."""
    n, level = container_size, 1
    while n > bottom_size:
        n //= 2
        level += 1
    return 3 if level == 2 else level


@dataclass
class Problem:
    """A synthetic workload: the cell density field plus boundary conditions."""

    name: str
    n: Tuple[int, int, int]          # container size in cells
    density: np.ndarray              # float64[nx,ny,nz] cell densities (0 = empty)
    dirichlet_cells: np.ndarray      # int32[k,3] cells whose 8 nodes are fixed in xyz
    forces: np.ndarray               # FORCE_DTYPE
    dx: float
    mg_level: int


def _blocks_from_density(density: np.ndarray):
    """4x4x4 blocks (grid coordinates) touching any node of a material cell."""
    nx, ny, nz = density.shape
    cells = density > 0
    nodes = np.zeros((nx + 1, ny + 1, nz + 1), bool)
    for a in (0, 1):
        for b in (0, 1):
            for c in (0, 1):
                nodes[a:a + nx, b:b + ny, c:c + nz] |= cells
    # node (i,j,k) in container coords -> grid coords + PADDING (a multiple of 4)
    bx = (nx + 1 + 3) // 4 + 1
    by = (ny + 1 + 3) // 4 + 1
    bz = (nz + 1 + 3) // 4 + 1
    pad = np.zeros((bx * 4, by * 4, bz * 4), bool)
    pad[:nx + 1, :ny + 1, :nz + 1] = nodes
    occ = pad.reshape(bx, 4, by, 4, bz, 4).any(axis=(1, 3, 5))
    bidx = np.argwhere(occ).astype(np.int32)
    base = bidx * 4 + PADDING
    # density payload in-block index i*16+j*4+k (fem_interface.h:150-152)
    dpad = np.zeros((bx * 4, by * 4, bz * 4), np.float64)
    dpad[:nx, :ny, :nz] = density
    blk = dpad.reshape(bx, 4, by, 4, bz, 4).transpose(0, 2, 4, 1, 3, 5)
    data = blk[bidx[:, 0], bidx[:, 1], bidx[:, 2]].reshape(-1, 64)
    return base.astype(np.int32), np.ascontiguousarray(data)


def dirichlet_nodes_from_cells(cells: np.ndarray, axes: str = "xyz") -> np.ndarray:
    """All corner nodes of the given cells, every listed axis, deduplicated."""
    if len(cells) == 0:
        return np.zeros(0, DIRICHLET_DTYPE)
    corners = np.array([[a, b, c] for a in (0, 1) for b in (0, 1) for c in (0, 1)], np.int32)
    nodes = (cells[:, None, :] + corners[None]).reshape(-1, 3)
    nodes = np.unique(nodes, axis=0)
    out = []
    for ax in range(3):
        if "xyz"[ax] not in axes:
            continue
        rec = np.zeros(len(nodes), DIRICHLET_DTYPE)
        rec["coord"] = nodes
        rec["axis"] = ax
        rec["value"] = 0.0
        out.append(rec)
    return np.concatenate(out)


def to_inputs(prob: Problem, *, E: float = 1e6, nu: float = 0.3, penalty: float = 3.0,
              minimum_stiffness: float = 1e-9, tolerance: float = 1e-4, max_iterations: int = 50,
              smoothing: int = 1, boundary_smoothing: int = 3, mg_level: Optional[int] = None) -> FEMInputs:
    """Pack a problem the way the driver does (spgrid_topo_opt.cpp:991-1228)."""
    mu, lam = lame(E, nu)
    base, data = _blocks_from_density(prob.density)
    # the driver never feeds exact zeros inside the container (spgrid_topo_opt.cpp:1122)
    p = FEMInputs()
    p.resolution = [int(PADDING + s + 6 * PADDING) for s in prob.n]
    p.dx = prob.dx
    p.global_mu, p.global_lambda = mu, lam
    p.use_density_only = True
    p.density = BlockedGrid(resolution=list(p.resolution), base=base, data=data)
    p.krylov = KrylovSolverParameters(tolerance, max_iterations, 0, False)
    p.extra_doubles["penalty"] = penalty
    p.extra_doubles["minimum_stiffness"] = minimum_stiffness
    p.extra_ints["boundary_smoothing"] = boundary_smoothing
    p.extra_ints["keep_state"] = 0
    p.extra_ints["forced_reuse"] = 1
    p.extra_ints["defect_correction_iter"] = 0
    p.extra_ints["defect_correction_cg_iter"] = 3
    p.extra_ints["solver_type"] = 1
    p.extra_doubles["min_fraction"] = 0.0
    p.mg_level = prob.mg_level if mg_level is None else mg_level
    p.explicit_mg_level = 0
    p.pre_and_post_smoothing_iter = smoothing
    p.bottom_smoothing_iter = 600
    p.jacobi_damping = 0.4
    cells = prob.dirichlet_cells.astype(np.int32) + PADDING
    p.dirichlet_nodes = dirichlet_nodes_from_cells(cells)
    f = prob.forces.copy()
    f["coord"] += PADDING
    p.forces = f
    p.caller_method = "spgrid_topo_opt_b200"
    p.preserve_output(base.shape[0])
    return p


# --------------------------------------------------------------------------
# Workloads
# --------------------------------------------------------------------------
def cantilever_box(n: int = 64, density=0.1, seed: Optional[int] = None,
                   bottom_size: int = 16) -> Problem:
    """Dense box of n^3 cells, x-min cell layer fixed, unit load (0,-1,0) at the
    x-max face centre node.  ``density`` is a constant or ``(lo, hi)`` for a
    seeded uniform field."""
    if isinstance(density, tuple):
        rng = np.random.default_rng(1234 if seed is None else seed)
        rho = rng.uniform(density[0], density[1], size=(n, n, n))
    else:
        rho = np.full((n, n, n), float(density))
    cells = np.argwhere(np.ones((1, n, n), bool)).astype(np.int32)
    f = np.zeros(1, FORCE_DTYPE)
    f["coord"][0] = (n, n // 2, n // 2)
    f["f"][0] = (0.0, -1.0, 0.0)
    return Problem(f"cantilever{n}", (n, n, n), rho, cells, f, 1.0 / n, mg_level_for(n, bottom_size))


def _smooth_noise(shape, seed: int, coarse: int = 8) -> np.ndarray:
    """Uniform[-1,1] noise on a coarse lattice, trilinearly interpolated."""
    rng = np.random.default_rng(seed)
    g = rng.uniform(-1, 1, size=(coarse + 1,) * 3)
    axes = [np.linspace(0, coarse, s, endpoint=False) + coarse / (2 * s) for s in shape]
    out = np.zeros(shape)
    i0 = [np.minimum(np.floor(a).astype(int), coarse - 1) for a in axes]
    t = [a - i for a, i in zip(axes, i0)]
    for dx in (0, 1):
        wx = t[0] if dx else 1 - t[0]
        for dy in (0, 1):
            wy = t[1] if dy else 1 - t[1]
            for dz in (0, 1):
                wz = t[2] if dz else 1 - t[2]
                out += (wx[:, None, None] * wy[None, :, None] * wz[None, None, :] *
                        g[np.ix_(i0[0] + dx, i0[1] + dy, i0[2] + dz)])
    return out


def sphere_shell(n: int = 256, r_in: float = 0.4, r_out: float = 0.5, seed: int = 1234,
                 bottom_size: int = 32) -> Problem:
    """Narrow-band sphere shell in an n^3 grid (sphere SDF of spgrid_topo_opt.cpp:440-455):
    cells whose centre lies at radius [r_in, r_out] of the unit box; density
    clamp(0.5 + 0.3*noise, 1e-3, 1); the lowest two cell layers of the shell
    are fixed; a downward unit load is spread over the top-cap nodes."""
    c = (np.arange(n) + 0.5) / n - 0.5
    r = np.sqrt(c[:, None, None] ** 2 + c[None, :, None] ** 2 + c[None, None, :] ** 2)
    shell = (r >= r_in) & (r <= r_out)
    rho = np.where(shell, np.clip(0.5 + 0.3 * _smooth_noise((n, n, n), seed), 1e-3, 1.0), 0.0)
    ys = np.argwhere(shell)[:, 1]
    ymin = ys.min()
    dcells = np.argwhere(shell & (np.arange(n)[None, :, None] <= ymin + 1)).astype(np.int32)
    # top cap: nodes of shell cells in the highest two cell layers
    ymax = ys.max()
    top = np.argwhere(shell & (np.arange(n)[None, :, None] >= ymax - 1))
    nodes = np.unique((top[:, None, :] + np.array([[a, 1, b] for a in (0, 1) for b in (0, 1)])[None]).reshape(-1, 3), axis=0)
    nodes = nodes[nodes[:, 1] == nodes[:, 1].max()]
    f = np.zeros(len(nodes), FORCE_DTYPE)
    f["coord"] = nodes
    f["f"][:, 1] = -1.0 / len(nodes)
    return Problem(f"shell{n}", (n, n, n), rho, dcells, f, 1.0 / n, mg_level_for(n, bottom_size))


def spheres_band_inputs(n: int = 1024, nspheres: int = 8, thickness: int = 12, seed: int = 7,
                        bottom_size: int = 16, **solver_kw) -> FEMInputs:
    """Narrow band of an n^3 grid, built block by block (no dense n^3 arrays): a
    ``thickness``-voxel shell around the union of ``nspheres`` seeded random
    spheres (centres in [0.3,0.7]^3, radii 0.1-0.3 of the box); cell density
    uniform [1e-3, 1] (seeded); every band cell of the lowest band cell layer is
    fixed (whole cells, xyz); 16 seeded unit point loads on band nodes."""
    rng = np.random.default_rng(seed)
    centres = rng.uniform(0.3, 0.7, size=(nspheres, 3))
    radii = rng.uniform(0.1, 0.3, size=nspheres)
    half = thickness / (2.0 * n)
    nb = n // 4

    def sdf(p):  # p: [..., 3] in unit-box coordinates
        d = np.full(p.shape[:-1], np.inf)
        for ctr, rad in zip(centres, radii):
            d = np.minimum(d, np.sqrt(((p - ctr) ** 2).sum(-1)) - rad)
        return d

    # candidate blocks: block centre within half + block half-diagonal of the surface
    g = (np.arange(nb) * 4 + 2.0) / n
    cand = []
    margin = half + np.sqrt(3) * 2.0 / n
    for bi in range(nb):
        pts = np.stack(np.broadcast_arrays(g[bi], g[:, None], g[None, :]), -1)
        near = np.abs(sdf(pts)) <= margin
        jj, kk = np.nonzero(near)
        if len(jj):
            cand.append(np.stack([np.full(len(jj), bi), jj, kk], 1))
    cand = np.concatenate(cand).astype(np.int64)
    # cell-level band test inside the candidate blocks
    off = np.array([[i, j, k] for i in range(4) for j in range(4) for k in range(4)], np.int64)  # i*16+j*4+k
    cells = cand[:, None, :] * 4 + off[None]                 # [nc, 64, 3] container cell coords
    band = np.abs(sdf((cells + 0.5) / n)) <= half
    keep = band.any(1)
    mat_blocks, band = cand[keep], band[keep]
    rho = np.where(band, rng.uniform(1e-3, 1.0, size=band.shape), 0.0)
    # node blocks: the +x/+y/+z neighbours of material blocks (zero density)
    fwd = np.array([[a, b, c] for a in (0, 1) for b in (0, 1) for c in (0, 1)], np.int64)
    allb = np.unique((mat_blocks[:, None, :] + fwd[None]).reshape(-1, 3), axis=0)
    # node blocks reach index nb on each axis: the key's stride is nb + 1 so that
    # a block past the box never shares a key with a material block
    key = lambda b: (b[:, 0] * (nb + 1) + b[:, 1]) * (nb + 1) + b[:, 2]
    mk = key(mat_blocks)
    order = np.argsort(mk)
    pos = np.searchsorted(mk[order], key(allb))
    pos = np.minimum(pos, len(mk) - 1)
    is_mat = mk[order][pos] == key(allb)
    data = np.zeros((len(allb), 64))
    data[is_mat] = rho[order][pos[is_mat]]
    base = (allb * 4 + PADDING).astype(np.int32)
    # Dirichlet: every band cell of the lowest band cell layer
    bc = (mat_blocks[:, None, :] * 4 + off[None])[band]
    ymin = bc[:, 1].min()
    dcells = bc[bc[:, 1] == ymin].astype(np.int32) + PADDING
    # loads: 16 seeded band cells, load on the cell's (1,1,1) corner node
    pick = bc[rng.choice(len(bc), 16, replace=False)] + 1 + PADDING
    f = np.zeros(16, FORCE_DTYPE)
    f["coord"] = pick
    v = rng.normal(size=(16, 3))
    f["f"] = v / np.linalg.norm(v, axis=1, keepdims=True)
    kw = dict(tolerance=1e-6)
    kw.update(solver_kw)
    mu, lam = lame(kw.pop("E", 1e6), kw.pop("nu", 0.3))
    p = FEMInputs()
    p.resolution = [n + 7 * PADDING] * 3
    p.dx = 1.0 / n
    p.global_mu, p.global_lambda = mu, lam
    p.density = BlockedGrid(resolution=list(p.resolution), base=base, data=data)
    p.krylov = KrylovSolverParameters(kw.get("tolerance", 1e-6), kw.get("max_iterations", 50), 0, False)
    p.extra_doubles.update({"penalty": kw.get("penalty", 3.0), "minimum_stiffness": kw.get("minimum_stiffness", 1e-9),
                            "min_fraction": 0.0})
    p.extra_ints.update({"boundary_smoothing": kw.get("boundary_smoothing", 3), "keep_state": 0, "forced_reuse": 1})
    p.mg_level = kw.get("mg_level", mg_level_for(n, bottom_size))
    p.pre_and_post_smoothing_iter = kw.get("smoothing", 1)
    p.dirichlet_nodes = dirichlet_nodes_from_cells(dcells)
    p.forces = f
    p.caller_method = "spgrid_topo_opt_b200"
    p.preserve_output(base.shape[0])
    return p


def bridge(nx: int = 512, ny: int = 128, nz: int = 256, density: float = 0.1, support_radius: float = 0.03,
           bottom_size: int = 16) -> Problem:
    """A bridge-like box domain of nx x ny x nz cells (x along the span, y up): the
    cells of the bottom layer within ``support_radius`` (a fraction of the
    largest extent) of the four bottom corners are fixed, and a uniform downward
    load of total magnitude 1 acts on the nodes of the top deck.  Every cell
    starts at ``density``.  A seeded-free synthetic stand-in for the reference's
    bridge script domain."""
    rho = np.full((nx, ny, nz), float(density))
    r = support_radius * max(nx, ny, nz)
    xs, zs = np.meshgrid(np.arange(nx) + 0.5, np.arange(nz) + 0.5, indexing="ij")
    near = np.zeros((nx, nz), bool)
    for cx in (0.0, float(nx)):
        for cz in (0.0, float(nz)):
            near |= (xs - cx) ** 2 + (zs - cz) ** 2 <= r * r
    ij = np.argwhere(near)
    cells = np.stack([ij[:, 0], np.zeros(len(ij), np.int64), ij[:, 1]], 1).astype(np.int32)
    top = np.argwhere(np.ones((nx + 1, nz + 1), bool))
    f = np.zeros(len(top), FORCE_DTYPE)
    f["coord"][:, 0] = top[:, 0]
    f["coord"][:, 1] = ny
    f["coord"][:, 2] = top[:, 1]
    f["f"][:, 1] = -1.0 / len(top)
    return Problem(f"bridge{nx}x{ny}x{nz}", (nx, ny, nz), rho, cells, f, 1.0 / max(nx, ny, nz),
                   mg_level_for(max(nx, ny, nz), bottom_size))
