// Kernels of the topology-optimization step that follows a solve in the
// reference's driver: the density-weighted sensitivity filter
// (topo_opt/spgrid_topo_opt.cpp:527-579) and the optimality-criteria density
// update (topo_opt/optimizer/optimality_criterion.cpp:19-145).  Both work on the
// input layout of FEMInputs: 4x4x4 blocks of cells, cell e = i*16 + j*4 + k,
// global cell index b*64 + e; a cell is inside the container when its density
// is positive (the driver sends 0 outside the container and at least
// minimum_density inside).
#pragma once
#include <cstdint>

namespace sgs {

// dc1 = sum_n w_n dc0_n rho_n / (sum_n w_n (rho + 1e-3)) over the container
// cells n within the cube of half width floor(filter_size), w = max(0,
// filter_size - |offset|), dc0 being scale times the given field (scale -1
// turns the compliance sensitivity dc into the driver's gradient).  Cells outside
// the container get 0 (the reference leaves them undefined; nothing reads them).
__global__ void filter_dc_kernel(int nin, const int* __restrict__ base, const int* __restrict__ grid, int gx, int gy,
                                 int gz, const double* __restrict__ rho, const double* __restrict__ dc0,
                                 double* __restrict__ dc1, double fsize, int half, double scale) {
  const long t = long(blockIdx.x) * blockDim.x + threadIdx.x;
  if (t >= long(nin) * 64) return;
  const int b = int(t >> 6), e = int(t & 63);
  const double r = rho[t];
  if (!(r > 0)) {
    dc1[t] = 0;
    return;
  }
  const int x = base[3 * b] + (e >> 4), y = base[3 * b + 1] + ((e >> 2) & 3), z = base[3 * b + 2] + (e & 3);
  double sum = 0, wsum = 0;
  for (int dx = -half; dx <= half; ++dx)
    for (int dy = -half; dy <= half; ++dy)
      for (int dz = -half; dz <= half; ++dz) {
        const int X = x + dx, Y = y + dy, Z = z + dz;
        if (X < 0 || Y < 0 || Z < 0) continue;
        const int bx = X >> 2, by = Y >> 2, bz = Z >> 2;
        if (bx >= gx || by >= gy || bz >= gz) continue;
        const int nb = grid[(long(bx) * gy + by) * gz + bz];
        if (nb < 0) continue;
        const long c = long(nb) * 64 + (X & 3) * 16 + (Y & 3) * 4 + (Z & 3);
        const double rn = rho[c];
        if (!(rn > 0)) continue;
        const double w = fmax(0.0, fsize - sqrt(double(dx * dx + dy * dy + dz * dz)));
        sum += w * (scale * dc0[c]) * rn;
        wsum += w;
      }
  dc1[t] = sum / (wsum * (r + 1e-3));
}

constexpr int OC_THREADS = 256, OC_BLOCKS = 592;

// New density of one cell at multiplier mid (optimality_criterion.cpp:88-97):
// old * sqrt(max(0, -dc0 - shift) / mid) clamped to old -+ step, then to
// [rho_min, 1].
__device__ __forceinline__ double oc_density(double old, double dc0, double mid, double shift, double step,
                                             double rho_min) {
  double nd = old * sqrt(fmax(0.0, -dc0 - shift) / mid);
  nd = fmin(fmax(nd, old - step), old + step);
  return fmin(fmax(nd, rho_min), 1.0);
}

// Per-CTA partials of a sum and a maximum (fixed order: warps, then the CTA's
// warps in sequence); one thread of the CTA writes them.
__device__ __forceinline__ void cta_sum_max(double sum, double chg, double* part_sum, double* part_change) {
  __shared__ double ss[OC_THREADS / 32], sc[OC_THREADS / 32];
  for (int o = 16; o; o >>= 1) {
    sum += __shfl_down_sync(0xffffffffu, sum, o);
    chg = fmax(chg, __shfl_down_sync(0xffffffffu, chg, o));
  }
  if ((threadIdx.x & 31) == 0) {
    ss[threadIdx.x >> 5] = sum;
    sc[threadIdx.x >> 5] = chg;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double a = 0, m = 0;
    for (int w = 0; w < OC_THREADS / 32; ++w) {
      a += ss[w];
      m = fmax(m, sc[w]);
    }
    part_sum[blockIdx.x] = a;
    part_change[blockIdx.x] = m;
  }
}

// One trial of the OC bisection at multiplier mid: the new density of every
// container cell, per-CTA partial sums of the counted densities and maxima of
// the change; with rho_out the densities are also written, at least DBL_MIN
// when keep_inside (a container cell stays in the container, as the driver's
// packing ensures, spgrid_topo_opt.cpp:1122).
__global__ void oc_trial_kernel(long n, const double* rho, const double* __restrict__ dc0,
                                const uint8_t* __restrict__ fixed, double mid, double shift, double step,
                                double rho_min, double fixed_rho, int exclude_fixed, double* rho_out,
                                double* __restrict__ part_sum, double* __restrict__ part_change, int keep_inside) {
  double sum = 0, chg = 0;
  for (long t = long(blockIdx.x) * blockDim.x + threadIdx.x; t < n; t += long(gridDim.x) * blockDim.x) {
    const double old = rho[t];
    if (!(old > 0)) continue;
    double nd = oc_density(old, dc0[t], mid, shift, step, rho_min);
    const bool fx = fixed && fixed[t];
    if (fx) nd = fixed_rho;
    if (!(exclude_fixed && fx)) sum += nd;
    chg = fmax(chg, fabs(nd - old));
    if (rho_out) rho_out[t] = keep_inside ? fmax(nd, 2.2250738585072014e-308) : nd;
  }
  cta_sum_max(sum, chg, part_sum, part_change);
}

// container cells, fixed container cells, and min over container cells of -dc0
__global__ void oc_stats_kernel(long n, const double* __restrict__ rho, const double* __restrict__ dc0,
                                const uint8_t* __restrict__ fixed, double* __restrict__ part) {
  __shared__ double s0[OC_THREADS / 32], s1[OC_THREADS / 32], s2[OC_THREADS / 32];
  double inside = 0, nfix = 0, mn = 1e30;
  for (long t = long(blockIdx.x) * blockDim.x + threadIdx.x; t < n; t += long(gridDim.x) * blockDim.x) {
    if (!(rho[t] > 0)) continue;
    inside += 1;
    if (fixed && fixed[t]) nfix += 1;
    mn = fmin(mn, -dc0[t]);
  }
  for (int o = 16; o; o >>= 1) {
    inside += __shfl_down_sync(0xffffffffu, inside, o);
    nfix += __shfl_down_sync(0xffffffffu, nfix, o);
    mn = fmin(mn, __shfl_down_sync(0xffffffffu, mn, o));
  }
  if ((threadIdx.x & 31) == 0) {
    s0[threadIdx.x >> 5] = inside;
    s1[threadIdx.x >> 5] = nfix;
    s2[threadIdx.x >> 5] = mn;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double a = 0, c = 0, m = 1e30;
    for (int w = 0; w < OC_THREADS / 32; ++w) {
      a += s0[w];
      c += s1[w];
      m = fmin(m, s2[w]);
    }
    part[3 * blockIdx.x] = a;
    part[3 * blockIdx.x + 1] = c;
    part[3 * blockIdx.x + 2] = m;
  }
}

// The SIMP map of the solver's input (fem_interface.h:343-353) from the design
// densities into the level-0 stiffness scales: E = (1 - Emin) max(rho_min, d)^p
// + Emin for d > 0 (d itself without penalty), 0 for the empty cells.
__global__ void simp_E_kernel(int nin, const int* __restrict__ in_block, const int* __restrict__ in_zoff,
                              const double* __restrict__ rho, double penalty, double emin, double rho_min,
                              double* __restrict__ E) {
  const long t = long(blockIdx.x) * blockDim.x + threadIdx.x;
  if (t >= long(nin) * 64) return;
  const int b = int(t >> 6), e = int(t & 63);
  const int blk = in_block[b];
  if (blk < 0) return;
  const double d = rho[t];
  double val = 0;
  if (d > 0) val = penalty != 0 ? (1 - emin) * pow(fmax(rho_min, d), penalty) + emin : d;
  E[long(blk) * 128 + (e >> 4) * 32 + ((e >> 2) & 3) * 8 + (e & 3) + in_zoff[b]] = val;
}

// ---------------------------------------------------------------------------
// The driver's step on a narrow band (container state, page maps): the solver
// session holds the fatter blocks; the sensitivity channels, the densities and
// the cell flags live on the container in the FEMInputs layout.
// ---------------------------------------------------------------------------
constexpr double DBL_MIN_D = 2.2250738585072014e-308;
constexpr uint8_t BAND_INSIDE = 1, BAND_FIXED = 4;  // SGS_CELL_INSIDE, SGS_CELL_FIXED

// Session cell <- container cell: the density the driver packs into FEMInputs
// (spgrid_topo_opt.cpp:1109-1125): max(d, DBL_MIN) for container cells of fat
// blocks, 0 for the rest of the fatter blocks.
__global__ void band_gather_kernel(long ncells, const int* __restrict__ map, const uint8_t* __restrict__ fat,
                                   const uint8_t* __restrict__ flags, const double* __restrict__ rho,
                                   double* __restrict__ out) {
  const long t = long(blockIdx.x) * blockDim.x + threadIdx.x;
  if (t >= ncells) return;
  const int c = map[t >> 6];
  const long cell = long(c) * 64 + (t & 63);
  out[t] = (fat[c] && (flags[cell] & BAND_INSIDE)) ? fmax(rho[cell], DBL_MIN_D) : 0.0;
}

// clear_gradients (spgrid_topo_opt.h:868-877): dc0 = 0 over the fat blocks
__global__ void band_clear_kernel(long ncells, const uint8_t* __restrict__ fat, double* __restrict__ dc0) {
  const long t = long(blockIdx.x) * blockDim.x + threadIdx.x;
  if (t < ncells && fat[t >> 6]) dc0[t] = 0;
}

// dc0 += grad with grad = -dc for the session's material cells (minimal_compliance.cpp:120-135)
__global__ void band_scatter_dc_kernel(long ncells, const int* __restrict__ map, const double* __restrict__ rho_s,
                                       const double* __restrict__ dc, double* __restrict__ dc0) {
  const long t = long(blockIdx.x) * blockDim.x + threadIdx.x;
  if (t >= ncells || !(rho_s[t] > 0)) return;
  const long cell = long(map[t >> 6]) * 64 + (t & 63);
  dc0[cell] += -dc[t];
}

// smooth_dc (spgrid_topo_opt.cpp:527-579) over the fat blocks: neighbours are the
// container cells of the whole band (their dc0 may date from an earlier
// iteration, as in the reference).  Cells outside the container get 0: their
// value is never read (the filter and the OC update visit container cells only).
__global__ void band_filter_kernel(long ncells, const int* __restrict__ base, const int* __restrict__ grid, int gx,
                                   int gy, int gz, const uint8_t* __restrict__ fat, const uint8_t* __restrict__ flags,
                                   const double* __restrict__ rho, const double* __restrict__ dc0,
                                   double* __restrict__ dc1, double fsize, int half) {
  const long t = long(blockIdx.x) * blockDim.x + threadIdx.x;
  if (t >= ncells) return;
  const int b = int(t >> 6), e = int(t & 63);
  if (!fat[b]) return;
  if (!(flags[t] & BAND_INSIDE)) {
    dc1[t] = 0;
    return;
  }
  const int x = base[3 * b] + (e >> 4), y = base[3 * b + 1] + ((e >> 2) & 3), z = base[3 * b + 2] + (e & 3);
  double sum = 0, wsum = 0;
  for (int dx = -half; dx <= half; ++dx)
    for (int dy = -half; dy <= half; ++dy)
      for (int dz = -half; dz <= half; ++dz) {
        const int X = x + dx, Y = y + dy, Z = z + dz;
        if (X < 0 || Y < 0 || Z < 0) continue;
        const int bx = X >> 2, by = Y >> 2, bz = Z >> 2;
        if (bx >= gx || by >= gy || bz >= gz) continue;
        const int nb = grid[(long(bx) * gy + by) * gz + bz];
        if (nb < 0) continue;
        const long c = long(nb) * 64 + (X & 3) * 16 + (Y & 3) * 4 + (Z & 3);
        if (!(flags[c] & BAND_INSIDE)) continue;
        const double w = fmax(0.0, fsize - sqrt(double(dx * dx + dy * dy + dz * dz)));
        sum += w * dc0[c] * rho[c];
        wsum += w;
      }
  dc1[t] = sum / (wsum * (rho[t] + 1e-3));
}

// the swap of dc0 and dc1 over the fat blocks (:571-578); only dc0 is read later
__global__ void band_copy_kernel(long ncells, const uint8_t* __restrict__ fat, const double* __restrict__ src,
                                 double* __restrict__ dst) {
  const long t = long(blockIdx.x) * blockDim.x + threadIdx.x;
  if (t < ncells && fat[t >> 6]) dst[t] = src[t];
}

// fixed container cells of the fat map and min over its container cells of -dc0
// (optimality_criterion.cpp:40-70)
__global__ void band_oc_stats_kernel(long ncells, const uint8_t* __restrict__ fat, const uint8_t* __restrict__ flags,
                                     const double* __restrict__ dc0, double* __restrict__ part_fix,
                                     double* __restrict__ part_min) {
  double nfix = 0, mn = 1e30;
  for (long t = long(blockIdx.x) * blockDim.x + threadIdx.x; t < ncells; t += long(gridDim.x) * blockDim.x) {
    if (!fat[t >> 6] || !(flags[t] & BAND_INSIDE)) continue;
    nfix += (flags[t] & BAND_FIXED) ? 1 : 0;
    mn = fmin(mn, -dc0[t]);
  }
  __shared__ double sf[OC_THREADS / 32], sm[OC_THREADS / 32];
  for (int o = 16; o; o >>= 1) {
    nfix += __shfl_down_sync(0xffffffffu, nfix, o);
    mn = fmin(mn, __shfl_down_sync(0xffffffffu, mn, o));
  }
  if ((threadIdx.x & 31) == 0) {
    sf[threadIdx.x >> 5] = nfix;
    sm[threadIdx.x >> 5] = mn;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double a = 0, m = 1e30;
    for (int w = 0; w < OC_THREADS / 32; ++w) {
      a += sf[w];
      m = fmin(m, sm[w]);
    }
    part_fix[blockIdx.x] = a;
    part_min[blockIdx.x] = m;
  }
}

// One OC trial over the container cells of the fat map (optimality_criterion.cpp:74-120);
// with rho_out the new densities are written.
__global__ void band_oc_trial_kernel(long ncells, const uint8_t* __restrict__ fat, const uint8_t* __restrict__ flags,
                                     const double* rho, const double* __restrict__ dc0, double mid, double shift,
                                     double step, double rho_min, double fixed_rho, int exclude_fixed, double* rho_out,
                                     double* __restrict__ part_sum, double* __restrict__ part_change) {
  double sum = 0, chg = 0;
  for (long t = long(blockIdx.x) * blockDim.x + threadIdx.x; t < ncells; t += long(gridDim.x) * blockDim.x) {
    if (!fat[t >> 6] || !(flags[t] & BAND_INSIDE)) continue;
    const double old = rho[t];
    double nd = oc_density(old, dc0[t], mid, shift, step, rho_min);
    const bool fx = (flags[t] & BAND_FIXED) != 0;
    if (fx) nd = fixed_rho;
    if (!(exclude_fixed && fx)) sum += nd;
    chg = fmax(chg, fabs(nd - old));
    if (rho_out) rho_out[t] = nd;
  }
  cta_sum_max(sum, chg, part_sum, part_change);
}

}  // namespace sgs
