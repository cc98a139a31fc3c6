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

// One trial of the OC bisection at multiplier mid: the new density of every
// container cell, per-CTA partial sums of the counted densities and maxima of
// the change; with rho_out the densities are also written, at least DBL_MIN
// when keep_inside (a container cell stays in the container, as the driver's
// packing ensures, spgrid_topo_opt.cpp:1122).
__global__ void oc_trial_kernel(long n, const double* rho, const double* __restrict__ dc0,
                                const uint8_t* __restrict__ fixed, double mid, double shift, double step,
                                double rho_min, double fixed_rho, int exclude_fixed, double* rho_out,
                                double* __restrict__ part_sum, double* __restrict__ part_change, int keep_inside) {
  __shared__ double ss[OC_THREADS / 32], sc[OC_THREADS / 32];
  double sum = 0, chg = 0;
  for (long t = long(blockIdx.x) * blockDim.x + threadIdx.x; t < n; t += long(gridDim.x) * blockDim.x) {
    const double old = rho[t];
    if (!(old > 0)) continue;
    double nd = old * sqrt(fmax(0.0, -dc0[t] - shift) / mid);
    nd = fmin(fmax(nd, old - step), old + step);
    nd = fmin(fmax(nd, rho_min), 1.0);
    const bool fx = fixed && fixed[t];
    if (fx) nd = fixed_rho;
    if (!(exclude_fixed && fx)) sum += nd;
    chg = fmax(chg, fabs(nd - old));
    if (rho_out) rho_out[t] = keep_inside ? fmax(nd, 2.2250738585072014e-308) : nd;
  }
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

}  // namespace sgs
