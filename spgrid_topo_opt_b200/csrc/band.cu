// Narrow-band page maps on the GPU; see band.hpp.  Kernels work on the
// container in the caller's block order: a warp per block for the per-cell
// passes (two cells a lane, coalesced 256-byte rows), a thread per block for the
// block passes, a lock-free union-find for the 6-connected components.
#include <cub/cub.cuh>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <memory>
#include <string>

#include "band.hpp"

namespace sgs {
namespace {

constexpr int BAND_WARPS = 8;  // warps per CTA of the warp-per-block kernels
enum {
  CNT_THIN = 0, CNT_FAT, CNT_FATTER, CNT_ACTIVE, CNT_COMPONENTS, CNT_BIG, CNT_BIG_ROOT, CNT_ERROR, CNT_FAT_CHANGED,
  CNT_VOXELS, CNT_REMOVED, CNT_SOLID, CNT_N
};

// Block of the container holding the cell block (bx, by, bz), or -1.
__device__ __forceinline__ int lookup(const int* __restrict__ grid, int gx, int gy, int gz, int bx, int by, int bz) {
  if (bx < 0 || by < 0 || bz < 0 || bx >= gx || by >= gy || bz >= gz) return -1;
  return grid[(long(bx) * gy + by) * gz + bz];
}

// Page key of block (bx, by, bz) of its 4x4x4 grid: bit 3m is
// bit m of bz, 3m+1 of by, 3m+2 of bx (SPGrid_Mask.h:38-47 with 64-byte
// elements and 4 KiB pages).  Sorting by it gives the driver's list order.
uint64_t driver_page_key(int bx, int by, int bz) {
  uint64_t key = 0;
  for (int m = 0; m < 21; ++m) {
    key |= uint64_t((bz >> m) & 1) << (3 * m);
    key |= uint64_t((by >> m) & 1) << (3 * m + 1);
    key |= uint64_t((bx >> m) & 1) << (3 * m + 2);
  }
  return key;
}

// Thin map (update_thin_page_map, spgrid_topo_opt.cpp:100-116): a block of the
// fat map stays when its largest density (BlockMeta starts at 0) reaches
// minimum_density + active_threshold or one of its cells carries a force.  The
// block's density sum is accumulated in region order (cell 0..63), one add at a
// time as in the reference, for the fraction_to_keep selection.
__global__ void band_thin_kernel(long n, const double* __restrict__ rho, const uint8_t* __restrict__ flags,
                                 const uint8_t* __restrict__ fat_prev, double threshold, uint8_t* __restrict__ thin,
                                 double* __restrict__ meta_sum, unsigned long long* __restrict__ cnt) {
  __shared__ double cells[BAND_WARPS][64];
  const int wl = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const long b = long(blockIdx.x) * BAND_WARPS + wl;
  if (b >= n) return;
  if (!fat_prev[b]) {
    if (lane == 0) thin[b] = 0;
    return;
  }
  const double d0 = rho[b * 64 + lane], d1 = rho[b * 64 + 32 + lane];
  const bool force = __any_sync(0xffffffffu, ((flags[b * 64 + lane] | flags[b * 64 + 32 + lane]) & SGS_CELL_FORCE) != 0);
  // std::max(m, d) keeps m when d is NaN; so does fmax
  double mx = fmax(0.0, fmax(d0, d1));
  for (int o = 16; o; o >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
  cells[wl][lane] = d0;
  cells[wl][lane + 32] = d1;
  __syncwarp();
  if (lane == 0) {
    double s = 0;
    for (int e = 0; e < 64; ++e) s += cells[wl][e];
    meta_sum[b] = s;
    const bool keep = mx >= threshold || force;
    thin[b] = keep;
    if (keep) atomicAdd(cnt + CNT_THIN, 1ull);
  }
}

// fraction_to_keep: driver list position p -> the fat flag, density sum and
// thin flag of the block at that position.
__global__ void band_list_kernel(long n, const int* __restrict__ morton, const uint8_t* __restrict__ fat,
                                 const uint8_t* __restrict__ thin, const double* __restrict__ meta_sum,
                                 uint8_t* __restrict__ fat_m, uint8_t* __restrict__ thin_m, double* __restrict__ sum_m) {
  const long p = long(blockIdx.x) * blockDim.x + threadIdx.x;
  if (p >= n) return;
  const int b = morton[p];
  fat_m[p] = fat[b];
  thin_m[p] = thin[b];
  sum_m[p] = meta_sum[b];
}

// The reference keeps the b-th block of the old thin list when block_meta[b] --
// the meta of the b-th block of the fat list -- has a density sum above the
// threshold (spgrid_topo_opt.cpp:140-147).
__global__ void band_keep_kernel(long n_thin, const int* __restrict__ thin_list, const double* __restrict__ fat_sums,
                                 const double* __restrict__ threshold, uint8_t* __restrict__ thin) {
  const long p = long(blockIdx.x) * blockDim.x + threadIdx.x;
  if (p >= n_thin) return;
  if (fat_sums[p] > *threshold) thin[thin_list[p]] = 1;
}

// ---- 6-connected components of the thin blocks (filter_isolated_blocks) ----
// Union-find with parent[x] <= x for every x: a root is hooked under a smaller
// root by compare-and-swap, path halving writes ancestors only, so every chain
// strictly decreases and each loop ends within n steps (the bound is checked).
__device__ __forceinline__ int uf_find(int* parent, int x, long n, unsigned long long* err) {
  for (long it = 0; it <= n; ++it) {
    const int p = __ldcg(parent + x);
    if (p == x) return x;
    const int g = __ldcg(parent + p);
    if (g == p) return p;
    __stcg(parent + x, g);
    x = g;
  }
  atomicExch(err, 1ull);
  return x;
}

__device__ __forceinline__ void uf_union(int* parent, int x, int y, long n, unsigned long long* err) {
  for (long it = 0;; ++it) {
    if (it > n) {
      atomicExch(err, 1ull);
      return;
    }
    x = uf_find(parent, x, n, err);
    y = uf_find(parent, y, n, err);
    if (x == y) return;
    if (x > y) {
      const int t = x;
      x = y;
      y = t;
    }
    if (atomicCAS(parent + y, y, x) == y) return;  // else y gained a parent meanwhile: retry
  }
}

__global__ void band_cc_init_kernel(long n, const uint8_t* __restrict__ thin, int* __restrict__ parent,
                                    int* __restrict__ size) {
  const long b = long(blockIdx.x) * blockDim.x + threadIdx.x;
  if (b >= n) return;
  parent[b] = thin[b] ? int(b) : -1;
  size[b] = 0;
}

__global__ void band_cc_hook_kernel(long n, const int* __restrict__ base, const int* __restrict__ grid, int gx, int gy,
                                    int gz, const uint8_t* __restrict__ thin, int* parent, unsigned long long* cnt) {
  const long b = long(blockIdx.x) * blockDim.x + threadIdx.x;
  if (b >= n || !thin[b]) return;
  const int bx = base[3 * b] >> 2, by = base[3 * b + 1] >> 2, bz = base[3 * b + 2] >> 2;
  const int nbx[3] = {bx + 1, bx, bx}, nby[3] = {by, by + 1, by}, nbz[3] = {bz, bz, bz + 1};
  for (int v = 0; v < 3; ++v) {
    const int c = lookup(grid, gx, gy, gz, nbx[v], nby[v], nbz[v]);
    if (c >= 0 && thin[c]) uf_union(parent, int(b), c, n, cnt + CNT_ERROR);
  }
}

__global__ void band_cc_flatten_kernel(long n, const uint8_t* __restrict__ thin, int* parent, int* __restrict__ size,
                                       unsigned long long* cnt) {
  const long b = long(blockIdx.x) * blockDim.x + threadIdx.x;
  if (b >= n || !thin[b]) return;
  const int r = uf_find(parent, int(b), n, cnt + CNT_ERROR);
  atomicAdd(size + r, 1);
}

// Components (roots) and those holding more than 30% of the thin blocks: the
// reference's fraction 1.0 * s / total in float64 compared with 0.3 (:1466-1480).
__global__ void band_cc_roots_kernel(long n, const uint8_t* __restrict__ thin, const int* __restrict__ parent,
                                     const int* __restrict__ size, unsigned long long* cnt) {
  const long b = long(blockIdx.x) * blockDim.x + threadIdx.x;
  if (b >= n || !thin[b] || __ldcg(parent + b) != int(b)) return;
  atomicAdd(cnt + CNT_COMPONENTS, 1ull);
  const double total = double(cnt[CNT_THIN]);
  if (1.0 * size[b] / total > 0.3) {
    atomicAdd(cnt + CNT_BIG, 1ull);
    atomicExch(cnt + CNT_BIG_ROOT, (unsigned long long)b);
  }
}

// No union runs any more: the walk to the root is read-only and ends within n steps.
__global__ void band_cc_keep_kernel(long n, const int* __restrict__ parent, int root, uint8_t* __restrict__ thin) {
  const long b = long(blockIdx.x) * blockDim.x + threadIdx.x;
  if (b >= n || !thin[b]) return;
  int r = int(b);
  for (long it = 0; it <= n; ++it) {
    const int p = parent[r];
    if (p == r) break;
    r = p;
  }
  if (r != root) thin[b] = 0;
}

// ---- 6-connected components of the container cells (filter_isolated_voxels) ----
// The same union-find over cells c = b * 64 + e of the thin blocks; a cell's +x,
// +y, +z neighbours lie in its own block or at the opposite face of the
// neighbouring block.
__device__ __forceinline__ bool vox_member(const uint8_t* __restrict__ thin, const uint8_t* __restrict__ flags,
                                           long c) {
  return thin[c >> 6] && (flags[c] & SGS_CELL_INSIDE);
}

// adds the warp's count of true predicates to *counter (every lane of the warp calls it)
__device__ __forceinline__ void warp_count(bool pred, unsigned long long* counter) {
  const unsigned m = __ballot_sync(0xffffffffu, pred);
  if ((threadIdx.x & 31) == 0 && m) atomicAdd(counter, (unsigned long long)__popc(m));
}

__global__ void vox_init_kernel(long N, const uint8_t* __restrict__ thin, const uint8_t* __restrict__ flags,
                                int* __restrict__ parent, int* __restrict__ size, unsigned long long* cnt) {
  const long c = long(blockIdx.x) * blockDim.x + threadIdx.x;
  const bool m = c < N && vox_member(thin, flags, c);
  if (c < N) {
    parent[c] = m ? int(c) : -1;
    size[c] = 0;
  }
  warp_count(m, cnt + CNT_VOXELS);
}

__global__ void vox_hook_kernel(long N, const int* __restrict__ base, const int* __restrict__ grid, int gx, int gy,
                                int gz, const uint8_t* __restrict__ thin, const uint8_t* __restrict__ flags,
                                int* parent, unsigned long long* cnt) {
  const long c = long(blockIdx.x) * blockDim.x + threadIdx.x;
  if (c >= N || !vox_member(thin, flags, c)) return;
  const long b = c >> 6;
  const int e = int(c & 63);
  const int q[3] = {e >> 4, (e >> 2) & 3, e & 3}, stride[3] = {16, 4, 1};
  for (int v = 0; v < 3; ++v) {
    long d = c + stride[v];
    if (q[v] == 3) {
      const int nb = lookup(grid, gx, gy, gz, (base[3 * b] >> 2) + (v == 0), (base[3 * b + 1] >> 2) + (v == 1),
                            (base[3 * b + 2] >> 2) + (v == 2));
      if (nb < 0) continue;
      d = long(nb) * 64 + e - 3 * stride[v];
    }
    if (vox_member(thin, flags, d)) uf_union(parent, int(c), int(d), N, cnt + CNT_ERROR);
  }
}

__global__ void vox_flatten_kernel(long N, const uint8_t* __restrict__ thin, const uint8_t* __restrict__ flags,
                                   int* parent, int* __restrict__ size, unsigned long long* cnt) {
  const long c = long(blockIdx.x) * blockDim.x + threadIdx.x;
  if (c >= N || !vox_member(thin, flags, c)) return;
  atomicAdd(size + uf_find(parent, int(c), N, cnt + CNT_ERROR), 1);
}

// Components and those above 30% of the cells searched (:1580-1606).
__global__ void vox_roots_kernel(long N, const int* __restrict__ parent, const int* __restrict__ size,
                                 unsigned long long* cnt) {
  const long c = long(blockIdx.x) * blockDim.x + threadIdx.x;
  if (c >= N || __ldcg(parent + c) != int(c)) return;
  atomicAdd(cnt + CNT_COMPONENTS, 1ull);
  if (1.0 * size[c] / double(cnt[CNT_VOXELS]) > 0.3) {
    atomicAdd(cnt + CNT_BIG, 1ull);
    atomicExch(cnt + CNT_BIG_ROOT, (unsigned long long)c);
  }
}

// Cells outside the kept component leave the container with density 0 (:1611-1626).
__global__ void vox_keep_kernel(long N, const uint8_t* __restrict__ thin, const int* __restrict__ parent, int root,
                                uint8_t* __restrict__ flags, double* __restrict__ rho, unsigned long long* cnt) {
  const long c = long(blockIdx.x) * blockDim.x + threadIdx.x;
  bool drop = false;
  if (c < N && vox_member(thin, flags, c)) {
    int r = int(c);
    for (long it = 0; it <= N; ++it) {
      const int p = parent[r];
      if (p == r) break;
      r = p;
    }
    drop = r != root;
    if (drop) {
      flags[c] = uint8_t(flags[c] & ~SGS_CELL_INSIDE);
      rho[c] = 0.0;
    }
  }
  warp_count(drop, cnt + CNT_REMOVED);
}

// threshold_and_kill (:1333-1340): container cells below the threshold leave it.
__global__ void vox_kill_kernel(long N, const double* __restrict__ rho, double threshold, uint8_t* __restrict__ flags,
                                unsigned long long* cnt) {
  const long c = long(blockIdx.x) * blockDim.x + threadIdx.x;
  const bool kill = c < N && (flags[c] & SGS_CELL_INSIDE) && rho[c] < threshold;
  if (kill) flags[c] = uint8_t(flags[c] & ~SGS_CELL_INSIDE);
  warp_count(kill, cnt + CNT_REMOVED);
}

// threshold_density_trail (:1756-1778): the cells of fat blocks (all 64, as the
// reference walks whole blocks) with density >= t or a fixed density count as
// solid; with apply their density becomes 1, else 0.
__global__ void band_threshold_kernel(long n, const uint8_t* __restrict__ fat, const uint8_t* __restrict__ flags,
                                      double* __restrict__ rho, double t, int apply, unsigned long long* cnt) {
  const int wl = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const long b = long(blockIdx.x) * BAND_WARPS + wl;
  if (b >= n || !fat[b]) return;
  int solid = 0;
  for (int h = 0; h < 2; ++h) {
    const long c = b * 64 + lane + 32 * h;
    const bool s = rho[c] >= t || (flags[c] & SGS_CELL_FIXED);
    solid += s;
    if (apply) rho[c] = s ? 1.0 : 0.0;
  }
  for (int o = 16; o; o >>= 1) solid += __shfl_xor_sync(0xffffffffu, solid, o);
  if (lane == 0 && solid) atomicAdd(cnt + CNT_SOLID, (unsigned long long)solid);
}

// Fat map (update_fat_page_map, :166-186): every cell of a thin block whose
// density exceeds active_threshold marks the pages of its 8 diagonal neighbours
// at fat_margin that belong to the container.  With fat_margin <= 4 those pages
// are among the block's 27 neighbours, so a warp ORs a 27-bit set over its 64
// cells and 27 lanes write the marks.
__global__ void band_fat_kernel(long n, const int* __restrict__ base, const int* __restrict__ grid, int gx, int gy,
                                int gz, const uint8_t* __restrict__ thin, const double* __restrict__ rho,
                                double active_threshold, int margin, uint8_t* __restrict__ fat) {
  const int wl = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const long b = long(blockIdx.x) * BAND_WARPS + wl;
  if (b >= n || !thin[b]) return;
  unsigned set = 0;
  for (int h = 0; h < 2; ++h) {
    const int e = lane + 32 * h;
    if (!(rho[b * 64 + e] > active_threshold)) continue;
    const int p[3] = {e >> 4, (e >> 2) & 3, e & 3};
    for (int s = 0; s < 8; ++s) {
      int bit = 0;
      for (int v = 0; v < 3; ++v) {
        const int q = p[v] + (((s >> (2 - v)) & 1) ? margin : -margin);
        bit = bit * 3 + (q < 0 ? 0 : q > 3 ? 2 : 1);
      }
      set |= 1u << bit;
    }
  }
  set = __reduce_or_sync(0xffffffffu, set);
  if (lane < 27 && ((set >> lane) & 1)) {
    const int c = lookup(grid, gx, gy, gz, (base[3 * b] >> 2) + lane / 9 - 1, (base[3 * b + 1] >> 2) + (lane / 3) % 3 - 1,
                         (base[3 * b + 2] >> 2) + lane % 3 - 1);
    if (c >= 0) fat[c] = 1;
  }
}

// Fatter map (:188-200): a fat block and its +1 neighbours in every combination
// of axes, within the container.
__global__ void band_fatter_kernel(long n, const int* __restrict__ base, const int* __restrict__ grid, int gx, int gy,
                                   int gz, const uint8_t* __restrict__ fat, uint8_t* __restrict__ fatter) {
  const long b = long(blockIdx.x) * blockDim.x + threadIdx.x;
  if (b >= n || !fat[b]) return;
  const int bx = base[3 * b] >> 2, by = base[3 * b + 1] >> 2, bz = base[3 * b + 2] >> 2;
  for (int s = 0; s < 8; ++s) {
    const int c = lookup(grid, gx, gy, gz, bx + ((s >> 2) & 1), by + ((s >> 1) & 1), bz + (s & 1));
    if (c >= 0) fatter[c] = 1;
  }
}

// Map sizes, the blocks whose fat flag changed (fat_old may be null) and the
// active voxels of the fatter map (:215-235).
__global__ void band_count_kernel(long n, const uint8_t* __restrict__ thin, const uint8_t* __restrict__ fat,
                                  const uint8_t* __restrict__ fatter, const uint8_t* __restrict__ fat_old,
                                  const uint8_t* __restrict__ flags, const double* __restrict__ rho,
                                  double active_threshold, unsigned long long* cnt) {
  const int wl = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const long b = long(blockIdx.x) * BAND_WARPS + wl;
  if (b >= n) return;
  if (lane == 0) {
    if (thin[b]) atomicAdd(cnt + CNT_THIN, 1ull);
    if (fat[b]) atomicAdd(cnt + CNT_FAT, 1ull);
    if (fatter[b]) atomicAdd(cnt + CNT_FATTER, 1ull);
    if (fat_old && (fat_old[b] != 0) != (fat[b] != 0)) atomicAdd(cnt + CNT_FAT_CHANGED, 1ull);
  }
  if (!fatter[b]) return;
  int a = 0;
  for (int h = 0; h < 2; ++h) {
    const long c = b * 64 + lane + 32 * h;
    a += (flags[c] & SGS_CELL_INSIDE) && rho[c] > active_threshold;
  }
  for (int o = 16; o; o >>= 1) a += __shfl_xor_sync(0xffffffffu, a, o);
  if (lane == 0 && a) atomicAdd(cnt + CNT_ACTIVE, (unsigned long long)a);
}

}  // namespace

Band::Band(const int32_t* base_h_in, int64_t nblocks, const int32_t res[3], const uint8_t* flags_in,
           const double* density_h) {
  if (nblocks <= 0 || !base_h_in || !res || !flags_in || !density_h) throw CudaError("empty container", SGS_ERR_INPUT);
  n = long(nblocks);
  for (int v = 0; v < 3; ++v) {
    if (res[v] <= 0) throw CudaError("resolution must be positive", SGS_ERR_INPUT);
    gdim[v] = (res[v] + 3) / 4;
  }
  std::vector<int32_t> g(size_t(gdim[0]) * gdim[1] * gdim[2], -1);
  std::vector<std::pair<uint64_t, int32_t>> keys(static_cast<size_t>(n));
  for (long b = 0; b < n; ++b) {
    int bi[3];
    for (int v = 0; v < 3; ++v) {
      const int c = base_h_in[3 * b + v];
      if (c < 0 || c % 4 || c >= res[v]) throw CudaError("container block outside the grid or not 4-aligned", SGS_ERR_GRID);
      bi[v] = c >> 2;
    }
    int32_t& slot = g[(size_t(bi[0]) * gdim[1] + bi[1]) * gdim[2] + bi[2]];
    if (slot >= 0) throw CudaError("duplicate container block", SGS_ERR_GRID);
    slot = int32_t(b);
    keys[size_t(b)] = {driver_page_key(bi[0], bi[1], bi[2]), int32_t(b)};
  }
  std::sort(keys.begin(), keys.end());
  std::vector<int32_t> order(static_cast<size_t>(n));
  for (long p = 0; p < n; ++p) order[size_t(p)] = keys[size_t(p)].second;
  base_h.assign(base_h_in, base_h_in + 3 * n);
  flags_h.assign(flags_in, flags_in + 64 * n);
  for (long c = 0; c < n * 64; ++c) total_inside += (flags_in[c] & SGS_CELL_INSIDE) ? 1 : 0;
  SGS_CUDA(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
  SGS_CUDA(cudaEventCreate(&ev[0]));
  SGS_CUDA(cudaEventCreate(&ev[1]));
  base.upload(base_h_in, size_t(n) * 3, stream);
  grid.upload(g, stream);
  morton.upload(order, stream);
  flags.upload(flags_in, size_t(n) * 64, stream);
  rho.upload(density_h, size_t(n) * 64, stream);
  thin.alloc(size_t(n));
  fat.alloc(size_t(n));
  fatter.alloc(size_t(n));
  for (auto* m : {&thin, &fat, &fatter}) SGS_CUDA(cudaMemsetAsync(m->p, 1, size_t(n), stream));
  meta_sum.alloc(size_t(n));
  parent.alloc(size_t(n));
  comp_size.alloc(size_t(n));
  counters.alloc(CNT_N);
  SGS_CUDA(cudaStreamSynchronize(stream));
}

Band::~Band() {
  if (stream) cudaStreamSynchronize(stream);
  for (auto& e : ev)
    if (e) cudaEventDestroy(e);
  if (stream) cudaStreamDestroy(stream);
}

void Band::set_density(const double* h) {
  SGS_CUDA(cudaMemcpyAsync(rho.p, h, size_t(n) * 64 * sizeof(double), cudaMemcpyHostToDevice, stream));
  g_h2d_bytes += size_t(n) * 64 * sizeof(double);
  SGS_CUDA(cudaStreamSynchronize(stream));
}

void Band::get_density(double* h) {
  SGS_CUDA(cudaMemcpyAsync(h, rho.p, size_t(n) * 64 * sizeof(double), cudaMemcpyDeviceToHost, stream));
  g_d2h_bytes += size_t(n) * 64 * sizeof(double);
  SGS_CUDA(cudaStreamSynchronize(stream));
}

void Band::set_fat(const uint8_t* h) {
  SGS_CUDA(cudaMemcpyAsync(fat.p, h, size_t(n), cudaMemcpyHostToDevice, stream));
  g_h2d_bytes += size_t(n);
  SGS_CUDA(cudaStreamSynchronize(stream));
}

void Band::maps(uint8_t* t, uint8_t* f, uint8_t* ff) {
  const uint8_t* src[3] = {thin.p, fat.p, fatter.p};
  uint8_t* dst[3] = {t, f, ff};
  for (int m = 0; m < 3; ++m)
    if (dst[m]) {
      SGS_CUDA(cudaMemcpyAsync(dst[m], src[m], size_t(n), cudaMemcpyDeviceToHost, stream));
      g_d2h_bytes += size_t(n);
    }
  SGS_CUDA(cudaStreamSynchronize(stream));
}

void Band::get_flags(uint8_t* h) {
  SGS_CUDA(cudaMemcpyAsync(h, flags.p, size_t(n) * 64, cudaMemcpyDeviceToHost, stream));
  g_d2h_bytes += size_t(n) * 64;
  SGS_CUDA(cudaStreamSynchronize(stream));
}

void Band::pull_flags() { get_flags(flags_h.data()); }

void Band::filter_voxels(sgs_band_voxel_stats* st) {
  const long N = n * 64;
  if (N > long(INT32_MAX)) throw CudaError("container too large for the voxel filter", SGS_ERR_INPUT);
  DevBuf<int32_t> vparent, vsize;
  vparent.alloc(size_t(N));
  vsize.alloc(size_t(N));
  const unsigned cgrid = blocks_for(N, 256);
  SGS_CUDA(cudaEventRecord(ev[0], stream));
  SGS_CUDA(cudaMemsetAsync(counters.p, 0, CNT_N * sizeof(unsigned long long), stream));
  vox_init_kernel<<<cgrid, 256, 0, stream>>>(N, thin.p, flags.p, vparent.p, vsize.p, counters.p);
  vox_hook_kernel<<<cgrid, 256, 0, stream>>>(N, base.p, grid.p, gdim[0], gdim[1], gdim[2], thin.p, flags.p, vparent.p,
                                              counters.p);
  vox_flatten_kernel<<<cgrid, 256, 0, stream>>>(N, thin.p, flags.p, vparent.p, vsize.p, counters.p);
  vox_roots_kernel<<<cgrid, 256, 0, stream>>>(N, vparent.p, vsize.p, counters.p);
  SGS_CUDA(cudaGetLastError());
  unsigned long long c[CNT_N];
  SGS_CUDA(cudaMemcpyAsync(c, counters.p, sizeof(c), cudaMemcpyDeviceToHost, stream));
  SGS_CUDA(cudaStreamSynchronize(stream));
  if (c[CNT_ERROR]) throw CudaError("union-find exceeded its step bound", SGS_ERR_INTERNAL);
  if (c[CNT_VOXELS] == 0) throw CudaError("no container voxels in the thin blocks", SGS_ERR_INPUT);
  const long components = long(c[CNT_COMPONENTS]);
  long removed = 0;
  if (components > 1) {
    if (c[CNT_BIG] != 1)
      throw CudaError(std::to_string(c[CNT_BIG]) + " voxel components hold more than 30% of the voxels",
                      SGS_ERR_INPUT);
    vox_keep_kernel<<<cgrid, 256, 0, stream>>>(N, thin.p, vparent.p, int(c[CNT_BIG_ROOT]), flags.p, rho.p,
                                               counters.p);
    SGS_CUDA(cudaGetLastError());
    SGS_CUDA(cudaMemcpyAsync(c + CNT_REMOVED, counters.p + CNT_REMOVED, sizeof(c[0]), cudaMemcpyDeviceToHost, stream));
    removed = long(c[CNT_REMOVED]);
  }
  SGS_CUDA(cudaEventRecord(ev[1], stream));
  if (removed) pull_flags();
  SGS_CUDA(cudaStreamSynchronize(stream));
  float ms = 0;
  SGS_CUDA(cudaEventElapsedTime(&ms, ev[0], ev[1]));
  if (st) {
    st->voxels = long(c[CNT_VOXELS]);
    st->components = components;
    st->kept = st->voxels - removed;
    st->removed = removed;
    st->device_seconds = ms * 1e-3;
  }
}

long Band::threshold_trail(double t, bool apply) {
  SGS_CUDA(cudaMemsetAsync(counters.p + CNT_SOLID, 0, sizeof(unsigned long long), stream));
  band_threshold_kernel<<<blocks_for(n, BAND_WARPS), 32 * BAND_WARPS, 0, stream>>>(n, fat.p, flags.p, rho.p, t,
                                                                                 apply ? 1 : 0, counters.p);
  SGS_CUDA(cudaGetLastError());
  unsigned long long c = 0;
  SGS_CUDA(cudaMemcpyAsync(&c, counters.p + CNT_SOLID, sizeof(c), cudaMemcpyDeviceToHost, stream));
  SGS_CUDA(cudaStreamSynchronize(stream));
  return long(c);
}

// threshold_density (:1780-1797): bisection on [0, 1] until lo + 1e-8 >= hi for
// the threshold whose solid count meets volume_fraction x total_container_voxels,
// then the design is thresholded at lo.  A threshold given (>= 0) is applied as is.
long Band::threshold_density(double volume_fraction, double threshold, double* used) {
  double t = threshold;
  if (!(threshold >= 0)) {
    const double target = volume_fraction * double(total_inside);
    double lo = 0, hi = 1;
    while (lo + 1e-8 < hi) {
      const double mid = (lo + hi) * 0.5;
      if (double(threshold_trail(mid, false)) > target)
        lo = mid;
      else
        hi = mid;
    }
    t = lo;
  }
  if (used) *used = t;
  return threshold_trail(t, true);
}

long Band::kill_below(double threshold) {
  const long N = n * 64;
  SGS_CUDA(cudaMemsetAsync(counters.p + CNT_REMOVED, 0, sizeof(unsigned long long), stream));
  vox_kill_kernel<<<blocks_for(N, 256), 256, 0, stream>>>(N, rho.p, threshold, flags.p, counters.p);
  SGS_CUDA(cudaGetLastError());
  unsigned long long killed = 0;
  SGS_CUDA(cudaMemcpyAsync(&killed, counters.p + CNT_REMOVED, sizeof(killed), cudaMemcpyDeviceToHost, stream));
  SGS_CUDA(cudaStreamSynchronize(stream));
  if (killed) pull_flags();
  return long(killed);
}

// fraction_to_keep (:121-151), with the reference's int(fraction * container
// blocks) target and its nth_element threshold over the fat blocks' sums.
void Band::keep_fraction(double fraction_to_keep, long n_thin) {
  const long keep = long(int(fraction_to_keep * double(n)));
  if (keep < n_thin) return;  // "constraint already satisfied"
  DevBuf<uint8_t> fat_m, thin_m;
  DevBuf<double> sum_m, fat_sums, sorted;
  DevBuf<int32_t> thin_list;
  DevBuf<int> nsel;
  fat_m.alloc(size_t(n));
  thin_m.alloc(size_t(n));
  sum_m.alloc(size_t(n));
  fat_sums.alloc(size_t(n));
  sorted.alloc(size_t(n));
  thin_list.alloc(size_t(n));
  nsel.alloc(2);
  band_list_kernel<<<blocks_for(n, 256), 256, 0, stream>>>(n, morton.p, fat.p, thin.p, meta_sum.p, fat_m.p, thin_m.p,
                                                            sum_m.p);
  SGS_CUDA(cudaGetLastError());
  size_t t1 = 0, t2 = 0, t3 = 0;
  SGS_CUDA(cub::DeviceSelect::Flagged(nullptr, t1, sum_m.p, fat_m.p, fat_sums.p, nsel.p, int(n), stream));
  SGS_CUDA(cub::DeviceSelect::Flagged(nullptr, t2, morton.p, thin_m.p, thin_list.p, nsel.p + 1, int(n), stream));
  SGS_CUDA(cub::DeviceRadixSort::SortKeys(nullptr, t3, fat_sums.p, sorted.p, int(n), 0, 64, stream));
  DevBuf<uint8_t> tmp;
  tmp.alloc(std::max(t1, std::max(t2, t3)));
  size_t tb = tmp.n;
  SGS_CUDA(cub::DeviceSelect::Flagged(tmp.p, tb, sum_m.p, fat_m.p, fat_sums.p, nsel.p, int(n), stream));
  tb = tmp.n;
  SGS_CUDA(cub::DeviceSelect::Flagged(tmp.p, tb, morton.p, thin_m.p, thin_list.p, nsel.p + 1, int(n), stream));
  int h[2];
  SGS_CUDA(cudaMemcpyAsync(h, nsel.p, sizeof(h), cudaMemcpyDeviceToHost, stream));
  SGS_CUDA(cudaStreamSynchronize(stream));
  const long n_fat = h[0];
  if (keep < 1 || keep > n_fat)
    throw CudaError("fraction_to_keep selects " + std::to_string(keep) + " blocks of a fat list of " +
                        std::to_string(n_fat),
                    SGS_ERR_INPUT);
  tb = tmp.n;
  SGS_CUDA(cub::DeviceRadixSort::SortKeys(tmp.p, tb, fat_sums.p, sorted.p, int(n_fat), 0, 64, stream));
  SGS_CUDA(cudaMemsetAsync(thin.p, 0, size_t(n), stream));
  band_keep_kernel<<<blocks_for(n_thin, 256), 256, 0, stream>>>(n_thin, thin_list.p, fat_sums.p,
                                                                 sorted.p + (keep - 1), thin.p);
  SGS_CUDA(cudaGetLastError());
  SGS_CUDA(cudaStreamSynchronize(stream));
}

void Band::update(const sgs_band_params& prm, sgs_band_stats* st) {
  if (prm.fat_margin < 0 || prm.fat_margin > 4) throw CudaError("fat_margin must be within 0..4", SGS_ERR_INPUT);
  const int gx = gdim[0], gy = gdim[1], gz = gdim[2];
  const unsigned wgrid = blocks_for(n, BAND_WARPS), tgrid = blocks_for(n, 256);
  // work on copies so that an update the reference would stop on leaves the maps as they were
  DevBuf<uint8_t> thin_new, fat_new, fatter_new;
  thin_new.alloc(size_t(n));
  fat_new.alloc(size_t(n));
  fatter_new.alloc(size_t(n));
  std::swap(thin.p, thin_new.p);  // thin_new holds the current thin map now
  SGS_CUDA(cudaEventRecord(ev[0], stream));
  SGS_CUDA(cudaMemsetAsync(counters.p, 0, CNT_N * sizeof(unsigned long long), stream));
  band_thin_kernel<<<wgrid, 32 * BAND_WARPS, 0, stream>>>(n, rho.p, flags.p, fat.p,
                                                         prm.minimum_density + prm.active_threshold, thin.p,
                                                         meta_sum.p, counters.p);
  SGS_CUDA(cudaGetLastError());
  unsigned long long c[CNT_N];
  auto read_counters = [&] {
    SGS_CUDA(cudaMemcpyAsync(c, counters.p, sizeof(c), cudaMemcpyDeviceToHost, stream));
    SGS_CUDA(cudaStreamSynchronize(stream));
  };
  auto fail = [&](const std::string& m) {
    std::swap(thin.p, thin_new.p);  // put the previous thin map back
    throw CudaError(m, SGS_ERR_INPUT);
  };
  read_counters();
  const long thin_before = long(c[CNT_THIN]);
  long n_thin = thin_before;
  if (prm.fraction_to_keep != 1.0) {
    try {
      keep_fraction(prm.fraction_to_keep, n_thin);
    } catch (const CudaError& e) {
      if (e.code != SGS_ERR_INPUT) throw;
      fail(e.what());
    }
    SGS_CUDA(cudaMemsetAsync(counters.p, 0, sizeof(unsigned long long), stream));
    band_count_kernel<<<wgrid, 32 * BAND_WARPS, 0, stream>>>(n, thin.p, fat.p, fatter.p, nullptr, flags.p, rho.p,
                                                              0.0, counters.p);
    SGS_CUDA(cudaGetLastError());
    read_counters();
    n_thin = long(c[CNT_THIN]);
    SGS_CUDA(cudaMemsetAsync(counters.p, 0, CNT_N * sizeof(unsigned long long), stream));
    SGS_CUDA(cudaMemcpyAsync(counters.p + CNT_THIN, c + CNT_THIN, sizeof(unsigned long long), cudaMemcpyHostToDevice,
                             stream));
  }
  long components = 0;
  if (prm.connectivity_filtering) {
    if (n_thin == 0) fail("no thin blocks left for the connectivity filter");
    band_cc_init_kernel<<<tgrid, 256, 0, stream>>>(n, thin.p, parent.p, comp_size.p);
    band_cc_hook_kernel<<<tgrid, 256, 0, stream>>>(n, base.p, grid.p, gx, gy, gz, thin.p, parent.p, counters.p);
    band_cc_flatten_kernel<<<tgrid, 256, 0, stream>>>(n, thin.p, parent.p, comp_size.p, counters.p);
    band_cc_roots_kernel<<<tgrid, 256, 0, stream>>>(n, thin.p, parent.p, comp_size.p, counters.p);
    SGS_CUDA(cudaGetLastError());
    read_counters();
    if (c[CNT_ERROR]) throw CudaError("union-find exceeded its step bound", SGS_ERR_INTERNAL);
    components = long(c[CNT_COMPONENTS]);
    if (components > 1) {
      if (c[CNT_BIG] != 1)
        fail(std::to_string(c[CNT_BIG]) + " block components hold more than 30% of the thin blocks");
      band_cc_keep_kernel<<<tgrid, 256, 0, stream>>>(n, parent.p, int(c[CNT_BIG_ROOT]), thin.p);
      SGS_CUDA(cudaGetLastError());
    }
  }
  SGS_CUDA(cudaMemsetAsync(fat_new.p, 0, size_t(n), stream));
  SGS_CUDA(cudaMemsetAsync(fatter_new.p, 0, size_t(n), stream));
  band_fat_kernel<<<wgrid, 32 * BAND_WARPS, 0, stream>>>(n, base.p, grid.p, gx, gy, gz, thin.p, rho.p,
                                                        prm.active_threshold, prm.fat_margin, fat_new.p);
  band_fatter_kernel<<<tgrid, 256, 0, stream>>>(n, base.p, grid.p, gx, gy, gz, fat_new.p, fatter_new.p);
  SGS_CUDA(cudaMemsetAsync(counters.p, 0, CNT_N * sizeof(unsigned long long), stream));
  band_count_kernel<<<wgrid, 32 * BAND_WARPS, 0, stream>>>(n, thin.p, fat_new.p, fatter_new.p, fat.p, flags.p,
                                                            rho.p, prm.active_threshold, counters.p);
  SGS_CUDA(cudaGetLastError());
  SGS_CUDA(cudaEventRecord(ev[1], stream));
  read_counters();
  std::swap(fat.p, fat_new.p);
  std::swap(fatter.p, fatter_new.p);
  float ms = 0;
  SGS_CUDA(cudaEventElapsedTime(&ms, ev[0], ev[1]));
  if (st) {
    st->container_blocks = n;
    st->thin_before_pruning = thin_before;
    st->thin_blocks = long(c[CNT_THIN]);
    st->fat_blocks = long(c[CNT_FAT]);
    st->fatter_blocks = long(c[CNT_FATTER]);
    st->components = components;
    st->active_voxels = long(c[CNT_ACTIVE]);
    st->fat_changed = long(c[CNT_FAT_CHANGED]);
    st->device_seconds = ms * 1e-3;
  }
}

}  // namespace sgs

// ===========================================================================
// C ABI
// ===========================================================================
using namespace sgs;

template <typename F>
static int band_call(sgs_band* h, F&& f) {
  if (!h || !h->band) return SGS_ERR_INPUT;
  try {
    f(*h->band);
  } catch (const CudaError& e) {
    h->error = e.what();
    return e.code;
  } catch (const std::exception& e) {
    h->error = e.what();
    return SGS_ERR_INTERNAL;
  }
  return 0;
}

SGS_API int sgs_band_create(const int32_t* block_base, int64_t nblocks, const int32_t resolution[3],
                            const uint8_t* cell_flags, const double* density, sgs_band** out, char* err,
                            int errlen) {
  if (!out) return SGS_ERR_INPUT;
  *out = nullptr;
  std::unique_ptr<sgs_band> h(new sgs_band());
  try {
    h->band.reset(new Band(block_base, nblocks, resolution, cell_flags, density));
  } catch (const CudaError& e) {
    if (err && errlen > 0) std::snprintf(err, size_t(errlen), "%s", e.what());
    return e.code;
  } catch (const std::exception& e) {
    if (err && errlen > 0) std::snprintf(err, size_t(errlen), "%s", e.what());
    return SGS_ERR_INTERNAL;
  }
  *out = h.release();
  return 0;
}

SGS_API void sgs_band_destroy(sgs_band* b) { delete b; }

SGS_API const char* sgs_band_last_error(sgs_band* b) { return b ? b->error.c_str() : "null band"; }

SGS_API int sgs_band_set_density(sgs_band* b, const double* density) {
  if (!density) return SGS_ERR_INPUT;
  return band_call(b, [&](Band& B) { B.set_density(density); });
}

SGS_API int sgs_band_get_density(sgs_band* b, double* density) {
  if (!density) return SGS_ERR_INPUT;
  return band_call(b, [&](Band& B) { B.get_density(density); });
}

SGS_API int sgs_band_set_fat(sgs_band* b, const uint8_t* fat) {
  if (!fat) return SGS_ERR_INPUT;
  return band_call(b, [&](Band& B) { B.set_fat(fat); });
}

SGS_API int sgs_band_update(sgs_band* b, const sgs_band_params* p, sgs_band_stats* stats) {
  if (!p) return SGS_ERR_INPUT;
  return band_call(b, [&](Band& B) { B.update(*p, stats); });
}

SGS_API int sgs_band_maps(sgs_band* b, uint8_t* thin, uint8_t* fat, uint8_t* fatter) {
  return band_call(b, [&](Band& B) { B.maps(thin, fat, fatter); });
}

SGS_API int sgs_band_get_flags(sgs_band* b, uint8_t* cell_flags) {
  if (!cell_flags) return SGS_ERR_INPUT;
  return band_call(b, [&](Band& B) { B.get_flags(cell_flags); });
}

SGS_API int sgs_band_filter_voxels(sgs_band* b, sgs_band_voxel_stats* stats) {
  return band_call(b, [&](Band& B) { B.filter_voxels(stats); });
}

SGS_API int sgs_band_kill_below(sgs_band* b, double threshold, int64_t* killed) {
  return band_call(b, [&](Band& B) {
    const long k = B.kill_below(threshold);
    if (killed) *killed = k;
  });
}

SGS_API int sgs_band_threshold_density(sgs_band* b, double volume_fraction, double threshold, double* threshold_used,
                                       int64_t* solid_voxels) {
  return band_call(b, [&](Band& B) {
    const long v = B.threshold_density(volume_fraction, threshold, threshold_used);
    if (solid_voxels) *solid_voxels = v;
  });
}
