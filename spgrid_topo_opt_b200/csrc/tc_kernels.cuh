// Level-0 FP32 operator on the 5th-generation tensor cores (tcgen05, sm_100a).
//
// The V-cycle's level-0 residual r = b - dx K u (SPGrid_Linear_Elasticity.h:214-344,
// in FP32 as the mixed-precision V-cycle runs it) recast as a GEMM per block of
// 4x4x8 nodes.  Every cell touching a node of the block (min corner in
// [-1,3]x[-1,3]x[-1,7], at most 225) with E != 0 becomes one row of
//     A[cell][24] = (u of its 8 corners, 3 components),
// and one MMA chain per 128 rows gives
//     D[cell][48] = A . [72 K_mu | 72 K_la]^T
// against the element matrices in exact integers (|entries| <= 32: exact in
// TF32).  A is split into TF32 high and low parts (a = hi + lo, hi = a with
// the 13 low mantissa bits cleared, lo = a - hi exact), two MMAs per K step,
// so the products keep ~22 bits: the result matches FP32 arithmetic.  The
// thread that owns a row forms y[I] = E (mu0 D[0:24] + lambda0 D[24:48]) / 72
// and stores it in shared memory; then every node sums the y of its 8 cells in
// a fixed corner order, so the result does not depend on scheduling.  Shared
// memory is the kernel's bottleneck, so its layouts avoid bank conflicts: A rows
// go out as 16-byte chunks, y is stored column-major.
//
// The CTA is persistent over blocks.  While one block is computed, the halo of
// the next one (its u/E nodes and b) is already in flight with cp.async into
// the other of two buffers, and the neighbour table of the block after that
// is loaded into registers, so the memory latency overlaps the MMA work.
//
// Shared memory holds A (hi and lo) and B in the canonical K-major layout of
// tcgen05 without swizzle: 8-row x 16-byte core matrices, the two 16-byte
// halves of a K step LBO = 128 bytes apart, 8-row groups SBO = 768 bytes apart
// (six 16-byte K chunks per row group).  D (128 rows x 48 FP32) lives in 64
// columns of tensor memory.  One thread issues the MMAs and commits them to an
// mbarrier; all threads wait on it for at most a second, and a timed-out wait
// sets an error word, ends the loop and frees the tensor memory instead of
// hanging.
#pragma once
#include <cstdint>

namespace sgs {

constexpr int TC_THREADS = 128;
constexpr int TC_ROWS = 128;                     // one M = 128 tile at a time
constexpr int TC_K = 24, TC_N = 48;
constexpr int TC_KCHUNKS = TC_K / 4;             // 16-byte chunks per row
constexpr int TC_GROUP_BYTES = TC_KCHUNKS * 128; // one 8-row group of all K chunks
constexpr int TC_A_BYTES = TC_ROWS / 8 * TC_GROUP_BYTES;  // 12 KiB per A copy
constexpr int TC_B_BYTES = TC_N / 8 * TC_GROUP_BYTES;     // 4.5 KiB
constexpr int TC_TMEM_COLS = 64;
constexpr int TC_HALO = 360;                     // nodes [-1,4]x[-1,4]x[-1,8]
constexpr int TC_CELLS = 225;                    // cells [-1,3]x[-1,3]x[-1,7]
constexpr uint64_t TC_WAIT_NS = 1000000000ull;   // an MMA wait gives up after one second

// dynamic shared memory layout (byte offsets from a 128-aligned base)
constexpr int TC_OFF_AHI = 0;                                  // also y[24][128] after the MMA
constexpr int TC_OFF_ALO = TC_OFF_AHI + TC_A_BYTES;
constexpr int TC_OFF_B = TC_OFF_ALO + TC_A_BYTES;
constexpr int TC_OFF_HALO = TC_OFF_B + TC_B_BYTES;             // 2 x 360 float4
constexpr int TC_OFF_BV = TC_OFF_HALO + 2 * TC_HALO * 16;      // 2 x 3 x 128 floats of b
constexpr int TC_OFF_ROW = TC_OFF_BV + 2 * 3 * 128 * 4;        // cell -> row (255: none), 225 bytes
constexpr int TC_OFF_CELL = TC_OFF_ROW + 256;                  // row -> cell, 256 bytes
constexpr int TC_OFF_MISC = TC_OFF_CELL + 256;                 // mbarrier, tensor memory address, counters
constexpr int TC_SMEM_BYTES = TC_OFF_MISC + 64 + 128;          // + alignment slack

__device__ __forceinline__ uint64_t tc_globaltimer() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

__device__ __forceinline__ uint32_t tc_smem_addr(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// canonical K-major, no-swizzle shared-memory descriptor (sm100 version 1)
__device__ __forceinline__ uint64_t tc_desc(uint32_t saddr) {
  uint64_t d = 0;
  d |= uint64_t((saddr >> 4) & 0x3FFF);                 // start address
  d |= uint64_t((128 >> 4) & 0x3FFF) << 16;             // leading byte offset: next 16-byte K chunk
  d |= uint64_t((TC_GROUP_BYTES >> 4) & 0x3FFF) << 32;  // stride byte offset: next 8-row group
  d |= uint64_t(1) << 46;                               // descriptor version for sm100
  return d;                                             // base offset 0, layout type 0 (no swizzle)
}

// instruction descriptor: D F32, A and B TF32, both K-major, N = 48, M = 128
constexpr uint32_t TC_IDESC = (1u << 4) | (2u << 7) | (2u << 10) | (uint32_t(TC_N >> 3) << 17) | (uint32_t(128 >> 4) << 24);

__device__ __forceinline__ float tc_hi(float a) { return __uint_as_float(__float_as_uint(a) & 0xFFFFE000u); }

// byte offset of element k of row r in a K-major operand
__device__ __forceinline__ int tc_off(int r, int k) {
  return (r >> 3) * TC_GROUP_BYTES + (k >> 2) * 128 + (r & 7) * 16 + (k & 3) * 4;
}

__device__ __forceinline__ void tc_cp16(void* dst, const void* src) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 16;" ::"r"(tc_smem_addr(dst)), "l"(src) : "memory");
}

// Issue the loads of block bi's halo (u/E nodes) and b into one buffer; nb27
// holds its neighbour table (the zero pad block where a neighbour is missing).
template <int OP>
__device__ __forceinline__ void tc_prefetch(int bi, const int* nb27, float4* halo, float* bv,
                                            const float4* __restrict__ u4, const float* __restrict__ b, long N) {
  for (int h = threadIdx.x; h < TC_HALO; h += TC_THREADS) {
    const int sx = h / 60, sy = (h / 10) % 6, sz = h % 10;
    const int lx = sx - 1, ly = sy - 1, lz = sz - 1;
    const int dxb = lx < 0 ? 0 : (lx > 3 ? 2 : 1), dyb = ly < 0 ? 0 : (ly > 3 ? 2 : 1), dzb = lz < 0 ? 0 : (lz > 7 ? 2 : 1);
    const int nb = nb27[dxb * 9 + dyb * 3 + dzb];
    tc_cp16(halo + h, u4 + (long(nb) * 128 + ((lx & 3) << 5) + ((ly & 3) << 3) + (lz & 7)));
  }
  if (OP == OP_RES && threadIdx.x < 96) {  // 3 planes x 32 chunks of 4 floats
    const int v = threadIdx.x >> 5, c = threadIdx.x & 31;
    tc_cp16(bv + v * 128 + 4 * c, b + long(bi) * 128 + v * N + 4 * c);
  }
  asm volatile("cp.async.commit_group;" ::: "memory");
}

template <int OP>  // OP_KU: out = dx K u; OP_RES: out = b - dx K u
__global__ void __launch_bounds__(TC_THREADS) level0_tc_kernel(int nblocks, const int* __restrict__ nbrz,
                                                              const float4* __restrict__ u4,
                                                              const float* __restrict__ b, float* __restrict__ out,
                                                              long N, float dx, float mu72, float la72,
                                                              int* __restrict__ error) {
  extern __shared__ uint8_t tc_raw[];
  uint8_t* sm = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(tc_raw) + 127) & ~uintptr_t(127));
  uint8_t* sA_hi = sm + TC_OFF_AHI;
  uint8_t* sA_lo = sm + TC_OFF_ALO;
  float* sY = reinterpret_cast<float*>(sm + TC_OFF_AHI);  // y[24][row] once the products are in
  uint8_t* sB = sm + TC_OFF_B;
  float4* halo_buf = reinterpret_cast<float4*>(sm + TC_OFF_HALO);
  float* bv_buf = reinterpret_cast<float*>(sm + TC_OFF_BV);
  uint8_t* cell_row = sm + TC_OFF_ROW;
  uint8_t* row_cell = sm + TC_OFF_CELL;
  uint64_t* mbar = reinterpret_cast<uint64_t*>(sm + TC_OFF_MISC);
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(sm + TC_OFF_MISC + 8);
  int* counts = reinterpret_cast<int*>(sm + TC_OFF_MISC + 16);  // [0..7] cells per (pass, warp), [8] abort
  __shared__ int snb2[2][27];
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;

  // B = [72 K_mu | 72 K_la] as [n = (I, v)][k = (J, w)], exact small integers
  for (int idx = tid; idx < TC_N * TC_K; idx += TC_THREADS) {
    const int n = idx / TC_K, k = idx % TC_K;
    const int I = (n % 24) / 3, v = n % 3, J = k / 3, w = k % 3;
    const int val = n < 24 ? q1_mu72(I, J, v, w) : q1_la72(I, J, v, w);
    *reinterpret_cast<float*>(sB + tc_off(n, k)) = float(val);
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(tc_smem_addr(tmem_slot)),
                 "r"(TC_TMEM_COLS));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  if (tid == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(tc_smem_addr(mbar)));
    counts[8] = 0;
  }
  // the neighbour tables of the first two blocks (constant during a solve: before the wait)
  const int first = blockIdx.x;
  if (tid < 27 && first < nblocks) snb2[0][tid] = nbrz[long(first) * 27 + tid];
  const int second = first + int(gridDim.x);
  int nb_ahead = (tid < 27 && second < nblocks) ? nbrz[long(second) * 27 + tid] : 0;
  asm volatile("tcgen05.fence::before_thread_sync;");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;");
  const uint32_t tmem = *tmem_slot;
  pdl_wait();
  if (first < nblocks) tc_prefetch<OP>(first, snb2[0], halo_buf, bv_buf, u4, b, N);
  uint32_t phase = 0;
  int buf = 0;

  for (int bi = first; bi < nblocks; bi += gridDim.x, buf ^= 1) {
    const int next = bi + int(gridDim.x);
    const float4* halo = halo_buf + buf * TC_HALO;
    const float* bv = bv_buf + buf * 384;
    // start the next block's loads, then wait for this block's
    if (next < nblocks) {
      if (tid < 27) snb2[buf ^ 1][tid] = nb_ahead;
      const int after = next + int(gridDim.x);
      nb_ahead = (tid < 27 && after < nblocks) ? nbrz[long(after) * 27 + tid] : 0;
      __syncthreads();
      tc_prefetch<OP>(next, snb2[buf ^ 1], halo_buf + (buf ^ 1) * TC_HALO, bv_buf + (buf ^ 1) * 384, u4, b, N);
      asm volatile("cp.async.wait_group 1;" ::: "memory");
    } else {
      asm volatile("cp.async.wait_group 0;" ::: "memory");
    }
    __syncthreads();
    // rows: the cells (min corner (cx, cy, cz) in [0,5)x[0,5)x[0,9) of the halo) with E != 0,
    // compacted in cell order; thread t tests cells t and t + 128
    int mycell[2];
#pragma unroll
    for (int q = 0; q < 2; ++q) {
      const int c = tid + q * TC_THREADS;
      bool on = false;
      if (c < TC_CELLS) on = halo[(c / 45) * 60 + ((c / 9) % 5) * 10 + c % 9].w != 0.f;
      const unsigned m = __ballot_sync(0xffffffffu, on);
      if (lane == 0) counts[warp + 4 * q] = __popc(m);
      mycell[q] = on ? (c | (__popc(m & ((1u << lane) - 1)) << 16)) : (c < TC_CELLS ? -1 - c : -1000);
    }
    __syncthreads();
    int rows;
    {
      int base[2][4];
      int run = 0;
#pragma unroll
      for (int q = 0; q < 2; ++q)
#pragma unroll
        for (int w = 0; w < 4; ++w) {
          base[q][w] = run;
          run += counts[w + 4 * q];
        }
      rows = run;
#pragma unroll
      for (int q = 0; q < 2; ++q) {
        if (mycell[q] >= 0) {
          const int c = mycell[q] & 0xFFFF, r = base[q][warp] + (mycell[q] >> 16);
          cell_row[c] = uint8_t(r);
          row_cell[r] = uint8_t(c);
        } else if (mycell[q] > -1000) {
          cell_row[-1 - mycell[q]] = 255;
        }
      }
    }
    __syncthreads();
    float f0 = 0.f, f1 = 0.f, f2 = 0.f;  // this thread's node, summed over the tiles
    const int ex = tid >> 5, ey = (tid >> 3) & 3, ez = tid & 7;
    for (int t0 = 0; t0 < rows; t0 += TC_ROWS) {
      const int nrow = min(TC_ROWS, rows - t0);
      // A rows of this tile: thread r builds row t0 + r in registers and stores it
      // as 16-byte chunks (8 consecutive rows of a chunk fill all 32 banks)
      if (tid < nrow) {
        const int c = row_cell[t0 + tid];
        const int cx = c / 45, cy = (c / 9) % 5, cz = c % 9;
        float a[TC_K];
#pragma unroll
        for (int J = 0; J < 8; ++J) {
          const float4 v = halo[(cx + (J >> 2)) * 60 + (cy + ((J >> 1) & 1)) * 10 + cz + (J & 1)];
          a[3 * J] = v.x;
          a[3 * J + 1] = v.y;
          a[3 * J + 2] = v.z;
        }
#pragma unroll
        for (int q = 0; q < TC_KCHUNKS; ++q) {
          const float4 hi = make_float4(tc_hi(a[4 * q]), tc_hi(a[4 * q + 1]), tc_hi(a[4 * q + 2]), tc_hi(a[4 * q + 3]));
          const float4 lo = make_float4(a[4 * q] - hi.x, a[4 * q + 1] - hi.y, a[4 * q + 2] - hi.z, a[4 * q + 3] - hi.w);
          const int off = tc_off(tid, 4 * q);
          *reinterpret_cast<float4*>(sA_hi + off) = hi;
          *reinterpret_cast<float4*>(sA_lo + off) = lo;
        }
      }
      // the MMA reads A through the async proxy
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      asm volatile("tcgen05.fence::before_thread_sync;");
      __syncthreads();
      asm volatile("tcgen05.fence::after_thread_sync;");
      if (tid == 0) {
        const uint32_t a_hi = tc_smem_addr(sA_hi), a_lo = tc_smem_addr(sA_lo), bb = tc_smem_addr(sB);
        const uint32_t zero_mask = 0;
#pragma unroll
        for (int s = 0; s < TC_K / 8; ++s) {
          const uint64_t db = tc_desc(bb + 256 * s);
          const uint64_t dah = tc_desc(a_hi + 256 * s);
          const uint64_t dal = tc_desc(a_lo + 256 * s);
          asm volatile(
              "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
              "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, {%5, %5, %5, %5}, p;\n\t}\n" ::"r"(tmem),
              "l"(dah), "l"(db), "r"(TC_IDESC), "r"(s > 0 ? 1u : 0u), "r"(zero_mask));
          asm volatile(
              "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
              "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, {%5, %5, %5, %5}, p;\n\t}\n" ::"r"(tmem),
              "l"(dal), "l"(db), "r"(TC_IDESC), "r"(1u), "r"(zero_mask));
        }
        asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                         tc_smem_addr(mbar))
                     : "memory");
      }
      // wait for the products, for at most TC_WAIT_NS of wall time
      const uint64_t tw = tc_globaltimer();
      uint32_t done = 0;
      while (true) {
        asm volatile(
            "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n\t}\n"
            : "=r"(done)
            : "r"(tc_smem_addr(mbar)), "r"(phase)
            : "memory");
        if (done || tc_globaltimer() - tw > TC_WAIT_NS) break;
      }
      if (!done) {
        atomicExch(error, 1);
        counts[8] = 1;
      }
      phase ^= 1u;
      asm volatile("tcgen05.fence::after_thread_sync;");
      // row tid of the tile is tensor-memory lane tid (warp w reads lanes 32w..32w+31)
      uint32_t d[48];
      const uint32_t taddr = tmem + (uint32_t(warp * 32) << 16);
#pragma unroll
      for (int c = 0; c < 3; ++c)
        asm volatile(
            "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, "
            "%14, %15}, [%16];"
            : "=r"(d[16 * c + 0]), "=r"(d[16 * c + 1]), "=r"(d[16 * c + 2]), "=r"(d[16 * c + 3]),
              "=r"(d[16 * c + 4]), "=r"(d[16 * c + 5]), "=r"(d[16 * c + 6]), "=r"(d[16 * c + 7]),
              "=r"(d[16 * c + 8]), "=r"(d[16 * c + 9]), "=r"(d[16 * c + 10]), "=r"(d[16 * c + 11]),
              "=r"(d[16 * c + 12]), "=r"(d[16 * c + 13]), "=r"(d[16 * c + 14]), "=r"(d[16 * c + 15])
            : "r"(taddr + uint32_t(16 * c)));
      asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
      asm volatile("tcgen05.fence::before_thread_sync;");
      __syncthreads();  // A is no longer read: y overwrites it
      // y stored column-major, sY[n][row]: the row owners write consecutive words
      if (tid < nrow) {
        const int c = row_cell[t0 + tid];
        const float E = halo[(c / 45) * 60 + ((c / 9) % 5) * 10 + c % 9].w;
#pragma unroll
        for (int n = 0; n < 24; ++n)
          sY[n * TC_ROWS + tid] = E * (mu72 * __uint_as_float(d[n]) + la72 * __uint_as_float(d[24 + n]));
      }
      __syncthreads();
      // node (ex, ey, ez) takes corner I of the cell (ex, ey, ez) - I: halo cell + 1 - I
#pragma unroll
      for (int I = 0; I < 8; ++I) {
        const int cx = ex + 1 - (I >> 2), cy = ey + 1 - ((I >> 1) & 1), cz = ez + 1 - (I & 1);
        const int r = int(cell_row[cx * 45 + cy * 9 + cz]) - t0;  // 255: no row
        if (cell_row[cx * 45 + cy * 9 + cz] != 255 && r >= 0 && r < nrow) {
          const float* yr = sY + 3 * I * TC_ROWS + r;
          f0 += yr[0];
          f1 += yr[TC_ROWS];
          f2 += yr[2 * TC_ROWS];
        }
      }
      asm volatile("tcgen05.fence::before_thread_sync;");
      __syncthreads();  // y is read: the next tile may overwrite A
    }
    const long g = long(bi) * 128 + tid;
    const float fv[3] = {f0 * dx, f1 * dx, f2 * dx};
#pragma unroll
    for (int v = 0; v < 3; ++v) out[g + v * N] = OP == OP_RES ? bv[v * 128 + tid] - fv[v] : fv[v];
    if (counts[8]) break;  // a wait gave up: leave the loop, release tensor memory
  }
  asm volatile("cp.async.wait_group 0;" ::: "memory");
  __syncthreads();
  if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TC_TMEM_COLS));
}

}  // namespace sgs
