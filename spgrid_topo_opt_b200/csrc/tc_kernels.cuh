// Level-0 FP32 operator on the 5th-generation tensor cores (tcgen05, sm_100a).
//
// The V-cycle's level-0 residual r = b - dx K u (SPGrid_Linear_Elasticity.h:214-344,
// in FP32 as the mixed-precision V-cycle runs it) recast as a GEMM per block of
// 4x4x8 nodes.  Every cell touching a node of the block (min corner in
// [-1,3]x[-1,3]x[-1,7], at most 225) with E != 0 becomes one row of
//     A[cell][24] = (u of its 8 corners, 3 components),
// and one MMA product per 128 rows gives
//     D[cell][48] = A . [72 K_mu | 72 K_la]^T
// against the element matrices in exact integers (|entries| <= 32: exact in
// TF32).  A is split into TF32 high and low parts (a = hi + lo, hi = a with
// the 13 low mantissa bits cleared, lo = a - hi exact), two MMAs per K step,
// so the products keep ~22 bits: the result matches FP32 arithmetic.  The
// epilogue forms y[I] = E (mu0 D[0:24] + lambda0 D[24:48]) / 72 per cell and
// adds it to the corner nodes inside the block in eight fixed phases (corner I
// of distinct cells lands on distinct nodes), so the sum is deterministic.
//
// Shared memory holds A (hi and lo) and B in the canonical K-major layout of
// tcgen05 without swizzle: 8-row x 16-byte core matrices, the two 16-byte
// halves of a K step LBO = 128 bytes apart, 8-row groups SBO = 768 bytes apart
// (six 16-byte K chunks per row group).  D lives in tensor memory: tile t (128
// rows) at column 64 t, 48 FP32 columns.  One thread issues the MMAs and
// commits them to an mbarrier; all threads wait on it for at most a second, and
// a timed-out wait sets an error word, ends the loop and frees the tensor
// memory instead of hanging.
#pragma once
#include <cstdint>

namespace sgs {

constexpr int TC_THREADS = 128;
constexpr int TC_MAX_ROWS = 256;                 // two M = 128 tiles (225 cells at most)
constexpr int TC_K = 24, TC_N = 48;
constexpr int TC_KCHUNKS = TC_K / 4;             // 16-byte chunks per row
constexpr int TC_GROUP_BYTES = TC_KCHUNKS * 128; // one 8-row group of all K chunks
constexpr int TC_A_BYTES = TC_MAX_ROWS / 8 * TC_GROUP_BYTES;  // 24 KiB per A copy
constexpr int TC_B_BYTES = TC_N / 8 * TC_GROUP_BYTES;         // 4.5 KiB
constexpr int TC_TMEM_COLS = 128;
constexpr uint64_t TC_WAIT_NS = 1000000000ull;   // an MMA wait gives up after one second

// dynamic shared memory layout (byte offsets, 1024-aligned base)
constexpr int TC_OFF_AHI = 0;
constexpr int TC_OFF_ALO = TC_OFF_AHI + TC_A_BYTES;
constexpr int TC_OFF_B = TC_OFF_ALO + TC_A_BYTES;
constexpr int TC_OFF_HALO = TC_OFF_B + TC_B_BYTES;                 // 360 float4
constexpr int TC_OFF_ACC = TC_OFF_HALO + 360 * 16;                 // 3 x 128 floats
constexpr int TC_OFF_ROWCELL = TC_OFF_ACC + 3 * 128 * 4;           // 256 shorts
constexpr int TC_OFF_MISC = TC_OFF_ROWCELL + TC_MAX_ROWS * 2;      // mbarrier, tmem address, counters
constexpr int TC_SMEM_BYTES = TC_OFF_MISC + 64 + 1024;             // + alignment slack

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
  d |= uint64_t((saddr >> 4) & 0x3FFF);          // start address
  d |= uint64_t((128 >> 4) & 0x3FFF) << 16;      // leading byte offset: next 16-byte K chunk
  d |= uint64_t((TC_GROUP_BYTES >> 4) & 0x3FFF) << 32;  // stride byte offset: next 8-row group
  d |= uint64_t(1) << 46;                        // descriptor version for sm100
  return d;                                      // base offset 0, layout type 0 (no swizzle)
}

// instruction descriptor: D F32, A and B TF32, both K-major, N = 48, M = 128
constexpr uint32_t TC_IDESC = (1u << 4) | (2u << 7) | (2u << 10) | (uint32_t(TC_N >> 3) << 17) | (uint32_t(128 >> 4) << 24);

__device__ __forceinline__ float tc_hi(float a) { return __uint_as_float(__float_as_uint(a) & 0xFFFFE000u); }

// byte offset of element k of row r in a K-major operand
__device__ __forceinline__ int tc_off(int r, int k) { return (r >> 3) * TC_GROUP_BYTES + (k >> 2) * 128 + (r & 7) * 16 + (k & 3) * 4; }

template <int OP>  // OP_KU: out = dx K u; OP_RES: out = b - dx K u
__global__ void __launch_bounds__(TC_THREADS) level0_tc_kernel(int nblocks, const int* __restrict__ nbrz,
                                                              const float4* __restrict__ u4,
                                                              const float* __restrict__ b, float* __restrict__ out,
                                                              long N, float dx, float mu72, float la72,
                                                              int* __restrict__ error) {
  extern __shared__ uint8_t tc_raw[];
  uint8_t* sm = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(tc_raw) + 1023) & ~uintptr_t(1023));
  uint8_t* sA_hi = sm + TC_OFF_AHI;
  uint8_t* sA_lo = sm + TC_OFF_ALO;
  uint8_t* sB = sm + TC_OFF_B;
  float4* halo = reinterpret_cast<float4*>(sm + TC_OFF_HALO);
  float* acc = reinterpret_cast<float*>(sm + TC_OFF_ACC);
  short* row_cell = reinterpret_cast<short*>(sm + TC_OFF_ROWCELL);
  uint64_t* mbar = reinterpret_cast<uint64_t*>(sm + TC_OFF_MISC);
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(sm + TC_OFF_MISC + 8);
  int* counts = reinterpret_cast<int*>(sm + TC_OFF_MISC + 16);  // [0..7] cells per (pass, warp), [8] abort
  __shared__ int snb[27];
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
  asm volatile("tcgen05.fence::before_thread_sync;");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;");
  const uint32_t tmem = *tmem_slot;
  pdl_wait();
  uint32_t phase = 0;

  for (int bi = blockIdx.x; bi < nblocks; bi += gridDim.x) {
    if (tid < 27) snb[tid] = nbrz[long(bi) * 27 + tid];
    __syncthreads();
    // stage the u/E halo: nodes [-1,4]x[-1,4]x[-1,8] as (sx, sy, sz) in [0,6)x[0,6)x[0,10)
    for (int h = tid; h < 360; h += TC_THREADS) {
      const int sx = h / 60, sy = (h / 10) % 6, sz = h % 10;
      const int lx = sx - 1, ly = sy - 1, lz = sz - 1;
      const int dxb = lx < 0 ? 0 : (lx > 3 ? 2 : 1), dyb = ly < 0 ? 0 : (ly > 3 ? 2 : 1), dzb = lz < 0 ? 0 : (lz > 7 ? 2 : 1);
      const int nb = snb[dxb * 9 + dyb * 3 + dzb];  // the zero pad block where there is none
      halo[h] = u4[long(nb) * 128 + ((lx & 3) << 5) + ((ly & 3) << 3) + (lz & 7)];
    }
    acc[tid] = 0.f;
    acc[128 + tid] = 0.f;
    acc[256 + tid] = 0.f;
    __syncthreads();
    // rows: the cells (min corner (cx, cy, cz) in [0,5)x[0,5)x[0,9) of the halo) with E != 0,
    // compacted in cell order; thread t tests cells t and t + 128
    int nmine = 0, mycell[2];
#pragma unroll
    for (int q = 0; q < 2; ++q) {
      const int c = tid + q * TC_THREADS;
      bool on = false;
      if (c < 225) {
        const int cx = c / 45, cy = (c / 9) % 5, cz = c % 9;
        on = halo[cx * 60 + cy * 10 + cz].w != 0.f;
      }
      const unsigned m = __ballot_sync(0xffffffffu, on);
      if (lane == 0) counts[warp + 4 * q] = __popc(m);
      mycell[q] = on ? (c | (__popc(m & ((1u << lane) - 1)) << 16)) : -1;
      nmine += on;
    }
    __syncthreads();
    int rows = 0;
    {
      int base[2][4];
      int run = 0;
#pragma unroll
      for (int q = 0; q < 2; ++q)
        for (int w = 0; w < 4; ++w) {
          base[q][w] = run;
          run += counts[w + 4 * q];
        }
      rows = run;
#pragma unroll
      for (int q = 0; q < 2; ++q) {
        if (mycell[q] < 0) continue;
        const int c = mycell[q] & 0xFFFF, r = base[q][warp] + (mycell[q] >> 16);
        row_cell[r] = short(c);
        const int cx = c / 45, cy = (c / 9) % 5, cz = c % 9;
#pragma unroll
        for (int J = 0; J < 8; ++J) {
          const float4 v = halo[(cx + (J >> 2)) * 60 + (cy + ((J >> 1) & 1)) * 10 + cz + (J & 1)];
          const float a[3] = {v.x, v.y, v.z};
#pragma unroll
          for (int w = 0; w < 3; ++w) {
            const float hi = tc_hi(a[w]);
            const int off = tc_off(r, J * 3 + w);
            *reinterpret_cast<float*>(sA_hi + off) = hi;
            *reinterpret_cast<float*>(sA_lo + off) = a[w] - hi;
          }
        }
      }
    }
    (void)nmine;
    const int ntiles = (rows + 127) >> 7;
    // the MMA reads A through the async proxy
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    asm volatile("tcgen05.fence::before_thread_sync;");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;");
    if (ntiles > 0) {
      if (tid == 0) {
        const uint32_t a_hi = tc_smem_addr(sA_hi), a_lo = tc_smem_addr(sA_lo), bb = tc_smem_addr(sB);
        const uint32_t zero_mask = 0;
        for (int t = 0; t < ntiles; ++t) {
          const uint32_t d = tmem + uint32_t(64 * t);
          for (int s = 0; s < TC_K / 8; ++s) {
            const uint64_t db = tc_desc(bb + 256 * s);
            const uint64_t dah = tc_desc(a_hi + t * 16 * TC_GROUP_BYTES + 256 * s);
            const uint64_t dal = tc_desc(a_lo + t * 16 * TC_GROUP_BYTES + 256 * s);
            asm volatile(
                "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
                "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, {%5, %5, %5, %5}, p;\n\t}\n" ::"r"(d),
                "l"(dah), "l"(db), "r"(TC_IDESC), "r"(s > 0 ? 1u : 0u), "r"(zero_mask));
            asm volatile(
                "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
                "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, {%5, %5, %5, %5}, p;\n\t}\n" ::"r"(d),
                "l"(dal), "l"(db), "r"(TC_IDESC), "r"(1u), "r"(zero_mask));
          }
        }
        asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                         tc_smem_addr(mbar))
                     : "memory");
      }
      // wait for the products, for at most TC_WAIT_NS of wall time
      const uint64_t t0 = tc_globaltimer();
      uint32_t done = 0;
      while (true) {
        asm volatile(
            "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n\t}\n"
            : "=r"(done)
            : "r"(tc_smem_addr(mbar)), "r"(phase)
            : "memory");
        if (done || tc_globaltimer() - t0 > TC_WAIT_NS) break;
      }
      if (!done) {
        atomicExch(error, 1);
        counts[8] = 1;
      }
      phase ^= 1u;
      asm volatile("tcgen05.fence::after_thread_sync;");
      // row tid of each tile: tensor-memory lane tid (warp w reads lanes 32w..32w+31)
      for (int t = 0; t < ntiles; ++t) {
        const int r = t * 128 + tid;
        uint32_t d[48];
        const uint32_t taddr = tmem + (uint32_t(warp * 32) << 16) + uint32_t(64 * t);
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
        const bool valid = r < rows;
        int cx = 0, cy = 0, cz = 0;
        float E = 0.f;
        if (valid) {
          const int c = row_cell[r];
          cx = c / 45;
          cy = (c / 9) % 5;
          cz = c % 9;
          E = halo[cx * 60 + cy * 10 + cz].w;
        }
        // corner I of the cell is node (cx + Ix - 1, cy + Iy - 1, cz + Iz - 1) of the block
#pragma unroll
        for (int I = 0; I < 8; ++I) {
          const int nx = cx + (I >> 2) - 1, ny = cy + ((I >> 1) & 1) - 1, nz = cz + (I & 1) - 1;
          const bool inside = valid && nx >= 0 && nx < 4 && ny >= 0 && ny < 4 && nz >= 0 && nz < 8;
          if (inside) {
            const int node = nx * 32 + ny * 8 + nz;
#pragma unroll
            for (int v = 0; v < 3; ++v)
              acc[v * 128 + node] += E * (mu72 * __uint_as_float(d[3 * I + v]) + la72 * __uint_as_float(d[24 + 3 * I + v]));
          }
          __syncthreads();  // one corner at a time: distinct cells, distinct nodes
        }
      }
    }
    asm volatile("tcgen05.fence::before_thread_sync;");
    __syncthreads();
    const long g = long(bi) * 128 + tid;
#pragma unroll
    for (int v = 0; v < 3; ++v) {
      const float f = acc[v * 128 + tid] * dx;
      out[g + v * N] = OP == OP_RES ? b[g + v * N] - f : f;
    }
    if (counts[8]) break;  // a wait gave up: leave the loop, release tensor memory
  }
  __syncthreads();
  if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TC_TMEM_COLS));
}

}  // namespace sgs
