// CUDA kernels of the narrow-band SPGrid elasticity MGPCG (sm_100a).
//
// Layout: a level holds nb active blocks of 4x4x8 nodes in SPGrid page order;
// node slot e = x*32 + y*8 + z inside a block, global node index b*128 + e.
// A 3-vector field is stored as three planes of N = nb*128 values ([3][N]).
// Level 0 carries the per-cell stiffness scale E (cell = its min-corner node,
// 0 = empty); the element matrix of a cell is E * (mu0*K_mu + lambda0*K_la).
// Coarse levels carry 27-point Galerkin stencils node-major, [N][243], entry
// ((i*3+j)*3+k)*9 + v*3 + w = row (node, v), column (node + (i,j,k) - 1, w).
#pragma once
#include <cstdint>

namespace sgs {

constexpr uint32_t ACTIVE_NODE = 0x10, DIR_X = 0x20, DIR_Y = 0x40, DIR_Z = 0x80, BOUNDARY_NODE = 0x1000;

// Combined element matrix Kc[I][J][v][w] = mu0*K_mu + lambda0*K_la (set per solve)
__constant__ double c_Kc64[8 * 8 * 9];
__constant__ float c_Kc32[8 * 8 * 9];

template <typename T>
__device__ __forceinline__ T kc(int idx);
template <>
__device__ __forceinline__ double kc<double>(int idx) { return c_Kc64[idx]; }
template <>
__device__ __forceinline__ float kc<float>(int idx) { return c_Kc32[idx]; }

__device__ __forceinline__ double round_to_float(double v) { return double(float(v)); }

// The element matrix in exact integers, 72 K_mu and 72 K_la of the Q1 hex on the
// unit cube (node a = 4x + 2y + z), from the 1D integrals of the linear shape
// functions times 6 (mass {2, 1}, derivative-mass {-3, 3}, stiffness {6, -6});
// the same formulas as element_tables() in solver.cu.  Up to sign the 576
// entries take 10 values (m, l), so Kc = (mu0 m + lambda0 l) / 72 is 10 numbers,
// which the single-precision level-0 kernels keep in registers (KcReg).
__host__ __device__ constexpr int q1_g(int a, int b, int i, int j) {
  int v = 1;
  for (int ax = 0; ax < 3; ++ax) {
    const int pa = (a >> (2 - ax)) & 1, pb = (b >> (2 - ax)) & 1;
    const bool da = ax == i, db = ax == j;
    v *= (da && db) ? (pa == pb ? 6 : -6) : da ? (pa ? 3 : -3) : db ? (pb ? 3 : -3) : (pa == pb ? 2 : 1);
  }
  return v;
}
__host__ __device__ constexpr int q1_mu72(int a, int b, int i, int j) {
  return (q1_g(a, b, j, i) + (i == j ? q1_g(a, b, 0, 0) + q1_g(a, b, 1, 1) + q1_g(a, b, 2, 2) : 0)) / 3;
}
__host__ __device__ constexpr int q1_la72(int a, int b, int i, int j) { return q1_g(a, b, i, j) / 3; }
// class of a sign-normalised pair (m > 0, or m = 0 and l >= 0); -1 if it is none of the 10
__host__ __device__ constexpr int q1_class(int m, int l) {
  return (m == 3 && l == -3) ? 0 : (m == 3 && l == 3) ? 1 : (m == 4 && l == -2) ? 2 : (m == 4 && l == 4) ? 3
       : (m == 6 && l == -6) ? 4 : (m == 6 && l == 6) ? 5 : (m == 8 && l == 2) ? 6 : (m == 8 && l == 8) ? 7
       : (m == 10 && l == 4) ? 8 : (m == 32 && l == 8) ? 9 : -1;
}
constexpr int Q1_CLASS_M[10] = {3, 3, 4, 4, 6, 6, 8, 8, 10, 32}, Q1_CLASS_L[10] = {-3, 3, -2, 4, -6, 6, 2, 8, 4, 8};
__constant__ float c_Kv32[10];   // (mu0 m_c + lambda0 l_c) / 72 per class, rounded like c_Kc32
__constant__ double c_Kv64[10];  // the same in double, equal to the entries of c_Kc64

template <typename T>
struct KcReg {
  T v[10];
  __device__ __forceinline__ void load() {
#pragma unroll
    for (int c = 0; c < 10; ++c) v[c] = sizeof(T) == 4 ? T(c_Kv32[c]) : T(c_Kv64[c]);
  }
  // Kc[I][J][r][s]; with constant arguments this folds to one register (and a sign)
  __device__ __forceinline__ T operator()(int I, int J, int r, int s) const {
    const int m = q1_mu72(I, J, r, s), l = q1_la72(I, J, r, s);
    const bool neg = m < 0 || (m == 0 && l < 0);
    const T k = v[q1_class(neg ? -m : m, neg ? -l : l)];
    return neg ? -k : k;
  }
};

// the packed node record of level 0: (u_x, u_y, u_z, E)
template <typename T>
struct Pack4;
template <>
struct Pack4<float> {
  using type = float4;
  static __device__ __forceinline__ float4 make(float a, float b, float c, float d) { return make_float4(a, b, c, d); }
};
template <>
struct Pack4<double> {
  using type = double4;
  static __device__ __forceinline__ double4 make(double a, double b, double c, double d) {
    return make_double4(a, b, c, d);
  }
};

// Programmatic dependent launch: kernels of the solve are launched so that they
// may start while their predecessor drains.  Each waits here until the
// predecessor has completed and its writes are visible, then lets its own
// successor be scheduled; code before the wait (a prologue) reads only data
// that no kernel of the solve writes (lists, neighbour tables, flags, E,
// stencils), since the predecessor may still be running.
__device__ __forceinline__ void pdl_wait() {
  asm volatile("griddepcontrol.wait;" ::: "memory");
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}

// ---------------------------------------------------------------------------
// Level-0 matrix-free operator on one block per CTA (128 threads, one node each;
// solver/CPU_Kernels/SPGrid_Linear_Elasticity.h:96-344): OP_KU: out = dx*K*u,
// OP_RES: out = b - dx*K*u.  u of the block plus a one-node halo and E of the
// cells around it are staged in shared memory; each node sums its 8 cells,
// g_I = sum_J Kc[I][J] u_J scaled by E_I.  Empty cells (E = 0) are skipped,
// which saves the work wherever a warp's nodes share them (band edges).
// ---------------------------------------------------------------------------
enum { OP_KU = 0, OP_RES = 1, OP_KUP = 2 };  // OP_KUP: K u with Project, and the CTA's partial u.(Ku)

// halo geometry: nodes [-1,4]x[-1,4]x[-1,8] (6x6x10), cells [-1,3]x[-1,3]x[-1,7] (5x5x9).
// In shared memory a y-row of the halo starts every HSY = 24 entries: a warp
// reads 4 consecutive rows of 8 consecutive z at once, and with the row starts
// at 0, 24, 48, 72 (mod 32 banks: 0, 24, 16, 8) those 32 words fall in distinct
// banks (FP32), or in distinct bank pairs per half-warp (FP64).  Rows of 10
// entries would put rows y and y+3 on the same banks.
constexpr int HU = 360, HE = 225;
constexpr int HSY = 24;
constexpr int HSX = 5 * HSY + 10, HN = 6 * HSX;   // node halo: x-plane stride, entries
constexpr int ESX = 4 * HSY + 9, HEN = 5 * ESX;   // cell halo

template <typename T, int OP>
__global__ void __launch_bounds__(128) level0_op_kernel(const int* __restrict__ block_list, int nblocks,
                                                        const int* __restrict__ nbr, const T* __restrict__ E,
                                                        const T* u, const T* __restrict__ b, T* __restrict__ out,
                                                        long N, T dx, const uint32_t* __restrict__ flags,
                                                        double* __restrict__ part) {
  pdl_wait();
  __shared__ T su[3][HN];
  __shared__ T sE[HEN];
  __shared__ int snb[27];
  const int bi = block_list ? block_list[blockIdx.x] : blockIdx.x;
  if (bi >= 0 && threadIdx.x < 27) snb[threadIdx.x] = nbr[long(bi) * 27 + threadIdx.x];
  __syncthreads();
  // stage u halo
  for (int h = threadIdx.x; h < HU; h += 128) {
    const int sx = h / 60, sy = (h / 10) % 6, sz = h % 10;
    const int lx = sx - 1, ly = sy - 1, lz = sz - 1;
    const int dxb = lx < 0 ? 0 : (lx > 3 ? 2 : 1), dyb = ly < 0 ? 0 : (ly > 3 ? 2 : 1), dzb = lz < 0 ? 0 : (lz > 7 ? 2 : 1);
    const int nb = snb[dxb * 9 + dyb * 3 + dzb];
    T a = 0, bb = 0, c = 0;
    if (nb >= 0) {
      const long idx = long(nb) * 128 + ((lx & 3) << 5) + ((ly & 3) << 3) + (lz & 7);
      a = u[idx];
      bb = u[idx + N];
      c = u[idx + 2 * N];
    }
    const int s = sx * HSX + sy * HSY + sz;
    su[0][s] = a;
    su[1][s] = bb;
    su[2][s] = c;
  }
  for (int h = threadIdx.x; h < HE; h += 128) {
    const int sx = h / 45, sy = (h / 9) % 5, sz = h % 9;
    const int lx = sx - 1, ly = sy - 1, lz = sz - 1;
    const int dxb = lx < 0 ? 0 : 1, dyb = ly < 0 ? 0 : 1, dzb = lz < 0 ? 0 : 1;
    const int nb = snb[dxb * 9 + dyb * 3 + dzb];
    sE[sx * ESX + sy * HSY + sz] = nb >= 0 ? E[long(nb) * 128 + ((lx & 3) << 5) + ((ly & 3) << 3) + (lz & 7)] : T(0);
  }
  __syncthreads();
  const int e = threadIdx.x;
  const int x = e >> 5, y = (e >> 3) & 3, z = e & 7;
  const long gidx = long(bi) * 128 + e;
  T f0 = 0, f1 = 0, f2 = 0;
#pragma unroll
  for (int I = 0; I < 8; ++I) {
    const int Ix = I >> 2, Iy = (I >> 1) & 1, Iz = I & 1;
    const int cx = x - Ix, cy = y - Iy, cz = z - Iz;  // cell, in [-1,3]x[-1,3]x[-1,7]
    const T Ec = sE[(cx + 1) * ESX + (cy + 1) * HSY + (cz + 1)];
    if (Ec == T(0)) continue;
    T g0 = 0, g1 = 0, g2 = 0;
#pragma unroll
    for (int J = 0; J < 8; ++J) {
      const int nx = cx + (J >> 2) + 1, ny = cy + ((J >> 1) & 1) + 1, nz = cz + (J & 1) + 1;
      const int h = nx * HSX + ny * HSY + nz;
      const T ux = su[0][h], uy = su[1][h], uz = su[2][h];
      const int k = (I * 8 + J) * 9;
      g0 += kc<T>(k + 0) * ux + kc<T>(k + 1) * uy + kc<T>(k + 2) * uz;
      g1 += kc<T>(k + 3) * ux + kc<T>(k + 4) * uy + kc<T>(k + 5) * uz;
      g2 += kc<T>(k + 6) * ux + kc<T>(k + 7) * uy + kc<T>(k + 8) * uz;
    }
    f0 += Ec * g0;
    f1 += Ec * g1;
    f2 += Ec * g2;
  }
  f0 *= dx;
  f1 *= dx;
  f2 *= dx;
  if (OP == OP_KU) {
    out[gidx] = f0;
    out[gidx + N] = f1;
    out[gidx + 2 * N] = f2;
  } else if (OP == OP_RES) {
    out[gidx] = b[gidx] - f0;
    out[gidx + N] = b[gidx + N] - f1;
    out[gidx + 2 * N] = b[gidx + 2 * N] - f2;
  } else {
    // the PCG matvec q = K s: Dirichlet components zeroed, and s.q summed per CTA
    const uint32_t fl = flags[gidx];
    if (fl & DIR_X) f0 = 0;
    if (fl & DIR_Y) f1 = 0;
    if (fl & DIR_Z) f2 = 0;
    out[gidx] = f0;
    out[gidx + N] = f1;
    out[gidx + 2 * N] = f2;
    const int hc = (x + 1) * HSX + (y + 1) * HSY + (z + 1);
    double d = double(su[0][hc]) * double(f0) + double(su[1][hc]) * double(f1) + double(su[2][hc]) * double(f2);
#pragma unroll
    for (int o = 16; o; o >>= 1) d += __shfl_down_sync(0xffffffffu, d, o);
    __shared__ double sd[4];
    if ((threadIdx.x & 31) == 0) sd[threadIdx.x >> 5] = d;
    __syncthreads();
    if (threadIdx.x == 0) part[blockIdx.x] = (sd[0] + sd[1]) + (sd[2] + sd[3]);
  }
}

// ---------------------------------------------------------------------------
// Level-0 Gauss-Seidel colour pass over a compact list of the colour's nodes
// (solver/CPU_Kernels/SPGrid_Gauss_Seidel.h:876-1180), one node per thread.
// The residual is accumulated cell by cell, g_I = sum_J Kc[I][J] u_J over the
// node's 8 cells and f = sum_I E_I g_I, visiting the 27 neighbours one x-plane
// (9 nodes) at a time; a cell is folded into f after its last plane.  Same-
// colour nodes share no cell, so a pass updates u in place.  List entries
// ~node (negative) name nodes the pass does not update: only their Dirichlet
// components are cleared.  MINB bounds the registers (resident CTAs per SM):
// the pass is latency-bound, so occupancy is worth a few spilled registers.
// ---------------------------------------------------------------------------

// Addressing of the 3x3x3 neighbourhood of a level-0 node: per axis, the terms
// of the neighbour-block selector (into the block's 27-entry nbr row) and of the
// slot inside that block, for the offsets -1, 0, +1.
struct Nbhd {
  const int* nb;
  int sx[3], sy[3], sz[3], lx[3], ly[3], lz[3];
  __device__ __forceinline__ void init(const int* __restrict__ nbr, int g) {
    const int bi = g >> 7, e = g & 127;
    const int x = e >> 5, y = (e >> 3) & 3, z = e & 7;
    nb = nbr + long(bi) * 27;
#pragma unroll
    for (int o = 0; o < 3; ++o) {
      const int xx = x + o - 1, yy = y + o - 1, zz = z + o - 1;
      sx[o] = (xx < 0 ? 0 : (xx > 3 ? 2 : 1)) * 9;
      sy[o] = (yy < 0 ? 0 : (yy > 3 ? 2 : 1)) * 3;
      sz[o] = zz < 0 ? 0 : (zz > 7 ? 2 : 1);
      lx[o] = (xx & 3) << 5;
      ly[o] = (yy & 3) << 3;
      lz[o] = zz & 7;
    }
  }
  // global index of the neighbour at offset (ix-1, iy-1, iz-1), -1 if its block is not active
  __device__ __forceinline__ int at(int ix, int iy, int iz) const {
    const int b = __ldg(nb + sx[ix] + sy[iy] + sz[iz]);
    return b < 0 ? -1 : (b << 7) + lx[ix] + ly[iy] + lz[iz];
  }
  // the same with a neighbour table whose missing blocks name an all-zero pad block
  __device__ __forceinline__ int at_padded(int ix, int iy, int iz) const {
    return (__ldg(nb + sx[ix] + sy[iy] + sz[iz]) << 7) + lx[ix] + ly[iy] + lz[iz];
  }
};

template <typename T, int MINB>
__global__ void __launch_bounds__(128, MINB) gs0_list_kernel(const int* __restrict__ list, int n,
                                                             const int* __restrict__ nbr, const T* __restrict__ E,
                                                             T* u, const T* __restrict__ b,
                                                             const uint32_t* __restrict__ flags, int N, T dx) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) {
    pdl_wait();
    return;
  }
  // prologue: list, flags, neighbour table and E do not change during a solve
  const int raw = list[t];
  const int g = raw >= 0 ? raw : ~raw;
  const uint32_t fl = flags[g];
  const bool fx = fl & DIR_X, fy = fl & DIR_Y, fz = fl & DIR_Z;
  Nbhd nh;
  nh.init(nbr, g);
  T Ec[8];
#pragma unroll
  for (int I = 0; I < 8; ++I) {  // the cell of corner I (min corner = node - I) sits at offset -I
    const int i = nh.at(1 - (I >> 2), 1 - ((I >> 1) & 1), 1 - (I & 1));
    Ec[I] = (raw < 0 || i < 0) ? T(0) : E[i];
  }
  pdl_wait();
  if (raw < 0) {
    if (fx) u[g] = T(0);
    if (fy) u[g + N] = T(0);
    if (fz) u[g + 2 * N] = T(0);
    return;
  }
  T gc[8][3], uc[3];
  T f[3] = {0, 0, 0}, dg[6] = {0, 0, 0, 0, 0, 0};
#pragma unroll
  for (int I = 0; I < 8; ++I) gc[I][0] = gc[I][1] = gc[I][2] = T(0);
#pragma unroll
  for (int px = 0; px < 3; ++px) {
    T up[9][3];
#pragma unroll
    for (int p = 0; p < 9; ++p) {
      const int iy = p / 3, iz = p % 3;
      const int i = (px == 1 && p == 4) ? g : nh.at(px, iy, iz);
      up[p][0] = i < 0 ? T(0) : u[i];
      up[p][1] = i < 0 ? T(0) : u[i + N];
      up[p][2] = i < 0 ? T(0) : u[i + 2 * N];
    }
    if (px == 1) {
      uc[0] = up[4][0];
      uc[1] = up[4][1];
      uc[2] = up[4][2];
    }
#pragma unroll
    for (int I = 0; I < 8; ++I) {
      const int Ix = I >> 2, Iy = (I >> 1) & 1, Iz = I & 1;
      const int Jx = px - 1 + Ix;
      if (Jx < 0 || Jx > 1) continue;
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const int Jy = q >> 1, Jz = q & 1;
        const int p = (Jy - Iy + 1) * 3 + (Jz - Iz + 1);
        const int k = (I * 8 + Jx * 4 + Jy * 2 + Jz) * 9;
#pragma unroll
        for (int v = 0; v < 3; ++v)
#pragma unroll
          for (int w = 0; w < 3; ++w) gc[I][v] = fma(kc<T>(k + v * 3 + w), up[p][w], gc[I][v]);
      }
      if (Jx == 1) {  // last plane of this cell
#pragma unroll
        for (int v = 0; v < 3; ++v) f[v] = fma(Ec[I], gc[I][v], f[v]);
        const int kd = (I * 8 + I) * 9;
        dg[0] = fma(kc<T>(kd + 0), Ec[I], dg[0]);
        dg[1] = fma(kc<T>(kd + 4), Ec[I], dg[1]);
        dg[2] = fma(kc<T>(kd + 8), Ec[I], dg[2]);
        dg[3] = fma(kc<T>(kd + 1), Ec[I], dg[3]);
        dg[4] = fma(kc<T>(kd + 2), Ec[I], dg[4]);
        dg[5] = fma(kc<T>(kd + 5), Ec[I], dg[5]);
      }
    }
  }
  // u += D^{-1} (b - K u), Dirichlet rows replaced by the identity
  const T r0 = b[g] - f[0] * dx, r1 = b[g + N] - f[1] * dx, r2 = b[g + 2 * N] - f[2] * dx;
  T d0 = dg[0] * dx, d1 = dg[1] * dx, d2 = dg[2] * dx, d3 = dg[3] * dx, d4 = dg[4] * dx, d5 = dg[5] * dx;
  if (fx) { d0 = 1; d3 = 0; d4 = 0; }
  if (fy) { d1 = 1; d3 = 0; d5 = 0; }
  if (fz) { d2 = 1; d4 = 0; d5 = 0; }
  const T m11 = d1 * d2 - d5 * d5, m12 = d5 * d4 - d2 * d3, m13 = d3 * d5 - d4 * d1;
  const T m22 = d2 * d0 - d4 * d4, m23 = d4 * d3 - d0 * d5, m33 = d0 * d1 - d3 * d3;
  const T inv = T(1) / (d0 * m11 + d3 * m12 + d4 * m13);
  T a0 = m11 * inv, a1 = m22 * inv, a2 = m33 * inv, a3 = m12 * inv, a4 = m13 * inv, a5 = m23 * inv;
  if (fx) { a0 = 0; a3 = 0; a4 = 0; }
  if (fy) { a1 = 0; a3 = 0; a5 = 0; }
  if (fz) { a2 = 0; a4 = 0; a5 = 0; }
  T v0 = uc[0] + r0 * a0 + r1 * a3 + r2 * a4;
  T v1 = uc[1] + r0 * a3 + r1 * a1 + r2 * a5;
  T v2 = uc[2] + r0 * a4 + r1 * a5 + r2 * a2;
  if (fx) v0 = 0;
  if (fy) v1 = 0;
  if (fz) v2 = 0;
  u[g] = v0;
  u[g + N] = v1;
  u[g + 2 * N] = v2;
}

// ---------------------------------------------------------------------------
// Packed level 0 of the V-cycle (mixed and FP64 modes).  The iterate of level 0
// is one record per node, (u_x, u_y, u_z, E of the node's cell): the 27-point
// gathers of the smoother and the halo staging of the residual then read a
// node's displacement and its cell's stiffness scale in one access (16 B in
// FP32, 32 B in FP64), the same bytes as three planes of u plus the E plane.
// ---------------------------------------------------------------------------

// u4 = (0, 0, 0, E): the zero start of the V-cycle's level-0 correction
template <typename T>
__global__ void reset_u4_kernel(typename Pack4<T>::type* __restrict__ u4, const T* __restrict__ E, long N) {
  pdl_wait();
  const long i = long(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i < N) u4[i] = Pack4<T>::make(T(0), T(0), T(0), E[i]);
}

// gs0_list_kernel on the packed iterate (one float4 gather per neighbour; the
// cells' E come with the nodes at offsets -I).  nbrz names the zero pad block
// (index nb) for missing neighbours, so the gathers need no test.
template <typename T, int MINB>
__global__ void __launch_bounds__(128, MINB) gs0_list4_kernel(const int* __restrict__ list, int n,
                                                              const int* __restrict__ nbrz,
                                                              typename Pack4<T>::type* u4, const T* __restrict__ b,
                                                              const uint32_t* __restrict__ flags, int N, T dx) {
  using V = typename Pack4<T>::type;
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) {
    pdl_wait();
    return;
  }
  const int raw = list[t];
  const int g = raw >= 0 ? raw : ~raw;
  const uint32_t fl = flags[g];
  const bool fx = fl & DIR_X, fy = fl & DIR_Y, fz = fl & DIR_Z;
  Nbhd nh;
  nh.init(nbrz, g);
  KcReg<T> K;
  K.load();
  pdl_wait();
  if (raw < 0) {
    V v = u4[g];
    if (fx) v.x = T(0);
    if (fy) v.y = T(0);
    if (fz) v.z = T(0);
    u4[g] = v;
    return;
  }
  T gc[8][3], Ec[8], uc[3];
  T f[3] = {0, 0, 0}, dg[6] = {0, 0, 0, 0, 0, 0};
#pragma unroll
  for (int I = 0; I < 8; ++I) gc[I][0] = gc[I][1] = gc[I][2] = T(0);
#pragma unroll
  for (int px = 0; px < 3; ++px) {
    T up[9][3];
#pragma unroll
    for (int p = 0; p < 9; ++p) {
      const int iy = p / 3, iz = p % 3;
      const V v = u4[(px == 1 && p == 4) ? g : nh.at_padded(px, iy, iz)];
      up[p][0] = v.x;
      up[p][1] = v.y;
      up[p][2] = v.z;
      if (px <= 1 && iy <= 1 && iz <= 1) Ec[(1 - px) * 4 + (1 - iy) * 2 + (1 - iz)] = v.w;
    }
    if (px == 1) {
      uc[0] = up[4][0];
      uc[1] = up[4][1];
      uc[2] = up[4][2];
    }
#pragma unroll
    for (int I = 0; I < 8; ++I) {
      const int Ix = I >> 2, Iy = (I >> 1) & 1, Iz = I & 1;
      const int Jx = px - 1 + Ix;
      if (Jx < 0 || Jx > 1) continue;
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const int Jy = q >> 1, Jz = q & 1;
        const int p = (Jy - Iy + 1) * 3 + (Jz - Iz + 1);
        const int J = Jx * 4 + Jy * 2 + Jz;
#pragma unroll
        for (int v = 0; v < 3; ++v)
#pragma unroll
          for (int w = 0; w < 3; ++w) gc[I][v] = fma(K(I, J, v, w), up[p][w], gc[I][v]);
      }
      if (Jx == 1) {
#pragma unroll
        for (int v = 0; v < 3; ++v) f[v] = fma(Ec[I], gc[I][v], f[v]);
        dg[0] = fma(K(I, I, 0, 0), Ec[I], dg[0]);
        dg[1] = fma(K(I, I, 1, 1), Ec[I], dg[1]);
        dg[2] = fma(K(I, I, 2, 2), Ec[I], dg[2]);
        dg[3] = fma(K(I, I, 0, 1), Ec[I], dg[3]);
        dg[4] = fma(K(I, I, 0, 2), Ec[I], dg[4]);
        dg[5] = fma(K(I, I, 1, 2), Ec[I], dg[5]);
      }
    }
  }
  const T r0 = b[g] - f[0] * dx, r1 = b[g + N] - f[1] * dx, r2 = b[g + 2 * N] - f[2] * dx;
  T d0 = dg[0] * dx, d1 = dg[1] * dx, d2 = dg[2] * dx, d3 = dg[3] * dx, d4 = dg[4] * dx, d5 = dg[5] * dx;
  if (fx) { d0 = 1; d3 = 0; d4 = 0; }
  if (fy) { d1 = 1; d3 = 0; d5 = 0; }
  if (fz) { d2 = 1; d4 = 0; d5 = 0; }
  const T m11 = d1 * d2 - d5 * d5, m12 = d5 * d4 - d2 * d3, m13 = d3 * d5 - d4 * d1;
  const T m22 = d2 * d0 - d4 * d4, m23 = d4 * d3 - d0 * d5, m33 = d0 * d1 - d3 * d3;
  const T inv = T(1) / (d0 * m11 + d3 * m12 + d4 * m13);
  T a0 = m11 * inv, a1 = m22 * inv, a2 = m33 * inv, a3 = m12 * inv, a4 = m13 * inv, a5 = m23 * inv;
  if (fx) { a0 = 0; a3 = 0; a4 = 0; }
  if (fy) { a1 = 0; a3 = 0; a5 = 0; }
  if (fz) { a2 = 0; a4 = 0; a5 = 0; }
  T v0 = uc[0] + r0 * a0 + r1 * a3 + r2 * a4;
  T v1 = uc[1] + r0 * a3 + r1 * a1 + r2 * a5;
  T v2 = uc[2] + r0 * a4 + r1 * a5 + r2 * a2;
  if (fx) v0 = 0;
  if (fy) v1 = 0;
  if (fz) v2 = 0;
  u4[g] = Pack4<T>::make(v0, v1, v2, Ec[0]);  // corner I = 0: the node's own cell
}

// gs0_list4_kernel for the short passes of the boundary band (about 10^3
// nodes): those are bound by one thread's chain of dependent loads, so eight
// threads share a node, thread I taking the cell of which the node is corner I.
// The Q1 element is symmetric under reflections, K(I, J) = S K(0, I^J) S with S
// = diag(-1 on the axes where I has its bit) (checked on the host at set-up);
// looping over J' = I^J keeps the coefficients K(0, J') compile-time register
// selections while the corner J a thread reads varies with I.  Per thread: 8
// gathers and 72 FMA; the cells' E g and diagonal blocks are summed over the
// eight threads with shuffles and thread 0 updates the node.  Same products as
// gs0_list4_kernel, summed in another order.
template <typename T>
__global__ void __launch_bounds__(128) gs0_cell4_kernel(const int* __restrict__ list, int n,
                                                        const int* __restrict__ nbrz,
                                                        typename Pack4<T>::type* u4, const T* __restrict__ b,
                                                        const uint32_t* __restrict__ flags, int N, T dx) {
  using V = typename Pack4<T>::type;
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  const int k = t >> 3, I = t & 7;  // groups of 8 threads never straddle a warp
  if (k >= n) {
    pdl_wait();
    return;
  }
  const int raw = list[k];
  const int g = raw >= 0 ? raw : ~raw;
  const uint32_t fl = flags[g];
  const bool fx = fl & DIR_X, fy = fl & DIR_Y, fz = fl & DIR_Z;
  // per axis: block selector and slot for offset 0 and for the offset 1 - 2 I_a
  // towards the cell's other corners
  const int bi = g >> 7, e = g & 127;
  const int x = e >> 5, y = (e >> 3) & 3, z = e & 7;
  const int Ix = I >> 2, Iy = (I >> 1) & 1, Iz = I & 1;
  const int x1 = x + 1 - 2 * Ix, y1 = y + 1 - 2 * Iy, z1 = z + 1 - 2 * Iz;
  const int sx[2] = {9, (x1 < 0 ? 0 : (x1 > 3 ? 2 : 1)) * 9}, lx[2] = {(x & 3) << 5, (x1 & 3) << 5};
  const int sy[2] = {3, (y1 < 0 ? 0 : (y1 > 3 ? 2 : 1)) * 3}, ly[2] = {(y & 3) << 3, (y1 & 3) << 3};
  const int sz[2] = {1, z1 < 0 ? 0 : (z1 > 7 ? 2 : 1)}, lz[2] = {z & 7, z1 & 7};
  const int* nb = nbrz + long(bi) * 27;
  int idx[8];
#pragma unroll
  for (int Jp = 0; Jp < 8; ++Jp) {
    const int a = Jp >> 2, c = (Jp >> 1) & 1, d = Jp & 1;
    idx[Jp] = (__ldg(nb + sx[a] + sy[c] + sz[d]) << 7) + lx[a] + ly[c] + lz[d];
  }
  KcReg<T> K;
  K.load();
  pdl_wait();
  if (raw < 0) {
    if (I == 0) {
      V v = u4[g];
      if (fx) v.x = T(0);
      if (fy) v.y = T(0);
      if (fz) v.z = T(0);
      u4[g] = v;
    }
    return;
  }
  if (sizeof(T) == 4 && I == 0) {  // the right-hand side, read after the shuffles, into L1 now
    asm volatile("prefetch.global.L1 [%0];" ::"l"(b + g));
    asm volatile("prefetch.global.L1 [%0];" ::"l"(b + g + N));
    asm volatile("prefetch.global.L1 [%0];" ::"l"(b + g + 2 * N));
  }
  const T s0 = Ix ? T(-1) : T(1), s1 = Iy ? T(-1) : T(1), s2 = Iz ? T(-1) : T(1);
  T gv[3] = {0, 0, 0}, Ec = 0, uc[3] = {0, 0, 0};
#pragma unroll
  for (int Jp = 0; Jp < 8; ++Jp) {
    const V v = u4[idx[Jp]];
    if (Jp == 0) {  // J = I: the node itself
      uc[0] = v.x;
      uc[1] = v.y;
      uc[2] = v.z;
    }
    if (Jp == I) Ec = v.w;  // J = 0: the cell's min corner carries its E
    const T w0 = s0 * v.x, w1 = s1 * v.y, w2 = s2 * v.z;
#pragma unroll
    for (int r = 0; r < 3; ++r)
      gv[r] = fma(K(0, Jp, r, 0), w0, fma(K(0, Jp, r, 1), w1, fma(K(0, Jp, r, 2), w2, gv[r])));
  }
  // this cell's share of the node's row and of its diagonal block
  T red[9] = {Ec * s0 * gv[0], Ec * s1 * gv[1], Ec * s2 * gv[2],
              Ec * K(0, 0, 0, 0), Ec * K(0, 0, 1, 1), Ec * K(0, 0, 2, 2),
              Ec * (s0 * s1) * K(0, 0, 0, 1), Ec * (s0 * s2) * K(0, 0, 0, 2), Ec * (s1 * s2) * K(0, 0, 1, 2)};
  // the eight threads of a node take the same branches: shuffle within the group only
  const unsigned group = 0xffu << (threadIdx.x & 24);
#pragma unroll
  for (int o = 4; o; o >>= 1)
#pragma unroll
    for (int q = 0; q < 9; ++q) red[q] += __shfl_xor_sync(group, red[q], o);
  if (I != 0) return;
  const T r0 = b[g] - red[0] * dx, r1 = b[g + N] - red[1] * dx, r2 = b[g + 2 * N] - red[2] * dx;
  T d0 = red[3] * dx, d1 = red[4] * dx, d2 = red[5] * dx, d3 = red[6] * dx, d4 = red[7] * dx, d5 = red[8] * dx;
  if (fx) { d0 = 1; d3 = 0; d4 = 0; }
  if (fy) { d1 = 1; d3 = 0; d5 = 0; }
  if (fz) { d2 = 1; d4 = 0; d5 = 0; }
  const T m11 = d1 * d2 - d5 * d5, m12 = d5 * d4 - d2 * d3, m13 = d3 * d5 - d4 * d1;
  const T m22 = d2 * d0 - d4 * d4, m23 = d4 * d3 - d0 * d5, m33 = d0 * d1 - d3 * d3;
  const T inv = T(1) / (d0 * m11 + d3 * m12 + d4 * m13);
  T a0 = m11 * inv, a1 = m22 * inv, a2 = m33 * inv, a3 = m12 * inv, a4 = m13 * inv, a5 = m23 * inv;
  if (fx) { a0 = 0; a3 = 0; a4 = 0; }
  if (fy) { a1 = 0; a3 = 0; a5 = 0; }
  if (fz) { a2 = 0; a4 = 0; a5 = 0; }
  T v0 = uc[0] + r0 * a0 + r1 * a3 + r2 * a4;
  T v1 = uc[1] + r0 * a3 + r1 * a1 + r2 * a5;
  T v2 = uc[2] + r0 * a4 + r1 * a5 + r2 * a2;
  if (fx) v0 = 0;
  if (fy) v1 = 0;
  if (fz) v2 = 0;
  u4[g] = Pack4<T>::make(v0, v1, v2, Ec);  // thread 0: the node's own cell
}

// level0_op_kernel<T, OP_RES> on the packed iterate: r = b - dx K u
template <typename T>
__global__ void __launch_bounds__(128) level0_res4_kernel(int nblocks, const int* __restrict__ nbrz,
                                                          const typename Pack4<T>::type* __restrict__ u4,
                                                          const T* __restrict__ b, T* __restrict__ out, long N, T dx) {
  pdl_wait();
  __shared__ T su[3][HN];
  __shared__ T sE[HN];
  __shared__ int snb[27];
  const int bi = blockIdx.x;
  KcReg<T> K;
  K.load();
  if (threadIdx.x < 27) snb[threadIdx.x] = nbrz[long(bi) * 27 + threadIdx.x];
  __syncthreads();
  for (int h = threadIdx.x; h < HU; h += 128) {
    const int sx = h / 60, sy = (h / 10) % 6, sz = h % 10;
    const int lx = sx - 1, ly = sy - 1, lz = sz - 1;
    const int dxb = lx < 0 ? 0 : (lx > 3 ? 2 : 1), dyb = ly < 0 ? 0 : (ly > 3 ? 2 : 1), dzb = lz < 0 ? 0 : (lz > 7 ? 2 : 1);
    const int nb = snb[dxb * 9 + dyb * 3 + dzb];  // the zero pad block where there is none
    const auto v = u4[long(nb) * 128 + ((lx & 3) << 5) + ((ly & 3) << 3) + (lz & 7)];
    const int s = sx * HSX + sy * HSY + sz;
    su[0][s] = v.x;
    su[1][s] = v.y;
    su[2][s] = v.z;
    sE[s] = v.w;
  }
  __syncthreads();
  const int e = threadIdx.x;
  const int x = e >> 5, y = (e >> 3) & 3, z = e & 7;
  const long gidx = long(bi) * 128 + e;
  T f0 = 0, f1 = 0, f2 = 0;
#pragma unroll
  for (int I = 0; I < 8; ++I) {
    const int Ix = I >> 2, Iy = (I >> 1) & 1, Iz = I & 1;
    const int cx = x - Ix, cy = y - Iy, cz = z - Iz;  // cell = its min-corner node, in the halo
    const T Ec = sE[(cx + 1) * HSX + (cy + 1) * HSY + (cz + 1)];
    if (Ec == T(0)) continue;
    T g0 = 0, g1 = 0, g2 = 0;
#pragma unroll
    for (int J = 0; J < 8; ++J) {
      const int nx = cx + (J >> 2) + 1, ny = cy + ((J >> 1) & 1) + 1, nz = cz + (J & 1) + 1;
      const int h = nx * HSX + ny * HSY + nz;
      const T ux = su[0][h], uy = su[1][h], uz = su[2][h];
      g0 += K(I, J, 0, 0) * ux + K(I, J, 0, 1) * uy + K(I, J, 0, 2) * uz;
      g1 += K(I, J, 1, 0) * ux + K(I, J, 1, 1) * uy + K(I, J, 1, 2) * uz;
      g2 += K(I, J, 2, 0) * ux + K(I, J, 2, 1) * uy + K(I, J, 2, 2) * uz;
    }
    f0 += Ec * g0;
    f1 += Ec * g1;
    f2 += Ec * g2;
  }
  out[gidx] = b[gidx] - f0 * dx;
  out[gidx + N] = b[gidx + N] - f1 * dx;
  out[gidx + 2 * N] = b[gidx + 2 * N] - f2 * dx;
}

// ---------------------------------------------------------------------------
// Coarse-level stencil operators (solver/MG/SPGrid_Stencil_Multiply.h:15-280)
// ---------------------------------------------------------------------------
struct GridView {
  const int* bgrid;  // dense block grid -> active block index or -1
  int gx, gy, gz;
  __device__ __forceinline__ long node(int x, int y, int z) const {
    if (x < 0 || y < 0 || z < 0) return -1;
    const int bx = x >> 2, by = y >> 2, bz = z >> 3;
    if (bx >= gx || by >= gy || bz >= gz) return -1;
    const int b = bgrid[(long(bx) * gy + by) * gz + bz];
    return b < 0 ? -1 : long(b) * 128 + ((x & 3) << 5) + ((y & 3) << 3) + (z & 7);
  }
};

enum { SOP_MUL = 0, SOP_RES = 1, SOP_GS = 2 };

// One warp per node: lane q < 27 multiplies the 3x3 block of spoke q with the
// neighbour's u, the warp sums the three components.  Stencils are node-major,
// A[node*243 + q*9 + v*3 + w]: lane q reads its nine entries, and the warp's
// reads together cover one contiguous row (972 bytes in FP32), which L1
// fetches once.  The neighbour's block comes from the level's 27-entry
// neighbour table (one load that needs only the block index, issued with the
// flags load), and the row is loaded whether or not the neighbour exists, so
// no load waits for another; a missing neighbour's spoke is skipped.  GS
// updates the nodes of a list: the active nodes of one colour, or the active
// boundary-band nodes of one colour (no node has a neighbour of its own
// colour, so the order inside a pass does not change the result).
// Results on Dirichlet components are zeroed (Project).  The reference
// projects the whole level after every colour; here only updated nodes are
// projected, which is the same because the V-cycle keeps u zero on Dirichlet
// components (cleared levels, projected transfers and updates).
template <typename T, int OP>
__global__ void __launch_bounds__(256) stencil_op_kernel(const int* __restrict__ list, int count,
                                                         const int* __restrict__ nbr,
                                                         const T* __restrict__ A, const uint32_t* __restrict__ flags,
                                                         const T* u, T* out_u, const T* __restrict__ b,
                                                         T* __restrict__ out, long N, int round_out) {
  const long w = (long(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;  // one warp per node
  const int lane = threadIdx.x & 31;
  // GS: node list[w] of the `count` listed; MUL / RES: node w of the first `count` blocks
  if (w >= (OP == SOP_GS ? long(count) : long(count) * 128)) {
    pdl_wait();
    return;
  }
  const long gidx = OP == SOP_GS ? long(list[w]) : w;
  const int bi = int(gidx >> 7), e = int(gidx & 127);
  // prologue: flags, neighbour table and stencil row do not change during a solve
  // neighbour (X, Y, Z) of the node in block coordinates, -1..4 x -1..4 x -1..8
  const int X = (e >> 5) + lane / 9 - 1, Y = ((e >> 3) & 3) + (lane / 3) % 3 - 1, Z = (e & 7) + lane % 3 - 1;
  const uint32_t fl = flags[gidx];
  const int nbk = lane < 27 ? nbr[long(bi) * 27 + (X < 0 ? 0 : (X > 3 ? 2 : 1)) * 9 + (Y < 0 ? 0 : (Y > 3 ? 2 : 1)) * 3 +
                                  (Z < 0 ? 0 : (Z > 7 ? 2 : 1))]
                            : -1;
  // an inactive node's row is all +0 (the operator build writes only the rows of
  // active nodes into zeroed storage): its zeros come from registers, and its
  // products with the neighbours' u are formed as before
  T a[9];
  if (lane < 27 && (OP == SOP_GS || (fl & ACTIVE_NODE))) {
    const T* ap = A + gidx * 243 + lane * 9;
#pragma unroll
    for (int k = 0; k < 9; ++k) a[k] = ap[k];
  } else {
#pragma unroll
    for (int k = 0; k < 9; ++k) a[k] = T(0);
  }
  const long n = nbk < 0 ? -1 : long(nbk) * 128 + ((X & 3) << 5) + ((Y & 3) << 3) + (Z & 7);
  T d0 = 0, d1 = 0, d2 = 0, d3 = 0, d4 = 0, d5 = 0;
  if (OP == SOP_GS && lane == 0) {
    const T* c = A + gidx * 243 + 13 * 9;
    d0 = c[0]; d1 = c[4]; d2 = c[8]; d3 = c[1]; d4 = c[2]; d5 = c[5];
  }
  pdl_wait();
  // lane 0 reads its right-hand side (and in GS its own u) after the warp's
  // reduction; prefetched here, after the wait, those loads find them in L1
  if (OP != SOP_MUL && lane == 0) {
    asm volatile("prefetch.global.L1 [%0];" ::"l"(b + gidx));
    asm volatile("prefetch.global.L1 [%0];" ::"l"(b + gidx + N));
    asm volatile("prefetch.global.L1 [%0];" ::"l"(b + gidx + 2 * N));
    if (OP == SOP_GS) {
      asm volatile("prefetch.global.L1 [%0];" ::"l"(u + gidx));
      asm volatile("prefetch.global.L1 [%0];" ::"l"(u + gidx + N));
      asm volatile("prefetch.global.L1 [%0];" ::"l"(u + gidx + 2 * N));
    }
  }
  T f0 = 0, f1 = 0, f2 = 0;
  if (n >= 0) {
    const T ux = u[n], uy = u[n + N], uz = u[n + 2 * N];
    f0 = a[0] * ux + a[1] * uy + a[2] * uz;
    f1 = a[3] * ux + a[4] * uy + a[5] * uz;
    f2 = a[6] * ux + a[7] * uy + a[8] * uz;
  }
#pragma unroll
  for (int o = 16; o; o >>= 1) {
    f0 += __shfl_down_sync(0xffffffffu, f0, o);
    f1 += __shfl_down_sync(0xffffffffu, f1, o);
    f2 += __shfl_down_sync(0xffffffffu, f2, o);
  }
  if (lane != 0) return;
  if (OP == SOP_MUL) {
    out[gidx] = (fl & DIR_X) ? T(0) : f0;
    out[gidx + N] = (fl & DIR_Y) ? T(0) : f1;
    out[gidx + 2 * N] = (fl & DIR_Z) ? T(0) : f2;
    return;
  }
  const T r0 = b[gidx] - f0, r1 = b[gidx + N] - f1, r2 = b[gidx + 2 * N] - f2;
  if (OP == SOP_RES) {
    T o0 = (fl & DIR_X) ? T(0) : r0, o1 = (fl & DIR_Y) ? T(0) : r1, o2 = (fl & DIR_Z) ? T(0) : r2;
    if (round_out) { o0 = T(round_to_float(o0)); o1 = T(round_to_float(o1)); o2 = T(round_to_float(o2)); }
    out[gidx] = o0;
    out[gidx + N] = o1;
    out[gidx + 2 * N] = o2;
    return;
  }
  const bool fx = fl & DIR_X, fy = fl & DIR_Y, fz = fl & DIR_Z;
  if (fx) { d0 = 1; d3 = 0; d4 = 0; }
  if (fy) { d1 = 1; d3 = 0; d5 = 0; }
  if (fz) { d2 = 1; d4 = 0; d5 = 0; }
  const T m11 = d1 * d2 - d5 * d5, m12 = d5 * d4 - d2 * d3, m13 = d3 * d5 - d4 * d1;
  const T m22 = d2 * d0 - d4 * d4, m23 = d4 * d3 - d0 * d5, m33 = d0 * d1 - d3 * d3;
  const T inv = T(1) / (d0 * m11 + d3 * m12 + d4 * m13);
  T a0 = m11 * inv, a1 = m22 * inv, a2 = m33 * inv, a3 = m12 * inv, a4 = m13 * inv, a5 = m23 * inv;
  if (fx) { a0 = 0; a3 = 0; a4 = 0; }
  if (fy) { a1 = 0; a3 = 0; a5 = 0; }
  if (fz) { a2 = 0; a4 = 0; a5 = 0; }
  T u0 = u[gidx] + (a0 * r0 + a3 * r1 + a4 * r2);
  T u1 = u[gidx + N] + (a3 * r0 + a1 * r1 + a5 * r2);
  T u2 = u[gidx + 2 * N] + (a4 * r0 + a5 * r1 + a2 * r2);
  if (fx) u0 = 0;
  if (fy) u1 = 0;
  if (fz) u2 = 0;
  out_u[gidx] = u0;
  out_u[gidx + N] = u1;
  out_u[gidx + 2 * N] = u2;
}

// ---------------------------------------------------------------------------
// Transfers (solver/MG/Restriction.h:52-88, solver/MG/Prolongation.h:151-193)
// ---------------------------------------------------------------------------
// coarse(c) = sum_{d in {-1,0,1}^3} w(d) fine(2c - (4,4,8) + d), w = prod (1/2,1,1/2);
// Dirichlet components zeroed afterwards.  One CTA per coarse block (launched
// with nb CTAs of 128 threads, thread = node): the 9x9x17 fine nodes the block
// reads are staged in shared memory once (the 27 fine blocks they lie in are
// looked up once), then every node sums its 27 in the reference's order; a
// missing fine node reads 0, which adds nothing.
template <typename T>
__global__ void __launch_bounds__(128) restrict_kernel(int nb, const int* __restrict__ coords,
                                                       const uint32_t* __restrict__ cflags, GridView fine,
                                                       const T* __restrict__ fin, long Nf, T* __restrict__ cout,
                                                       long Nc) {
  constexpr int RX = 9, RY = 9, RZ = 17, RN = RX * RY * RZ;
  __shared__ T sf[3][RN];
  __shared__ int sblk[27];
  const int bi = blockIdx.x, e = threadIdx.x;
  if (bi >= nb) return;
  const int CX = coords[3 * bi], CY = coords[3 * bi + 1], CZ = coords[3 * bi + 2];
  const int x0 = 2 * CX - 5, y0 = 2 * CY - 5, z0 = 2 * CZ - 9;  // fine region origin
  const int bx0 = x0 >> 2, by0 = y0 >> 2, bz0 = z0 >> 3;
  if (e < 27) {  // block indices are fixed during a solve: looked up before the wait
    const int bx = bx0 + e / 9, by = by0 + (e / 3) % 3, bz = bz0 + e % 3;
    const long n = fine.node(bx * 4, by * 4, bz * 8);
    sblk[e] = n < 0 ? -1 : int(n >> 7);
  }
  pdl_wait();
  __syncthreads();
  for (int h = e; h < RN; h += 128) {
    const int fx = x0 + h / (RY * RZ), fy = y0 + (h / RZ) % RY, fz = z0 + h % RZ;
    const int b = sblk[((fx >> 2) - bx0) * 9 + ((fy >> 2) - by0) * 3 + ((fz >> 3) - bz0)];
    T a = 0, c = 0, d = 0;
    if (b >= 0) {
      const long n = long(b) * 128 + ((fx & 3) << 5) + ((fy & 3) << 3) + (fz & 7);
      a = fin[n];
      c = fin[n + Nf];
      d = fin[n + 2 * Nf];
    }
    sf[0][h] = a;
    sf[1][h] = c;
    sf[2][h] = d;
  }
  __syncthreads();
  const int lx = e >> 5, ly = (e >> 3) & 3, lz = e & 7;
  T v0 = 0, v1 = 0, v2 = 0;
  for (int q = 0; q < 27; ++q) {
    const int i = q / 9, j = (q / 3) % 3, k = q % 3;
    const int h = (2 * lx + i) * (RY * RZ) + (2 * ly + j) * RZ + (2 * lz + k);
    const T w = T((i == 1 ? 1.0 : 0.5) * (j == 1 ? 1.0 : 0.5) * (k == 1 ? 1.0 : 0.5));
    v0 += w * sf[0][h];
    v1 += w * sf[1][h];
    v2 += w * sf[2][h];
  }
  const long t = long(bi) * 128 + e;
  const uint32_t fl = cflags[t];
  cout[t] = (fl & DIR_X) ? T(0) : v0;
  cout[t + Nc] = (fl & DIR_Y) ? T(0) : v1;
  cout[t + 2 * Nc] = (fl & DIR_Z) ? T(0) : v2;
}

// The 3x3x5 coarse nodes that the 4x4x8 fine nodes of a fine block interpolate
// from ((f + (4,4,8)) >> 1 + {0,1}^3), staged in shared memory by one CTA per
// fine block (128 threads, thread = node); missing coarse nodes read 0.
template <typename T>
__device__ __forceinline__ void stage_coarse_patch(T (*sc)[45], int FX, int FY, int FZ, GridView coarse,
                                                   const T* __restrict__ cin, long Nc) {
  const int e = threadIdx.x;
  if (e < 45) {
    const long n = coarse.node(FX / 2 + 2 + e / 15, FY / 2 + 2 + (e / 5) % 3, FZ / 2 + 4 + e % 5);
    sc[0][e] = n < 0 ? T(0) : cin[n];
    sc[1][e] = n < 0 ? T(0) : cin[n + Nc];
    sc[2][e] = n < 0 ? T(0) : cin[n + 2 * Nc];
  }
  __syncthreads();
}

// fine(f) += sum of trilinear weights * coarse(((f + (4,4,8)) >> 1) + {0,1}^3); then
// Project (Dirichlet), optional float rounding, Project_Null_Space (inactive nodes),
// as Run_VCycle does after Prolongate (solver/MG/Multigrid_Hierarchy.h:600-603).
template <typename T>
__global__ void __launch_bounds__(128) prolongate_kernel(int nb, const int* __restrict__ coords,
                                                         const uint32_t* __restrict__ fflags, GridView coarse,
                                                         const T* __restrict__ cin, long Nc, T* __restrict__ fu,
                                                         long Nf, int round_out) {
  __shared__ T sc[3][45];
  const int bi = blockIdx.x, e = threadIdx.x;
  if (bi >= nb) return;
  const int FX = coords[3 * bi], FY = coords[3 * bi + 1], FZ = coords[3 * bi + 2];
  pdl_wait();
  stage_coarse_patch<T>(sc, FX, FY, FZ, coarse, cin, Nc);
  const int lx = e >> 5, ly = (e >> 3) & 3, lz = e & 7;
  const long t = long(bi) * 128 + e;
  T v0 = fu[t], v1 = fu[t + Nf], v2 = fu[t + 2 * Nf];
  for (int q = 0; q < 8; ++q) {
    const int ii = q >> 2, jj = (q >> 1) & 1, kk = q & 1;
    const double wx = (lx & 1) ? 0.5 : (ii ? 0.0 : 1.0);
    const double wy = (ly & 1) ? 0.5 : (jj ? 0.0 : 1.0);
    const double wz = (lz & 1) ? 0.5 : (kk ? 0.0 : 1.0);
    const T w = T(wx * wy * wz);
    if (!(w > T(0))) continue;
    const int h = ((lx >> 1) + ii) * 15 + ((ly >> 1) + jj) * 5 + (lz >> 1) + kk;
    v0 += w * sc[0][h];
    v1 += w * sc[1][h];
    v2 += w * sc[2][h];
  }
  const uint32_t fl = fflags[t];
  if (fl & DIR_X) v0 = 0;
  if (fl & DIR_Y) v1 = 0;
  if (fl & DIR_Z) v2 = 0;
  if (round_out) { v0 = T(round_to_float(v0)); v1 = T(round_to_float(v1)); v2 = T(round_to_float(v2)); }
  if (!(fl & ACTIVE_NODE)) v0 = v1 = v2 = 0;
  fu[t] = v0;
  fu[t + Nf] = v1;
  fu[t + 2 * Nf] = v2;
}

// prolongate_kernel into the packed level-0 iterate (E in .w is kept).  Only
// active nodes are read and written: the V-cycle starts from u = 0 and no
// kernel before this one writes an inactive node's displacement, so those
// slots already hold the zeros that the projection would write.
template <typename T>
__global__ void __launch_bounds__(128) prolongate4_kernel(int nb, const int* __restrict__ coords,
                                                          const uint32_t* __restrict__ fflags, GridView coarse,
                                                          const T* __restrict__ cin, long Nc,
                                                          typename Pack4<T>::type* __restrict__ fu4) {
  __shared__ T sc[3][45];
  const int bi = blockIdx.x, e = threadIdx.x;
  if (bi >= nb) return;
  const int FX = coords[3 * bi], FY = coords[3 * bi + 1], FZ = coords[3 * bi + 2];
  const long t = long(bi) * 128 + e;
  const uint32_t fl = fflags[t];
  pdl_wait();
  stage_coarse_patch<T>(sc, FX, FY, FZ, coarse, cin, Nc);
  if (!(fl & ACTIVE_NODE)) return;
  const int lx = e >> 5, ly = (e >> 3) & 3, lz = e & 7;
  auto v = fu4[t];
  for (int q = 0; q < 8; ++q) {
    const int ii = q >> 2, jj = (q >> 1) & 1, kk = q & 1;
    const double wx = (lx & 1) ? 0.5 : (ii ? 0.0 : 1.0);
    const double wy = (ly & 1) ? 0.5 : (jj ? 0.0 : 1.0);
    const double wz = (lz & 1) ? 0.5 : (kk ? 0.0 : 1.0);
    const T w = T(wx * wy * wz);
    if (!(w > T(0))) continue;
    const int h = ((lx >> 1) + ii) * 15 + ((ly >> 1) + jj) * 5 + (lz >> 1) + kk;
    v.x += w * sc[0][h];
    v.y += w * sc[1][h];
    v.z += w * sc[2][h];
  }
  if (fl & DIR_X) v.x = 0;
  if (fl & DIR_Y) v.y = 0;
  if (fl & DIR_Z) v.z = 0;
  fu4[t] = v;
}

// ---------------------------------------------------------------------------
// Elementwise helpers
// ---------------------------------------------------------------------------
template <typename T>
__global__ void round_float_kernel(T* p, long n) {
  pdl_wait();
  long t = long(blockIdx.x) * blockDim.x + threadIdx.x;
  if (t < n) p[t] = T(round_to_float(p[t]));
}

template <typename T>
__global__ void zero_list_kernel(T* p, const int* __restrict__ idx, int n) {
  pdl_wait();
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t < n) p[idx[t]] = T(0);
}

// zero the three components of nodes without ACTIVE_NODE (Project_Null_Space.h:223-232)
template <typename T>
__global__ void project_null_kernel(T* p, const uint32_t* __restrict__ flags, long N) {
  pdl_wait();
  long t = long(blockIdx.x) * blockDim.x + threadIdx.x;
  if (t < N && !(flags[t] & ACTIVE_NODE)) p[t] = p[t + N] = p[t + 2 * N] = T(0);
}

template <typename TD, typename TS>
__global__ void convert_kernel(TD* __restrict__ d, const TS* __restrict__ s, long n) {
  pdl_wait();
  long t = long(blockIdx.x) * blockDim.x + threadIdx.x;
  if (t < n) d[t] = TD(s[t]);
}

}  // namespace sgs
