// Set-up kernels: Galerkin coarse operators, Dirichlet deletion, dense bottom
// operator and its inverse.
#pragma once
#include "kernels.cuh"

namespace sgs {

// ---------------------------------------------------------------------------
// Galerkin operator of a coarse level at `depth` (solver/MG/Galerkin_Coarsen.h:40-100).
// The reference prolongates a unit vector cell by cell down to the finest level,
// applies the finest element matrices and restricts back.  The same quantity is
// assembled here in two steps.  For a coarse cell C and a finest cell p inside
// it, table[p][a][b][v][w] = sum_ij W_p[i][a] W_p[j][b] Kc[i][j][v][w] (W_p: the
// trilinear weights of C's corners at p's nodes), so the 24x24 cell matrix is
//     K_C[(a,v),(b,w)] = sum_p E_p * table[p][a][b][v][w],
// one row of a GEMM [cells x 8^depth] x [8^depth x 576].  Each active coarse
// node then sums the row blocks of its corner from its 8 incident cells.
// ---------------------------------------------------------------------------

// table[p][(a*8+b)*9 + v*3 + w], one thread per (p, a, b)
__global__ void galerkin_table_kernel(int depth, double* __restrict__ table) {
  const long t = long(blockIdx.x) * blockDim.x + threadIdx.x;
  const int side = 1 << depth;
  const long npos = long(side) * side * side;
  if (t >= npos * 64) return;
  const long p = t >> 6;
  const int a = int(t >> 3) & 7, b = int(t) & 7;
  const int pc[3] = {int(p / (long(side) * side)), int((p / side) % side), int(p % side)};
  double Wa[8], Wb[8];
  for (int i = 0; i < 8; ++i) {
    double wa = 1, wb = 1;
    for (int ax = 0; ax < 3; ++ax) {
      const double tpos = double(pc[ax] + ((i >> (2 - ax)) & 1)) / side;
      wa *= ((a >> (2 - ax)) & 1) ? tpos : 1 - tpos;
      wb *= ((b >> (2 - ax)) & 1) ? tpos : 1 - tpos;
    }
    Wa[i] = wa;
    Wb[i] = wb;
  }
  double acc[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
  for (int i = 0; i < 8; ++i) {
    if (Wa[i] == 0) continue;
    for (int j = 0; j < 8; ++j) {
      const double w = Wa[i] * Wb[j];
      if (w == 0) continue;
      for (int m = 0; m < 9; ++m) acc[m] += w * c_Kc64[(i * 8 + j) * 9 + m];
    }
  }
  double* out = table + p * 576 + (a * 8 + b) * 9;
  for (int m = 0; m < 9; ++m) out[m] = acc[m];
}

// Cell matrices: C[cell][576] = sum_p E(origin_cell + p) * table[p][576], 64x64
// output tiles, the E operand gathered from the finest level on the fly.
constexpr int GT = 64;
__global__ void __launch_bounds__(256) galerkin_cell_kernel(int ncells, const int* __restrict__ origin, int depth,
                                                           GridView g0, const double* __restrict__ E0,
                                                           const double* __restrict__ table, double* __restrict__ C) {
  extern __shared__ double gsm[];
  double* sA = gsm;            // [64 cells][65]
  double* sB = gsm + GT * 65;  // [64 p][65]
  const int col0 = blockIdx.x * GT;
  const int cell0 = blockIdx.y * GT;
  const int side = 1 << depth;
  const long npos = long(side) * side * side;
  const int t = threadIdx.x, ty = t / 16, tx = t % 16;
  double acc[4][4] = {};
  for (long p0 = 0; p0 < npos; p0 += GT) {
    for (int i = t; i < GT * GT; i += 256) {
      const int r = i / GT, k = i % GT;
      const int cell = cell0 + r;
      const long p = p0 + k;
      double ev = 0;
      if (cell < ncells && p < npos) {
        const int px = int(p / (long(side) * side)), py = int((p / side) % side), pz = int(p % side);
        const long n = g0.node(origin[3 * cell] + px, origin[3 * cell + 1] + py, origin[3 * cell + 2] + pz);
        if (n >= 0) ev = E0[n];
      }
      sA[r * 65 + k] = ev;
    }
    __syncthreads();
    for (int i = t; i < GT * GT; i += 256) {
      const int k = i / GT, c = i % GT;
      const long p = p0 + k;
      sB[k * 65 + c] = p < npos ? table[p * 576 + col0 + c] : 0.0;
    }
    __syncthreads();
    for (int k = 0; k < GT; ++k) {
      double av[4], bv[4];
#pragma unroll
      for (int r = 0; r < 4; ++r) av[r] = sA[(ty + 16 * r) * 65 + k];
#pragma unroll
      for (int s = 0; s < 4; ++s) bv[s] = sB[k * 65 + tx + 16 * s];
#pragma unroll
      for (int r = 0; r < 4; ++r)
#pragma unroll
        for (int s = 0; s < 4; ++s) acc[r][s] += av[r] * bv[s];
    }
    __syncthreads();
  }
#pragma unroll
  for (int r = 0; r < 4; ++r) {
    const int cell = cell0 + ty + 16 * r;
    if (cell >= ncells) continue;
#pragma unroll
    for (int s = 0; s < 4; ++s) C[long(cell) * 576 + col0 + tx + 16 * s] = acc[r][s];
  }
}

// Cell matrices of the next coarser level from this level's: a coarse cell
// covers 2x2x2 cells of the finer level (child d at finer cell 2c - (4,4,8) + d),
// and the trilinear basis of its corners restricted to a child is the child's
// basis times w_d[i][a], the weight of coarse corner a at child corner i (a
// product of 0, 1/2, 1 per axis, exact).  So
//     K_C[(a,v),(b,w)] = sum_d sum_ij w_d[i][a] w_d[j][b] K_d[(i,v),(j,w)],
// which equals the sum over the finest cells of galerkin_cell_kernel up to
// rounding, at 8 children instead of 8^depth positions per coarse cell.  One
// CTA of 576 threads per coarse cell, one output entry per thread, children in
// fixed order.
__global__ void __launch_bounds__(576) galerkin_coarsen_kernel(const int* __restrict__ ccoord, GridView gf,
                                                              const int* __restrict__ fine_cell_of_slot,
                                                              const double* __restrict__ Cf, double* __restrict__ Cc) {
  __shared__ double sK[8][576];
  __shared__ double sw[8][64];  // sw[d][i * 8 + a]
  __shared__ int child[8];
  const int cell = blockIdx.x, t = threadIdx.x;
  if (t < 8) {
    const int fx = 2 * ccoord[3 * cell] - 4 + ((t >> 2) & 1), fy = 2 * ccoord[3 * cell + 1] - 4 + ((t >> 1) & 1),
              fz = 2 * ccoord[3 * cell + 2] - 8 + (t & 1);
    const long n = gf.node(fx, fy, fz);
    child[t] = n >= 0 ? fine_cell_of_slot[n] : -1;
  }
  if (t < 512) {
    const int d = t >> 6, i = (t >> 3) & 7, a = t & 7;
    double w = 1;
    for (int ax = 0; ax < 3; ++ax) {
      const int sh = 2 - ax;
      const double pos = 0.5 * double(((d >> sh) & 1) + ((i >> sh) & 1));  // child corner in the coarse cell
      w *= ((a >> sh) & 1) ? pos : 1 - pos;
    }
    sw[d][i * 8 + a] = w;
  }
  __syncthreads();
  for (int d = 0; d < 8; ++d) sK[d][t] = child[d] >= 0 ? Cf[long(child[d]) * 576 + t] : 0.0;
  __syncthreads();
  const int a = t / 72, b = (t / 9) & 7, m = t % 9;
  double acc = 0;
  for (int d = 0; d < 8; ++d) {
    if (child[d] < 0) continue;
    for (int i = 0; i < 8; ++i) {
      const double wa = sw[d][i * 8 + a];
      if (wa == 0) continue;
      for (int j = 0; j < 8; ++j) {
        const double wab = wa * sw[d][j * 8 + b];
        if (wab != 0) acc = __fma_rn(wab, sK[d][(i * 8 + j) * 9 + m], acc);
      }
    }
  }
  Cc[long(cell) * 576 + t] = acc;
}

// Node stencils from the cell matrices: entry (q, v, w) sums the (corner, neighbour)
// blocks of the incident cells in a fixed order; spoke q is active when any of
// those blocks has a non-zero entry (Galerkin_Coarsen.h:79-93).  One CTA per node.
__global__ void __launch_bounds__(256) galerkin_assemble_kernel(const int* __restrict__ coords,
                                                               const uint32_t* __restrict__ flags,
                                                               const int* __restrict__ cell_of_slot, GridView g,
                                                               const double* __restrict__ C, double* __restrict__ A,
                                                               uint32_t* __restrict__ spokes, double dx) {
  __shared__ int scell[8];
  const long gidx = blockIdx.x;
  if (!(flags[gidx] & ACTIVE_NODE)) return;
  const int bi = int(gidx >> 7), e = int(gidx & 127);
  const int x = coords[3 * bi] + (e >> 5), y = coords[3 * bi + 1] + ((e >> 3) & 3), z = coords[3 * bi + 2] + (e & 7);
  const int t = threadIdx.x;
  if (t < 8) {
    const long n = g.node(x + (t >> 2) - 1, y + ((t >> 1) & 1) - 1, z + (t & 1) - 1);
    scell[t] = n >= 0 ? cell_of_slot[n] : -1;
  }
  __syncthreads();
  if (t < 243) {
    const int q = t / 9, vw = t % 9;
    const int qi = q / 9, qj = (q / 3) % 3, qk = q % 3;
    double s = 0;
    for (int c = 0; c < 8; ++c) {
      const int bx = qi - (c >> 2), by = qj - ((c >> 1) & 1), bz = qk - (c & 1);
      if (bx < 0 || bx > 1 || by < 0 || by > 1 || bz < 0 || bz > 1 || scell[c] < 0) continue;
      s += C[long(scell[c]) * 576 + ((7 - c) * 8 + ((bx << 2) | (by << 1) | bz)) * 9 + vw];
    }
    A[gidx * 243 + t] = s * dx;
  }
  if (t < 32) {
    bool nz = false;
    if (t < 27) {
      const int qi = t / 9, qj = (t / 3) % 3, qk = t % 3;
      for (int c = 0; c < 8; ++c) {
        const int bx = qi - (c >> 2), by = qj - ((c >> 1) & 1), bz = qk - (c & 1);
        if (bx < 0 || bx > 1 || by < 0 || by > 1 || bz < 0 || bz > 1 || scell[c] < 0) continue;
        const double* blk = C + long(scell[c]) * 576 + ((7 - c) * 8 + ((bx << 2) | (by << 1) | bz)) * 9;
        for (int k = 0; k < 9; ++k) nz |= blk[k] != 0.0;
      }
    }
    const unsigned m = __ballot_sync(0xffffffffu, nz);
    if (t == 0) spokes[gidx] = m & 0x07ffffffu;
  }
}

// Delete_Dirichlet_Equations (solver/MG/Delete_Dirichlet_Equations.h:24-50)
__global__ void delete_dirichlet_kernel(int nb, const int* __restrict__ coords, const uint32_t* __restrict__ flags,
                                        const uint32_t* __restrict__ spokes, GridView g, double* __restrict__ A, long N) {
  const long gidx = long(blockIdx.x) * blockDim.x + threadIdx.x;
  if (gidx >= long(nb) * 128) return;
  const uint32_t fl = flags[gidx];
  if (!(fl & ACTIVE_NODE)) return;
  const uint32_t sp = spokes[gidx];
  const int bi = int(gidx >> 7), e = int(gidx & 127);
  const int x = coords[3 * bi] + (e >> 5), y = coords[3 * bi + 1] + ((e >> 3) & 3), z = coords[3 * bi + 2] + (e & 7);
  for (int q = 0; q < 27; ++q) {
    if (!(sp & (1u << q))) continue;
    const long n = g.node(x + q / 9 - 1, y + (q / 3) % 3 - 1, z + q % 3 - 1);
    const uint32_t nf = n >= 0 ? flags[n] : 0u;
    for (int v = 0; v < 3; ++v)
      for (int w = 0; w < 3; ++w) {
        double* a = A + gidx * 243 + q * 9 + v * 3 + w;
        if (fl & (DIR_X << v)) *a = (v == w && q == 13) ? 1.0 : 0.0;
        else if ((nf & ACTIVE_NODE) && (nf & (DIR_X << w))) *a = 0.0;
      }
  }
}

// Dense bottom operator over the DOF nodes (nodes with an active spoke), the way
// Build_CSR_Matrix forms PARDISO's upper triangle (solver/MG/Elasticity_Matrix.cpp:98-161):
// entry (r,c), r <= c, comes from row r's stencil; Dirichlet rows/columns become identity.
__global__ void bottom_assemble_kernel(int ndof_nodes, const int* __restrict__ dof_node, const int* __restrict__ node_dof,
                                       const int* __restrict__ coords, const uint32_t* __restrict__ flags,
                                       const uint32_t* __restrict__ spokes, GridView g, const double* __restrict__ A,
                                       long N, double* __restrict__ M, long ld) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= ndof_nodes) return;
  const long gidx = dof_node[i];
  const uint32_t fl = flags[gidx], sp = spokes[gidx];
  const bool fact = fl & ACTIVE_NODE;
  const int bi = int(gidx >> 7), e = int(gidx & 127);
  const int x = coords[3 * bi] + (e >> 5), y = coords[3 * bi + 1] + ((e >> 3) & 3), z = coords[3 * bi + 2] + (e & 7);
  for (int q = 0; q < 27; ++q) {
    if (!(sp & (1u << q))) continue;
    const long n = g.node(x + q / 9 - 1, y + (q / 3) % 3 - 1, z + q % 3 - 1);
    if (n < 0) continue;
    const int j = node_dof[n];
    if (j < 0) continue;
    const uint32_t nf = flags[n];
    for (int v = 0; v < 3; ++v)
      for (int w = 0; w < 3; ++w) {
        const long r = 3L * i + v, c = 3L * j + w;
        if (r > c) continue;
        double val = A[gidx * 243 + q * 9 + v * 3 + w];
        const bool dr = fact && (fl & (DIR_X << v));
        const bool dc = (nf & ACTIVE_NODE) && (nf & (DIR_X << w));
        if (dr || dc) val = (r == c) ? 1.0 : 0.0;
        M[r * ld + c] = val;
        M[c * ld + r] = val;
      }
  }
}

__global__ void identity_pad_kernel(double* M, long ld, long n0) {
  long i = n0 + long(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i < ld) M[i * ld + i] = 1.0;
}

// ---------------------------------------------------------------------------
// Blocked Gauss-Jordan inversion of the (padded) bottom matrix, 64x64 tiles.
// Sweeping pivot block K: P' = P^-1, A_KJ' = P^-1 A_KJ, A_IJ' = A_IJ - A_IK A_KJ',
// A_IK' = -A_IK P^-1.  After all pivots the matrix holds its inverse.
// ---------------------------------------------------------------------------
constexpr int GJ = 64;

__global__ void __launch_bounds__(256) gj_pivot_kernel(double* M, long ld, int K, double* Pinv, int* bad) {
  extern __shared__ double sP[];  // 64x65
  const int t = threadIdx.x;
  for (int i = t; i < GJ * GJ; i += 256) sP[(i / GJ) * 65 + i % GJ] = M[(long(K) * GJ + i / GJ) * ld + long(K) * GJ + i % GJ];
  __syncthreads();
  for (int k = 0; k < GJ; ++k) {
    const double piv = sP[k * 65 + k];
    __syncthreads();
    if (t == 0 && !(piv > 0)) *bad = 1;
    const double ip = 1.0 / piv;
    if (t < GJ) sP[k * 65 + t] = (t == k) ? ip : sP[k * 65 + t] * ip;
    __syncthreads();
    for (int idx = t; idx < GJ * GJ; idx += 256) {
      const int i = idx / GJ, j = idx % GJ;
      if (i == k) continue;
      const double f = sP[i * 65 + k];
      if (j == k) continue;
      sP[i * 65 + j] -= f * sP[k * 65 + j];
    }
    __syncthreads();
    if (t < GJ && t != k) sP[t * 65 + k] = -sP[t * 65 + k] * sP[k * 65 + k];
    __syncthreads();
  }
  for (int i = t; i < GJ * GJ; i += 256) Pinv[i] = sP[(i / GJ) * 65 + i % GJ];
}

// C = alpha * A(tile) x B(tile) [+ C if accumulate]; tiles addressed by (row tile, col tile)
// mode 0: row panel  A_KJ <- Pinv * A_KJ        (grid.x = tile J, skip K)
// mode 1: update     A_IJ <- A_IJ - A_IK*A_KJ   (grid = (J, I), skip K)
// mode 2: col panel  A_IK <- -A_IK * Pinv       (grid.x = tile I, skip K)
__global__ void __launch_bounds__(256) gj_tile_kernel(double* M, long ld, int K, const double* __restrict__ Pinv, int mode) {
  extern __shared__ double sm[];
  double* sA = sm;             // 64 x 65
  double* sB = sm + GJ * 65;   // 64 x 65
  int I, J;
  const double* srcA;
  const double* srcB;
  long lda, ldb;
  if (mode == 0) {
    J = blockIdx.x; if (J == K) return; I = K;
    srcA = Pinv; lda = GJ; srcB = M + long(K) * GJ * ld + long(J) * GJ; ldb = ld;
  } else if (mode == 1) {
    J = blockIdx.x; I = blockIdx.y; if (I == K || J == K) return;
    srcA = M + long(I) * GJ * ld + long(K) * GJ; lda = ld; srcB = M + long(K) * GJ * ld + long(J) * GJ; ldb = ld;
  } else {
    I = blockIdx.x; if (I == K) return; J = K;
    srcA = M + long(I) * GJ * ld + long(K) * GJ; lda = ld; srcB = Pinv; ldb = GJ;
  }
  const int t = threadIdx.x;
  for (int i = t; i < GJ * GJ; i += 256) {
    sA[(i / GJ) * 65 + i % GJ] = srcA[long(i / GJ) * lda + i % GJ];
    sB[(i / GJ) * 65 + i % GJ] = srcB[long(i / GJ) * ldb + i % GJ];
  }
  __syncthreads();
  const int ty = t / 16, tx = t % 16;
  double acc[4][4] = {};
  for (int k = 0; k < GJ; ++k) {
    double av[4], bv[4];
#pragma unroll
    for (int r = 0; r < 4; ++r) av[r] = sA[(ty + 16 * r) * 65 + k];
#pragma unroll
    for (int s = 0; s < 4; ++s) bv[s] = sB[k * 65 + tx + 16 * s];
#pragma unroll
    for (int r = 0; r < 4; ++r)
#pragma unroll
      for (int s = 0; s < 4; ++s) acc[r][s] += av[r] * bv[s];
  }
  double* C = M + long(I) * GJ * ld + long(J) * GJ;
#pragma unroll
  for (int r = 0; r < 4; ++r)
#pragma unroll
    for (int s = 0; s < 4; ++s) {
      double* cp = C + long(ty + 16 * r) * ld + tx + 16 * s;
      if (mode == 0) *cp = acc[r][s];
      else if (mode == 1) *cp -= acc[r][s];
      else *cp = -acc[r][s];
    }
}

__global__ void gj_store_pivot_kernel(double* M, long ld, int K, const double* __restrict__ Pinv) {
  for (int i = threadIdx.x; i < GJ * GJ; i += blockDim.x) M[(long(K) * GJ + i / GJ) * ld + long(K) * GJ + i % GJ] = Pinv[i];
}

// ---------------------------------------------------------------------------
// Symmetric blocked Gauss-Jordan with 128-wide pivot panels.  The bottom matrix
// is SPD, and after pivots 0..K-1 tile (I, J) equals the transpose of tile
// (J, I), negated when exactly one of I, J has been pivoted.  So only the lower
// tiles (I >= J) are updated; the panels a step needs are gathered from them:
//   row panel  R_J = A_KJ  (J < K), A_KK, A_JK^T (J > K)
//   col panel  C_I = A_IK  (I > K), A_KK, -A_KI^T (I < K)
// then T = P^-1 R, lower tiles A_IJ -= C_I T_J, A_IK = -C_I P^-1 (I > K),
// A_KJ = T_J (J < K), A_KK = P^-1.  After the last pivot the lower tiles hold
// the lower half of M^-1 and are mirrored.  FP64 GEMM tiles of 128 x 128, a
// thread computing 8 x 8 entries from k-chunks staged in shared memory.
// ---------------------------------------------------------------------------
constexpr int SGJ = 128, SGJ_K = 16;

__global__ void sgj_gather_kernel(const double* __restrict__ M, long ld, int K, double* __restrict__ R,
                                  double* __restrict__ Cp, double* __restrict__ P) {
  const long t = long(blockIdx.x) * blockDim.x + threadIdx.x;
  if (t >= long(SGJ) * ld) return;
  const long k0 = long(K) * SGJ;
  {  // R[r][c], r < 128, c < ld
    const long r = t / ld, c = t % ld, J = c / SGJ;
    R[t] = (J <= K) ? M[(k0 + r) * ld + c] : M[c * ld + k0 + r];
  }
  {  // Cp[i][q], i < ld, q < 128
    const long i = t / SGJ, q = t % SGJ, I = i / SGJ;
    Cp[t] = (I >= K) ? M[i * ld + k0 + q] : -M[(k0 + q) * ld + i];
  }
  if (P && t < long(SGJ) * SGJ) P[t] = M[(k0 + t / SGJ) * ld + k0 + t % SGJ];
}

// One FP64 tensor-core MMA (m16n8k8): D = A B + D on a 16 x 8 tile.  With
// g = lane / 4 and t = lane % 4, a lane holds A[g][t], A[g+8][t], A[g][t+4],
// A[g+8][t+4]; B[t][g], B[t+4][g]; D[g][2t], D[g][2t+1], D[g+8][2t], D[g+8][2t+1].
__device__ __forceinline__ void dmma_16x8x8(double (&d)[4], const double (&a)[4], const double (&b)[2]) {
  asm volatile(
      "mma.sync.aligned.m16n8k8.row.col.f64.f64.f64.f64 {%0, %1, %2, %3}, {%4, %5, %6, %7}, {%8, %9}, "
      "{%0, %1, %2, %3};\n"
      : "+d"(d[0]), "+d"(d[1]), "+d"(d[2]), "+d"(d[3])
      : "d"(a[0]), "d"(a[1]), "d"(a[2]), "d"(a[3]), "d"(b[0]), "d"(b[1]));
}

// C(tile) = alpha * A(tile rows, 0:k) * B(0:k, tile cols) + beta * C(tile) on
// 128 x 128 tiles: sixteen warps of 32 x 32 (four per SM sub-partition, to hide
// the MMA latency), k staged through shared memory in chunks of 16, FP64 MMAs.
// Tiles: SGJ_DENSE (blockIdx.y, blockIdx.x); SGJ_LOWER the tiles I >= J of a
// square grid (blockIdx.x), leaving out row and column `skip` (none if < 0);
// SGJ_CROSS the lower tiles of row and column `skip` (blockIdx.x = J for
// J <= skip, else I).
constexpr int SGJ_THREADS = 512;          // sixteen warps of 32 x 32 per 128 x 128 tile
constexpr int SGJ_AS = 20, SGJ_BS = 132;  // padded strides (4 mod 16 doubles): conflict-free fragment loads
constexpr int SGJ_STAGE = SGJ * SGJ_AS + SGJ_K * SGJ_BS;  // doubles per pipeline stage
constexpr size_t SGJ_SMEM = 2 * SGJ_STAGE * sizeof(double);
enum { SGJ_DENSE = 0, SGJ_LOWER = 1, SGJ_CROSS = 2 };

__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
  const unsigned s = unsigned(__cvta_generic_to_shared(smem));
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
__device__ __forceinline__ void cp_async_wait_prior() { asm volatile("cp.async.wait_group 1;\n" ::); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;\n" ::); }

// k staged through two shared-memory stages filled by cp.async: the copy of
// chunk c + 1 runs while chunk c is multiplied.
__global__ void __launch_bounds__(SGJ_THREADS, 1) sgj_gemm_kernel(int k, const double* __restrict__ A, long lda,
                                                          const double* __restrict__ B, long ldb, double* C, long ldc,
                                                          double alpha, double beta, int mode, int skip) {
  extern __shared__ __align__(16) double sg[];
  long I, J;
  if (mode == SGJ_LOWER) {
    const long t = blockIdx.x;
    long i = long((sqrt(8.0 * double(t) + 1.0) - 1.0) * 0.5);
    while ((i + 1) * (i + 2) / 2 <= t) ++i;
    while (i * (i + 1) / 2 > t) --i;
    I = i;
    J = t - i * (i + 1) / 2;
    if (I == skip || J == skip) return;
  } else if (mode == SGJ_CROSS) {
    const long b = blockIdx.x;
    I = b <= skip ? skip : b;
    J = b <= skip ? b : skip;
  } else {
    I = blockIdx.y;
    J = blockIdx.x;
  }
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int wr = (warp >> 2) * 32, wc = (warp & 3) * 32;  // the warp's 32 x 32 sub-tile
  if (beta != 0) {  // the epilogue reads this C tile: bring it into L2 while the products run
    const double* quarter_row = C + (I * SGJ + (tid >> 2)) * ldc + J * SGJ + (tid & 3) * 32;
#pragma unroll
    for (int q = 0; q < 2; ++q) asm volatile("prefetch.global.L2 [%0];" ::"l"(quarter_row + 16 * q));
  }
  const int fr = lane >> 2, fc = lane & 3;
  const double* Ab = A + I * SGJ * lda;
  const double* Bb = B + J * SGJ;
  const int ar = tid >> 2, ak = (tid & 3) * 4;    // A chunk: row, first k
  const int bk = tid >> 5, bc = (tid & 31) * 4;   // B chunk: k, first column
  auto stage = [&](int k0, int st) {
    double* As = sg + st * SGJ_STAGE;
    double* Bs = As + SGJ * SGJ_AS;
    const double* a = Ab + long(ar) * lda + k0 + ak;
    const double* b = Bb + long(k0 + bk) * ldb + bc;
#pragma unroll
    for (int q = 0; q < 2; ++q) {
      cp_async16(&As[ar * SGJ_AS + ak + 2 * q], a + 2 * q);
      cp_async16(&Bs[bk * SGJ_BS + bc + 2 * q], b + 2 * q);
    }
    cp_async_commit();
  };
  double acc[2][4][4];
#pragma unroll
  for (int i = 0; i < 2; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) acc[i][j][0] = acc[i][j][1] = acc[i][j][2] = acc[i][j][3] = 0;
  const int nchunks = k / SGJ_K;
  stage(0, 0);
  for (int c = 0; c < nchunks; ++c) {
    if (c + 1 < nchunks) {
      stage((c + 1) * SGJ_K, (c + 1) & 1);
      cp_async_wait_prior();
    } else {
      cp_async_wait_all();
    }
    __syncthreads();
    const double* As = sg + (c & 1) * SGJ_STAGE;
    const double* Bs = As + SGJ * SGJ_AS;
#pragma unroll
    for (int k8 = 0; k8 < SGJ_K; k8 += 8) {
      double a[2][4], b[4][2];
#pragma unroll
      for (int i = 0; i < 2; ++i) {
        const double* r = As + (wr + 16 * i + fr) * SGJ_AS + k8 + fc;
        a[i][0] = r[0];
        a[i][1] = r[8 * SGJ_AS];
        a[i][2] = r[4];
        a[i][3] = r[8 * SGJ_AS + 4];
      }
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        b[j][0] = Bs[(k8 + fc) * SGJ_BS + wc + 8 * j + fr];
        b[j][1] = Bs[(k8 + fc + 4) * SGJ_BS + wc + 8 * j + fr];
      }
#pragma unroll
      for (int i = 0; i < 2; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) dmma_16x8x8(acc[i][j], a[i], b[j]);
    }
    __syncthreads();  // the stage is refilled two chunks later
  }
#pragma unroll
  for (int i = 0; i < 2; ++i)
#pragma unroll
    for (int hr = 0; hr < 2; ++hr) {
      double* row = C + (I * SGJ + wr + 16 * i + 8 * hr + fr) * ldc + J * SGJ + wc + 2 * fc;
#pragma unroll
      for (int j = 0; j < 4; ++j)
#pragma unroll
        for (int h = 0; h < 2; ++h) {
          double* p = row + 8 * j + h;
          *p = (beta != 0 ? beta * *p : 0.0) + alpha * acc[i][j][2 * hr + h];
        }
    }
}

// mirror the lower triangle into the upper one
__global__ void sgj_mirror_kernel(double* M, long ld) {
  __shared__ double tile[32][33];
  const int bx = blockIdx.x, by = blockIdx.y;  // source tile (row by, col bx), by > bx
  if (by <= bx) {
    if (by < bx) return;
    // diagonal 32x32 tile: copy lower to upper in place
    for (int i = threadIdx.y; i < 32; i += blockDim.y) {
      const int j = threadIdx.x;
      if (j > i) M[(long(by) * 32 + i) * ld + long(bx) * 32 + j] = M[(long(bx) * 32 + j) * ld + long(by) * 32 + i];
    }
    return;
  }
  for (int i = threadIdx.y; i < 32; i += blockDim.y)
    tile[i][threadIdx.x] = M[(long(by) * 32 + i) * ld + long(bx) * 32 + threadIdx.x];
  __syncthreads();
  for (int i = threadIdx.y; i < 32; i += blockDim.y)
    M[(long(bx) * 32 + i) * ld + long(by) * 32 + threadIdx.x] = tile[threadIdx.x][i];
}

// ---------------------------------------------------------------------------
// Bottom solve (Exact_Solve, solver/MG/Multigrid_Hierarchy.h:346-372): nodes of
// the level take b, DOF nodes then get the exact solution x = M^-1 b.
// ---------------------------------------------------------------------------
template <typename T>
__global__ void bottom_gather_kernel(int ndof, const int* __restrict__ dof_node, const T* __restrict__ b, long N,
                                     double* __restrict__ xb) {
  pdl_wait();
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= ndof) return;
  long n = dof_node[i];
  xb[3 * i] = double(b[n]);
  xb[3 * i + 1] = double(b[n + N]);
  xb[3 * i + 2] = double(b[n + 2 * N]);
}

// y = M x, one warp per row
__global__ void gemv_kernel(const double* __restrict__ M, long ld, long n, const double* __restrict__ x,
                            double* __restrict__ y) {
  pdl_wait();
  const long row = (long(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (row >= n) return;
  const double* m = M + row * ld;
  double s = 0;
  for (long c = lane; c < n; c += 32) s += m[c] * x[c];
  for (int o = 16; o; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
  if (lane == 0) y[row] = s;
}

// y = M x with an FP32 copy of M (ld a multiple of 128, rows 16-byte aligned),
// 32 rows per CTA of 1024 threads, one warp per row.  x is staged once per CTA
// in shared memory as FP32 (exact: in mixed precision it is gathered from an
// FP32 right-hand side), so the loop streams only M.
constexpr int GEMV32_ROWS = 32;
__global__ void __launch_bounds__(1024) gemv32_kernel(const float* __restrict__ M, long ld, long n,
                                                      const double* __restrict__ x, double* __restrict__ y) {
  extern __shared__ float4 xs4[];
  float* xs = reinterpret_cast<float*>(xs4);
  pdl_wait();
  for (long c = threadIdx.x; c < n; c += blockDim.x) xs[c] = float(x[c]);
  __syncthreads();
  const long row = long(blockIdx.x) * GEMV32_ROWS + (threadIdx.x >> 5);
  const int lane = threadIdx.x & 31;
  if (row >= n) return;
  const float4* m = reinterpret_cast<const float4*>(M + row * ld);
  float s0 = 0.f, s1 = 0.f;
  for (long c = lane; c < n / 4; c += 32) {
    const float4 a = __ldcs(m + c);  // read once per application: do not keep it in L2
    const float4 v = xs4[c];
    s0 = fmaf(a.x, v.x, s0);
    s1 = fmaf(a.y, v.y, s1);
    s0 = fmaf(a.z, v.z, s0);
    s1 = fmaf(a.w, v.w, s1);
  }
  double s = double(s0) + double(s1);
  for (int o = 16; o; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
  if (lane == 0) y[row] = s;
}

template <typename T>
__global__ void bottom_scatter_kernel(int ndof, const int* __restrict__ dof_node, const double* __restrict__ xs,
                                      T* __restrict__ u, long N) {
  pdl_wait();
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= ndof) return;
  long n = dof_node[i];
  u[n] = T(xs[3 * i]);
  u[n + N] = T(xs[3 * i + 1]);
  u[n + 2 * N] = T(xs[3 * i + 2]);
}

}  // namespace sgs
