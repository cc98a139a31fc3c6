// Set-up kernels: Galerkin coarse operators, Dirichlet deletion, dense bottom
// operator and its inverse.
#pragma once
#include "kernels.cuh"

namespace sgs {

// ---------------------------------------------------------------------------
// Galerkin operator of a coarse level at `depth` (solver/MG/Galerkin_Coarsen.h:40-100).
// The reference prolongates a unit vector cell by cell down to the finest level,
// applies the finest element matrices and restricts back.  Here the same
// quantity is assembled directly: for coarse cell C and fine cell p inside it,
// table[p][a][b][v][w] = sum_ij W_p[i][a] W_p[j][b] Kc[i][j][v][w] with W_p the
// trilinear weights of C's corners at p's nodes, so
//     K_C[(a,v),(b,w)] = sum_p E_p * table[p][a][b][v][w].
// One CTA (576 threads: 8 cells x 8 corners x 9 components) per coarse node.
// ---------------------------------------------------------------------------
constexpr int GAL_CHUNK = 64;

__global__ void __launch_bounds__(576) galerkin_kernel(const int* __restrict__ coords, const uint32_t* __restrict__ flags,
                                                       int depth, GridView g0, const double* __restrict__ E0,
                                                       const double* __restrict__ table, double* __restrict__ A,
                                                       uint32_t* __restrict__ spokes, long N, double dx) {
  __shared__ double sE[8][GAL_CHUNK];
  __shared__ double contrib[8][72];
  __shared__ int sorigin[8][3];
  const long gidx = blockIdx.x;
  if (!(flags[gidx] & ACTIVE_NODE)) return;
  const int bi = int(gidx >> 7), e = int(gidx & 127);
  const int x = coords[3 * bi] + (e >> 5), y = coords[3 * bi + 1] + ((e >> 3) & 3), z = coords[3 * bi + 2] + (e & 7);
  const int t = threadIdx.x;
  const int c = t / 72, b = (t / 9) % 8, vw = t % 9;
  const int a = 7 - c;
  const int side = 1 << depth;
  if (t < 8) {
    // min corner of coarse cell t on the finest level: 2^d * cell - (2^d - 1) * (4,4,8)
    const int ccx = x + (t >> 2) - 1, ccy = y + ((t >> 1) & 1) - 1, ccz = z + (t & 1) - 1;
    sorigin[t][0] = side * ccx - (side - 1) * 4;
    sorigin[t][1] = side * ccy - (side - 1) * 4;
    sorigin[t][2] = side * ccz - (side - 1) * 8;
  }
  __syncthreads();
  const long npos = long(side) * side * side;
  double acc = 0;
  for (long p0 = 0; p0 < npos; p0 += GAL_CHUNK) {
    if (t < 8 * GAL_CHUNK) {
      const int cc = t / GAL_CHUNK;
      const long p = p0 + t % GAL_CHUNK;
      double ev = 0;
      if (p < npos) {
        const int px = int(p / (long(side) * side)), py = int((p / side) % side), pz = int(p % side);
        const long n = g0.node(sorigin[cc][0] + px, sorigin[cc][1] + py, sorigin[cc][2] + pz);
        if (n >= 0) ev = E0[n];
      }
      sE[cc][t % GAL_CHUNK] = ev;
    }
    __syncthreads();
    const int np = int(min(long(GAL_CHUNK), npos - p0));
    const double* tb = table + ((p0 * 8 + a) * 8 + b) * 9 + vw;
    for (int q = 0; q < np; ++q) {
      const double ev = sE[c][q];
      if (ev != 0) acc += ev * tb[long(q) * 576];
    }
    __syncthreads();
  }
  contrib[c][b * 9 + vw] = acc;
  __syncthreads();
  if (t < 243) {
    const int q = t / 9, w9 = t % 9;
    const int qi = q / 9, qj = (q / 3) % 3, qk = q % 3;
    double s = 0;
    for (int cc = 0; cc < 8; ++cc) {
      const int bx = qi - (cc >> 2), by = qj - ((cc >> 1) & 1), bz = qk - (cc & 1);
      if (bx < 0 || bx > 1 || by < 0 || by > 1 || bz < 0 || bz > 1) continue;
      s += contrib[cc][((bx << 2) | (by << 1) | bz) * 9 + w9];
    }
    A[gidx * 243 + q * 9 + w9] = s * dx;
  }
  if (t < 27) {
    const int qi = t / 9, qj = (t / 3) % 3, qk = t % 3;
    bool nz = false;
    for (int cc = 0; cc < 8; ++cc) {
      const int bx = qi - (cc >> 2), by = qj - ((cc >> 1) & 1), bz = qk - (cc & 1);
      if (bx < 0 || bx > 1 || by < 0 || by > 1 || bz < 0 || bz > 1) continue;
      for (int k = 0; k < 9; ++k) nz |= contrib[cc][((bx << 2) | (by << 1) | bz) * 9 + k] != 0.0;
    }
    unsigned m = __ballot_sync(0x07ffffffu, nz);
    if (t == 0) spokes[gidx] = m;
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
// Bottom solve (Exact_Solve, solver/MG/Multigrid_Hierarchy.h:346-372): nodes of
// the level take b, DOF nodes then get the exact solution x = M^-1 b.
// ---------------------------------------------------------------------------
template <typename T>
__global__ void bottom_gather_kernel(int ndof, const int* __restrict__ dof_node, const T* __restrict__ b, long N,
                                     double* __restrict__ xb) {
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
  const long row = (long(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (row >= n) return;
  const double* m = M + row * ld;
  double s = 0;
  for (long c = lane; c < n; c += 32) s += m[c] * x[c];
  for (int o = 16; o; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
  if (lane == 0) y[row] = s;
}

template <typename T>
__global__ void bottom_scatter_kernel(int ndof, const int* __restrict__ dof_node, const double* __restrict__ xs,
                                      T* __restrict__ u, long N) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= ndof) return;
  long n = dof_node[i];
  u[n] = T(xs[3 * i]);
  u[n + N] = T(xs[3 * i + 1]);
  u[n + 2 * N] = T(xs[3 * i + 2]);
}

}  // namespace sgs
