// ORACLE — test infrastructure only.  CPU restatement of the reference solver
// path of yuanming-hu/spgrid_topo_opt (solver/SPGrid_CPU_Solver.cpp and the
// CG/, MG/, CPU_Kernels/ code it calls).  Only tests/, __graft_entry__.smoke()
// and bench.py's CPU-baseline leg load this library, and only as the checker.
//
// What it restates (reference file:line):
//   * SPGrid page ordering: blocks of 4x4x8 nodes ordered by the page index of
//     their Morton offset (external/SPGrid/Core/SPGrid_Mask.h:38-47,142;
//     SPGrid_Page_Map.h:117-124).  Memory semantics follow SPGrid: every
//     address of a level reads as zero until written, writes outside active
//     pages persist ("ghost" blocks here) but are never iterated.
//   * density -> mu/lambda through the SIMP map (fem_interface.h:343-353,
//     SPGrid_CPU_Solver.cpp:100-136);
//   * Dirichlet node -> cell rule (SPGrid_CPU_Solver.cpp:147-192);
//   * flags: Flaging/Flag_Nodes/Flag_Boundary_Nodes/Get_Boundary_Blocks/
//     Create_Dirichlet_List (CPU_Kernels/Flaging.h:31-173), hierarchy flags
//     (MG/Multigrid_Hierarchy.h:122-214);
//   * matrix-free K*u and residual (CPU_Kernels/SPGrid_Linear_Elasticity.h:22-344);
//   * coloured Gauss-Seidel on level 0 (CPU_Kernels/SPGrid_Gauss_Seidel.h:762-1180);
//   * restriction / accumulating prolongation (MG/Restriction.h:52-88,
//     MG/Prolongation.h:151-193);
//   * Galerkin coarse operators by recursive cell prolongation
//     (MG/Galerkin_Coarsen.h:40-100, MG/Linear_Elasticity_SIMD_Cell_Multiply.h:72-161,
//     MG/Trilinear_Cell_Transfer_Operators_SIMD.h:152-281), Dirichlet deletion
//     (MG/Delete_Dirichlet_Equations.h:24-50);
//   * coarse stencil multiply / coloured smoothing (MG/SPGrid_Stencil_Multiply.h:15-280);
//   * exact bottom solve (MG/Elasticity_Matrix.cpp:16-269, PARDISO replaced by a
//     banded Cholesky: both are exact SPD solves);
//   * V-cycle (MG/Multigrid_Hierarchy.h:569-619) and PCG
//     (CG/CONJUGATE_GRADIENT.cpp:21-61, CG/CG_SYSTEM.cpp:136-320,
//     CG/CG_VECTOR.cpp:15-145, CG/KRYLOV_SYSTEM_BASE.cpp:25-31);
//   * the SIMP compliance sensitivity (topo_opt/objective/minimal_compliance.cpp:86-146).
//
// Precision modes: REF reproduces the reference's float rounding of CG axpys
// (CG_VECTOR.cpp:25-30,108-113) and its Cast_To_Float inside the V-cycle
// (Multigrid_Hierarchy.h:439-451); FP64 leaves every value in double.
#include <algorithm>
#include <array>
#include <cfloat>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <limits>
#include <memory>
#include <unordered_set>
#include <vector>

#ifdef _OPENMP
#include <omp.h>
#endif

namespace orc {

// ---------------------------------------------------------------------------
// Flag bits (solver/Flags.h:10-24)
// ---------------------------------------------------------------------------
constexpr uint64_t ACTIVE_NODE = 0x10, DIRICHLET_NODE_X = 0x20, DIRICHLET_NODE_Y = 0x40,
                   DIRICHLET_NODE_Z = 0x80, DIRICHLET_NODE = 0xE0, ACTIVE_CELL = 0x100,
                   DIRICHLET_CELL_X = 0x200, DIRICHLET_CELL = 0xE00, BOUNDARY_NODE = 0x1000,
                   BOUNDARY_NODE_TEMP = 0x2000;

constexpr int BX = 4, BY = 4, BZ = 8, NPB = 128;  // solver block: 4x4x8 nodes
enum { CH_U0 = 0, CH_F0 = 3, CH_S0 = 6, CH_Q0 = 9, CH_MU = 12, CH_LA = 13, NCH = 15 };

enum Mode { MODE_REF = 0, MODE_FP64 = 1 };

// ---------------------------------------------------------------------------
// Stiffness tables derived from the Q1 element: K_mu[a][b][i][j] =
// int( delta_ij grad N_a . grad N_b + d_j N_a d_i N_b ), K_la = int d_i N_a d_j N_b
// on the unit cube; node index a = 4x+2y+z.  Exact rationals k/72.
// ---------------------------------------------------------------------------
static double K_mu[8][8][3][3], K_la[8][8][3][3];
static bool tables_ready = false;

static void build_tables() {
  if (tables_ready) return;
  // 1D integrals on [0,1] for phi_0 = 1-t, phi_1 = t, times 6 to stay integral:
  // M[a][b] = 6*int phi_a phi_b, D[a][b] = 6*int phi'_a phi_b, S[a][b] = 6*int phi'_a phi'_b
  const int M[2][2] = {{2, 1}, {1, 2}};
  const int D[2][2] = {{-3, -3}, {3, 3}};  // D[a][b]: derivative on a
  const int S[2][2] = {{6, -6}, {-6, 6}};
  auto bit = [](int n, int axis) { return (n >> (2 - axis)) & 1; };
  // g(a,b,i,j) = 216 * int d_i N_a d_j N_b
  auto g = [&](int a, int b, int i, int j) {
    long v = 1;
    for (int ax = 0; ax < 3; ++ax) {
      int pa = bit(a, ax), pb = bit(b, ax);
      bool da = (ax == i), db = (ax == j);
      int f;
      if (da && db) f = S[pa][pb];
      else if (da) f = D[pa][pb];
      else if (db) f = D[pb][pa];
      else f = M[pa][pb];
      v *= f;
    }
    return v;
  };
  for (int a = 0; a < 8; ++a)
    for (int b = 0; b < 8; ++b)
      for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) {
          long lam = g(a, b, i, j);
          long mu = g(a, b, j, i);
          if (i == j)
            for (int k = 0; k < 3; ++k) mu += g(a, b, k, k);
          // entries are multiples of 3/216 = 1/72
          K_la[a][b][i][j] = double(lam / 3) / 72.0;
          K_mu[a][b][i][j] = double(mu / 3) / 72.0;
        }
  tables_ready = true;
}

// ---------------------------------------------------------------------------
// SPGrid-like level storage
// ---------------------------------------------------------------------------
static inline uint64_t page_key(int bi, int bj, int bk) {
  // Page index bits of the Morton offset: bit 3m <- bj_m, 3m+1 <- bi_m, 3m+2 <- bk_m
  uint64_t key = 0;
  for (int m = 0; m < 21; ++m) {
    key |= uint64_t((bj >> m) & 1) << (3 * m);
    key |= uint64_t((bi >> m) & 1) << (3 * m + 1);
    key |= uint64_t((bk >> m) & 1) << (3 * m + 2);
  }
  return key;
}

struct Block {
  double ch[NCH][NPB];
  uint64_t flags[NPB];
};

static inline int lidx(int x, int y, int z) { return x * 32 + y * 8 + z; }

struct Level {
  int size[3] = {0, 0, 0};
  int nb[3] = {0, 0, 0};  // block grid dims
  std::vector<int32_t> bmap;  // block grid -> pool index, -1 when never touched
  std::vector<std::unique_ptr<Block>> pool;
  std::vector<uint8_t> active_page;  // per block-grid cell
  std::vector<int> active;           // pool indices of active blocks, page order
  std::vector<std::array<int, 3>> pool_base;
  std::vector<int> boundary;         // pool indices of boundary blocks
  std::array<std::vector<std::pair<int, int>>, 3> dirichlet;  // (pool, elem) per axis

  void init(int sx, int sy, int sz) {
    size[0] = sx; size[1] = sy; size[2] = sz;
    nb[0] = sx / BX + 3; nb[1] = sy / BY + 3; nb[2] = sz / BZ + 3;
    bmap.assign(size_t(nb[0]) * nb[1] * nb[2], -1);
    active_page.assign(bmap.size(), 0);
  }
  inline long cell_of(int x, int y, int z) const {
    if (x < 0 || y < 0 || z < 0) return -1;
    int bi = x >> 2, bj = y >> 2, bk = z >> 3;
    if (bi >= nb[0] || bj >= nb[1] || bk >= nb[2]) return -1;
    return (long(bi) * nb[1] + bj) * nb[2] + bk;
  }
  inline Block* find(int x, int y, int z) const {
    long c = cell_of(x, y, z);
    if (c < 0) return nullptr;
    int p = bmap[c];
    return p < 0 ? nullptr : pool[p].get();
  }
  Block* touch(int x, int y, int z) {
    long c = cell_of(x, y, z);
    if (c < 0) return nullptr;
    int p = bmap[c];
    if (p < 0) {
      p = int(pool.size());
      pool.emplace_back(new Block());
      std::memset(pool.back().get(), 0, sizeof(Block));
      pool_base.push_back({x & ~3, y & ~3, z & ~7});
      bmap[c] = p;
    }
    return pool[p].get();
  }
  void set_page(int x, int y, int z) {
    long c = cell_of(x, y, z);
    if (c < 0) return;
    touch(x, y, z);
    active_page[c] = 1;
  }
  bool test_page(int x, int y, int z) const {
    long c = cell_of(x, y, z);
    return c >= 0 && active_page[c];
  }
  void update_blocks() {
    std::vector<std::pair<uint64_t, int>> keys;
    for (long c = 0; c < long(bmap.size()); ++c)
      if (active_page[c]) {
        int p = bmap[c];
        auto& b = pool_base[p];
        keys.push_back({page_key(b[0] >> 2, b[1] >> 2, b[2] >> 3), p});
      }
    std::sort(keys.begin(), keys.end());
    active.clear();
    for (auto& k : keys) active.push_back(k.second);
  }
  inline double get(int ch, int x, int y, int z) const {
    Block* b = find(x, y, z);
    return b ? b->ch[ch][lidx(x & 3, y & 3, z & 7)] : 0.0;
  }
  inline uint64_t getf(int x, int y, int z) const {
    Block* b = find(x, y, z);
    return b ? b->flags[lidx(x & 3, y & 3, z & 7)] : 0;
  }
  // Writes outside the level's address range are dropped (SPGrid would fault).
  inline uint64_t& flag_ref(int x, int y, int z) {
    static thread_local uint64_t sink;
    Block* b = touch(x, y, z);
    if (!b) { sink = 0; return sink; }
    return b->flags[lidx(x & 3, y & 3, z & 7)];
  }
  inline double& ref(int ch, int x, int y, int z) {
    static thread_local double sink;
    Block* b = touch(x, y, z);
    if (!b) { sink = 0; return sink; }
    return b->ch[ch][lidx(x & 3, y & 3, z & 7)];
  }
};

// Galerkin stencil record (MG/Elasticity_Matrix.h:212-217), kept per active node
struct StencilLevel {
  std::vector<double> data;      // [active block][elem][243]
  std::vector<uint32_t> flags;   // spoke / dirichlet flags per node
  std::vector<int> block_of_pool;  // pool index -> active block ordinal (or -1)
};
constexpr uint32_t COORD_DIRICHLET[3] = {0x10000000u, 0x20000000u, 0x40000000u};
// Spoke<di,dj,dk>::Active = 1 << (9di+3dj+dk+13), di in {-1,0,1} (MG/Elasticity_Matrix.h:175-178)
static inline uint32_t spoke_bit(int i, int j, int k) { return 1u << (9 * i + 3 * j + k); }

static inline double to_float(double v) { return double(float(v)); }

// ---------------------------------------------------------------------------
// Exact SPD band solver for the bottom level
// ---------------------------------------------------------------------------
struct BandCholesky {
  long n = 0, bw = 0;
  std::vector<double> L;  // row-major band: L[i*(bw+1) + (j - i + bw)] for j in [i-bw, i]
  bool ok = false;
  double& at(long i, long j) { return L[size_t(i) * (bw + 1) + (j - i + bw)]; }
  bool factor() {
    for (long j = 0; j < n; ++j) {
      double d = at(j, j);
      long k0 = std::max(0L, j - bw);
      for (long k = k0; k < j; ++k) d -= at(j, k) * at(j, k);
      if (!(d > 0)) return false;
      d = std::sqrt(d);
      at(j, j) = d;
      long iend = std::min(n - 1, j + bw);
#pragma omp parallel for schedule(static)
      for (long i = j + 1; i <= iend; ++i) {
        double s = at(i, j);
        long kk0 = std::max(k0, i - bw);
        for (long k = kk0; k < j; ++k) s -= at(i, k) * at(j, k);
        at(i, j) = s / d;
      }
    }
    ok = true;
    return true;
  }
  void solve(std::vector<double>& x) {
    for (long i = 0; i < n; ++i) {
      double s = x[i];
      for (long k = std::max(0L, i - bw); k < i; ++k) s -= at(i, k) * x[k];
      x[i] = s / at(i, i);
    }
    for (long i = n - 1; i >= 0; --i) {
      double s = x[i];
      for (long k = i + 1; k <= std::min(n - 1, i + bw); ++k) s -= at(k, i) * x[k];
      x[i] = s / at(i, i);
    }
  }
};

// ---------------------------------------------------------------------------
// Solver state
// ---------------------------------------------------------------------------
struct Params {
  int resolution[3];
  double dx, global_mu, global_lambda, penalty, minimum_stiffness, minimum_density;
  int mg_level, smoothing_iter, boundary_smoothing, max_iterations, mode, explicit_level;
  double tolerance;
};

struct Solver {
  Params P;
  std::vector<Level> L;
  std::vector<StencilLevel> S;
  // bottom
  std::vector<std::pair<int, int>> bottom_nodes;  // (pool, elem) with DOF index 3*k
  BandCholesky chol;
  std::vector<long> bottom_perm;  // dof -> band position
  // inputs
  std::vector<std::array<int, 3>> in_base;
  std::vector<std::array<int, 3>> f_coord;
  std::vector<std::array<double, 3>> f_val;
  std::vector<std::array<int, 3>> d_coord;
  std::vector<int> d_axis;
  std::vector<double> d_val;
  bool disable_mg = false;
  int status = 0;
  char err[256] = {0};
  // stats
  int iterations = 0;
  double initial_residual = 0, final_residual = 0;
  std::vector<double> history;
};

#define ORC_FAIL(S, code, ...)                             \
  do {                                                     \
    (S).status = (code);                                   \
    std::snprintf((S).err, sizeof((S).err), __VA_ARGS__); \
    return false;                                          \
  } while (0)

// ---------------------------------------------------------------------------
// Level-0 operators
// ---------------------------------------------------------------------------
// f = dx * K u for every node of the listed blocks (SPGrid_Linear_Elasticity.h:96-213).
static void multiply_node(const Level& l, int x, int y, int z, int uch, double dx, double f[3]) {
  f[0] = f[1] = f[2] = 0;
  for (int I = 0; I < 8; ++I) {
    int Ix = I >> 2, Iy = (I >> 1) & 1, Iz = I & 1;
    int cx = x - Ix, cy = y - Iy, cz = z - Iz;
    double mu = l.get(CH_MU, cx, cy, cz), la = l.get(CH_LA, cx, cy, cz);
    for (int J = 0; J < 8; ++J) {
      int Jx = J >> 2, Jy = (J >> 1) & 1, Jz = J & 1;
      int nx = cx + Jx, ny = cy + Jy, nz = cz + Jz;
      double u[3] = {l.get(uch, nx, ny, nz), l.get(uch + 1, nx, ny, nz), l.get(uch + 2, nx, ny, nz)};
      for (int v = 0; v < 3; ++v)
        for (int w = 0; w < 3; ++w) f[v] += (mu * K_mu[I][J][v][w] + la * K_la[I][J][v][w]) * u[w];
    }
  }
  for (int v = 0; v < 3; ++v) f[v] *= dx;
}

static void ku(Level& l, int uch, int fch, double dx) {
  const int nb = int(l.active.size());
#pragma omp parallel for schedule(static)
  for (int b = 0; b < nb; ++b) {
    int p = l.active[b];
    auto base = l.pool_base[p];
    Block* blk = l.pool[p].get();
    for (int e = 0; e < NPB; ++e) {
      int x = base[0] + (e >> 5), y = base[1] + ((e >> 3) & 3), z = base[2] + (e & 7);
      double f[3];
      multiply_node(l, x, y, z, uch, dx, f);
      for (int v = 0; v < 3; ++v) blk->ch[fch + v][e] = f[v];
    }
  }
}

// r = b - dx*K u (SPGrid_Linear_Elasticity.h:214-344); r may alias b.
static void residual0(Level& l, int uch, int bch, int rch, double dx) {
  const int nb = int(l.active.size());
  std::vector<double> tmp(size_t(nb) * NPB * 3);
#pragma omp parallel for schedule(static)
  for (int b = 0; b < nb; ++b) {
    int p = l.active[b];
    auto base = l.pool_base[p];
    Block* blk = l.pool[p].get();
    for (int e = 0; e < NPB; ++e) {
      int x = base[0] + (e >> 5), y = base[1] + ((e >> 3) & 3), z = base[2] + (e & 7);
      double f[3];
      multiply_node(l, x, y, z, uch, dx, f);
      for (int v = 0; v < 3; ++v) tmp[(size_t(b) * NPB + e) * 3 + v] = blk->ch[bch + v][e] - f[v];
    }
  }
  for (int b = 0; b < nb; ++b) {
    Block* blk = l.pool[l.active[b]].get();
    for (int e = 0; e < NPB; ++e)
      for (int v = 0; v < 3; ++v) blk->ch[rch + v][e] = tmp[(size_t(b) * NPB + e) * 3 + v];
  }
}

// One colour of the level-0 Gauss-Seidel smoother (SPGrid_Gauss_Seidel.h:876-1180).
static void gs_color0(Level& l, const std::vector<int>& blocks, int color, int uch, int bch, double dx,
                      bool boundary) {
  const int px = (color >> 2) & 1, py = (color >> 1) & 1, pz = color & 1;
  const int nb = int(blocks.size());
#pragma omp parallel for schedule(static)
  for (int b = 0; b < nb; ++b) {
    int p = blocks[b];
    auto base = l.pool_base[p];
    Block* blk = l.pool[p].get();
    for (int i = px; i < BX; i += 2)
      for (int j = py; j < BY; j += 2)
        for (int k = pz; k < BZ; k += 2) {
          int e = lidx(i, j, k);
          int x = base[0] + i, y = base[1] + j, z = base[2] + k;
          uint64_t fl = blk->flags[e];
          double u0[3] = {blk->ch[uch][e], blk->ch[uch + 1][e], blk->ch[uch + 2][e]};
          double u[3] = {u0[0], u0[1], u0[2]};
          bool act = (fl & ACTIVE_NODE) && (!boundary || (fl & BOUNDARY_NODE));
          if (act) {
            double f[3] = {0, 0, 0}, d[6] = {0, 0, 0, 0, 0, 0};
            for (int I = 0; I < 8; ++I) {
              int Ix = I >> 2, Iy = (I >> 1) & 1, Iz = I & 1;
              int cx = x - Ix, cy = y - Iy, cz = z - Iz;
              double mu = l.get(CH_MU, cx, cy, cz), la = l.get(CH_LA, cx, cy, cz);
              for (int J = 0; J < 8; ++J) {
                int nx = cx + (J >> 2), ny = cy + ((J >> 1) & 1), nz = cz + (J & 1);
                double un[3] = {l.get(uch, nx, ny, nz), l.get(uch + 1, nx, ny, nz),
                                l.get(uch + 2, nx, ny, nz)};
                double K[3][3];
                for (int v = 0; v < 3; ++v)
                  for (int w = 0; w < 3; ++w) K[v][w] = mu * K_mu[I][J][v][w] + la * K_la[I][J][v][w];
                for (int v = 0; v < 3; ++v) f[v] += K[v][0] * un[0] + K[v][1] * un[1] + K[v][2] * un[2];
                if (J == I) {
                  d[0] += K[0][0]; d[1] += K[1][1]; d[2] += K[2][2];
                  d[3] += K[0][1]; d[4] += K[0][2]; d[5] += K[1][2];
                }
              }
            }
            double r[3];
            for (int v = 0; v < 3; ++v) r[v] = blk->ch[bch + v][e] - f[v] * dx;
            for (int q = 0; q < 6; ++q) d[q] *= dx;
            const bool dxf = fl & DIRICHLET_NODE_X, dyf = fl & DIRICHLET_NODE_Y, dzf = fl & DIRICHLET_NODE_Z;
            if (dxf) { d[0] = 1; d[3] = 0; d[4] = 0; }
            if (dyf) { d[1] = 1; d[3] = 0; d[5] = 0; }
            if (dzf) { d[2] = 1; d[4] = 0; d[5] = 0; }
            double m11 = d[1] * d[2] - d[5] * d[5], m12 = d[5] * d[4] - d[2] * d[3],
                   m13 = d[3] * d[5] - d[4] * d[1], m22 = d[2] * d[0] - d[4] * d[4],
                   m23 = d[4] * d[3] - d[0] * d[5], m33 = d[0] * d[1] - d[3] * d[3];
            double det = d[0] * m11 + d[3] * m12 + d[4] * m13;
            double inv = 1.0 / det;
            double a[6] = {m11 * inv, m22 * inv, m33 * inv, m12 * inv, m13 * inv, m23 * inv};
            if (dxf) { a[0] = 0; a[3] = 0; a[4] = 0; }
            if (dyf) { a[1] = 0; a[3] = 0; a[5] = 0; }
            if (dzf) { a[2] = 0; a[4] = 0; a[5] = 0; }
            u[0] += r[0] * a[0] + r[1] * a[3] + r[2] * a[4];
            u[1] += r[0] * a[3] + r[1] * a[1] + r[2] * a[5];
            u[2] += r[0] * a[4] + r[1] * a[5] + r[2] * a[2];
          }
          if (fl & DIRICHLET_NODE_X) u[0] = 0;
          if (fl & DIRICHLET_NODE_Y) u[1] = 0;
          if (fl & DIRICHLET_NODE_Z) u[2] = 0;
          for (int v = 0; v < 3; ++v) blk->ch[uch + v][e] = u[v];
        }
  }
}

// ---------------------------------------------------------------------------
// Transfers (MG/Restriction.h:52-88, MG/Prolongation.h:151-193)
// ---------------------------------------------------------------------------
static void restrict_level(Level& coarse, const Level& fine, int cch, int fch) {
  const double w[3] = {0.5, 1.0, 0.5};
  const int nb = int(coarse.active.size());
#pragma omp parallel for schedule(static)
  for (int b = 0; b < nb; ++b) {
    int p = coarse.active[b];
    auto base = coarse.pool_base[p];
    Block* blk = coarse.pool[p].get();
    for (int e = 0; e < NPB; ++e) {
      int x = base[0] + (e >> 5), y = base[1] + ((e >> 3) & 3), z = base[2] + (e & 7);
      int fx = 2 * x - BX, fy = 2 * y - BY, fz = 2 * z - BZ;
      double v[3] = {0, 0, 0};
      for (int ii = 0; ii < 3; ++ii)
        for (int jj = 0; jj < 3; ++jj)
          for (int kk = 0; kk < 3; ++kk) {
            double wt = w[ii] * w[jj] * w[kk];
            for (int c = 0; c < 3; ++c) v[c] += wt * fine.get(fch + c, fx + ii - 1, fy + jj - 1, fz + kk - 1);
          }
      for (int c = 0; c < 3; ++c) blk->ch[cch + c][e] = v[c];
    }
  }
}

static void prolongate_level(Level& fine, const Level& coarse, int fch, int cch) {
  const int nb = int(fine.active.size());
#pragma omp parallel for schedule(static)
  for (int b = 0; b < nb; ++b) {
    int p = fine.active[b];
    auto base = fine.pool_base[p];
    Block* blk = fine.pool[p].get();
    for (int e = 0; e < NPB; ++e) {
      int i = e >> 5, j = (e >> 3) & 3, k = e & 7;
      int x = base[0] + i, y = base[1] + j, z = base[2] + k;
      int cx = (x + BX) >> 1, cy = (y + BY) >> 1, cz = (z + BZ) >> 1;
      double v[3] = {blk->ch[fch][e], blk->ch[fch + 1][e], blk->ch[fch + 2][e]};
      for (int ii = 0; ii < 2; ++ii) {
        double wi = (i & 1) ? 0.5 : (ii == 0 ? 1.0 : 0.0);
        for (int jj = 0; jj < 2; ++jj) {
          double wj = (j & 1) ? 0.5 : (jj == 0 ? 1.0 : 0.0);
          for (int kk = 0; kk < 2; ++kk) {
            double wk = (k & 1) ? 0.5 : (kk == 0 ? 1.0 : 0.0);
            double wt = wi * wj * wk;
            if (wt > 0)
              for (int c = 0; c < 3; ++c) v[c] += wt * coarse.get(cch + c, cx + ii, cy + jj, cz + kk);
          }
        }
      }
      for (int c = 0; c < 3; ++c) blk->ch[fch + c][e] = v[c];
    }
  }
}

// Zero Dirichlet components (CG_SYSTEM.cpp:242-255, CPU_Kernels/Project.h)
static void project(Level& l, int ch) {
  for (int v = 0; v < 3; ++v)
    for (auto& pe : l.dirichlet[v]) l.pool[pe.first]->ch[ch + v][pe.second] = 0;
}

// Zero non-active nodes (Project_Null_Space.h:223-232)
static void project_null(Level& l, int ch) {
  for (int p : l.active) {
    Block* b = l.pool[p].get();
    for (int e = 0; e < NPB; ++e)
      if (!(b->flags[e] & ACTIVE_NODE)) b->ch[ch][e] = b->ch[ch + 1][e] = b->ch[ch + 2][e] = 0;
  }
}

static void clear3(Level& l, int ch) {
  for (int p : l.active) {
    Block* b = l.pool[p].get();
    for (int v = 0; v < 3; ++v) std::memset(b->ch[ch + v], 0, sizeof(double) * NPB);
  }
}

static void cast3(Level& l, int ch) {
  for (int p : l.active) {
    Block* b = l.pool[p].get();
    for (int v = 0; v < 3; ++v)
      for (int e = 0; e < NPB; ++e) b->ch[ch + v][e] = to_float(b->ch[ch + v][e]);
  }
}

// ---------------------------------------------------------------------------
// Galerkin coarse operators
// ---------------------------------------------------------------------------
// f[v][w][n] for a cell of depth `depth` whose min-corner node is (x,y,z) on the
// level of that depth; input: scalar nodal field u[8] placed in component w.
static void galerkin_cell(const Level& l0, const double u[8], int x, int y, int z, int depth,
                          double f[3][3][8]) {
  if (depth == 0) {
    for (int v = 0; v < 3; ++v)
      for (int w = 0; w < 3; ++w)
        for (int n = 0; n < 8; ++n) f[v][w][n] = 0;
    if (!l0.test_page(x, y, z)) return;
    double mu = l0.get(CH_MU, x, y, z), la = l0.get(CH_LA, x, y, z);
    for (int node = 0; node < 8; ++node) {
      double mu_u = u[node] * mu, la_u = u[node] * la;
      for (int v = 0; v < 3; ++v)
        for (int w = 0; w < 3; ++w)
          for (int n = 0; n < 8; ++n)
            f[v][w][n] += K_mu[n][node][v][w] * mu_u + K_la[n][node][v][w] * la_u;
    }
    return;
  }
  // prolongate the cell's 8 nodal values onto its 8 children (trilinear)
  double uf[8][8];
  for (int c = 0; c < 8; ++c) {
    int cxp = c >> 2, cyp = (c >> 1) & 1, czp = c & 1;
    for (int n = 0; n < 8; ++n) {
      // fine node position in half-units of the coarse cell
      double px = 0.5 * (cxp + (n >> 2)), py = 0.5 * (cyp + ((n >> 1) & 1)), pz = 0.5 * (czp + (n & 1));
      double s = 0;
      for (int a = 0; a < 8; ++a) {
        double wx = (a >> 2) ? px : 1 - px, wy = ((a >> 1) & 1) ? py : 1 - py, wz = (a & 1) ? pz : 1 - pz;
        s += wx * wy * wz * u[a];
      }
      uf[c][n] = s;
    }
  }
  const int fx = 2 * x - BX, fy = 2 * y - BY, fz = 2 * z - BZ;
  double fc[8][3][3][8];
  for (int c = 0; c < 8; ++c) galerkin_cell(l0, uf[c], fx + (c >> 2), fy + ((c >> 1) & 1), fz + (c & 1), depth - 1, fc[c]);
  // restrict: transpose of the prolongation above
  for (int v = 0; v < 3; ++v)
    for (int w = 0; w < 3; ++w)
      for (int a = 0; a < 8; ++a) {
        double s = 0;
        for (int c = 0; c < 8; ++c) {
          int cxp = c >> 2, cyp = (c >> 1) & 1, czp = c & 1;
          for (int n = 0; n < 8; ++n) {
            double px = 0.5 * (cxp + (n >> 2)), py = 0.5 * (cyp + ((n >> 1) & 1)), pz = 0.5 * (czp + (n & 1));
            double wx = (a >> 2) ? px : 1 - px, wy = ((a >> 1) & 1) ? py : 1 - py, wz = (a & 1) ? pz : 1 - pz;
            s += wx * wy * wz * fc[c][v][w][n];
          }
        }
        f[v][w][a] = s;
      }
}

// Walk down the level maps: cell (x,y,z) of level `depth` expressed on level depth-1 is 2c-B.
static void build_stencils(Solver& s, int level) {
  Level& l = s.L[level];
  const Level& l0 = s.L[0];
  StencilLevel& st = s.S[level];
  const int nb = int(l.active.size());
  st.data.assign(size_t(nb) * NPB * 243, 0.0);
  st.flags.assign(size_t(nb) * NPB, 0u);
  st.block_of_pool.assign(l.pool.size(), -1);
  for (int b = 0; b < nb; ++b) st.block_of_pool[l.active[b]] = b;
  const double dx = s.P.dx;
#pragma omp parallel for schedule(dynamic)
  for (int b = 0; b < nb; ++b) {
    int p = l.active[b];
    auto base = l.pool_base[p];
    Block* blk = l.pool[p].get();
    for (int e = 0; e < NPB; ++e) {
      if (!(blk->flags[e] & ACTIVE_NODE)) continue;
      int x = base[0] + (e >> 5), y = base[1] + ((e >> 3) & 3), z = base[2] + (e & 7);
      double stencil[3][3][3][3][3] = {};
      uint32_t sflags = 0;
      for (int cell = 0; cell < 8; ++cell) {
        int cxp = cell >> 2, cyp = (cell >> 1) & 1, czp = cell & 1;
        double u[8] = {0, 0, 0, 0, 0, 0, 0, 0};
        u[7 - cell] = 1.0;
        double f[3][3][8];
        galerkin_cell(l0, u, x + cxp - 1, y + cyp - 1, z + czp - 1, level, f);
        for (int node = 0; node < 8; ++node) {
          int si = cxp + (node >> 2), sj = cyp + ((node >> 1) & 1), sk = czp + (node & 1);
          bool nz = false;
          for (int v = 0; v < 3; ++v)
            for (int w = 0; w < 3; ++w) {
              // stencil row: our node, comp v; column: neighbour, comp w (= f[w][v] by symmetry)
              double a = f[w][v][node];
              if (a != 0) nz = true;
              stencil[si][sj][sk][v][w] += a;
            }
          if (nz) sflags |= spoke_bit(si, sj, sk);
        }
      }
      for (int v = 0; v < 3; ++v)
        if (blk->flags[e] & (DIRICHLET_NODE_X << v)) sflags |= COORD_DIRICHLET[v];
      double* out = &st.data[(size_t(b) * NPB + e) * 243];
      const double* flat = &stencil[0][0][0][0][0];
      for (int q = 0; q < 243; ++q) out[q] = flat[q] * dx;
      st.flags[size_t(b) * NPB + e] = sflags;
    }
  }
}

static inline const double* stencil_at(const Solver& s, int level, int x, int y, int z, uint32_t* fl) {
  const Level& l = s.L[level];
  long c = l.cell_of(x, y, z);
  if (c < 0 || l.bmap[c] < 0 || size_t(l.bmap[c]) >= s.S[level].block_of_pool.size()) {
    if (fl) *fl = 0;
    return nullptr;
  }
  int ab = s.S[level].block_of_pool[l.bmap[c]];
  if (ab < 0) { if (fl) *fl = 0; return nullptr; }
  size_t idx = size_t(ab) * NPB + lidx(x & 3, y & 3, z & 7);
  if (fl) *fl = s.S[level].flags[idx];
  return &s.S[level].data[idx * 243];
}

// Delete_Dirichlet_Equations.h:24-50
static void delete_dirichlet(Solver& s, int level) {
  Level& l = s.L[level];
  StencilLevel& st = s.S[level];
  const int nb = int(l.active.size());
  for (int b = 0; b < nb; ++b) {
    auto base = l.pool_base[l.active[b]];
    for (int e = 0; e < NPB; ++e) {
      size_t idx = size_t(b) * NPB + e;
      uint32_t fl = st.flags[idx];
      double* sd = &st.data[idx * 243];
      int x = base[0] + (e >> 5), y = base[1] + ((e >> 3) & 3), z = base[2] + (e & 7);
      for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j)
          for (int k = 0; k < 3; ++k) {
            if (!(fl & spoke_bit(i, j, k))) continue;
            uint32_t nfl = 0;
            stencil_at(s, level, x + i - 1, y + j - 1, z + k - 1, &nfl);
            for (int v = 0; v < 3; ++v)
              for (int w = 0; w < 3; ++w) {
                double& a = sd[(((i * 3 + j) * 3 + k) * 3 + v) * 3 + w];
                if (fl & COORD_DIRICHLET[v]) a = (v == w && i == 1 && j == 1 && k == 1) ? 1.0 : 0.0;
                else if (nfl & COORD_DIRICHLET[w]) a = 0.0;
              }
          }
    }
  }
}

// r = A u (stencil) on every node of the active blocks (SPGrid_Stencil_Multiply.h:30-69)
static void stencil_multiply(Solver& s, int level, int uch, int rch) {
  Level& l = s.L[level];
  const int nb = int(l.active.size());
  std::vector<double> tmp(size_t(nb) * NPB * 3);
#pragma omp parallel for schedule(static)
  for (int b = 0; b < nb; ++b) {
    auto base = l.pool_base[l.active[b]];
    for (int e = 0; e < NPB; ++e) {
      int x = base[0] + (e >> 5), y = base[1] + ((e >> 3) & 3), z = base[2] + (e & 7);
      const double* sd = &s.S[level].data[(size_t(b) * NPB + e) * 243];
      double f[3] = {0, 0, 0};
      for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j)
          for (int k = 0; k < 3; ++k) {
            double u[3] = {l.get(uch, x + i - 1, y + j - 1, z + k - 1), l.get(uch + 1, x + i - 1, y + j - 1, z + k - 1),
                           l.get(uch + 2, x + i - 1, y + j - 1, z + k - 1)};
            const double* a = sd + ((i * 3 + j) * 3 + k) * 9;
            for (int v = 0; v < 3; ++v)
              for (int w = 0; w < 3; ++w) f[v] += u[w] * a[v * 3 + w];
          }
      for (int v = 0; v < 3; ++v) tmp[(size_t(b) * NPB + e) * 3 + v] = f[v];
    }
  }
  for (int b = 0; b < nb; ++b) {
    Block* blk = l.pool[l.active[b]].get();
    for (int e = 0; e < NPB; ++e)
      for (int v = 0; v < 3; ++v) blk->ch[rch + v][e] = tmp[(size_t(b) * NPB + e) * 3 + v];
  }
}

// SPGrid_Stencil_Colored_Smooth (SPGrid_Stencil_Multiply.h:161-279) + Project
static void stencil_smooth_color(Solver& s, int level, const std::vector<int>& blocks, int color, int uch,
                                 int bch, bool boundary) {
  Level& l = s.L[level];
  const int px = (color >> 2) & 1, py = (color >> 1) & 1, pz = color & 1;
  const int nb = int(blocks.size());
#pragma omp parallel for schedule(static)
  for (int b = 0; b < nb; ++b) {
    int p = blocks[b];
    auto base = l.pool_base[p];
    Block* blk = l.pool[p].get();
    for (int i = px; i < BX; i += 2)
      for (int j = py; j < BY; j += 2)
        for (int k = pz; k < BZ; k += 2) {
          int e = lidx(i, j, k);
          uint64_t fl = blk->flags[e];
          if (!(fl & ACTIVE_NODE)) continue;
          if (boundary && !(fl & BOUNDARY_NODE)) continue;
          int x = base[0] + i, y = base[1] + j, z = base[2] + k;
          const double* sd = stencil_at(s, level, x, y, z, nullptr);
          double st[243];
          if (sd) std::memcpy(st, sd, sizeof(st));
          else std::memset(st, 0, sizeof(st));
          double r[3] = {blk->ch[bch][e], blk->ch[bch + 1][e], blk->ch[bch + 2][e]};
          const double* c = st + 13 * 9;
          double d[6] = {c[0], c[4], c[8], c[1], c[2], c[5]};
          if (fl & DIRICHLET_NODE_X) { d[0] = 1; d[3] = 0; d[4] = 0; }
          if (fl & DIRICHLET_NODE_Y) { d[1] = 1; d[3] = 0; d[5] = 0; }
          if (fl & DIRICHLET_NODE_Z) { d[2] = 1; d[4] = 0; d[5] = 0; }
          double m11 = d[1] * d[2] - d[5] * d[5], m12 = d[5] * d[4] - d[2] * d[3],
                 m13 = d[3] * d[5] - d[4] * d[1], m22 = d[2] * d[0] - d[4] * d[4],
                 m23 = d[4] * d[3] - d[0] * d[5], m33 = d[0] * d[1] - d[3] * d[3];
          double det = d[0] * m11 + d[3] * m12 + d[4] * m13;
          double inv = 1.0 / det;
          double a[6] = {m11 * inv, m22 * inv, m33 * inv, m12 * inv, m13 * inv, m23 * inv};
          if (fl & DIRICHLET_NODE_X) { a[0] = 0; a[3] = 0; a[4] = 0; }
          if (fl & DIRICHLET_NODE_Y) { a[1] = 0; a[3] = 0; a[5] = 0; }
          if (fl & DIRICHLET_NODE_Z) { a[2] = 0; a[4] = 0; a[5] = 0; }
          for (int ii = 0; ii < 3; ++ii)
            for (int jj = 0; jj < 3; ++jj)
              for (int kk = 0; kk < 3; ++kk) {
                double u[3] = {l.get(uch, x + ii - 1, y + jj - 1, z + kk - 1),
                               l.get(uch + 1, x + ii - 1, y + jj - 1, z + kk - 1),
                               l.get(uch + 2, x + ii - 1, y + jj - 1, z + kk - 1)};
                const double* m = st + ((ii * 3 + jj) * 3 + kk) * 9;
                for (int v = 0; v < 3; ++v)
                  for (int w = 0; w < 3; ++w) r[v] -= u[w] * m[v * 3 + w];
              }
          double dl[3];
          dl[0] = a[0] * r[0] + a[3] * r[1] + a[4] * r[2];
          dl[1] = a[3] * r[0] + a[1] * r[1] + a[5] * r[2];
          dl[2] = a[4] * r[0] + a[5] * r[1] + a[2] * r[2];
          for (int v = 0; v < 3; ++v) blk->ch[uch + v][e] += dl[v];
        }
  }
}

// ---------------------------------------------------------------------------
// Setup
// ---------------------------------------------------------------------------
static void flag_nodes(Level& l) {
  // Flag_Nodes (Flaging.h:65-80): serial, OR the cell's flags (>>4) into its 8 corners
  for (int p : l.active) {
    auto base = l.pool_base[p];
    for (int e = 0; e < NPB; ++e) {
      uint64_t nf = (l.pool[p]->flags[e] & (ACTIVE_CELL | DIRICHLET_CELL)) >> 4;
      int x = base[0] + (e >> 5), y = base[1] + ((e >> 3) & 3), z = base[2] + (e & 7);
      for (int c = 0; c < 8; ++c) l.flag_ref(x + (c >> 2), y + ((c >> 1) & 1), z + (c & 1)) |= nf;
    }
  }
}

static void flag_boundary(Level& l, int band = 3) {
  for (int pass = 0; pass < band; ++pass) {
    for (int p : l.active) {
      auto base = l.pool_base[p];
      for (int e = 0; e < NPB; ++e) {
        uint64_t& f = l.pool[p]->flags[e];
        if (f & DIRICHLET_NODE) continue;
        if (!(f & ACTIVE_NODE)) continue;
        int x = base[0] + (e >> 5), y = base[1] + ((e >> 3) & 3), z = base[2] + (e & 7);
        bool hit = false;
        for (int i = -1; i <= 1 && !hit; ++i)
          for (int j = -1; j <= 1 && !hit; ++j)
            for (int k = -1; k <= 1 && !hit; ++k)
              if (l.getf(x + i, y + j, z + k) & (DIRICHLET_NODE | BOUNDARY_NODE)) hit = true;
        if (hit) f |= BOUNDARY_NODE_TEMP;
      }
    }
    for (int p : l.active)
      for (int e = 0; e < NPB; ++e) {
        uint64_t& f = l.pool[p]->flags[e];
        if (f & BOUNDARY_NODE_TEMP) { f -= BOUNDARY_NODE_TEMP; f |= BOUNDARY_NODE; }
      }
  }
  l.boundary.clear();
  for (int p : l.active)
    for (int e = 0; e < NPB; ++e)
      if (l.pool[p]->flags[e] & BOUNDARY_NODE) { l.boundary.push_back(p); break; }
}

static void dirichlet_lists(Level& l) {
  for (int v = 0; v < 3; ++v) l.dirichlet[v].clear();
  for (int p : l.active)
    for (int e = 0; e < NPB; ++e)
      for (int v = 0; v < 3; ++v)
        if (l.pool[p]->flags[e] & (DIRICHLET_NODE_X << v)) l.dirichlet[v].push_back({p, e});
}

static bool setup(Solver& s, int nblocks, const int32_t* base, const double* density) {
  build_tables();
  const Params& P = s.P;
  if (P.mg_level == 2) ORC_FAIL(s, 3, "mg_level = 2 is not supported");
  // mg_level 0 disables the preconditioner (SPGrid_CPU_Solver.cpp:217-235)
  s.disable_mg = P.mg_level <= 0;
  int nlev = P.mg_level < 1 ? 1 : P.mg_level;
  s.L.resize(nlev);
  s.S.resize(nlev);
  s.L[0].init(P.resolution[0], P.resolution[1], P.resolution[2]);
  Level& l0 = s.L[0];
  // page activation + SIMP map (SPGrid_CPU_Solver.cpp:102-136)
  for (int b = 0; b < nblocks; ++b) {
    int bx = base[3 * b], by = base[3 * b + 1], bz = base[3 * b + 2];
    s.in_base.push_back({bx, by, bz});
    if (bx < 0 || by < 0 || bz < 0 || l0.cell_of(bx, by, bz) < 0) ORC_FAIL(s, 4, "block base outside the grid");
    l0.set_page(bx, by, bz);
    for (int e = 0; e < 64; ++e) {
      int ii = e >> 4, jj = (e >> 2) & 3, kk = e & 3;
      double d = density[size_t(b) * 64 + e];
      if (d > 0) {
        double E = P.penalty ? (1 - P.minimum_stiffness) * std::pow(std::max(P.minimum_density, d), P.penalty) +
                                   P.minimum_stiffness
                             : d;
        l0.ref(CH_MU, bx + ii, by + jj, bz + kk) = E * P.global_mu;
        l0.ref(CH_LA, bx + ii, by + jj, bz + kk) = E * P.global_lambda;
      }
    }
  }
  l0.update_blocks();
  // Validate_With_Density (Validate_Blocks.h:311-335)
  for (int p : l0.active) {
    auto bb = l0.pool_base[p];
    for (int e = 0; e < NPB; ++e) {
      if (!(l0.pool[p]->ch[CH_MU][e] > 0)) continue;
      int x = bb[0] + (e >> 5), y = bb[1] + ((e >> 3) & 3), z = bb[2] + (e & 7);
      for (int c = 1; c < 8; ++c)
        if (!l0.test_page(x + (c >> 2), y + ((c >> 1) & 1), z + (c & 1)))
          ORC_FAIL(s, 5, "block activation check failed at (%d,%d,%d)", x, y, z);
    }
  }
  // Dirichlet node -> cell rule (SPGrid_CPU_Solver.cpp:169-192)
  for (int v = 0; v < 3; ++v) {
    std::unordered_set<uint64_t> set;
    auto key = [](int x, int y, int z) { return (uint64_t(uint32_t(x)) << 42) | (uint64_t(uint32_t(y)) << 21) | uint32_t(z); };
    for (size_t i = 0; i < s.d_coord.size(); ++i)
      if (s.d_axis[i] == v) set.insert(key(s.d_coord[i][0], s.d_coord[i][1], s.d_coord[i][2]));
    for (size_t i = 0; i < s.d_coord.size(); ++i) {
      if (s.d_axis[i] != v) continue;
      auto c = s.d_coord[i];
      bool all = true;
      for (int n = 1; n < 8 && all; ++n)
        all = set.count(key(c[0] + (n >> 2), c[1] + ((n >> 1) & 1), c[2] + (n & 1))) > 0;
      if (all) {
        // Flaging with Dirichlet cells (Flaging.h:45-52)
        if (l0.cell_of(c[0], c[1], c[2]) >= 0) l0.flag_ref(c[0], c[1], c[2]) |= (DIRICHLET_CELL_X << v);
      }
    }
  }
  // ACTIVE_CELL from mu != 0 (Flaging.h:31-44)
  for (int p : l0.active)
    for (int e = 0; e < NPB; ++e)
      if (l0.pool[p]->ch[CH_MU][e] != 0) l0.pool[p]->flags[e] |= ACTIVE_CELL;
  // coarse levels (Multigrid_Hierarchy.h:122-144, 158-195)
  for (int lev = 1; lev < nlev; ++lev) {
    int sz[3];
    const int pad[3] = {2 * BX, 2 * BY, 2 * BZ};
    for (int v = 0; v < 3; ++v) {
      int fine = s.L[lev - 1].size[v] + 1 - pad[v];
      sz[v] = pad[v] + fine / 2 + (fine % 2 ? 1 : 0);
    }
    s.L[lev].init(sz[0], sz[1], sz[2]);
    Level& f = s.L[lev - 1];
    Level& c = s.L[lev];
    for (int p : f.active) {
      auto bb = f.pool_base[p];
      for (int e = 0; e < NPB; ++e) {
        uint64_t ff = f.pool[p]->flags[e];
        int x = bb[0] + (e >> 5), y = bb[1] + ((e >> 3) & 3), z = bb[2] + (e & 7);
        int cx = (x + BX) >> 1, cy = (y + BY) >> 1, cz = (z + BZ) >> 1;
        if (ff & ACTIVE_CELL) {
          c.flag_ref(cx, cy, cz) |= ACTIVE_CELL;
          for (int n = 0; n < 8; ++n) c.set_page(cx + (n >> 2), cy + ((n >> 1) & 1), cz + (n & 1));
        }
        for (int v = 0; v < 3; ++v)
          if (ff & (DIRICHLET_CELL_X << v)) {
            c.flag_ref(cx, cy, cz) |= (DIRICHLET_CELL_X << v);
            for (int n = 1; n < 8; ++n) c.set_page(cx + (n >> 2), cy + ((n >> 1) & 1), cz + (n & 1));
          }
      }
    }
    c.update_blocks();
  }
  for (int lev = 0; lev < nlev; ++lev) flag_nodes(s.L[lev]);
  for (int lev = 0; lev < nlev; ++lev) flag_boundary(s.L[lev]);
  for (int lev = 0; lev < nlev; ++lev) dirichlet_lists(s.L[lev]);
  // Check_Padding (Multigrid_Hierarchy.h:145-157)
  for (int p : l0.active) {
    auto bb = l0.pool_base[p];
    const int bs[3] = {BX, BY, BZ};
    for (int v = 0; v < 3; ++v)
      if (bb[v] < bs[v] || bb[v] >= l0.size[v] - 2 * bs[v]) ORC_FAIL(s, 6, "padding violated at block (%d,%d,%d)", bb[0], bb[1], bb[2]);
  }
  // Galerkin operators (Multigrid_Hierarchy.h:215-226)
  int first = (nlev == 1) ? 0 : P.explicit_level;
  if (s.disable_mg) return true;
  for (int lev = first; lev < nlev; ++lev) {
    build_stencils(s, lev);
    delete_dirichlet(s, lev);
  }
  // bottom factorization: DOFs = nodes with any active spoke (Elasticity_Matrix.cpp:39-96)
  {
    int lev = nlev - 1;
    Level& l = s.L[lev];
    StencilLevel& st = s.S[lev];
    s.bottom_nodes.clear();
    int mn[3] = {1 << 30, 1 << 30, 1 << 30}, mx[3] = {-1, -1, -1};
    for (size_t b = 0; b < l.active.size(); ++b)
      for (int e = 0; e < NPB; ++e)
        if (st.flags[b * NPB + e] & 0x07ffffffu) {
          s.bottom_nodes.push_back({l.active[b], e});
          auto bb = l.pool_base[l.active[b]];
          int c[3] = {bb[0] + (e >> 5), bb[1] + ((e >> 3) & 3), bb[2] + (e & 7)};
          for (int v = 0; v < 3; ++v) { mn[v] = std::min(mn[v], c[v]); mx[v] = std::max(mx[v], c[v]); }
        }
    long nn = long(s.bottom_nodes.size());
    if (nn > 0) {
      // lexicographic order with the largest extent slowest
      int ext[3] = {mx[0] - mn[0] + 1, mx[1] - mn[1] + 1, mx[2] - mn[2] + 1};
      int ax[3] = {0, 1, 2};
      std::sort(ax, ax + 3, [&](int a, int b) { return ext[a] > ext[b]; });
      std::vector<std::pair<long, long>> order(nn);
      for (long i = 0; i < nn; ++i) {
        auto& pe = s.bottom_nodes[i];
        auto bb = l.pool_base[pe.first];
        int c[3] = {bb[0] + (pe.second >> 5) - mn[0], bb[1] + ((pe.second >> 3) & 3) - mn[1], bb[2] + (pe.second & 7) - mn[2]};
        long key = (long(c[ax[0]]) * ext[ax[1]] + c[ax[1]]) * ext[ax[2]] + c[ax[2]];
        order[i] = {key, i};
      }
      std::sort(order.begin(), order.end());
      std::vector<long> pos_of(nn);
      for (long i = 0; i < nn; ++i) pos_of[order[i].second] = i;
      // node lookup by coordinate for the band assembly
      long bw_nodes = 0;
      std::vector<long> key_of(nn);
      for (long i = 0; i < nn; ++i) key_of[order[i].second] = order[i].first;
      // bandwidth in nodes: max |pos difference| among coupled nodes
      auto find_node = [&](int x, int y, int z) -> long {
        long c = l.cell_of(x, y, z);
        if (c < 0 || l.bmap[c] < 0) return -1;
        int ab = st.block_of_pool[l.bmap[c]];
        if (ab < 0) return -1;
        return long(ab) * NPB + lidx(x & 3, y & 3, z & 7);
      };
      std::vector<long> node_dof(l.active.size() * NPB, -1);
      for (long i = 0; i < nn; ++i) {
        auto& pe = s.bottom_nodes[i];
        node_dof[size_t(st.block_of_pool[pe.first]) * NPB + pe.second] = pos_of[i];
      }
      for (long i = 0; i < nn; ++i) {
        auto& pe = s.bottom_nodes[i];
        auto bb = l.pool_base[pe.first];
        int x = bb[0] + (pe.second >> 5), y = bb[1] + ((pe.second >> 3) & 3), z = bb[2] + (pe.second & 7);
        uint32_t fl = st.flags[size_t(st.block_of_pool[pe.first]) * NPB + pe.second];
        for (int q = 0; q < 27; ++q)
          if (fl & spoke_bit(q / 9, (q / 3) % 3, q % 3)) {
            long nd = find_node(x + q / 9 - 1, y + (q / 3) % 3 - 1, z + q % 3 - 1);
            if (nd >= 0 && node_dof[nd] >= 0) bw_nodes = std::max(bw_nodes, std::labs(node_dof[nd] - pos_of[i]));
          }
      }
      BandCholesky& C = s.chol;
      C.n = 3 * nn;
      C.bw = 3 * bw_nodes + 2;
      C.L.assign(size_t(C.n) * (C.bw + 1), 0.0);
      for (long i = 0; i < nn; ++i) {
        auto& pe = s.bottom_nodes[i];
        auto bb = l.pool_base[pe.first];
        int x = bb[0] + (pe.second >> 5), y = bb[1] + ((pe.second >> 3) & 3), z = bb[2] + (pe.second & 7);
        size_t idx = size_t(st.block_of_pool[pe.first]) * NPB + pe.second;
        uint32_t fl = st.flags[idx];
        const double* sd = &st.data[idx * 243];
        long row0 = 3 * pos_of[i];
        for (int q = 0; q < 27; ++q) {
          if (!(fl & spoke_bit(q / 9, (q / 3) % 3, q % 3))) continue;
          long nd = find_node(x + q / 9 - 1, y + (q / 3) % 3 - 1, z + q % 3 - 1);
          if (nd < 0 || node_dof[nd] < 0) continue;
          uint32_t nfl = st.flags[nd];
          long col0 = 3 * node_dof[nd];
          for (int v = 0; v < 3; ++v)
            for (int w = 0; w < 3; ++w) {
              long r = row0 + v, cidx = col0 + w;
              if (cidx > r) continue;  // lower triangle
              double a = sd[q * 9 + v * 3 + w];
              if ((fl & COORD_DIRICHLET[v]) || (nfl & COORD_DIRICHLET[w])) a = (r == cidx) ? 1.0 : 0.0;
              C.at(r, cidx) = a;
            }
        }
      }
      s.bottom_perm.assign(nn, 0);
      for (long i = 0; i < nn; ++i) s.bottom_perm[i] = pos_of[i];
      if (!C.factor()) ORC_FAIL(s, 7, "bottom operator is not positive definite");
    }
  }
  return true;
}

// Exact_Solve (Multigrid_Hierarchy.h:346-372): nodes without DOFs take b
static void bottom_solve(Solver& s, int uch, int bch) {
  int lev = int(s.L.size()) - 1;
  Level& l = s.L[lev];
  for (int p : l.active) {
    Block* b = l.pool[p].get();
    for (int v = 0; v < 3; ++v) std::memcpy(b->ch[uch + v], b->ch[bch + v], sizeof(double) * NPB);
  }
  long nn = long(s.bottom_nodes.size());
  if (nn == 0) return;
  std::vector<double> x(3 * nn);
  for (long i = 0; i < nn; ++i) {
    auto& pe = s.bottom_nodes[i];
    for (int v = 0; v < 3; ++v) x[3 * s.bottom_perm[i] + v] = l.pool[pe.first]->ch[bch + v][pe.second];
  }
  s.chol.solve(x);
  for (long i = 0; i < nn; ++i) {
    auto& pe = s.bottom_nodes[i];
    for (int v = 0; v < 3; ++v) l.pool[pe.first]->ch[uch + v][pe.second] = x[3 * s.bottom_perm[i] + v];
  }
}

static void smooth_level(Solver& s, int level, int uch, int bch, bool forward, bool boundary) {
  Level& l = s.L[level];
  const std::vector<int>& blocks = boundary ? l.boundary : l.active;
  if (level == 0) {
    for (int q = 0; q < 8; ++q) gs_color0(l, blocks, forward ? q : 7 - q, uch, bch, s.P.dx, boundary);
    return;
  }
  static const int order[2][8] = {{1, 5, 4, 6, 7, 3, 2, 0}, {0, 2, 3, 7, 6, 4, 5, 1}};
  const int* c = forward ? order[0] : order[1];
  for (int q = 0; q < 8; ++q) {
    stencil_smooth_color(s, level, blocks, c[q], uch, bch, boundary);
    project(l, uch);
  }
}

// Run_VCycle (Multigrid_Hierarchy.h:569-619); u = ch9-11, b = ch3-5, r = ch6-8
static void vcycle(Solver& s) {
  const int U = CH_Q0, B = CH_F0, R = CH_S0;
  const int n = int(s.L.size());
  const bool ref = s.P.mode == MODE_REF;
  const int ns = s.P.smoothing_iter, nbs = s.P.boundary_smoothing, ex = s.P.explicit_level;
  auto sweeps = [&](int level, bool fwd) {
    for (int t = 0; t < nbs; ++t) { smooth_level(s, level, U, B, fwd, true); if (ref) cast3(s.L[level], U); }
    for (int t = 0; t < ns; ++t) { smooth_level(s, level, U, B, fwd, false); if (ref) cast3(s.L[level], U); }
    for (int t = 0; t < nbs; ++t) { smooth_level(s, level, U, B, fwd, true); if (ref) cast3(s.L[level], U); }
  };
  for (int level = 0; level < n - 1; ++level) {
    bool smooth = level == 0 || level >= ex;
    if (smooth) sweeps(level, true);
    clear3(s.L[level + 1], U);
    clear3(s.L[level + 1], B);
    if (smooth) {
      if (level == 0) residual0(s.L[0], U, B, R, s.P.dx);
      else {
        stencil_multiply(s, level, U, R);
        Level& l = s.L[level];
        for (int p : l.active)
          for (int v = 0; v < 3; ++v)
            for (int e = 0; e < NPB; ++e) l.pool[p]->ch[R + v][e] = l.pool[p]->ch[B + v][e] - l.pool[p]->ch[R + v][e];
        project(l, R);
      }
      if (ref) cast3(s.L[level], R);
      restrict_level(s.L[level + 1], s.L[level], B, R);
    } else {
      restrict_level(s.L[level + 1], s.L[level], B, B);
    }
    project(s.L[level + 1], B);
  }
  bottom_solve(s, U, B);
  if (ref) cast3(s.L[n - 1], U);
  for (int level = n - 2; level >= 0; --level) {
    prolongate_level(s.L[level], s.L[level + 1], U, U);
    project(s.L[level], U);
    if (ref) cast3(s.L[level], U);
    project_null(s.L[level], U);
    if (level == 0 || level >= ex) sweeps(level, false);
  }
}

// ---------------------------------------------------------------------------
// PCG (CONJUGATE_GRADIENT.cpp:21-61) on level-0 channel triples
// ---------------------------------------------------------------------------
static double dot3(Level& l, int a, int b) {
  double s = 0;
  for (int v = 0; v < 3; ++v) {
    double part = 0;
    const int nb = int(l.active.size());
#pragma omp parallel for reduction(+ : part) schedule(static)
    for (int q = 0; q < nb; ++q) {
      Block* blk = l.pool[l.active[q]].get();
      for (int e = 0; e < NPB; ++e) part += blk->ch[a + v][e] * blk->ch[b + v][e];
    }
    s += part;
  }
  return s;
}

static double linf3(Level& l, int a) {
  double m = 0;
  for (int p : l.active) {
    Block* blk = l.pool[p].get();
    for (int v = 0; v < 3; ++v)
      for (int e = 0; e < NPB; ++e) m = std::max(m, std::fabs(blk->ch[a + v][e]));
  }
  return m;
}

// dst = c*x + y with the reference's optional float rounding (CG_VECTOR.cpp:96-114)
static void axpy3(Level& l, int dst, double c, int x, int y, bool fl) {
  for (int p : l.active) {
    Block* b = l.pool[p].get();
    for (int v = 0; v < 3; ++v)
      for (int e = 0; e < NPB; ++e) {
        if (fl) {
          float t = float(c) * float(b->ch[x + v][e]) + float(b->ch[y + v][e]);
          b->ch[dst + v][e] = t;
        } else {
          b->ch[dst + v][e] = c * b->ch[x + v][e] + b->ch[y + v][e];
        }
      }
  }
}

static void precondition(Solver& s, int r, int z) {
  Level& l0 = s.L[0];
  if (s.disable_mg) {  // z = r (CG_SYSTEM.cpp:319-320)
    for (int p : l0.active)
      for (int v = 0; v < 3; ++v) std::memcpy(l0.pool[p]->ch[z + v], l0.pool[p]->ch[r + v], sizeof(double) * NPB);
    project(l0, z);
    project_null(l0, z);
    return;
  }
  // Apply_Preconditioner (CG_SYSTEM.cpp:218-257): the V-cycle works on r (b), z (u), ch6-8 (scratch)
  std::vector<double> sbk(l0.active.size() * NPB * 3);
  for (size_t q = 0; q < l0.active.size(); ++q)
    for (int v = 0; v < 3; ++v)
      std::memcpy(&sbk[(q * 3 + v) * NPB], l0.pool[l0.active[q]]->ch[CH_S0 + v], sizeof(double) * NPB);
  clear3(l0, z);
  if (r != CH_F0) return;  // the V-cycle reads its right-hand side from ch3-5
  vcycle(s);
  for (size_t q = 0; q < l0.active.size(); ++q)
    for (int v = 0; v < 3; ++v)
      std::memcpy(l0.pool[l0.active[q]]->ch[CH_S0 + v], &sbk[(q * 3 + v) * NPB], sizeof(double) * NPB);
  // Precondition(): Project(z); Project_Nullspace(z)
  project(l0, z);
  project_null(l0, z);
}

static bool solve(Solver& s) {
  Level& l0 = s.L[0];
  const double dx = s.P.dx;
  const bool fl = s.P.mode == MODE_REF;
  const int U = CH_U0, F = CH_F0, S = CH_S0, Q = CH_Q0;
  // u = g on every listed Dirichlet node, zero elsewhere (SPGrid_CPU_Solver.cpp:241-285)
  clear3(l0, U);
  for (size_t i = 0; i < s.d_coord.size(); ++i) {
    auto c = s.d_coord[i];
    if (l0.cell_of(c[0], c[1], c[2]) >= 0) l0.ref(U + s.d_axis[i], c[0], c[1], c[2]) = s.d_val[i];
  }
  // s = forces; Project; Project_Nullspace; f = s - K u; Project (SPGrid_CPU_Solver.cpp:287-301)
  clear3(l0, S);
  for (size_t i = 0; i < s.f_coord.size(); ++i) {
    auto c = s.f_coord[i];
    if (l0.cell_of(c[0], c[1], c[2]) < 0) continue;
    for (int v = 0; v < 3; ++v) l0.ref(S + v, c[0], c[1], c[2]) = s.f_val[i][v];
  }
  project(l0, S);
  project_null(l0, S);
  residual0(l0, U, S, F, dx);
  project(l0, F);
  project(l0, F);
  // backup u (the Dirichlet lift) and solve for the correction
  std::vector<double> ubk(l0.active.size() * NPB * 3);
  for (size_t q = 0; q < l0.active.size(); ++q)
    for (int v = 0; v < 3; ++v) std::memcpy(&ubk[(q * 3 + v) * NPB], l0.pool[l0.active[q]]->ch[U + v], sizeof(double) * NPB);
  clear3(l0, Q);
  clear3(l0, S);
  s.initial_residual = linf3(l0, F);
  const double tol = s.P.tolerance * s.initial_residual;
  clear3(l0, U);
  // CONJUGATE_GRADIENT_4Ch::Solve
  project(l0, U);
  ku(l0, U, Q, dx);
  // r -= q (CG_VECTOR operator-=, float-rounded in REF mode)
  for (int p : l0.active) {
    Block* b = l0.pool[p].get();
    for (int v = 0; v < 3; ++v)
      for (int e = 0; e < NPB; ++e) {
        if (fl) { float t = float(b->ch[F + v][e]) - float(b->ch[Q + v][e]); b->ch[F + v][e] = t; }
        else b->ch[F + v][e] -= b->ch[Q + v][e];
      }
  }
  project(l0, F);
  double rho_old = FLT_MAX;
  const double small = std::numeric_limits<double>::epsilon();
  int it;
  double norm = 0;
  s.history.clear();
  for (it = 0;; ++it) {
    project_null(l0, F);
    norm = linf3(l0, F);
    s.history.push_back(norm);
    if (norm <= tol && (it >= 0 || norm < small)) break;
    if (it == s.P.max_iterations) break;
    precondition(s, F, Q);  // z aliases q (SPGrid_CPU_Solver.cpp:91-92)
    double rho = dot3(l0, Q, F);
    axpy3(l0, S, rho / rho_old, S, Q, fl);
    ku(l0, S, Q, dx);
    project(l0, Q);
    double sq = dot3(l0, S, Q);
    if (sq <= 0) {
      s.iterations = it;
      s.final_residual = norm;
      s.status = 8;
      std::snprintf(s.err, sizeof(s.err), "CG detected an indefinite or singular operator");
      return false;
    }
    double alpha = rho / sq;
    axpy3(l0, U, alpha, S, U, fl);
    axpy3(l0, F, -alpha, Q, F, fl);
    rho_old = rho;
  }
  s.iterations = it;
  s.final_residual = norm;
  for (size_t q = 0; q < l0.active.size(); ++q)
    for (int v = 0; v < 3; ++v)
      for (int e = 0; e < NPB; ++e) l0.pool[l0.active[q]]->ch[U + v][e] += ubk[(q * 3 + v) * NPB + e];
  return true;
}

}  // namespace orc

// ===========================================================================
// C ABI for the Python test harness
// ===========================================================================
using namespace orc;

extern "C" {

struct OracleParams {
  int32_t resolution[3];
  int32_t mg_level;
  double dx, global_mu, global_lambda, penalty, minimum_stiffness, minimum_density, tolerance;
  int32_t smoothing_iter, boundary_smoothing, max_iterations, mode;
  int32_t explicit_level, num_threads;
};

void* oracle_create(const OracleParams* p, int nblocks, const int32_t* base, const double* density, int nforces,
                    const int32_t* fcoord, const double* fval, int ndir, const int32_t* dcoord, const int32_t* daxis,
                    const double* dval, int* status, char* err, int errlen) {
#ifdef _OPENMP
  if (p->num_threads > 0) omp_set_num_threads(p->num_threads);
#endif
  Solver* s = new Solver();
  s->P.resolution[0] = p->resolution[0];
  s->P.resolution[1] = p->resolution[1];
  s->P.resolution[2] = p->resolution[2];
  s->P.dx = p->dx;
  s->P.global_mu = p->global_mu;
  s->P.global_lambda = p->global_lambda;
  s->P.penalty = p->penalty;
  s->P.minimum_stiffness = p->minimum_stiffness;
  s->P.minimum_density = p->minimum_density;
  s->P.mg_level = p->mg_level;
  s->P.smoothing_iter = p->smoothing_iter;
  s->P.boundary_smoothing = p->boundary_smoothing;
  s->P.max_iterations = p->max_iterations;
  s->P.mode = p->mode;
  s->P.explicit_level = p->explicit_level;
  s->P.tolerance = p->tolerance;
  for (int i = 0; i < nforces; ++i) {
    s->f_coord.push_back({fcoord[3 * i], fcoord[3 * i + 1], fcoord[3 * i + 2]});
    s->f_val.push_back({fval[3 * i], fval[3 * i + 1], fval[3 * i + 2]});
  }
  for (int i = 0; i < ndir; ++i) {
    s->d_coord.push_back({dcoord[3 * i], dcoord[3 * i + 1], dcoord[3 * i + 2]});
    s->d_axis.push_back(daxis[i]);
    s->d_val.push_back(dval[i]);
  }
  bool ok = setup(*s, nblocks, base, density);
  *status = ok ? 0 : s->status;
  if (!ok && err && errlen > 0) std::snprintf(err, errlen, "%s", s->err);
  return s;
}

void oracle_destroy(void* h) { delete static_cast<Solver*>(h); }

int oracle_levels(void* h) { return int(static_cast<Solver*>(h)->L.size()); }

// Active blocks of a level in page order; returns count, fills base coords when non-null.
int oracle_level_blocks(void* h, int level, int32_t* coords) {
  Level& l = static_cast<Solver*>(h)->L[level];
  if (coords)
    for (size_t b = 0; b < l.active.size(); ++b)
      for (int v = 0; v < 3; ++v) coords[3 * b + v] = l.pool_base[l.active[b]][v];
  return int(l.active.size());
}

int oracle_level_size(void* h, int level, int32_t* size) {
  Level& l = static_cast<Solver*>(h)->L[level];
  for (int v = 0; v < 3; ++v) size[v] = l.size[v];
  return 0;
}

int oracle_boundary_blocks(void* h, int level, int32_t* ordinals) {
  Level& l = static_cast<Solver*>(h)->L[level];
  std::vector<int> ord(l.pool.size(), -1);
  for (size_t b = 0; b < l.active.size(); ++b) ord[l.active[b]] = int(b);
  if (ordinals)
    for (size_t i = 0; i < l.boundary.size(); ++i) ordinals[i] = ord[l.boundary[i]];
  return int(l.boundary.size());
}

void oracle_get_flags(void* h, int level, uint32_t* out) {
  Level& l = static_cast<Solver*>(h)->L[level];
  for (size_t b = 0; b < l.active.size(); ++b)
    for (int e = 0; e < NPB; ++e) out[b * NPB + e] = uint32_t(l.pool[l.active[b]]->flags[e]);
}

// channel triple <-> compact arrays [3][nb*128]
static void put3(Level& l, int ch, const double* in) {
  size_t n = l.active.size() * NPB;
  for (size_t b = 0; b < l.active.size(); ++b)
    for (int v = 0; v < 3; ++v) std::memcpy(l.pool[l.active[b]]->ch[ch + v], in + v * n + b * NPB, sizeof(double) * NPB);
}
static void get3(Level& l, int ch, double* out) {
  size_t n = l.active.size() * NPB;
  for (size_t b = 0; b < l.active.size(); ++b)
    for (int v = 0; v < 3; ++v) std::memcpy(out + v * n + b * NPB, l.pool[l.active[b]]->ch[ch + v], sizeof(double) * NPB);
}

void oracle_get_material(void* h, double* mu, double* la) {
  Level& l = static_cast<Solver*>(h)->L[0];
  for (size_t b = 0; b < l.active.size(); ++b) {
    std::memcpy(mu + b * NPB, l.pool[l.active[b]]->ch[CH_MU], sizeof(double) * NPB);
    std::memcpy(la + b * NPB, l.pool[l.active[b]]->ch[CH_LA], sizeof(double) * NPB);
  }
}

// Unit operators on compact arrays; see the op codes below.
//  0: level-0 K*u            in=u            out=dx*K u
//  1: level-0 residual       in=u, in2=b     out=b - dx*K u
//  2: smoothing sweep        in=u, in2=b     out=u after one sweep; arg bit0 forward, bit1 boundary
//  3: restriction            in=fine (level) out=coarse (level+1), then Dirichlet projection
//  4: prolongation           in=coarse(level+1), in2=fine(level) out=fine + P coarse, then the
//                            Dirichlet projection, the float cast (REF) and the null-space projection
//  5: stencil multiply       in=u (level)    out=A u with Dirichlet components zeroed
//  6: bottom solve           in=b (last level) out=u
//  7: V-cycle                in=r (level 0)  out=z (projected), scratch restored
int oracle_apply(void* h, int op, int level, int arg, const double* in, const double* in2, double* out) {
  Solver& s = *static_cast<Solver*>(h);
  if (level < 0 || level >= int(s.L.size())) return -1;
  Level& l = s.L[level];
  const int A = CH_Q0, B = CH_F0, C = CH_S0;
  switch (op) {
    case 0: put3(l, A, in); ku(l, A, C, s.P.dx); get3(l, C, out); return 0;
    case 1: put3(l, A, in); put3(l, B, in2); residual0(l, A, B, C, s.P.dx); get3(l, C, out); return 0;
    case 2: put3(l, A, in); put3(l, B, in2); smooth_level(s, level, A, B, arg & 1, (arg >> 1) & 1); get3(l, A, out); return 0;
    case 3:
      if (level + 1 >= int(s.L.size())) return -1;
      put3(l, C, in); restrict_level(s.L[level + 1], l, B, C); project(s.L[level + 1], B); get3(s.L[level + 1], B, out);
      return 0;
    case 4:
      if (level + 1 >= int(s.L.size())) return -1;
      put3(s.L[level + 1], A, in); put3(l, C, in2); prolongate_level(l, s.L[level + 1], C, A); project(l, C);
      if (s.P.mode == MODE_REF) cast3(l, C);
      project_null(l, C);
      get3(l, C, out);
      return 0;
    case 5: put3(l, A, in); stencil_multiply(s, level, A, C); project(l, C); get3(l, C, out); return 0;
    case 6: put3(l, B, in); bottom_solve(s, A, B); get3(l, A, out); return 0;
    case 7: put3(l, B, in); precondition(s, B, A); get3(l, A, out); return 0;
  }
  return -2;
}

// Galerkin stencils of a level: out[nb*128*243], flags[nb*128]
int oracle_get_stencils(void* h, int level, double* out, uint32_t* flags) {
  Solver& s = *static_cast<Solver*>(h);
  if (s.S[level].data.empty()) return -1;
  std::memcpy(out, s.S[level].data.data(), s.S[level].data.size() * sizeof(double));
  if (flags) std::memcpy(flags, s.S[level].flags.data(), s.S[level].flags.size() * sizeof(uint32_t));
  return 0;
}

// Full solve. disp: [nblocks_in][64][4] in input block order (SPGrid_CPU_Solver.cpp:343-364);
// stats: [iterations, initial L-inf residual, final L-inf residual]; history of L-inf norms.
int oracle_solve(void* h, double* disp, double* stats, double* history, int hist_cap, char* err, int errlen) {
  Solver& s = *static_cast<Solver*>(h);
  bool ok = solve(s);
  stats[0] = s.iterations;
  stats[1] = s.initial_residual;
  stats[2] = s.final_residual;
  for (int i = 0; i < hist_cap && i < int(s.history.size()); ++i) history[i] = s.history[i];
  if (!ok) {
    if (err && errlen > 0) std::snprintf(err, errlen, "%s", s.err);
    return s.status;
  }
  Level& l0 = s.L[0];
  for (size_t b = 0; b < s.in_base.size(); ++b) {
    auto bb = s.in_base[b];
    for (int e = 0; e < 64; ++e) {
      int x = bb[0] + (e >> 4), y = bb[1] + ((e >> 2) & 3), z = bb[2] + (e & 3);
      double* o = disp + (b * 64 + e) * 4;
      double r = 0;
      for (int v = 0; v < 3; ++v) {
        o[v] = l0.get(CH_U0 + v, x, y, z);
        r = std::max(r, std::fabs(l0.get(CH_F0 + v, x, y, z)));
      }
      o[3] = r;
    }
  }
  return 0;
}

// Stiffness tables: out_mu/out_la [8][8][3][3]
void oracle_tables(double* out_mu, double* out_la) {
  build_tables();
  std::memcpy(out_mu, K_mu, sizeof(K_mu));
  std::memcpy(out_la, K_la, sizeof(K_la));
}

// Morton page keys of block coordinates (block units)
void oracle_page_keys(int n, const int32_t* bijk, uint64_t* keys) {
  for (int i = 0; i < n; ++i) keys[i] = page_key(bijk[3 * i], bijk[3 * i + 1], bijk[3 * i + 2]);
}

// SIMP sensitivity (minimal_compliance.cpp:86-146): for every cell with density > 0
// of the input blocks, sum = u_e^T K0 u_e with K0 = mu0*K_mu + lambda0*K_la (no dx);
// dc = sum * p * rho^(p-1) * (1 - Emin); objective += sum * (Emin + rho^p (1 - Emin)).
// u: [nblocks][64][3] nodal displacement for each input block's nodes plus the +1 layer
// is read through the level-0 grid after a solve, so this must follow oracle_solve.
double oracle_sensitivity(void* h, const double* density, double* dc_out, double* sum_out) {
  Solver& s = *static_cast<Solver*>(h);
  build_tables();
  Level& l0 = s.L[0];
  const double p = s.P.penalty, emin = s.P.minimum_stiffness;
  double objective = 0;
  for (size_t b = 0; b < s.in_base.size(); ++b) {
    auto bb = s.in_base[b];
    for (int e = 0; e < 64; ++e) {
      double rho = density[b * 64 + e];
      double sum = 0;
      if (rho > 0) {
        int x = bb[0] + (e >> 4), y = bb[1] + ((e >> 2) & 3), z = bb[2] + (e & 3);
        double u[8][3];
        for (int a = 0; a < 8; ++a)
          for (int v = 0; v < 3; ++v) u[a][v] = l0.get(CH_U0 + v, x + (a >> 2), y + ((a >> 1) & 1), z + (a & 1));
        for (int a = 0; a < 8; ++a)
          for (int bn = 0; bn < 8; ++bn)
            for (int i = 0; i < 3; ++i)
              for (int j = 0; j < 3; ++j)
                sum += u[a][i] * (K_mu[a][bn][i][j] * s.P.global_mu + K_la[a][bn][i][j] * s.P.global_lambda) * u[bn][j];
        objective += sum * (emin + std::pow(rho, p) * (1 - emin));
        dc_out[b * 64 + e] = sum * std::pow(rho, p - 1.0) * p * (1 - emin);
      } else {
        dc_out[b * 64 + e] = 0;
      }
      if (sum_out) sum_out[b * 64 + e] = sum;
    }
  }
  return objective;
}

}  // extern "C"
