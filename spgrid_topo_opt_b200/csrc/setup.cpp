// Host-side hierarchy construction; see setup.hpp.
//
// Follows the reference's set-up sequence: page activation and the SIMP map
// (solver/SPGrid_CPU_Solver.cpp:100-145), the Dirichlet node->cell rule (:147-192),
// cell/node flags and the boundary band (solver/CPU_Kernels/Flaging.h:31-173),
// the coarse levels (solver/MG/Multigrid_Hierarchy.h:122-214) and the padding
// check (:145-157).
#include "setup.hpp"

#include <chrono>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <memory>
#include <parallel/algorithm>
#include <unordered_set>

#include <omp.h>

namespace sgs {

uint64_t page_key(int bi, int bj, int bk) {
  uint64_t key = 0;
  for (int m = 0; m < 21; ++m) {
    key |= uint64_t((bj >> m) & 1) << (3 * m);
    key |= uint64_t((bi >> m) & 1) << (3 * m + 1);
    key |= uint64_t((bk >> m) & 1) << (3 * m + 2);
  }
  return key;
}

static inline int node_slot(int x, int y, int z) { return (x & 3) * 32 + (y & 3) * 8 + (z & 7); }

long HostLevel::cell(int x, int y, int z) const {
  if (x < 0 || y < 0 || z < 0) return -1;
  int bi = x >> 2, bj = y >> 2, bk = z >> 3;
  if (bi >= grid[0] || bj >= grid[1] || bk >= grid[2]) return -1;
  return (long(bi) * grid[1] + bj) * grid[2] + bk;
}

int HostLevel::block_at(int x, int y, int z) const {
  long c = cell(x, y, z);
  return c < 0 ? -1 : bgrid[c];
}

int HostLevel::active_block_at(int x, int y, int z) const {
  int b = block_at(x, y, z);
  return (b >= 0 && b < nb) ? b : -1;
}

int HostLevel::touch(int x, int y, int z, bool with_flags) {
  long c = cell(x, y, z);
  if (c < 0) return -1;
  int b = bgrid[c];
  if (b < 0) {
    b = int(coords.size() / 3);
    bgrid[c] = b;
    coords.push_back(x & ~3);
    coords.push_back(y & ~3);
    coords.push_back(z & ~7);
    if (with_flags) flags.resize(flags.size() + NODES_PER_BLOCK, 0u);
  }
  return b;
}

namespace {

// A level under construction.  Its blocks are numbered as the reference's
// page order has them: the active blocks (pages) in page-key order first, then
// the ghost blocks (touched, not pages) in the order they were created; see
// number_blocks.  Blocks touched after numbering are ghosts and are appended.
struct Builder {
  HostLevel L;

  void init(int sx, int sy, int sz) {
    L.size[0] = sx; L.size[1] = sy; L.size[2] = sz;
    L.grid[0] = sx / BLK_X + 3; L.grid[1] = sy / BLK_Y + 3; L.grid[2] = sz / BLK_Z + 3;
    const long ncell = long(L.grid[0]) * L.grid[1] * L.grid[2];
    L.bgrid.resize(size_t(ncell));  // uninitialised: filled below, in parallel
    L.active_page.resize(size_t(ncell));
    int32_t* g = L.bgrid.data();
    uint8_t* a = L.active_page.data();
#pragma omp parallel for schedule(static)
    for (long c = 0; c < ncell; ++c) {
      g[c] = -1;
      a[c] = 0;
    }
  }
  bool test_page(int x, int y, int z) const {
    long c = L.cell(x, y, z);
    return c >= 0 && L.active_page[c];
  }
  uint32_t* flag(int x, int y, int z) {
    int b = L.touch(x, y, z);
    return b < 0 ? nullptr : &L.flags[size_t(b) * NODES_PER_BLOCK + node_slot(x, y, z)];
  }
};

// The cells c of a block grid of ncell cells with key_of(c) != NONE, as (key,
// cell) pairs sorted by key; the grid is scanned in one chunk per thread
// (counted, then gathered) and the pairs sorted in parallel.
constexpr uint64_t NONE = ~uint64_t(0);
template <typename KeyOf>
std::vector<std::pair<uint64_t, long>> sorted_cells(long ncell, const KeyOf& key_of) {
  const int nt = std::max(1, omp_get_max_threads());
  const long chunk = (ncell + nt - 1) / nt;
  std::vector<long> start(size_t(nt) + 1, 0);
#pragma omp parallel for schedule(static, 1) num_threads(nt)
  for (int t = 0; t < nt; ++t) {
    long n = 0;
    for (long c = long(t) * chunk; c < std::min(ncell, long(t + 1) * chunk); ++c) n += key_of(c) != NONE;
    start[size_t(t) + 1] = n;
  }
  for (int t = 0; t < nt; ++t) start[size_t(t) + 1] += start[size_t(t)];
  std::vector<std::pair<uint64_t, long>> out(static_cast<size_t>(start[size_t(nt)]));
#pragma omp parallel for schedule(static, 1) num_threads(nt)
  for (int t = 0; t < nt; ++t) {
    long k = start[size_t(t)];
    for (long c = long(t) * chunk; c < std::min(ncell, long(t + 1) * chunk); ++c) {
      const uint64_t key = key_of(c);
      if (key != NONE) out[size_t(k++)] = {key, c};
    }
  }
  __gnu_parallel::sort(out.begin(), out.end());
  return out;
}

// Numbers the blocks of a level under construction: the active blocks (cells
// `act`, in page-key order) first, the ghost blocks (`ghost`, in creation
// order) after; coordinates set, flags zeroed.
void number_blocks(HostLevel& L, const std::vector<std::pair<uint64_t, long>>& act,
                   const std::vector<std::pair<uint64_t, long>>& ghost) {
  const long na = long(act.size()), nall = na + long(ghost.size());
  const long g12 = long(L.grid[1]) * L.grid[2];
  L.coords.resize(3 * size_t(nall));
#pragma omp parallel for schedule(static)
  for (long i = 0; i < nall; ++i) {
    const long c = i < na ? act[size_t(i)].second : ghost[size_t(i - na)].second;
    L.bgrid[size_t(c)] = int32_t(i);
    L.coords[3 * size_t(i)] = int(c / g12) * BLK_X;
    L.coords[3 * size_t(i) + 1] = int((c / L.grid[2]) % L.grid[1]) * BLK_Y;
    L.coords[3 * size_t(i) + 2] = int(c % L.grid[2]) * BLK_Z;
  }
  L.nb = int(na);
  L.flags.resize(size_t(nall) * NODES_PER_BLOCK);  // uninitialised
  uint32_t* f = L.flags.data();
#pragma omp parallel for schedule(static)
  for (long i = 0; i < nall * NODES_PER_BLOCK; ++i) f[i] = 0u;
}

// the page key of a block-grid cell
uint64_t cell_key(const HostLevel& L, long c) {
  const long g12 = long(L.grid[1]) * L.grid[2];
  return page_key(int(c / g12), int((c / L.grid[2]) % L.grid[1]), int(c % L.grid[2]));
}

// The 27 blocks (active or ghost) around block b, -1 where there is none;
// entry (dx+1)*9 + (dy+1)*3 + (dz+1).
static void block_ring(const HostLevel& L, int b, int ring[27]) {
  const int bx = L.coords[3 * b], by = L.coords[3 * b + 1], bz = L.coords[3 * b + 2];
  for (int d = 0; d < 27; ++d)
    ring[d] = L.block_at(bx + (d / 9 - 1) * BLK_X, by + ((d / 3) % 3 - 1) * BLK_Y, bz + (d % 3 - 1) * BLK_Z);
}

void flag_nodes(HostLevel& L) {
  // Flaging.h:65-80 — each active block's cells OR (flags >> 4) into their 8
  // corner nodes; nodes in untouched pages get ghost blocks.  The OR is order
  // free, so it runs as a gather: first the ghost blocks that some cell of an
  // active block reaches are created (serially), then every node ORs the bits
  // of its 8 incident cells in active blocks (in parallel).
  const uint32_t CELL = F_ACTIVE_CELL | F_DIRICHLET_CELL;
  // bit (dx*4+dy*2+dz) of corner_reach[e]: the corners of cell e reach the block at +(dx, dy, dz)
  uint8_t corner_reach[NODES_PER_BLOCK];
  for (int e = 0; e < NODES_PER_BLOCK; ++e) {
    const int kx = (e >> 5) == 3, ky = ((e >> 3) & 3) == 3, kz = (e & 7) == 7;
    unsigned m = 0;
    for (int c = 1; c < 8; ++c)
      if ((!(c & 4) || kx) && (!(c & 2) || ky) && (!(c & 1) || kz)) m |= 1u << c;
    corner_reach[e] = uint8_t(m);
  }
  std::vector<uint8_t> reach(size_t(L.nb), 0);  // per block: the OR over its cells with a CELL bit
#pragma omp parallel for schedule(static)
  for (int b = 0; b < L.nb; ++b) {
    const uint32_t* f = L.flags.data() + size_t(b) * NODES_PER_BLOCK;
    unsigned m = 0;
    for (int e = 0; e < NODES_PER_BLOCK; ++e) m |= (f[e] & CELL) ? corner_reach[e] : 0u;
    reach[size_t(b)] = uint8_t(m);
  }
  for (int b = 0; b < L.nb; ++b)
    for (int c = 1; c < 8; ++c)
      if (reach[size_t(b)] >> c & 1)
        L.touch(L.coords[3 * b] + (c >> 2) * BLK_X, L.coords[3 * b + 1] + ((c >> 1) & 1) * BLK_Y,
                L.coords[3 * b + 2] + (c & 1) * BLK_Z);
  // The node bits are ORed into the flags in place: other threads read only the
  // cell bits of a word, which these writes leave as they are (relaxed atomic
  // loads and stores, one writer per word).
  const int nall = int(L.coords.size() / 3);
  uint32_t* flags = L.flags.data();
  auto cell_bits = [&](size_t i) { return __atomic_load_n(&flags[i], __ATOMIC_RELAXED); };
#pragma omp parallel for schedule(static)
  for (int b = 0; b < nall; ++b) {
    // the blocks at offsets -(c>>2, (c>>1)&1, c&1) that hold a node's cells; only
    // cells of active blocks spread their flags
    int src[8];
    const int bx = L.coords[3 * b], by = L.coords[3 * b + 1], bz = L.coords[3 * b + 2];
    for (int c = 0; c < 8; ++c) {
      const int nb = c ? L.block_at(bx - (c >> 2) * BLK_X, by - ((c >> 1) & 1) * BLK_Y, bz - (c & 1) * BLK_Z) : b;
      src[c] = (nb >= 0 && nb < L.nb) ? nb : -1;
    }
    // the cell bits of cells x-1..3, y-1..3, z-1..7 (index +1), then ORed along
    // z, y and x in place: entry (x+1, y+1, z+1) ends as the OR of the 8 cells
    // of node (x, y, z)
    // z-column (ax, ay): entry 0 from the -z block's z = 7, entries 1-8 from z = 0-7
    uint32_t A[5][5][9];
    for (int ax = 0; ax < 5; ++ax)
      for (int ay = 0; ay < 5; ++ay) {
        const int s = (ax == 0 ? 4 : 0) | (ay == 0 ? 2 : 0);
        const size_t col = size_t(((ax + 3) & 3) * 32 + ((ay + 3) & 3) * 8);
        const int below = src[s | 1], own = src[s];
        A[ax][ay][0] = below >= 0 ? cell_bits(size_t(below) * NODES_PER_BLOCK + col + 7) & CELL : 0u;
        for (int z = 0; z < 8; ++z)
          A[ax][ay][z + 1] = own >= 0 ? cell_bits(size_t(own) * NODES_PER_BLOCK + col + size_t(z)) & CELL : 0u;
      }
    for (int ax = 0; ax < 5; ++ax)
      for (int ay = 0; ay < 5; ++ay)
        for (int az = 8; az > 0; --az) A[ax][ay][az] |= A[ax][ay][az - 1];
    for (int ax = 0; ax < 5; ++ax)
      for (int ay = 4; ay > 0; --ay)
        for (int az = 1; az < 9; ++az) A[ax][ay][az] |= A[ax][ay - 1][az];
    for (int ax = 4; ax > 0; --ax)
      for (int ay = 1; ay < 5; ++ay)
        for (int az = 1; az < 9; ++az) A[ax][ay][az] |= A[ax - 1][ay][az];
    const size_t out = size_t(b) * NODES_PER_BLOCK;
    for (int e = 0; e < NODES_PER_BLOCK; ++e) {
      const uint32_t add = A[(e >> 5) + 1][((e >> 3) & 3) + 1][(e & 7) + 1] >> 4;
      if (add) __atomic_store_n(&flags[out + size_t(e)], cell_bits(out + size_t(e)) | add, __ATOMIC_RELAXED);
    }
  }
}

void flag_boundary(HostLevel& L, int band = 3) {
  // Flaging.h:93-147: three Jacobi-style passes growing a band of active,
  // non-Dirichlet nodes around the Dirichlet nodes.  A pass can only reach
  // blocks next to a block that already holds a Dirichlet or band node, so
  // each pass visits those blocks alone: the neighbours of the seeded blocks
  // (the neighbour relation is symmetric), whose 27-block rings are looked up
  // when they first become candidates.
  const uint32_t SEED = F_DIRICHLET_NODE | F_BOUNDARY_NODE;
  const int nall = int(L.coords.size() / 3);
  HostBuf<std::array<int, 27>> rings(static_cast<size_t>(L.nb));  // entries filled on first use
  std::vector<uint8_t> have_ring(static_cast<size_t>(L.nb), 0), banded(static_cast<size_t>(L.nb), 0);
  std::vector<uint8_t> seeded(static_cast<size_t>(nall), 0), is_cand(static_cast<size_t>(L.nb), 0);
  auto flag_at = [&](const int* ring, int x, int y, int z) -> uint32_t {
    const int nb = ring[(x < 0 ? 0 : (x > 3 ? 2 : 1)) * 9 + (y < 0 ? 0 : (y > 3 ? 2 : 1)) * 3 + (z < 0 ? 0 : (z > 7 ? 2 : 1))];
    return nb < 0 ? 0u : L.flags[size_t(nb) * NODES_PER_BLOCK + node_slot(x, y, z)];
  };
  // blocks holding a Dirichlet or band node (ghost blocks included)
#pragma omp parallel for schedule(static)
  for (int b = 0; b < nall; ++b) {
    uint8_t s = 0;
    for (int e = 0; e < NODES_PER_BLOCK && !s; ++e) s = (L.flags[size_t(b) * NODES_PER_BLOCK + e] & SEED) != 0;
    seeded[size_t(b)] = s;
  }
  std::vector<int> seeds, cand;
  for (int b = 0; b < nall; ++b)
    if (seeded[size_t(b)]) seeds.push_back(b);
  for (int pass = 0; pass < band; ++pass) {
    // candidates: the active blocks among the seeded blocks' 27 neighbours, ascending
    std::fill(is_cand.begin(), is_cand.end(), uint8_t(0));
#pragma omp parallel for schedule(static)
    for (long k = 0; k < long(seeds.size()); ++k) {
      int ring[27];
      block_ring(L, seeds[size_t(k)], ring);
      for (int d = 0; d < 27; ++d)
        if (ring[d] >= 0 && ring[d] < L.nb) __atomic_store_n(&is_cand[size_t(ring[d])], uint8_t(1), __ATOMIC_RELAXED);
    }
    cand.clear();
    for (int b = 0; b < L.nb; ++b)
      if (is_cand[size_t(b)]) cand.push_back(b);
#pragma omp parallel for schedule(dynamic, 16)
    for (long k = 0; k < long(cand.size()); ++k) {
      const int b = cand[size_t(k)];
      if (!have_ring[size_t(b)]) {
        block_ring(L, b, rings[size_t(b)].data());
        have_ring[size_t(b)] = 1;
      }
      const int* ring = rings[size_t(b)].data();
      for (int e = 0; e < NODES_PER_BLOCK; ++e) {
        uint32_t& f = L.flags[size_t(b) * NODES_PER_BLOCK + e];
        if ((f & F_DIRICHLET_NODE) || !(f & F_ACTIVE_NODE)) continue;
        const int x = e >> 5, y = (e >> 3) & 3, z = e & 7;
        bool hit = false;
        for (int d = 0; d < 27 && !hit; ++d) hit = flag_at(ring, x + d / 9 - 1, y + (d / 3) % 3 - 1, z + d % 3 - 1) & SEED;
        if (hit) f |= F_BOUNDARY_TEMP;
      }
    }
#pragma omp parallel for schedule(static)
    for (long k = 0; k < long(cand.size()); ++k)
      for (int e = 0; e < NODES_PER_BLOCK; ++e) {
        uint32_t& f = L.flags[size_t(cand[size_t(k)]) * NODES_PER_BLOCK + e];
        if (f & F_BOUNDARY_TEMP) {
          f = (f & ~F_BOUNDARY_TEMP) | F_BOUNDARY_NODE;
          banded[size_t(cand[size_t(k)])] = 1;
        }
      }
    for (int b : cand)  // the blocks that gained band nodes seed the next pass
      if (banded[size_t(b)] && !seeded[size_t(b)]) {
        seeded[size_t(b)] = 1;
        seeds.push_back(b);
      }
  }
  // the blocks with a boundary-band node: only candidates gain them
  L.boundary.clear();
  for (int b = 0; b < L.nb; ++b)
    if (banded[size_t(b)]) L.boundary.push_back(b);
}

void finish_level(HostLevel& L) {
  // Dirichlet node lists in ascending node order: per-block counts, a prefix
  // over the blocks, then a parallel fill of the few blocks that hold one
  std::vector<int32_t> cnt(size_t(L.nb) * 3, 0);
  const uint32_t DIR = F_DIRICHLET_NODE_X | (F_DIRICHLET_NODE_X << 1) | (F_DIRICHLET_NODE_X << 2);
#pragma omp parallel for schedule(static)
  for (int b = 0; b < L.nb; ++b) {
    const uint32_t* f = L.flags.data() + size_t(b) * NODES_PER_BLOCK;
    uint32_t any = 0;
    for (int e = 0; e < NODES_PER_BLOCK; ++e) any |= f[e];
    if (!(any & DIR)) continue;
    for (int e = 0; e < NODES_PER_BLOCK; ++e)
      for (int v = 0; v < 3; ++v) cnt[size_t(b) * 3 + v] += (f[e] & (F_DIRICHLET_NODE_X << v)) ? 1 : 0;
  }
  std::vector<int> holders;
  for (int b = 0; b < L.nb; ++b)
    if (cnt[size_t(b) * 3] | cnt[size_t(b) * 3 + 1] | cnt[size_t(b) * 3 + 2]) holders.push_back(b);
  for (int v = 0; v < 3; ++v) {
    int32_t total = 0;
    for (int b : holders) {
      const int32_t c = cnt[size_t(b) * 3 + v];
      cnt[size_t(b) * 3 + v] = total;
      total += c;
    }
    L.dirichlet[v].assign(size_t(total), 0);
  }
#pragma omp parallel for schedule(static)
  for (long k = 0; k < long(holders.size()); ++k) {
    const int b = holders[size_t(k)];
    for (int e = 0; e < NODES_PER_BLOCK; ++e) {
      const uint32_t f = L.flags[size_t(b) * NODES_PER_BLOCK + e];
      for (int v = 0; v < 3; ++v)
        if (f & (F_DIRICHLET_NODE_X << v)) L.dirichlet[v][size_t(cnt[size_t(b) * 3 + v]++)] = b * NODES_PER_BLOCK + e;
    }
  }
}

}  // namespace

std::string build_problem(const FEMInputs& in, Problem& P, int* error_code) {
  char msg[256];
  auto fail = [&](int code, const char* m) {
    *error_code = code;
    return std::string(m);
  };
  *error_code = 0;
  if (!in.use_density_only) return fail(2, "Unsupported mode: only use_density_only=true inputs are accepted");
  if (in.mg_level == 2) return fail(3, "mg_level = 2 is not supported (the caller bumps it to 3)");
  for (int v = 0; v < 3; ++v)
    if (in.resolution[v] <= 0 || in.resolution[v] > (1 << 20)) return fail(4, "resolution out of range");
  P.resolution[0] = in.resolution[0]; P.resolution[1] = in.resolution[1]; P.resolution[2] = in.resolution[2];
  P.dx = in.dx;
  P.mu0 = in.global_mu;
  P.lambda0 = in.global_lambda;
  P.disable_mg = in.mg_level <= 0;
  P.mg_levels = in.mg_level <= 0 ? 1 : in.mg_level;
  P.dense_bottom_max = in.get_int("sgs_dense_bottom_max", 24576);
  P.smoothing = in.pre_and_post_smoothing_iter;
  P.boundary_smoothing = in.get_int("boundary_smoothing", 5);
  P.inner_smoothing = std::max(1, in.get_int("sgs_inner_smoothing", P.inner_smoothing));
  P.inner_boundary_smoothing = std::max(0, in.get_int("sgs_inner_boundary_smoothing", P.inner_boundary_smoothing));
  P.tolerance = in.krylov.tolerance;
  const double penalty = in.get_double("penalty", 0.0), emin = in.get_double("minimum_stiffness", 0.0),
               rho_min = in.get_double("minimum_density", 0.0);
  P.penalty = penalty;
  P.minimum_stiffness = emin;
  P.minimum_density = rho_min;

  using hclk = std::chrono::steady_clock;
  auto tmark = hclk::now();
  auto phase_done = [&](int k) {
    const auto t = hclk::now();
    P.host_phase[k] = std::chrono::duration<double>(t - tmark).count();
    tmark = t;
  };
  // ---- level 0: page activation and stiffness (SPGrid_CPU_Solver.cpp:102-136)
  Builder b0;
  b0.init(in.resolution[0], in.resolution[1], in.resolution[2]);
  const size_t nin = in.density.num_blocks();
  // Each 4x4x4 input block fills one z half of a 4x4x8 solver block.  The
  // solver blocks are the distinct pages of the input blocks, numbered in page
  // order: the pages are marked in the block grid, listed, sorted by page key
  // and numbered, in parallel.  Blocks touched later (ghosts) follow them in
  // creation order.  The per-cell work then
  // runs per input block in parallel, which writes disjoint slots unless an
  // input block is repeated: then the cells go in input order, the last write
  // winning.
  std::vector<int32_t> in_slot(nin);
  std::vector<uint8_t> halves;  // per block: bit h set when an input block fills its z half h
  bool repeated = false;
  {
    HostLevel& L = b0.L;
    std::vector<long> cell_of(nin);
    std::vector<uint8_t> bad(nin);
#pragma omp parallel for schedule(static)
    for (long b = 0; b < long(nin); ++b) {
      const int x = in.density.base[3 * b], y = in.density.base[3 * b + 1], z = in.density.base[3 * b + 2];
      const bool aligned = !((x & 3) || (y & 3) || (z & 3));
      cell_of[size_t(b)] = aligned ? L.cell(x, y, z) : -1;
      bad[size_t(b)] = !aligned ? 1 : (cell_of[size_t(b)] < 0 ? 2 : 0);
    }
    for (size_t b = 0; b < nin; ++b)  // the first failure in input order
      if (bad[b]) return fail(4, bad[b] == 1 ? "density block base is not a multiple of 4" : "density block outside the grid");
    uint8_t* page = L.active_page.data();
#pragma omp parallel for schedule(static)
    for (long b = 0; b < long(nin); ++b) __atomic_store_n(&page[cell_of[size_t(b)]], uint8_t(1), __ATOMIC_RELAXED);
    const auto pages = sorted_cells(long(L.active_page.size()), [&](long c) { return page[c] ? cell_key(L, c) : NONE; });
    number_blocks(L, pages, {});
    const int nb = L.nb;
    halves.assign(size_t(nb), 0);
    int rep = 0;
#pragma omp parallel for schedule(static) reduction(| : rep)
    for (long b = 0; b < long(nin); ++b) {
      const int z = in.density.base[3 * b + 2];
      const int bk = L.bgrid[size_t(cell_of[size_t(b)])];
      in_slot[size_t(b)] = bk * NODES_PER_BLOCK + node_slot(in.density.base[3 * b], in.density.base[3 * b + 1], z);
      const uint8_t h = uint8_t(1u << ((z >> 2) & 1));
      rep |= (__atomic_fetch_or(&halves[size_t(bk)], h, __ATOMIC_RELAXED) & h) ? 1 : 0;
    }
    repeated = rep != 0;
  }
  // The SIMP map of every input cell, once (fem_interface.h:343-353).  It goes
  // straight to the cell's slot of the level-0 stiffness scales P.E (zero where
  // there is no material), where every input cell has a slot of its own; when
  // input blocks repeat, the values are kept per input cell first and the last
  // input block's win in P.E below.
  // input cell e = i*16 + j*4 + k sits at slot offset i*32 + j*8 + k from the block's slot
  auto cell_slot = [](int e) { return (e >> 4) * 32 + ((e >> 2) & 3) * 8 + (e & 3); };
  auto simp = [&](double d) {
    return d > 0 ? (penalty ? (1 - emin) * std::pow(std::max(rho_min, d), penalty) + emin : d) : 0.0;
  };
  // A material cell's corners leave its page only across a +face of the page,
  // so an input block needs at most the 7 pages beyond its +faces.  Bit n of
  // face_need[zl][e] is set when input cell e reaches the page at offset
  // (n>>2, (n>>1)&1, n&1); zl = 1 for an input block in the upper z half of its page.
  uint8_t face_need[2][64];
  for (int zl = 0; zl < 2; ++zl)
    for (int e = 0; e < 64; ++e) {
      const int ex = (e >> 4) == 3, ey = ((e >> 2) & 3) == 3, ez = zl && (e & 3) == 3;
      unsigned m = 0;
      for (int n = 1; n < 8; ++n)
        if ((!(n & 4) || ex) && (!(n & 2) || ey) && (!(n & 1) || ez)) m |= 1u << n;
      face_need[zl][e] = uint8_t(m);
    }
  P.E.resize(size_t(b0.L.nb) * NODES_PER_BLOCK);
  {
    // without repeated input blocks every z half that an input block covers is
    // written in full below: only the other halves are cleared here
    double* E = P.E.data();
#pragma omp parallel for schedule(static)
    for (long b = 0; b < long(b0.L.nb); ++b)
      for (int h = 0; h < 2; ++h)
        if (repeated || !((halves[size_t(b)] >> h) & 1))
          for (int xy = 0; xy < 16; ++xy)
            for (int k = 0; k < 4; ++k) E[size_t(b) * NODES_PER_BLOCK + size_t(xy * 8 + 4 * h + k)] = 0.0;
  }
  std::unique_ptr<double[]> Ein;
  std::vector<uint8_t> need(nin, 0);  // per input block: the +face pages its material cells need
  if (repeated) {
    Ein.reset(new double[nin * 64]);
#pragma omp parallel for schedule(static)
    for (long c = 0; c < long(nin) * 64; ++c) Ein[size_t(c)] = simp(in.density.data[size_t(c)]);
#pragma omp parallel for schedule(static)
    for (long b = 0; b < long(nin); ++b) {
      const int zl = (in.density.base[3 * b + 2] & 4) != 0;
      unsigned m = 0;
      for (int e = 0; e < 64; ++e)
        if (Ein[size_t(b) * 64 + size_t(e)] * P.mu0 > 0) m |= face_need[zl][e];
      need[size_t(b)] = uint8_t(m);
    }
  } else {
    // one pass over the input cells: the stiffness scale, the pages the
    // material needs, and ACTIVE_CELL where the density is positive and
    // mu != 0 (Flaging.h:31-44), written before renumbering (a failed
    // validation below discards the level)
    double* E = P.E.data();
    uint32_t* flags = b0.L.flags.data();
#pragma omp parallel for schedule(static)
    for (long b = 0; b < long(nin); ++b) {
      const size_t base = size_t(in_slot[size_t(b)]);
      const int zl = (in.density.base[3 * b + 2] & 4) != 0;
      unsigned m = 0;
      for (int e = 0; e < 64; ++e) {
        const double d = in.density.data[size_t(b) * 64 + size_t(e)];
        const double Ev = simp(d);
        const size_t slot = base + size_t(cell_slot(e));
        E[slot] = Ev;
        if (Ev * P.mu0 > 0) m |= face_need[zl][e];
        if (d > 0 && Ev * P.mu0 != 0) flags[slot] |= F_ACTIVE_CELL;
      }
      need[size_t(b)] = uint8_t(m);
    }
  }
  auto cell_E = [&](size_t b, int e) {
    return repeated ? Ein[b * 64 + size_t(e)] : P.E[size_t(in_slot[b]) + size_t(cell_slot(e))];
  };
  // Validate_With_Density (solver/CPU_Kernels/Validate_Blocks.h:311-335): every
  // material cell needs its +1 neighbour pages; the first failure in input order
  // is reported.  The pages an input block needs are tested once, and only a
  // block that misses one is searched cell by cell.
  long first_bad = -1;
  {
    std::vector<long> bad(nin, -1);
#pragma omp parallel for schedule(static)
    for (long b = 0; b < long(nin); ++b) {
      const int x = in.density.base[3 * b], y = in.density.base[3 * b + 1], z = in.density.base[3 * b + 2];
      const unsigned nb_need = need[size_t(b)];
      bool ok = true;
      for (int n = 1; n < 8 && ok; ++n)
        if (nb_need >> n & 1) ok = b0.test_page(x + (n >> 2) * 4, y + ((n >> 1) & 1) * 4, z + (n & 1) * 4);
      if (ok) continue;
      for (int e = 0; e < 64 && bad[size_t(b)] < 0; ++e) {
        if (!(cell_E(size_t(b), e) * P.mu0 > 0)) continue;
        const int cx = x + (e >> 4), cy = y + ((e >> 2) & 3), cz = z + (e & 3);
        for (int n = 1; n < 8; ++n)
          if (!b0.test_page(cx + (n >> 2), cy + ((n >> 1) & 1), cz + (n & 1))) {
            bad[size_t(b)] = long(b) * 64 + e;
            break;
          }
      }
    }
    for (size_t b = 0; b < nin && first_bad < 0; ++b) first_bad = bad[b];
  }
  if (first_bad >= 0) {
    const size_t b = size_t(first_bad / 64);
    const int e = int(first_bad % 64);
    std::snprintf(msg, sizeof msg, "Block activation check failed at cell (%d, %d, %d)", in.density.base[3 * b] + (e >> 4),
                  in.density.base[3 * b + 1] + ((e >> 2) & 3), in.density.base[3 * b + 2] + (e & 3));
    return fail(5, msg);
  }
  // ACTIVE_CELL with repeated input blocks: serially, since copies of a block share slots
  if (repeated)
    for (size_t b = 0; b < nin; ++b)
      for (int e = 0; e < 64; ++e)
        if (in.density.data[b * 64 + size_t(e)] > 0 && cell_E(b, e) * P.mu0 != 0)
          b0.L.flags[size_t(in_slot[b] + cell_slot(e))] |= F_ACTIVE_CELL;
  // Dirichlet node -> cell: a cell is fixed on axis v when all 8 corners are
  // listed on axis v (SPGrid_CPU_Solver.cpp:169-192)
  for (int v = 0; v < 3; ++v) {
    std::unordered_set<uint64_t> set;
    auto key = [](int x, int y, int z) {
      return (uint64_t(uint32_t(x) & 0x1fffff) << 42) | (uint64_t(uint32_t(y) & 0x1fffff) << 21) | (uint32_t(z) & 0x1fffff);
    };
    for (auto& d : in.dirichlet_nodes)
      if (d.axis == v) set.insert(key(d.coord[0], d.coord[1], d.coord[2]));
    for (auto& d : in.dirichlet_nodes) {
      if (d.axis != v) continue;
      bool all = true;
      for (int n = 1; n < 8 && all; ++n)
        all = set.count(key(d.coord[0] + (n >> 2), d.coord[1] + ((n >> 1) & 1), d.coord[2] + (n & 1))) > 0;
      if (all) {
        uint32_t* f = b0.flag(d.coord[0], d.coord[1], d.coord[2]);
        if (f) *f |= (F_DIRICHLET_CELL_X << v);
      }
    }
  }
  for (auto& d : in.dirichlet_nodes)
    if (d.axis < 0 || d.axis > 2) return fail(4, "Dirichlet axis out of range");
  P.levels.clear();
  P.levels.push_back(std::move(b0.L));
  // repeated input blocks: the last one's material wins, as a serial pass
  // over the input blocks leaves it
  if (repeated)
    for (size_t b = 0; b < nin; ++b) {
      const size_t base = size_t(in_slot[b]);
      for (int e = 0; e < 64; ++e)
        if (in.density.data[b * 64 + e] > 0) P.E[base + size_t(cell_slot(e))] = Ein[b * 64 + size_t(e)];
    }

  phase_done(0);
  // ---- coarse levels (Multigrid_Hierarchy.h:122-195)
  const int pad[3] = {2 * BLK_X, 2 * BLK_Y, 2 * BLK_Z};
  auto coarsen = [&](const HostLevel& F) {
    int sz[3];
    for (int v = 0; v < 3; ++v) {
      int fine = F.size[v] + 1 - pad[v];
      sz[v] = pad[v] + fine / 2 + (fine % 2 ? 1 : 0);
    }
    Builder bc;
    bc.init(sz[0], sz[1], sz[2]);
    // The cells of a fine block map into one coarse block: a 2x2x4 patch at
    // ((bx+4)/2, (by+4)/2, (bz+8)/2).  Per fine block (in parallel) the OR of the
    // cell flags landing on each patch cell and the set of coarse pages the
    // cells' corners cx + n reach: a +1 offset leaves the patch's page only on
    // an axis where the cell is on the page's last layer (bit dx*4 + dy*2 + dz of
    // the page offset); n = 0 is excluded for Dirichlet cells.  The blocks are
    // then created and marked in fine-block order, as a serial pass over the
    // cells would.
    struct Patch {
      uint32_t flags[16];
      uint8_t pages;
      bool any;
    };
    // Whether a cell's coarse image lies on its page's last layer depends on the
    // cell's slot e and on the parity of the fine block's coordinates (x/4, y/4,
    // z/8 mod 2) alone: the patch cell, the reached pages and the reached pages
    // without n = 0 are tabulated per parity p (bit 4: x/4 odd, 2: y/4, 1: z/8),
    // from a representative block of each parity.
    uint8_t patch_cell[NODES_PER_BLOCK], reach_tab[8][NODES_PER_BLOCK], no_self_tab[8][NODES_PER_BLOCK];
    for (int p = 0; p < 8; ++p)
      for (int e = 0; e < NODES_PER_BLOCK; ++e) {
        const int bx = (p >> 2) * BLK_X, by = ((p >> 1) & 1) * BLK_Y, bz = (p & 1) * BLK_Z;
        const int cx = (bx + (e >> 5) + BLK_X) >> 1, cy = (by + ((e >> 3) & 3) + BLK_Y) >> 1,
                  cz = (bz + (e & 7) + BLK_Z) >> 1;
        const int kx = (cx & 3) == 3, ky = (cy & 3) == 3, kz = (cz & 7) == 7;
        unsigned reach = 0;
        for (int dx = 0; dx <= kx; ++dx)
          for (int dy = 0; dy <= ky; ++dy)
            for (int dz = 0; dz <= kz; ++dz) reach |= 1u << (dx * 4 + dy * 2 + dz);
        reach_tab[p][e] = uint8_t(reach);
        no_self_tab[p][e] = uint8_t((kx && ky && kz) ? (reach & ~1u) : reach);
        patch_cell[e] = uint8_t(((e >> 5) >> 1) * 8 + (((e >> 3) & 3) >> 1) * 4 + ((e & 7) >> 1));
      }
    std::vector<Patch> patch(static_cast<size_t>(F.nb));
#pragma omp parallel for schedule(static)
    for (int b = 0; b < F.nb; ++b) {
      Patch& pt = patch[size_t(b)];
      std::fill(pt.flags, pt.flags + 16, 0u);
      const int p = (((F.coords[3 * b] / BLK_X) & 1) << 2) | (((F.coords[3 * b + 1] / BLK_Y) & 1) << 1) |
                    ((F.coords[3 * b + 2] / BLK_Z) & 1);
      const uint32_t* fl = F.flags.data() + size_t(b) * NODES_PER_BLOCK;
      unsigned pages = 0, any = 0;
      for (int e = 0; e < NODES_PER_BLOCK; ++e) {
        const uint32_t ff = fl[e] & (F_ACTIVE_CELL | F_DIRICHLET_CELL);
        if (!ff) continue;
        pt.flags[patch_cell[e]] |= ff;
        pages |= (ff & F_ACTIVE_CELL) ? reach_tab[p][e] : no_self_tab[p][e];
        any = 1;
      }
      pt.pages = uint8_t(pages);
      pt.any = any != 0;
    }
    // The coarse blocks are the patch blocks and the reached pages.  A serial
    // pass in fine-block order would create them in that order; the pages
    // (active) then go in page-key order and the rest (ghosts, created only as
    // a patch block) in creation order, i.e. in the order of the first fine
    // block whose patch lies in them.  That numbering is made directly:
    // pages marked and patch blocks' first fine block found (atomic minimum)
    // in parallel, both lists sorted, and the patch flags ORed into their
    // blocks, each fine block's patch being a disjoint 2x2x4 part of one
    // coarse block.
    HostLevel& C = bc.L;
    const long ncell = long(C.bgrid.size());
    std::vector<long> own(static_cast<size_t>(F.nb), -1);
    std::vector<int32_t> first(static_cast<size_t>(ncell), INT32_MAX);
    uint8_t* page = C.active_page.data();
#pragma omp parallel for schedule(static)
    for (int b = 0; b < F.nb; ++b) {
      const Patch& pt = patch[size_t(b)];
      if (!pt.any) continue;
      const int cx0 = (F.coords[3 * b] + BLK_X) >> 1, cy0 = (F.coords[3 * b + 1] + BLK_Y) >> 1,
                cz0 = (F.coords[3 * b + 2] + BLK_Z) >> 1;
      const long c = C.cell(cx0, cy0, cz0);
      own[size_t(b)] = c;
      if (c >= 0) {
        int32_t cur = __atomic_load_n(&first[size_t(c)], __ATOMIC_RELAXED);
        while (b < cur && !__atomic_compare_exchange_n(&first[size_t(c)], &cur, int32_t(b), false, __ATOMIC_RELAXED,
                                                       __ATOMIC_RELAXED)) {
        }
      }
      for (int d = 0; d < 8; ++d)
        if (pt.pages >> d & 1) {
          const long pc = C.cell(cx0 + ((d >> 2) & 1) * BLK_X, cy0 + ((d >> 1) & 1) * BLK_Y, cz0 + (d & 1) * BLK_Z);
          if (pc >= 0) __atomic_store_n(&page[pc], uint8_t(1), __ATOMIC_RELAXED);
        }
    }
    const auto act = sorted_cells(ncell, [&](long c) { return page[c] ? cell_key(C, c) : NONE; });
    const auto ghost = sorted_cells(
        ncell, [&](long c) { return !page[c] && first[size_t(c)] != INT32_MAX ? uint64_t(first[size_t(c)]) : NONE; });
    number_blocks(C, act, ghost);
#pragma omp parallel for schedule(static)
    for (int b = 0; b < F.nb; ++b) {
      if (own[size_t(b)] < 0) continue;
      const Patch& pt = patch[size_t(b)];
      const int cx0 = (F.coords[3 * b] + BLK_X) >> 1, cy0 = (F.coords[3 * b + 1] + BLK_Y) >> 1,
                cz0 = (F.coords[3 * b + 2] + BLK_Z) >> 1;
      uint32_t* f = &C.flags[size_t(C.bgrid[size_t(own[size_t(b)])]) * NODES_PER_BLOCK];
      for (int l = 0; l < 16; ++l)
        if (pt.flags[l]) f[node_slot(cx0 + (l >> 3), cy0 + ((l >> 2) & 1), cz0 + (l & 3))] |= pt.flags[l];
    }
    return std::move(bc.L);
  };
  for (int lev = 1; lev < P.mg_levels; ++lev) P.levels.push_back(coarsen(P.levels[lev - 1]));
  phase_done(1);
  for (auto& L : P.levels) flag_nodes(L);
  for (auto& L : P.levels) flag_boundary(L);
  for (auto& L : P.levels) finish_level(L);
  phase_done(2);
  // levels below a bottom too large for the dense inverse: the bottom is then
  // solved by CG with V-cycles over them (same coarsening rule, Galerkin
  // operators down to depth 6)
  if (!P.disable_mg) {
    auto active_nodes = [](const HostLevel& L) {
      long n = 0;
      for (long i = 0; i < long(L.nb) * NODES_PER_BLOCK; ++i) n += (L.flags[size_t(i)] & F_ACTIVE_NODE) ? 1 : 0;
      return n;
    };
    while (P.levels.size() < 7 && 3 * active_nodes(P.levels.back()) > P.dense_bottom_max) {
      HostLevel L = coarsen(P.levels.back());
      flag_nodes(L);
      flag_boundary(L);
      finish_level(L);
      P.levels.push_back(std::move(L));
    }
  }

  // ---- padding check (Multigrid_Hierarchy.h:145-157)
  {
    HostLevel& L = P.levels[0];
    const int bs[3] = {BLK_X, BLK_Y, BLK_Z};
    for (int b = 0; b < L.nb; ++b)
      for (int v = 0; v < 3; ++v) {
        int c = L.coords[3 * b + v];
        if (c < bs[v] || c >= L.size[v] - 2 * bs[v]) {
          std::snprintf(msg, sizeof msg, "Padding violated by block (%d, %d, %d)", L.coords[3 * b], L.coords[3 * b + 1],
                        L.coords[3 * b + 2]);
          return fail(6, msg);
        }
      }
  }

  // ---- input-block map, forces and the Dirichlet lift on level 0
  HostLevel& L0 = P.levels[0];
  P.in_block.resize(nin);
  P.in_zoff.resize(nin);
  P.in_base.assign(in.density.base.begin(), in.density.base.end());
  for (size_t b = 0; b < nin; ++b) {
    int x = in.density.base[3 * b], y = in.density.base[3 * b + 1], z = in.density.base[3 * b + 2];
    P.in_block[b] = L0.active_block_at(x, y, z);
    P.in_zoff[b] = z & 4;
  }
  // forces are assigned, the last entry of a node wins (SPGrid_CPU_Solver.cpp:290-296)
  P.force_node.clear();
  P.force_val.clear();
  for (auto& f : in.forces) {
    int bk = L0.active_block_at(f.coord[0], f.coord[1], f.coord[2]);
    if (bk < 0) continue;  // outside the active pages: the projections zero it
    P.force_node.push_back(bk * NODES_PER_BLOCK + node_slot(f.coord[0], f.coord[1], f.coord[2]));
    for (int v = 0; v < 3; ++v) {
      if (!std::isfinite(f.f[v])) return fail(4, "non-finite force");
      P.force_val.push_back(f.f[v]);
    }
  }
  P.lift_node.clear();
  P.lift_axis.clear();
  P.lift_val.clear();
  for (auto& d : in.dirichlet_nodes) {
    int bk = L0.active_block_at(d.coord[0], d.coord[1], d.coord[2]);
    if (bk < 0) continue;  // values on inactive pages never reach an active cell
    if (!std::isfinite(d.value)) return fail(4, "non-finite Dirichlet value");
    P.lift_node.push_back(bk * NODES_PER_BLOCK + node_slot(d.coord[0], d.coord[1], d.coord[2]));
    P.lift_axis.push_back(d.axis);
    P.lift_val.push_back(d.value);
  }
  phase_done(3);
  return std::string();
}

}  // namespace sgs
