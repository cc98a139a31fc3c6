// Host-side construction of the multigrid hierarchy on SPGrid blocks.
//
// A level stores its active blocks of 4x4x8 nodes in SPGrid page order (the
// page index of the block's Morton offset: bit 3m <- y-block bit m, 3m+1 <-
// x-block bit m, 3m+2 <- z-block bit m; external/SPGrid/Core/SPGrid_Mask.h:38-47,
// SPGrid_Page_Map.h:117-124).  Node (x,y,z) of block b lives at index
// b*128 + (x&3)*32 + (y&3)*8 + (z&7).  Blocks that were written but never
// activated ("ghost" blocks) follow the active ones: SPGrid keeps such writes in
// memory and later reads see them, which matters for the boundary band.
#pragma once
#include <array>
#include <cstdint>
#include <string>
#include <memory>
#include <utility>
#include <vector>

#include "wire.hpp"

namespace sgs {

constexpr uint32_t F_ACTIVE_NODE = 0x10, F_DIRICHLET_NODE_X = 0x20, F_DIRICHLET_NODE = 0xE0,
                   F_ACTIVE_CELL = 0x100, F_DIRICHLET_CELL_X = 0x200, F_DIRICHLET_CELL = 0xE00,
                   F_BOUNDARY_NODE = 0x1000, F_BOUNDARY_TEMP = 0x2000;  // solver/Flags.h:10-24
constexpr int BLK_X = 4, BLK_Y = 4, BLK_Z = 8, NODES_PER_BLOCK = 128;

uint64_t page_key(int bi, int bj, int bk);

struct HostLevel {
  int size[3] = {0, 0, 0};            // allocator size (nodes per axis)
  int grid[3] = {0, 0, 0};            // block-grid dims
  HostBuf<int32_t> bgrid;             // block grid -> block index (active or ghost), -1 if untouched
  int nb = 0;                         // active blocks (first nb entries of coords/flags)
  std::vector<int32_t> coords;        // block base coordinates, [nb_all*3]
  HostBuf<uint32_t> flags;            // [nb_all*128]
  HostBuf<uint8_t> active_page;       // per block-grid cell
  std::vector<int32_t> boundary;      // active blocks with a boundary-band node
  std::array<std::vector<int32_t>, 3> dirichlet;  // node indices with a Dirichlet component

  long cell(int x, int y, int z) const;
  int block_at(int x, int y, int z) const;       // active or ghost, -1 if none
  int active_block_at(int x, int y, int z) const;  // active only
  int touch(int x, int y, int z, bool with_flags = true);  // create a ghost block when needed
};


struct Problem {
  // inputs
  int resolution[3] = {0, 0, 0};
  double dx = 1, mu0 = 0, lambda0 = 0;
  double penalty = 0, minimum_stiffness = 0, minimum_density = 0;  // SIMP parameters (fem_interface.h:318-353)
  int mg_levels = 3;          // levels of the V-cycle after the mg_level=0 rewrite
  bool disable_mg = false;
  // A bottom level (levels[mg_levels - 1]) with more unknowns than this is
  // solved by CG preconditioned with V-cycles over further levels, which then
  // follow it in `levels` (at most 7 levels in all); smaller ones are inverted.
  long dense_bottom_max = 24576;
  // host set-up phase times (seconds): level 0 (pages, SIMP map, checks,
  // Dirichlet cells, stiffness scales), coarsening, node flags and boundary
  // bands, the rest (inner levels, padding check, forces, Dirichlet lift)
  double host_phase[4] = {0, 0, 0, 0};
  int explicit_level = 2;
  int smoothing = 1, boundary_smoothing = 5;
  // the inner bottom CG's V-cycle (this library's replacement of the exact
  // bottom factorisation, so its preconditioner is free): full and
  // boundary-band sweeps per level and direction.  Three full sweeps and no
  // band sweeps took half the time of the outer V-cycle's schedule on narrow
  // bands and boxes (the solve converges to the same round-off either way).
  int inner_smoothing = 3, inner_boundary_smoothing = 0;
  double tolerance = 1e-4;
  int max_iterations = 500;
  // level data
  std::vector<HostLevel> levels;
  HostBuf<double> E;          // level-0 stiffness scale per cell slot (0 = empty)
  // input blocks: level-0 block index and the z offset (0 or 4) inside it
  std::vector<int32_t> in_block, in_zoff;
  std::vector<int32_t> in_base;
  // forces and Dirichlet values mapped to level-0 node indices
  std::vector<int32_t> force_node;
  std::vector<double> force_val;  // [n*3]
  std::vector<int32_t> lift_node, lift_axis;
  std::vector<double> lift_val;
};

// Build the problem from decoded inputs.  Returns an empty string on success,
// else a message (the caller reports it through FEMOutputs.success/error_code).
std::string build_problem(const FEMInputs& in, Problem& P, int* error_code);

}  // namespace sgs
