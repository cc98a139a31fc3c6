// Reference-side SPGrid harness (test infrastructure).  Compiled by
// oracle/Makefile from the reference's external/SPGrid/Core sources and the
// solver's own headers where they lie.  It pins:
//   * the page (block) order the solver iterates in: Set_Page on block bases,
//     Update_Block_Offsets, then LinearToCoord of every block
//     (external/SPGrid/Core/SPGrid_Page_Map.h:66-124, SPGrid_Mask.h:142-181);
//   * the element offsets of the solver's field mask (SPGrid_Mask.h:142);
//   * the level maps DownsampleOffset/UpsampleOffset with origin (4,4,8)
//     (SPGrid_Mask.h:184-227);
//   * the element stiffness tables K_mu/K_la (solver/CPU_Kernels/Stiffness_Matrices.h)
//     and Km_cell/Kl_cell (solver/MG/Linear_Elasticity_Stiffness_Matrix.h).
//
//   * the block order of the optimizer driver's grid (64-byte nodes, 4 KiB pages:
//     4x4x4 blocks, topo_opt/spgrid_topo_opt.h:45-94), which its page maps
//     (thin/fat/fatter) list their blocks in;
//
//   spgrid_harness order <size> <coords.txt>   block bases (x y z per line) -> page order
//   spgrid_harness order4 <size> <coords.txt>  the same on the driver's 4x4x4 grid
//   spgrid_harness offsets <coords.txt>         element offsets and level maps of nodes
//   spgrid_harness tables <out.bin>             K_mu, K_la, Km_cell, Kl_cell as float64
#include <array>
#include <cstdint>
#include <cstdio>
#include <fstream>
#include <iostream>
#include <vector>

#include <SPGrid/Core/SPGrid_Allocator.h>
#include <SPGrid/Core/SPGrid_Page_Map.h>
using namespace SPGrid;
#include "Elasticity_Solver_Data.h"
#include "CPU_Kernels/Stiffness_Matrices.h"
#include "MG/Linear_Elasticity_Stiffness_Matrix.h"

using Struct = Elasticity_Solver_Data<double, uint64_t>;
using Alloc = SPGrid_Allocator<Struct, 3, 14>;
using PageMap = SPGrid_Page_Map<14>;
using Mask = Alloc::Array_mask<double>;
struct DriverNode {
  double field[8];
};
using DriverAlloc = SPGrid_Allocator<DriverNode, 3, 12>;
using DriverPageMap = SPGrid_Page_Map<12>;
using DriverMask = DriverAlloc::Array_mask<double>;

static std::vector<std::array<int, 3>> read_coords(const char* fn) {
  std::vector<std::array<int, 3>> out;
  std::ifstream f(fn);
  int x, y, z;
  while (f >> x >> y >> z) out.push_back({x, y, z});
  return out;
}

int main(int argc, char** argv) {
  if (argc < 3) return 2;
  std::string cmd = argv[1];
  if (cmd == "order" && argc >= 4) {
    int size = std::atoi(argv[2]);
    Alloc alloc(size, size, size);
    PageMap pm(alloc);
    for (auto& c : read_coords(argv[3])) pm.Set_Page(Mask::Linear_Offset(c[0], c[1], c[2]));
    pm.Update_Block_Offsets();
    auto blocks = pm.Get_Blocks();
    for (unsigned b = 0; b < blocks.second; ++b) {
      auto c = Mask::LinearToCoord(blocks.first[b]);
      std::printf("%d %d %d\n", c[0], c[1], c[2]);
    }
    return 0;
  }
  if (cmd == "order4" && argc >= 4) {
    int size = std::atoi(argv[2]);
    DriverAlloc alloc(size, size, size);
    DriverPageMap pm(alloc);
    for (auto& c : read_coords(argv[3])) pm.Set_Page(DriverMask::Linear_Offset(c[0], c[1], c[2]));
    pm.Update_Block_Offsets();
    auto blocks = pm.Get_Blocks();
    for (unsigned b = 0; b < blocks.second; ++b) {
      auto c = DriverMask::LinearToCoord(blocks.first[b]);
      std::printf("%d %d %d\n", c[0], c[1], c[2]);
    }
    return 0;
  }
  if (cmd == "offsets") {
    for (auto& c : read_coords(argv[2])) {
      uint64_t off = Mask::Linear_Offset(c[0], c[1], c[2]);
      auto dn = Mask::LinearToCoord(Mask::DownsampleOffset<4, 4, 8>(off));
      auto up = Mask::LinearToCoord(Mask::UpsampleOffset<4, 4, 8>(off));
      std::printf("%d %d %d %llu %d %d %d %d %d %d\n", c[0], c[1], c[2], (unsigned long long)off, dn[0], dn[1], dn[2],
                  up[0], up[1], up[2]);
    }
    return 0;
  }
  if (cmd == "tables") {
    std::ofstream f(argv[2], std::ios::binary);
    f.write(reinterpret_cast<const char*>(&K_mu<double>[0][0][0][0]), sizeof(double) * 576);
    f.write(reinterpret_cast<const char*>(&K_la<double>[0][0][0][0]), sizeof(double) * 576);
    f.write(reinterpret_cast<const char*>(&Km_cell<double>[0][0][0][0]), sizeof(double) * 576);
    f.write(reinterpret_cast<const char*>(&Kl_cell<double>[0][0][0][0]), sizeof(double) * 576);
    return 0;
  }
  return 2;
}
