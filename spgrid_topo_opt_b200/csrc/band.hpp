// Narrow-band page maps of the optimizer driver on the GPU.
//
// The driver keeps four page maps over its 4x4x4-block grid
// (topo_opt/spgrid_topo_opt.h:116-134): the container, and inside it the thin
// map (blocks that still hold material), the fat map (cells the optimizer
// updates) and the fatter map (the blocks handed to fem_solve).  One update runs
// Opt::update_thin_page_map (topo_opt/spgrid_topo_opt.cpp:92-152),
// Opt::filter_isolated_blocks (:1404-1510) and Opt::update_fat_page_map
// (:154-241); the voxel-level Opt::filter_isolated_voxels (:1512-1633) and the
// kill of Opt::threshold_and_kill (:1333-1344) change the cell flags.  Band
// holds the container on the device (block bases, a dense block lookup, per-cell
// flags and densities) and the three maps as byte masks in the caller's block
// order; only the driver's list order (its Morton page order, needed where the
// reference indexes one list by another's positions) is kept as a permutation.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <memory>
#include <string>
#include <vector>

#include "common.cuh"

namespace sgs {

class Band {
 public:
  Band(const int32_t* base, int64_t nblocks, const int32_t resolution[3], const uint8_t* cell_flags,
       const double* density);
  ~Band();
  Band(const Band&) = delete;
  Band& operator=(const Band&) = delete;

  void set_density(const double* density);  // host, [nblocks][64]
  void get_density(double* density);
  void set_fat(const uint8_t* fat);          // host, [nblocks]
  void update(const sgs_band_params& p, sgs_band_stats* stats);
  void maps(uint8_t* thin, uint8_t* fat, uint8_t* fatter);
  void get_flags(uint8_t* flags);
  void filter_voxels(sgs_band_voxel_stats* stats);
  long kill_below(double threshold);
  long threshold_density(double volume_fraction, double threshold, double* used);

  long n = 0;                 // container blocks
  int gdim[3] = {0, 0, 0};    // dense block lookup extent (blocks per axis)
  cudaStream_t stream = nullptr;
  DevBuf<int32_t> base;       // [n][3] block bases (cells)
  DevBuf<int32_t> grid;       // [gx][gy][gz] -> block or -1
  DevBuf<int32_t> morton;     // driver list position -> block
  DevBuf<uint8_t> flags;      // [n][64] SGS_CELL_* bits
  DevBuf<double> rho;         // [n][64]
  DevBuf<uint8_t> thin, fat, fatter;
  DevBuf<double> meta_sum;    // density sum of every fat block (BlockMeta::density_sum)
  DevBuf<int32_t> parent, comp_size;
  DevBuf<unsigned long long> counters;
  cudaEvent_t ev[2] = {nullptr, nullptr};

  // the driver's optimizer state on the container, for the band step
  std::vector<int32_t> base_h;     // host copy of the block bases
  std::vector<uint8_t> flags_h;    // host copy of the cell flags
  long total_inside = 0;           // total_container_voxels
  DevBuf<double> dc0, dc1;         // sensitivity channels; dc0 persists outside the fat map
  DevBuf<int32_t> sess_map;        // attached session's input block -> container block
  const void* attached = nullptr;  // the solver sess_map belongs to

 private:
  void keep_fraction(double fraction_to_keep, long n_thin);
  void pull_flags();  // device flags -> flags_h after a change on the device
  long threshold_trail(double t, bool apply);
};

}  // namespace sgs

struct sgs_band {
  std::unique_ptr<sgs::Band> band;
  std::string error;
};
