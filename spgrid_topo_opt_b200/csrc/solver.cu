// Narrow-band SPGrid linear-elasticity MGPCG on one B200.
//
// Host orchestration of the kernels in kernels.cuh / setup_kernels.cuh and the
// C ABI declared in include/spgrid_fem.h.  The solve follows the reference's
// fem_solve (solver/SPGrid_CPU_Solver.cpp:26-409): Dirichlet lift, PCG with one
// V-cycle per iteration (solver/CG/CONJUGATE_GRADIENT.cpp:21-61,
// solver/MG/Multigrid_Hierarchy.h:569-619), L-infinity stopping rule relative
// to the zero-guess residual, output packing per input block.
#include <cuda_runtime.h>
#include <sys/mman.h>

#include <cub/cub.cuh>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <functional>
#include <memory>
#include <mutex>
#include <new>
#include <string>
#include <thread>
#include <map>
#include <unordered_map>
#include <vector>

#include "../../include/spgrid_fem.h"
#include "band.hpp"
#include "common.cuh"
#include "kernels.cuh"
#include "setup.hpp"
#include "setup_kernels.cuh"
#include "tc_kernels.cuh"
#include "topo_kernels.cuh"
#include "wire.hpp"

namespace sgs {


// Element stiffness of the Q1 hex on the unit cube: K_mu = int(delta_ij grad Na.grad Nb
// + d_j Na d_i Nb), K_la = int d_i Na d_j Nb; node index a = 4x + 2y + z.  These are
// the exact rationals k/72 of solver/CPU_Kernels/Stiffness_Matrices.h.
static void element_tables(double Kmu[8][8][3][3], double Kla[8][8][3][3]) {
  const int M[2][2] = {{2, 1}, {1, 2}}, D[2][2] = {{-3, -3}, {3, 3}}, S[2][2] = {{6, -6}, {-6, 6}};
  auto g = [&](int a, int b, int i, int j) {
    long v = 1;
    for (int ax = 0; ax < 3; ++ax) {
      int pa = (a >> (2 - ax)) & 1, pb = (b >> (2 - ax)) & 1;
      bool da = ax == i, db = ax == j;
      v *= (da && db) ? S[pa][pb] : da ? D[pa][pb] : db ? D[pb][pa] : M[pa][pb];
    }
    return v;  // 216 * integral
  };
  for (int a = 0; a < 8; ++a)
    for (int b = 0; b < 8; ++b)
      for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) {
          long lam = g(a, b, i, j), mu = g(a, b, j, i);
          if (i == j)
            for (int k = 0; k < 3; ++k) mu += g(a, b, k, k);
          Kla[a][b][i][j] = double(lam / 3) / 72.0;
          Kmu[a][b][i][j] = double(mu / 3) / 72.0;
        }
}

// ---------------------------------------------------------------------------
// Device level
// ---------------------------------------------------------------------------
template <typename T>
struct Level {
  int nb = 0;
  long N = 0;
  DevBuf<int> coords, nbr, bgrid, boundary, dir[3];
  DevBuf<uint32_t> flags, spokes;
  GridView grid{};
  int nbound = 0, ndir[3] = {0, 0, 0};
  DevBuf<T> u, b, r;   // [3N] each
  DevBuf<T> A;         // [243][N] stencils (levels with Galerkin operators)
  bool has_matrix = false;
  // level 0: node lists of the Gauss-Seidel passes, full sweep colours 0..7
  // then boundary sweep colours 8..15, concatenated; list k is gs_off[k]..gs_off[k+1]
  DevBuf<int> gs_list;
  int gs_off[17] = {0};
  // levels with stencils: node lists of the Gauss-Seidel passes, active nodes of
  // colour c (list c) and active boundary-band nodes of colour c (list 8 + c),
  // each ascending; list k is sgs_off[k]..sgs_off[k+1]
  DevBuf<int> sgs_list;
  int sgs_off[17] = {0};
  // level 0 of the V-cycle (mixed and FP64 modes): the iterate packed as (u, E) per
  // node, followed by one all-zero pad block (index nb) that nbrz names for missing neighbours
  DevBuf<typename Pack4<T>::type> u4;
  DevBuf<int> nbrz;
};

struct Bottom {
  int ndof_nodes = 0;
  long n = 0, ld = 0;
  DevBuf<int> dof_node, node_dof;
  DevBuf<double> Minv, xb, xs;
  DevBuf<float> Minv32;  // mixed precision: the FP32 V-cycle applies an FP32 copy of Minv
};

enum Precision { PREC_REFERENCE = 0, PREC_FP64 = 1, PREC_MIXED = 2 };

// Unknowns of a bottom level are the nodes with an active spoke (the rows of
// Build_CSR_Matrix, Elasticity_Matrix.cpp:16-164): out = in there, 0 elsewhere
// (in-place allowed).
__global__ void inner_mask_kernel(double* out, const double* in, const uint32_t* __restrict__ spokes, long N) {
  pdl_wait();
  const long i = long(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= N) return;
  const bool on = spokes[i] & 0x07ffffffu;
#pragma unroll
  for (int v = 0; v < 3; ++v) out[i + v * N] = on ? in[i + v * N] : 0.0;
}

// The inner solve's result on the unknowns, b elsewhere (PARDISO_Solve writes
// back only the rows it solved, Elasticity_Matrix.cpp:238-269).
template <typename T>
__global__ void inner_select_kernel(T* __restrict__ out, const double* __restrict__ x, const double* __restrict__ b,
                                    const uint32_t* __restrict__ spokes, long N) {
  pdl_wait();
  const long i = long(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= N) return;
  const bool on = spokes[i] & 0x07ffffffu;
#pragma unroll
  for (int v = 0; v < 3; ++v) out[i + v * N] = T(on ? x[i + v * N] : b[i + v * N]);
}

// The packed level-0 iterate from planar fields: (u_x, u_y, u_z, E) per node slot.
template <typename T>
__global__ void pack_u4_kernel(typename Pack4<T>::type* __restrict__ u4, const T* __restrict__ u, const T* __restrict__ E,
                               long N) {
  const long i = long(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i < N) u4[i] = Pack4<T>::make(u[i], u[i + N], u[i + 2 * N], E[i]);
}

// Node lists of the level-0 Gauss-Seidel passes, built on the device (see
// Solver::colour_lists).  Sub-list of a slot: 2k for the updates of list k,
// 2k + 1 for its Dirichlet-only clears; lists 0..7 the full sweep's colours,
// 8..15 the boundary sweep's (blocks of the boundary list only).
__device__ __forceinline__ void colour_sub(uint32_t fl, int e, bool band_block, int& full, int& band) {
  const int c = ((e >> 5) & 1) << 2 | ((e >> 3) & 1) << 1 | (e & 1);
  const bool act = fl & ACTIVE_NODE, dir = fl & (DIR_X | DIR_Y | DIR_Z);
  full = act ? 2 * c : (dir ? 2 * c + 1 : -1);
  band = -1;
  if (band_block) band = (act && (fl & BOUNDARY_NODE)) ? 2 * (8 + c) : (dir ? 2 * (8 + c) + 1 : -1);
}

// per block (CTA of 128 threads, thread = slot): entries of each of the 32
// sub-lists, stored sub-list major, cnt[l * nb + b]
__global__ void colour_count_kernel(int nb, const uint32_t* __restrict__ flags, const uint8_t* __restrict__ band_block,
                                    int* __restrict__ cnt) {
  __shared__ int sc[32];
  const int b = blockIdx.x, e = threadIdx.x;
  if (e < 32) sc[e] = 0;
  __syncthreads();
  int full, band;
  colour_sub(flags[long(b) * 128 + e], e, band_block[b] != 0, full, band);
  if (full >= 0) atomicAdd(&sc[full], 1);
  if (band >= 0) atomicAdd(&sc[band], 1);
  __syncthreads();
  if (e < 32) cnt[long(e) * nb + b] = sc[e];
}

// Write every entry at its sub-list's start for the block (exclusive scan of
// the counts) plus its rank among the block's earlier slots of the same
// sub-list, so each sub-list ascends: blocks in order, slots in order.
__global__ void colour_fill_kernel(int nb, const uint32_t* __restrict__ flags, const uint8_t* __restrict__ band_block,
                                   const int* __restrict__ pos, int* __restrict__ out) {
  __shared__ int8_t sfull[128], sband[128];
  const int b = blockIdx.x, e = threadIdx.x;
  const long g = long(b) * 128 + e;
  int full, band;
  colour_sub(flags[g], e, band_block[b] != 0, full, band);
  sfull[e] = int8_t(full);
  sband[e] = int8_t(band);
  __syncthreads();
  int rf = 0, rb = 0;
  for (int k = 0; k < e; ++k) {
    rf += (full >= 0) && (sfull[k] == full || sband[k] == full);
    rb += (band >= 0) && (sfull[k] == band || sband[k] == band);
  }
  if (full >= 0) out[pos[long(full) * nb + b] + rf] = (full & 1) ? ~int(g) : int(g);
  if (band >= 0) out[pos[long(band) * nb + b] + rb] = (band & 1) ? ~int(g) : int(g);
}

// Neighbour table of a level: entry (dx+1)*9 + (dy+1)*3 + (dz+1) of block b is
// the active block at offset (dx, dy, dz) blocks, -1 where there is none or
// only a ghost block (the block grid names active blocks only).
__global__ void block_neighbours_kernel(int nb, const int* __restrict__ coords, GridView g, int* __restrict__ nbr) {
  const long t = long(blockIdx.x) * blockDim.x + threadIdx.x;
  if (t >= long(nb) * 27) return;
  const int b = int(t / 27), d = int(t % 27);
  const long n = g.node(coords[3 * b] + (d / 9 - 1) * BLK_X, coords[3 * b + 1] + ((d / 3) % 3 - 1) * BLK_Y,
                        coords[3 * b + 2] + (d % 3 - 1) * BLK_Z);
  nbr[t] = n < 0 ? -1 : int(n >> 7);
}

// block grid entries naming ghost blocks (index >= nb) become -1; neighbour
// tables with the zero pad block (index nb) in place of missing neighbours
__global__ void active_grid_kernel(int* __restrict__ g, long n, int nb) {
  const long i = long(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i < n && g[i] >= nb) g[i] = -1;
}
__global__ void pad_neighbours_kernel(int* __restrict__ z, const int* __restrict__ nbr, long n, int nb) {
  const long i = long(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i < n) z[i] = nbr[i] < 0 ? nb : nbr[i];
}

__global__ void mark_blocks_kernel(const int* __restrict__ list, int n, uint8_t* __restrict__ mark) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) mark[list[i]] = 1;
}

// Scratch of the allocation-free sensitivity entry point (sgs_sensitivity_static):
// per-CTA partial sums of the objective in a static device array that every GPU
// loading the library holds until the process exits.
static __device__ __align__(256) double g_sensitivity_partials[SGS_SENSITIVITY_STATIC_MAX_PARTIALS];

// ---------------------------------------------------------------------------
// The solver: device hierarchy + PCG
// ---------------------------------------------------------------------------
// Scratch for the Galerkin set-up's cell matrices, per device and kept for the
// process (grown when a larger problem needs it): two buffers of up to
// gigabytes (the level being built and the one above it), which a fresh
// allocation from the stream-ordered pool could take a tenth of a second to
// map whenever the pool's free memory was fragmented.  One set-up uses it at
// a time per device (cell_scratch_lock).
struct CellScratch {
  double* p[2] = {nullptr, nullptr};
  size_t n[2] = {0, 0};
};
static std::mutex g_cell_scratch_mutex;
static std::map<int, CellScratch> g_cell_scratch;
static std::unique_lock<std::mutex> cell_scratch_lock() { return std::unique_lock<std::mutex>(g_cell_scratch_mutex); }
// buffer `slot` of the current device's scratch, at least `count` doubles (the caller holds the lock)
static double* cell_scratch(int slot, size_t count) {
  int dev = 0;
  SGS_CUDA(cudaGetDevice(&dev));
  CellScratch& c = g_cell_scratch[dev];
  if (c.n[slot] < count) {
    if (c.p[slot]) SGS_CUDA(cudaFree(c.p[slot]));
    c.p[slot] = nullptr;
    c.n[slot] = 0;
    SGS_CUDA(cudaMalloc(reinterpret_cast<void**>(&c.p[slot]), count * sizeof(double)));
    c.n[slot] = count;
  }
  return c.p[slot];
}

class Solver {
 public:
  Problem P;
  int precision = PREC_REFERENCE;
  int device = -1;                    // CUDA device of the session (current at set-up)
  double* static_partials = nullptr;  // device address of g_sensitivity_partials on that device
  // the FP32 level-0 residual of the mixed V-cycle on the tensor cores (level0_tc_kernel);
  // off by default: measured slower than the CUDA-core kernel (shared-memory bound)
  bool tensor_cores = false;
  int tc_grid = 0;
  DevBuf<int> tc_err;  // set by a tensor-core kernel whose wait gave up
  cudaStream_t stream = nullptr;
  // level data (double for reference/fp64, float for the mixed V-cycle)
  std::vector<std::unique_ptr<Level<double>>> L64;
  std::vector<std::unique_ptr<Level<float>>> L32;
  Bottom bottom;
  DevBuf<double> E64;
  DevBuf<float> E32;
  // CG vectors [3N0]
  DevBuf<double> x, f, s, q, ubk, scratch;
  DevBuf<int> lift_node, lift_axis, force_node;
  DevBuf<double> lift_val, force_val;
  DevBuf<int> load_node;     // loaded nodes, once each (the compliance f.u)
  DevBuf<double> load_val;
  DevBuf<double> red;      // reduction partials
  DevBuf<double> scal;     // device scalars: 0 rho, 1 rho_old, 2 sq, 3 norm, 4 beta, 5 alpha, 6 -alpha, 7 breakdown
  double* h_scal = nullptr;  // pinned mirror
  // input block map for packing
  DevBuf<int> in_block, in_zoff;
  DevBuf<double> out_disp;
  // stats
  int iterations = 0;
  double initial_residual = 0, final_residual = 0, setup_seconds = 0, solve_seconds = 0;
  // warm start (SPGrid_CPU_Solver.cpp:240-321): a previous solution gathered
  // into the level-0 layout, the residual the stopping rule is relative to
  // (the zero-guess residual of the call that created the kept state), and
  // whether the previous solution was reused
  DevBuf<double> warm_u;
  double warm_reference = 0, warm_residual = 0;
  bool forced_reuse = false, warm_reused = false;
  std::vector<double> history;
  std::string error;
  int error_code = 0;
  // graph of one PCG iteration, launched by the host per iteration (with an
  // inner bottom solve, whose iteration count the host decides, or where
  // conditional graph nodes are unavailable)
  cudaGraphExec_t iter_graph = nullptr;
  // the whole PCG loop as one graph: the convergence test, then a WHILE node
  // whose body is one iteration followed by the test (no host round trip per
  // iteration); loop_buf holds the loop record and the residual history
  cudaGraphExec_t loop_graph = nullptr;
  DevBuf<double> loop_buf;
  double* h_loop = nullptr;  // pinned mirror of loop_buf
  bool loop_unavailable = false;
  std::string loop_note;     // why the device loop is not used, if it is not
  int loop_history = 1024;   // residuals one launch records (2 .. LOOP_HIST)
  long launches_per_iteration = 0;
  long launch_counter = 0;   // kernels launched (or captured) by this solver
  long solve_launches = 0;   // kernels executed by the last solve
  double solve_device_seconds = 0;
  cudaEvent_t ev_start = nullptr, ev_end = nullptr;

  ~Solver() {
    if (ev_start) cudaEventDestroy(ev_start);
    if (ev_end) cudaEventDestroy(ev_end);
    if (iter_graph) cudaGraphExecDestroy(iter_graph);
    if (loop_graph) cudaGraphExecDestroy(loop_graph);
    if (h_scal) cudaFreeHost(h_scal);
    if (h_loop) cudaFreeHost(h_loop);
    if (stream) cudaStreamDestroy(stream);
  }

  long N0() const { return long(P.levels[0].nb) * NODES_PER_BLOCK; }
  long active_nodes0 = 0;  // level-0 nodes flagged active: the problem has 3x as many DOF

  // Launch on the solver stream with programmatic stream serialization (the
  // kernel begins with pdl_wait(), so it may be scheduled while its
  // predecessor finishes).
  template <typename... KArgs, typename... Args>
  void launch(void (*kernel)(KArgs...), dim3 grid, dim3 block, size_t smem, Args... args) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = stream;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    SGS_CUDA(cudaLaunchKernelEx(&cfg, kernel, KArgs(args)...));
  }
  bool mixed() const { return precision == PREC_MIXED; }
  // the mixed and FP64 V-cycles keep their level-0 iterate packed (see
  // reset_u4_kernel); the reference-rounding mode rounds planar fields
  bool packed0() const { return (mixed() || precision == PREC_FP64) && nout() > 1; }
  bool round_ref() const { return precision == PREC_REFERENCE; }
  // levels on the device: the V-cycle's (the reference's mg_level) followed by
  // the levels of the inner solve of a large bottom, if any
  int nlev() const { return int(P.levels.size()); }
  int nout() const { return std::min(P.mg_levels, nlev()); }
  bool inner() const { return !P.disable_mg && nlev() > nout(); }

  void init(int prec) {
    precision = prec;
    // the device the session lives on (current at set-up); entry points that
    // take caller-owned device buffers check that it is current again
    SGS_CUDA(cudaGetDevice(&device));
    SGS_CUDA(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
    {
      int sms = 0;
      SGS_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
      tc_grid = 5 * sms;  // five 44 KB CTAs per SM
      SGS_CUDA(cudaFuncSetAttribute(level0_tc_kernel<OP_RES>, cudaFuncAttributeMaxDynamicSharedMemorySize, TC_SMEM_BYTES));
      SGS_CUDA(cudaFuncSetAttribute(level0_tc_kernel<OP_KU>, cudaFuncAttributeMaxDynamicSharedMemorySize, TC_SMEM_BYTES));
      tc_err.alloc(1);
      tc_err.zero(stream);
    }
    // the host-side name of a __device__ array is not its device address:
    // resolve it here, once per session, with the session's device current
    {
      void* p = nullptr;
      SGS_CUDA(cudaGetSymbolAddress(&p, g_sensitivity_partials));
      static_partials = static_cast<double*>(p);
    }
    SGS_CUDA(cudaMallocHost(&h_scal, 16 * sizeof(double)));
    using clk = std::chrono::steady_clock;
    auto t0 = clk::now();
    auto mark = [&](double* slot) {
      SGS_CUDA(cudaStreamSynchronize(stream));
      const auto t = clk::now();
      *slot = std::chrono::duration<double>(t - t0).count();
      t0 = t;
    };
    const auto start = t0;
    upload_constants();
    build_levels();
    mark(&setup_phase[0]);
    build_operators();
    mark(&setup_phase[1]);
    build_bottom();
    mark(&setup_phase[2]);
    alloc_cg();
    mark(&setup_phase[3]);
    setup_seconds = std::chrono::duration<double>(clk::now() - start).count();
  }
  // device set-up phases: levels and lists, Galerkin operators, bottom inverse, CG vectors
  double setup_phase[4] = {0, 0, 0, 0};
  double host_setup_seconds = 0;

  void upload_constants() {
    double Kmu[8][8][3][3], Kla[8][8][3][3];
    element_tables(Kmu, Kla);
    double kc64[576];
    float kc32[576];
    for (int I = 0; I < 8; ++I)
      for (int J = 0; J < 8; ++J)
        for (int v = 0; v < 3; ++v)
          for (int w = 0; w < 3; ++w) {
            double val = P.mu0 * Kmu[I][J][v][w] + P.lambda0 * Kla[I][J][v][w];
            kc64[(I * 8 + J) * 9 + v * 3 + w] = val;
            kc32[(I * 8 + J) * 9 + v * 3 + w] = float(val);
          }
    // the 10 sign classes of the entries (q1_class); the integer formulas must
    // reproduce the element tables
    float kv[10];
    double kv64[10];
    for (int c = 0; c < 10; ++c) {
      kv64[c] = P.mu0 * (double(Q1_CLASS_M[c]) / 72.0) + P.lambda0 * (double(Q1_CLASS_L[c]) / 72.0);
      kv[c] = float(kv64[c]);
    }
    for (int I = 0; I < 8; ++I)
      for (int J = 0; J < 8; ++J)
        for (int v = 0; v < 3; ++v)
          for (int w = 0; w < 3; ++w) {
            const int m = q1_mu72(I, J, v, w), l = q1_la72(I, J, v, w);
            const bool neg = m < 0 || (m == 0 && l < 0);
            const int c = q1_class(neg ? -m : m, neg ? -l : l);
            if (c < 0 || double(m) / 72.0 != Kmu[I][J][v][w] || double(l) / 72.0 != Kla[I][J][v][w] ||
                (neg ? -kv[c] : kv[c]) != kc32[(I * 8 + J) * 9 + v * 3 + w] ||
                (neg ? -kv64[c] : kv64[c]) != kc64[(I * 8 + J) * 9 + v * 3 + w])
              throw CudaError("element table classes are inconsistent", SGS_ERR_INTERNAL);
            // the reflection symmetry gs0_cell4_kernel relies on: K(I, J) = S K(0, I^J) S
            const double sg = ((I >> (2 - v)) & 1 ? -1.0 : 1.0) * ((I >> (2 - w)) & 1 ? -1.0 : 1.0);
            if (Kmu[I][J][v][w] != sg * Kmu[0][I ^ J][v][w] || Kla[I][J][v][w] != sg * Kla[0][I ^ J][v][w])
              throw CudaError("element table lacks the reflection symmetry", SGS_ERR_INTERNAL);
          }
    SGS_CUDA(cudaMemcpyToSymbolAsync(c_Kv32, kv, sizeof(kv), 0, cudaMemcpyHostToDevice, stream));
    SGS_CUDA(cudaMemcpyToSymbolAsync(c_Kv64, kv64, sizeof(kv64), 0, cudaMemcpyHostToDevice, stream));
    SGS_CUDA(cudaMemcpyToSymbolAsync(c_Kc64, kc64, sizeof(kc64), 0, cudaMemcpyHostToDevice, stream));
    SGS_CUDA(cudaMemcpyToSymbolAsync(c_Kc32, kc32, sizeof(kc32), 0, cudaMemcpyHostToDevice, stream));
  }

  template <typename T>
  void upload_level(Level<T>& d, const HostLevel& h) {
    d.nb = h.nb;
    d.N = long(h.nb) * NODES_PER_BLOCK;
    d.coords.upload(h.coords.data(), size_t(h.nb) * 3, stream);
    d.flags.upload(h.flags.data(), size_t(d.N), stream);
    // the block grid names active blocks only (ghost blocks become -1, on the device)
    d.bgrid.upload(h.bgrid, stream);
    if (d.bgrid.n)
      active_grid_kernel<<<blocks_for(long(d.bgrid.n), 256), 256, 0, stream>>>(d.bgrid.p, long(d.bgrid.n), h.nb);
    d.grid = GridView{d.bgrid.p, h.grid[0], h.grid[1], h.grid[2]};
    // the 27 neighbour blocks of every active block, from the block grid
    d.nbr.alloc(size_t(h.nb) * 27);
    if (h.nb)
      block_neighbours_kernel<<<blocks_for(long(h.nb) * 27, 256), 256, 0, stream>>>(h.nb, d.coords.p, d.grid, d.nbr.p);
    SGS_CUDA(cudaGetLastError());
    d.boundary.upload(h.boundary, stream);
    d.nbound = int(h.boundary.size());
    for (int v = 0; v < 3; ++v) {
      std::vector<int32_t> lst(h.dirichlet[v].begin(), h.dirichlet[v].end());
      for (auto& i : lst) i += v * int(d.N);  // index into the [3][N] planes
      d.dir[v].upload(lst, stream);
      d.ndir[v] = int(lst.size());
    }
    d.u.alloc(3 * d.N);
    d.b.alloc(3 * d.N);
    d.r.alloc(3 * d.N);
    d.u.zero(stream);
    d.b.zero(stream);
    d.r.zero(stream);
  }

  // The single-precision copy of a level's index data comes from the
  // double-precision level already on the device (device-to-device copies).
  template <typename TD, typename TS>
  void clone_level(Level<TD>& d, const Level<TS>& src) {
    auto copy = [&](auto& dst, const auto& from) {
      dst.alloc(from.n);
      if (from.n)
        SGS_CUDA(cudaMemcpyAsync(dst.p, from.p, from.n * sizeof(*from.p), cudaMemcpyDeviceToDevice, stream));
    };
    d.nb = src.nb;
    d.N = src.N;
    copy(d.coords, src.coords);
    copy(d.nbr, src.nbr);
    copy(d.flags, src.flags);
    copy(d.bgrid, src.bgrid);
    copy(d.boundary, src.boundary);
    d.grid = GridView{d.bgrid.p, src.grid.gx, src.grid.gy, src.grid.gz};
    d.nbound = src.nbound;
    for (int v = 0; v < 3; ++v) {
      copy(d.dir[v], src.dir[v]);
      d.ndir[v] = src.ndir[v];
    }
    d.u.alloc(3 * d.N);
    d.b.alloc(3 * d.N);
    d.r.alloc(3 * d.N);
    d.u.zero(stream);
    d.b.zero(stream);
    d.r.zero(stream);
  }

  // Node lists of the level-0 Gauss-Seidel passes.  A node's colour is the
  // parity of its coordinates (blocks have even extents, so the slot's parity
  // is the global one).  A pass visits the colour's nodes of all blocks (full
  // sweep) or of the boundary blocks (boundary sweep), updates the active
  // (active boundary-band) ones and clears the Dirichlet components of the
  // rest; those come last in a list, encoded as ~node.  Lists ascend, so a
  // warp's threads work on neighbouring nodes of few blocks.  Built on the
  // device from the uploaded flags: per-block counts of the 32 sub-lists (16
  // lists x {update, clear}), an exclusive scan over (sub-list, block), and a
  // fill that ranks each entry among its block's earlier slots.
  void colour_lists(Level<double>& d) {
    const int nb = d.nb;
    if (nb == 0) {
      std::fill(d.gs_off, d.gs_off + 17, 0);
      return;
    }
    DevBuf<uint8_t> band_block;
    band_block.alloc(size_t(nb));
    band_block.zero(stream);
    if (d.nbound > 0)
      mark_blocks_kernel<<<blocks_for(d.nbound, 256), 256, 0, stream>>>(d.boundary.p, d.nbound, band_block.p);
    DevBuf<int> cnt, pos;
    const long n = 32L * nb;
    cnt.alloc(size_t(n) + 1);
    pos.alloc(size_t(n) + 1);
    colour_count_kernel<<<nb, 128, 0, stream>>>(nb, d.flags.p, band_block.p, cnt.p);
    SGS_CUDA(cudaMemsetAsync(cnt.p + n, 0, sizeof(int), stream));
    size_t tmp_bytes = 0;
    SGS_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, tmp_bytes, cnt.p, pos.p, int(n + 1), stream));
    DevBuf<uint8_t> tmp;
    tmp.alloc(tmp_bytes);
    SGS_CUDA(cub::DeviceScan::ExclusiveSum(tmp.p, tmp_bytes, cnt.p, pos.p, int(n + 1), stream));
    // list k starts where sub-list 2k does (block 0); the end is the total
    for (int k = 0; k < 16; ++k)
      SGS_CUDA(cudaMemcpyAsync(&d.gs_off[k], pos.p + long(2 * k) * nb, sizeof(int), cudaMemcpyDeviceToHost, stream));
    SGS_CUDA(cudaMemcpyAsync(&d.gs_off[16], pos.p + n, sizeof(int), cudaMemcpyDeviceToHost, stream));
    SGS_CUDA(cudaStreamSynchronize(stream));
    d.gs_list.alloc(size_t(d.gs_off[16]));
    if (d.gs_off[16] > 0)
      colour_fill_kernel<<<nb, 128, 0, stream>>>(nb, d.flags.p, band_block.p, pos.p, d.gs_list.p);
    SGS_CUDA(cudaGetLastError());
    SGS_CUDA(cudaStreamSynchronize(stream));  // the temporaries go out of scope
  }

  // the packed level-0 iterate with its zero pad block, and the neighbour table naming it
  template <typename T>
  void alloc_packed(Level<T>& d) {
    d.u4.alloc(size_t(d.N) + NODES_PER_BLOCK);
    SGS_CUDA(cudaMemsetAsync(d.u4.p + d.N, 0, NODES_PER_BLOCK * sizeof(typename Pack4<T>::type), stream));
    d.nbrz.alloc(d.nbr.n);
    if (d.nbr.n)
      pad_neighbours_kernel<<<blocks_for(long(d.nbr.n), 256), 256, 0, stream>>>(d.nbrz.p, d.nbr.p, long(d.nbr.n), d.nb);
  }

  void build_levels() {
    // the level-0 kernels index the [3][N] planes with 32-bit integers
    if (3 * long(P.levels[0].nb) * NODES_PER_BLOCK >= long(INT32_MAX))
      throw CudaError("the finest level has too many blocks for 32-bit node indices", SGS_ERR_INPUT);
    long active = 0;
    const long n0 = N0();
    const uint32_t* fl0 = P.levels[0].flags.data();
#pragma omp parallel for reduction(+ : active) schedule(static)
    for (long i = 0; i < n0; ++i) active += (fl0[i] & ACTIVE_NODE) ? 1 : 0;
    active_nodes0 = active;
    for (auto& h : P.levels) {
      const bool first = &h == &P.levels[0];
      L64.emplace_back(new Level<double>());
      upload_level(*L64.back(), h);
      if (first) {
        colour_lists(*L64.back());
        if (precision == PREC_FP64 && nout() > 1) alloc_packed(*L64.back());
      }
      if (mixed()) {
        L32.emplace_back(new Level<float>());
        clone_level(*L32.back(), *L64.back());
        if (first) {
          auto& g32 = L32.back()->gs_list;
          g32.alloc(L64.back()->gs_list.n);
          if (g32.n)
            SGS_CUDA(cudaMemcpyAsync(g32.p, L64.back()->gs_list.p, g32.n * sizeof(int), cudaMemcpyDeviceToDevice,
                                     stream));
          std::copy(L64.back()->gs_off, L64.back()->gs_off + 17, L32.back()->gs_off);
          if (nout() > 1) alloc_packed(*L32.back());
        }
      }
    }
    E64.upload(P.E.data(), P.E.size(), stream);
    if (mixed()) {
      E32.alloc(P.E.size());
      launch(convert_kernel<float, double>, blocks_for(long(P.E.size()), 256), 256, 0, E32.p, E64.p, long(P.E.size()));
    }
  }

  // Galerkin operators of the levels >= explicit_level (all on the GPU):
  // table of the depth, cell matrices as a GEMM over the finest cells, node
  // stencils, Dirichlet deletion (Multigrid_Hierarchy.h:215-226).
  // The node lists of a stencil level's Gauss-Seidel passes, from the host
  // flags: per-block counts of the 16 lists, a prefix over (list, block), and
  // a parallel fill, so each list ascends.  A node's colour is the parity of
  // its slot (blocks have even extents).
  void stencil_lists(Level<double>& d, const HostLevel& h) {
    const int nb = d.nb;
    std::vector<int32_t> pos(16 * size_t(nb) + 1, 0);
    auto colour = [](int e) { return ((e >> 5) & 1) * 4 + ((e >> 3) & 1) * 2 + (e & 1); };
#pragma omp parallel for schedule(static)
    for (int b = 0; b < nb; ++b)
      for (int e = 0; e < NODES_PER_BLOCK; ++e) {
        const uint32_t fl = h.flags[size_t(b) * NODES_PER_BLOCK + size_t(e)];
        if (!(fl & F_ACTIVE_NODE)) continue;
        const int c = colour(e);
        ++pos[size_t(c) * nb + size_t(b) + 1];
        if (fl & F_BOUNDARY_NODE) ++pos[size_t(8 + c) * nb + size_t(b) + 1];
      }
    for (size_t i = 1; i < pos.size(); ++i) pos[i] += pos[i - 1];
    std::vector<int32_t> list(size_t(pos.back()));
#pragma omp parallel for schedule(static)
    for (int b = 0; b < nb; ++b) {
      int32_t at[16];
      for (int k = 0; k < 16; ++k) at[k] = pos[size_t(k) * nb + size_t(b)];
      for (int e = 0; e < NODES_PER_BLOCK; ++e) {
        const uint32_t fl = h.flags[size_t(b) * NODES_PER_BLOCK + size_t(e)];
        if (!(fl & F_ACTIVE_NODE)) continue;
        const int c = colour(e), node = b * NODES_PER_BLOCK + e;
        list[size_t(at[c]++)] = node;
        if (fl & F_BOUNDARY_NODE) list[size_t(at[8 + c]++)] = node;
      }
    }
    for (int k = 0; k <= 16; ++k) d.sgs_off[k] = pos[size_t(k) * nb];
    d.sgs_list.upload(list, stream);
  }

  void build_operators() {
    if (P.disable_mg) return;
    const int n = nlev();
    // levels >= explicit_level, or every level when the V-cycle has one level
    // (its bottom is level 0, factored from the depth-0 stencil as in
    // Multigrid_Hierarchy.h:215-226); the inner-solve levels are all >= them
    const int first = (nout() == 1) ? 0 : P.explicit_level;
    // the previous level's cell matrices: the next level's come from them
    // (galerkin_coarsen_kernel) except in the reference-rounding mode, which
    // sums every level from the finest cells as the reference does; both
    // levels' matrices live in the process's cell scratch (buffers `cur` and
    // 1 - `cur`)
    auto scratch = cell_scratch_lock();
    int cur = 0;
    double* prev_cellmat = nullptr;
    DevBuf<int32_t> prev_cell;
    int prev_lev = -1;
    for (int lev = first; lev < n; ++lev) {
      Level<double>& d = *L64[lev];
      if (lev > 6) throw CudaError("multigrid depth above 6 is not supported", SGS_ERR_INPUT);
      const HostLevel& h = P.levels[lev];
      const int side = 1 << lev;
      const long npos = long(side) * side * side;
      // active coarse cells (the only ones with finest material) numbered in
      // slot order, and their coordinates and finest origin: per-block counts,
      // a prefix over the blocks, then a parallel fill
      const int nblk = int(d.N / NODES_PER_BLOCK);
      std::vector<int32_t> first_cell(size_t(nblk) + 1, 0);
#pragma omp parallel for schedule(static)
      for (int b = 0; b < nblk; ++b) {
        int k = 0;
        for (int e = 0; e < NODES_PER_BLOCK; ++e) k += (h.flags[size_t(b) * NODES_PER_BLOCK + e] & F_ACTIVE_CELL) ? 1 : 0;
        first_cell[size_t(b) + 1] = k;
      }
      for (int b = 0; b < nblk; ++b) first_cell[size_t(b) + 1] += first_cell[size_t(b)];
      const int ncells = first_cell[size_t(nblk)];
      std::vector<int32_t> origin(3 * size_t(ncells)), ccoord(3 * size_t(ncells));
      HostBuf<int32_t> cell_of_slot(size_t(d.N));
      const int B[3] = {BLK_X, BLK_Y, BLK_Z};
#pragma omp parallel for schedule(static)
      for (int b = 0; b < nblk; ++b) {
        int k = first_cell[size_t(b)];
        for (int e = 0; e < NODES_PER_BLOCK; ++e) {
          const size_t slot = size_t(b) * NODES_PER_BLOCK + size_t(e);
          if (!(h.flags[slot] & F_ACTIVE_CELL)) {
            cell_of_slot[slot] = -1;
            continue;
          }
          const int c[3] = {h.coords[3 * b] + (e >> 5), h.coords[3 * b + 1] + ((e >> 3) & 3), h.coords[3 * b + 2] + (e & 7)};
          for (int v = 0; v < 3; ++v) {
            origin[3 * size_t(k) + size_t(v)] = side * c[v] - (side - 1) * B[v];
            ccoord[3 * size_t(k) + size_t(v)] = c[v];
          }
          cell_of_slot[slot] = k++;
        }
      }
      const bool recursive = !round_ref() && prev_lev == lev - 1 && lev > 0;
      d.A.alloc(243 * size_t(d.N));
      d.A.zero(stream);
      d.spokes.alloc(size_t(d.N));
      d.spokes.zero(stream);
      d.has_matrix = true;
      stencil_lists(d, h);
      if (ncells > 0) {
        DevBuf<int32_t> dcell;
        dcell.upload(cell_of_slot, stream);
        double* cellmat = cell_scratch(cur, size_t(ncells) * 576);
        if (recursive) {
          DevBuf<int32_t> dcc;
          dcc.upload(ccoord, stream);
          galerkin_coarsen_kernel<<<unsigned(ncells), 576, 0, stream>>>(dcc.p, L64[lev - 1]->grid, prev_cell.p,
                                                                     prev_cellmat, cellmat);
          SGS_CUDA(cudaGetLastError());
          SGS_CUDA(cudaStreamSynchronize(stream));  // dcc goes out of scope
        } else {
          DevBuf<double> table;
          DevBuf<int32_t> dorigin;
          table.alloc(size_t(npos) * 576);
          galerkin_table_kernel<<<blocks_for(npos * 64, 128), 128, 0, stream>>>(lev, table.p);
          dorigin.upload(origin, stream);
          const size_t smem = 2 * GT * 65 * sizeof(double);
          SGS_CUDA(cudaFuncSetAttribute(galerkin_cell_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)));
          galerkin_cell_kernel<<<dim3(576 / GT, (ncells + GT - 1) / GT), 256, smem, stream>>>(
              ncells, dorigin.p, lev, L64[0]->grid, E64.p, table.p, cellmat);
          SGS_CUDA(cudaGetLastError());
          SGS_CUDA(cudaStreamSynchronize(stream));  // the temporaries go out of scope
        }
        galerkin_assemble_kernel<<<unsigned(d.N), 256, 0, stream>>>(d.coords.p, d.flags.p, dcell.p, d.grid, cellmat, d.A.p,
                                                                   d.spokes.p, P.dx);
        SGS_CUDA(cudaGetLastError());
        delete_dirichlet_kernel<<<blocks_for(d.N, 128), 128, 0, stream>>>(d.nb, d.coords.p, d.flags.p, d.spokes.p, d.grid,
                                                                         d.A.p, d.N);
        SGS_CUDA(cudaGetLastError());
        SGS_CUDA(cudaStreamSynchronize(stream));
        prev_cellmat = cellmat;
        cur = 1 - cur;
        std::swap(prev_cell.p, dcell.p);
        std::swap(prev_cell.n, dcell.n);
        prev_lev = lev;
      } else {
        prev_lev = -1;
      }
      if (mixed()) {
        Level<float>& m = *L32[lev];
        m.A.alloc(243 * size_t(d.N));
        launch(convert_kernel<float, double>, blocks_for(243 * d.N, 256), 256, 0, m.A.p, d.A.p, 243 * d.N);
        m.spokes.alloc(size_t(d.N));
        SGS_CUDA(cudaMemcpyAsync(m.spokes.p, d.spokes.p, d.N * 4, cudaMemcpyDeviceToDevice, stream));
        m.sgs_list.alloc(d.sgs_list.n);
        if (d.sgs_list.n)
          SGS_CUDA(cudaMemcpyAsync(m.sgs_list.p, d.sgs_list.p, d.sgs_list.n * sizeof(int), cudaMemcpyDeviceToDevice,
                                   stream));
        std::copy(d.sgs_off, d.sgs_off + 17, m.sgs_off);
        m.has_matrix = true;
      }
    }
  }

  void build_bottom() {
    if (P.disable_mg) return;
    Level<double>& d = *L64[nlev() - 1];
    std::vector<uint32_t> sp(size_t(d.N));
    if (d.N) SGS_CUDA(cudaMemcpyAsync(sp.data(), d.spokes.p, d.N * 4, cudaMemcpyDeviceToHost, stream));
    SGS_CUDA(cudaStreamSynchronize(stream));
    std::vector<int32_t> dof_node, node_dof(size_t(d.N), -1);
    for (long i = 0; i < d.N; ++i)
      if (sp[i] & 0x07ffffffu) {
        node_dof[i] = int(dof_node.size());
        dof_node.push_back(int(i));
      }
    bottom.ndof_nodes = int(dof_node.size());
    bottom.n = 3L * bottom.ndof_nodes;
    bottom.ld = ((bottom.n + SGJ - 1) / SGJ) * SGJ;
    const long max_dense = 24576;  // 4.8 GB of FP64
    if (bottom.n > max_dense) {
      char m[160];
      std::snprintf(m, sizeof m,
                    "the deepest level has %ld unknowns; the dense bottom solve supports at most %ld (the hierarchy "
                    "cannot be deeper than 7 levels)",
                    bottom.n, max_dense);
      throw CudaError(m, SGS_ERR_INPUT);
    }
    bottom.dof_node.upload(dof_node, stream);
    bottom.node_dof.upload(node_dof, stream);
    bottom.xb.alloc(size_t(bottom.ld));
    bottom.xs.alloc(size_t(bottom.ld));
    bottom.xb.zero(stream);
    bottom.xs.zero(stream);
    if (bottom.n == 0) return;
    bottom.Minv.alloc(size_t(bottom.ld) * bottom.ld);
    bottom.Minv.zero(stream);
    bottom_assemble_kernel<<<blocks_for(bottom.ndof_nodes, 128), 128, 0, stream>>>(
        bottom.ndof_nodes, bottom.dof_node.p, bottom.node_dof.p, d.coords.p, d.flags.p, d.spokes.p, d.grid, d.A.p, d.N,
        bottom.Minv.p, bottom.ld);
    if (bottom.ld > bottom.n)
      identity_pad_kernel<<<blocks_for(bottom.ld - bottom.n, 64), 64, 0, stream>>>(bottom.Minv.p, bottom.ld, bottom.n);
    SGS_CUDA(cudaGetLastError());
    invert_dense(bottom.Minv.p, bottom.ld);
    if (mixed()) {
      SGS_CUDA(cudaFuncSetAttribute(gemv32_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    int(bottom.ld * sizeof(float))));
      bottom.Minv32.alloc(bottom.Minv.n);
      convert_kernel<float, double><<<blocks_for(long(bottom.Minv.n), 256), 256, 0, stream>>>(
          bottom.Minv32.p, bottom.Minv.p, long(bottom.Minv.n));
      SGS_CUDA(cudaGetLastError());
      // Minv stays allocated until the session ends: released here, its block
      // would be split by later allocations of the set-up, and the next
      // session's inverse would then grow the memory pool through the driver
    }
  }

  // In-place inverse of the SPD bottom matrix (ld a multiple of SGJ): symmetric
  // blocked Gauss-Jordan over 128-wide pivots (lower tiles only, see
  // setup_kernels.cuh); each 128 x 128 pivot block is inverted by the 64-wide
  // Gauss-Jordan kernels on a second stream, one step ahead: as soon as step K
  // has updated the row and column of pivot K+1, that block is inverted while
  // the rest of step K's update runs.
  void invert_dense(double* M, long ld) {
    const int nt = int(ld / SGJ);
    DevBuf<double> R, T, Cp, P[2], pinv;
    R.alloc(size_t(SGJ) * ld);
    T.alloc(size_t(SGJ) * ld);
    Cp.alloc(size_t(SGJ) * ld);
    P[0].alloc(size_t(SGJ) * SGJ);
    P[1].alloc(size_t(SGJ) * SGJ);
    pinv.alloc(GJ * GJ);
    DevBuf<int> bad;
    bad.alloc(1);
    bad.zero(stream);
    const size_t tile_smem = 2 * GJ * 65 * sizeof(double);
    SGS_CUDA(cudaFuncSetAttribute(gj_tile_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(tile_smem)));
    SGS_CUDA(cudaFuncSetAttribute(sgj_gemm_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(SGJ_SMEM)));
    const long nel = long(SGJ) * ld;
    const size_t row = size_t(ld) * sizeof(double), tile_row = SGJ * sizeof(double);
    // the look-ahead pivot inversion runs beside the update, whose CTAs fill the
    // SMs: its stream has the highest priority so that it takes the first free SM
    cudaStream_t aux;
    int prio_low = 0, prio_high = 0;
    SGS_CUDA(cudaDeviceGetStreamPriorityRange(&prio_low, &prio_high));
    SGS_CUDA(cudaStreamCreateWithPriority(&aux, cudaStreamNonBlocking, prio_high));
    cudaEvent_t crossed, inverted;
    SGS_CUDA(cudaEventCreateWithFlags(&crossed, cudaEventDisableTiming));
    SGS_CUDA(cudaEventCreateWithFlags(&inverted, cudaEventDisableTiming));
    // P <- (diagonal tile K)^-1 on stream st
    auto invert_pivot = [&](int K, double* Pk, cudaStream_t st) {
      SGS_CUDA(cudaMemcpy2DAsync(Pk, tile_row, M + size_t(K) * SGJ * ld + size_t(K) * SGJ, row, tile_row, SGJ,
                                 cudaMemcpyDeviceToDevice, st));
      for (int k = 0; k < SGJ / GJ; ++k) {
        gj_pivot_kernel<<<1, 256, GJ * 65 * sizeof(double), st>>>(Pk, SGJ, k, pinv.p, bad.p);
        gj_tile_kernel<<<SGJ / GJ, 256, tile_smem, st>>>(Pk, SGJ, k, pinv.p, 0);
        gj_tile_kernel<<<dim3(SGJ / GJ, SGJ / GJ), 256, tile_smem, st>>>(Pk, SGJ, k, pinv.p, 1);
        gj_tile_kernel<<<SGJ / GJ, 256, tile_smem, st>>>(Pk, SGJ, k, pinv.p, 2);
        gj_store_pivot_kernel<<<1, 256, 0, st>>>(Pk, SGJ, k, pinv.p);
      }
    };
    invert_pivot(0, P[0].p, stream);
    for (int K = 0; K < nt; ++K) {
      double* Pk = P[K & 1].p;
      if (K > 0) SGS_CUDA(cudaStreamWaitEvent(stream, inverted, 0));
      sgj_gather_kernel<<<blocks_for(nel, 256), 256, 0, stream>>>(M, ld, K, R.p, Cp.p, nullptr);
      // T = P^-1 R
      sgj_gemm_kernel<<<dim3(nt, 1), SGJ_THREADS, SGJ_SMEM, stream>>>(SGJ, Pk, SGJ, R.p, ld, T.p, ld, 1.0, 0.0, SGJ_DENSE, -1);
      const int next = K + 1 < nt ? K + 1 : -1;
      if (next >= 0) {
        // the row and column of the next pivot first, then its inverse on the side stream
        sgj_gemm_kernel<<<nt, SGJ_THREADS, SGJ_SMEM, stream>>>(SGJ, Cp.p, SGJ, T.p, ld, M, ld, -1.0, 1.0, SGJ_CROSS, next);
        SGS_CUDA(cudaEventRecord(crossed, stream));
        SGS_CUDA(cudaStreamWaitEvent(aux, crossed, 0));
        invert_pivot(next, P[next & 1].p, aux);
        SGS_CUDA(cudaEventRecord(inverted, aux));
      }
      // the other lower tiles: M -= Cp T
      sgj_gemm_kernel<<<unsigned(long(nt) * (nt + 1) / 2), SGJ_THREADS, SGJ_SMEM, stream>>>(SGJ, Cp.p, SGJ, T.p, ld, M, ld, -1.0,
                                                                             1.0, SGJ_LOWER, next);
      // A_IK = -Cp_I P^-1 below the pivot
      if (K + 1 < nt)
        sgj_gemm_kernel<<<dim3(1, nt - K - 1), SGJ_THREADS, SGJ_SMEM, stream>>>(SGJ, Cp.p + size_t(K + 1) * SGJ * SGJ, SGJ, Pk, SGJ,
                                                                 M + size_t(K + 1) * SGJ * ld + size_t(K) * SGJ, ld,
                                                                 -1.0, 0.0, SGJ_DENSE, -1);
      // A_KJ = T_J left of the pivot, A_KK = P^-1
      if (K > 0)
        SGS_CUDA(cudaMemcpy2DAsync(M + size_t(K) * SGJ * ld, row, T.p, row, size_t(K) * SGJ * sizeof(double), SGJ,
                                   cudaMemcpyDeviceToDevice, stream));
      SGS_CUDA(cudaMemcpy2DAsync(M + size_t(K) * SGJ * ld + size_t(K) * SGJ, row, Pk, tile_row, tile_row, SGJ,
                                 cudaMemcpyDeviceToDevice, stream));
    }
    SGS_CUDA(cudaStreamSynchronize(aux));
    cudaEventDestroy(crossed);
    cudaEventDestroy(inverted);
    cudaStreamDestroy(aux);
    sgj_mirror_kernel<<<dim3(unsigned(ld / 32), unsigned(ld / 32)), dim3(32, 8), 0, stream>>>(M, ld);
    SGS_CUDA(cudaGetLastError());
    int hbad = 0;
    SGS_CUDA(cudaMemcpyAsync(&hbad, bad.p, sizeof(int), cudaMemcpyDeviceToHost, stream));
    SGS_CUDA(cudaStreamSynchronize(stream));
    if (hbad) throw CudaError("bottom operator is not positive definite", SGS_ERR_BREAKDOWN);
  }

  void alloc_cg() {
    const long n3 = 3 * N0();
    for (DevBuf<double>* v : {&x, &f, &s, &q, &ubk, &scratch}) {
      v->alloc(size_t(n3));
      v->zero(stream);
    }
    lift_node.upload(P.lift_node, stream);
    lift_axis.upload(P.lift_axis, stream);
    lift_val.upload(P.lift_val, stream);
    force_node.upload(P.force_node, stream);
    force_val.upload(P.force_val, stream);
    {
      // the loads as the solve assembles them: one value per node, the last entry wins
      std::unordered_map<int32_t, size_t> at;
      std::vector<int32_t> nodes;
      std::vector<double> vals;
      for (size_t k = 0; k < P.force_node.size(); ++k) {
        auto it = at.find(P.force_node[k]);
        size_t slot;
        if (it == at.end()) {
          slot = nodes.size();
          at.emplace(P.force_node[k], slot);
          nodes.push_back(P.force_node[k]);
          vals.resize(vals.size() + 3);
        } else {
          slot = it->second;
        }
        for (int v = 0; v < 3; ++v) vals[3 * slot + size_t(v)] = P.force_val[3 * k + size_t(v)];
      }
      load_node.upload(nodes, stream);
      load_val.upload(vals, stream);
    }
    red.alloc(size_t(std::max<long>(2048, P.levels[0].nb)));  // reduction partials (one per level-0 block at most)
    scal.alloc(16);
    scal.zero(stream);
    in_block.upload(P.in_block, stream);
    in_zoff.upload(P.in_zoff, stream);
    out_disp.alloc(P.in_block.size() * 64 * 4);
  }

  // ------------------------------------------------------------------ kernels
  template <typename T>
  Level<T>& lev(int l);

  template <typename T>
  const T* Edev();

  template <typename T>
  void project(Level<T>& d, T* v) {
    for (int c = 0; c < 3; ++c)
      if (d.ndir[c]) {
        launch(zero_list_kernel<T>, blocks_for(d.ndir[c], 256), 256, 0, v, d.dir[c].p, d.ndir[c]);
        ++launch_counter;
      }
  }

  template <typename T>
  void project_null(Level<T>& d, T* v) {
    launch(project_null_kernel<T>, blocks_for(d.N, 256), 256, 0, v, d.flags.p, d.N);
    ++launch_counter;
  }

  template <typename T>
  void round3(Level<T>& d, T* v) {
    launch(round_float_kernel<T>, blocks_for(3 * d.N, 256), 256, 0, v, 3 * d.N);
    ++launch_counter;
  }

  // out = dx K u (OP_KU), b - dx K u (OP_RES) or the projected PCG matvec with
  // per-block partial products u.out in red (OP_KUP) over all level-0 blocks
  template <typename T, int OP>
  void level0(const T* u, const T* b, T* out) {
    Level<T>& d = lev<T>(0);
    if (d.nb <= 0) return;
    launch(level0_op_kernel<T, OP>, d.nb, 128, 0, nullptr, d.nb, d.nbr.p, Edev<T>(), u, b, out, d.N, T(P.dx),
           d.flags.p, red.p);
    ++launch_counter;
  }

  // SOP_GS: `list` names `count` nodes; SOP_MUL / SOP_RES: all nodes of the
  // level's `count` blocks (list == nullptr)
  template <typename T, int OP>
  void stencil(int l, const int* list, int count, const T* u, T* uo, const T* b, T* out, int round_out) {
    Level<T>& d = lev<T>(l);
    if (count <= 0) return;
    const long nodes = OP == SOP_GS ? long(count) : long(count) * NODES_PER_BLOCK;
    launch(stencil_op_kernel<T, OP>, blocks_for(nodes * 32, 256), 256, 0, list, count, d.nbr.p, d.A.p, d.flags.p, u,
           uo, b, out, d.N, round_out);
    ++launch_counter;
  }

  // one full smoothing sweep (8 colours) of level l on u given b
  template <typename T>
  void sweep(int l, T* u, const T* b, bool forward, bool boundary, bool matrix_free = true) {
    Level<T>& d = lev<T>(l);
    if ((boundary ? d.nbound : d.nb) == 0) return;
    if (l == 0 && matrix_free) {
      for (int k = 0; k < 8; ++k) {
        const int c = (boundary ? 8 : 0) + (forward ? k : 7 - k);
        const int lo = d.gs_off[c], cnt = d.gs_off[c + 1] - lo;
        if (cnt == 0) continue;
        if (!u && boundary) {  // boundary band: few nodes, eight threads per node
          launch(gs0_cell4_kernel<T>, blocks_for(long(cnt) * 8, 128), 128, 0, d.gs_list.p + lo, cnt, d.nbrz.p, d.u4.p,
                 b, d.flags.p, int(d.N), T(P.dx));
          ++launch_counter;
          continue;
        }
        if (!u) {  // the packed iterate of the V-cycle
          // single precision: 64 registers, 8 CTAs per SM (faster than 6 or 10
          // despite a few spilled bytes); double: 128, 4 per SM
          if constexpr (sizeof(T) == 4)
            launch(gs0_list4_kernel<T, 8>, blocks_for(cnt, 128), 128, 0, d.gs_list.p + lo, cnt, d.nbrz.p, d.u4.p, b,
                   d.flags.p, int(d.N), T(P.dx));
          else
            launch(gs0_list4_kernel<T, 4>, blocks_for(cnt, 128), 128, 0, d.gs_list.p + lo, cnt, d.nbrz.p, d.u4.p, b,
                   d.flags.p, int(d.N), T(P.dx));
          ++launch_counter;
          continue;
        }
        // single precision: 80 registers, 6 CTAs per SM; double: 128, 4 per SM
        if constexpr (sizeof(T) == 4)
          launch(gs0_list_kernel<T, 6>, blocks_for(cnt, 128), 128, 0, d.gs_list.p + lo, cnt, d.nbr.p, Edev<T>(), u, b,
                 d.flags.p, int(d.N), T(P.dx));
        else
          launch(gs0_list_kernel<T, 4>, blocks_for(cnt, 128), 128, 0, d.gs_list.p + lo, cnt, d.nbr.p, Edev<T>(), u, b,
                 d.flags.p, int(d.N), T(P.dx));
        ++launch_counter;
      }
      return;
    }
    static const int order[2][8] = {{1, 5, 4, 6, 7, 3, 2, 0}, {0, 2, 3, 7, 6, 4, 5, 1}};
    for (int k = 0; k < 8; ++k) {
      const int li = (boundary ? 8 : 0) + (forward ? order[0][k] : order[1][k]);
      stencil<T, SOP_GS>(l, d.sgs_list.p + d.sgs_off[li], d.sgs_off[li + 1] - d.sgs_off[li], u, u, b, nullptr, 0);
    }
  }

  template <typename T>
  void sweeps(int l, T* u, const T* b, bool forward) {
    const bool rr = round_ref();
    for (int t = 0; t < P.boundary_smoothing; ++t) {
      sweep<T>(l, u, b, forward, true);
      if (rr) round3(lev<T>(l), u);
    }
    for (int t = 0; t < P.smoothing; ++t) {
      sweep<T>(l, u, b, forward, false);
      if (rr) round3(lev<T>(l), u);
    }
    for (int t = 0; t < P.boundary_smoothing; ++t) {
      sweep<T>(l, u, b, forward, true);
      if (rr) round3(lev<T>(l), u);
    }
  }

  template <typename T>
  void restrict_to(int lc, const T* fine_field) {
    Level<T>& c = lev<T>(lc);
    Level<T>& fl = lev<T>(lc - 1);
    if (c.N == 0) return;
    launch(restrict_kernel<T>, blocks_for(c.N, 128), 128, 0, c.nb, c.coords.p, c.flags.p, fl.grid, fine_field, fl.N,
                                                                c.b.p, c.N);
    ++launch_counter;
  }

  template <typename T>
  void prolongate_to(int lf, T* fine_u, int round = -1) {
    Level<T>& fl = lev<T>(lf);
    Level<T>& c = lev<T>(lf + 1);
    if (fl.N == 0) return;
    if (!fine_u) {  // into the packed level-0 iterate
      launch(prolongate4_kernel<T>, blocks_for(fl.N, 128), 128, 0, fl.nb, fl.coords.p, fl.flags.p, c.grid, c.u.p, c.N,
             fl.u4.p);
      ++launch_counter;
      return;
    }
    launch(prolongate_kernel<T>, blocks_for(fl.N, 128), 128, 0, fl.nb, fl.coords.p, fl.flags.p, c.grid, c.u.p, c.N,
                                                                   fine_u, fl.N, round < 0 ? (round_ref() ? 1 : 0) : round);
    ++launch_counter;
  }

  // the V-cycle's bottom: the dense inverse, or the inner solve of a large bottom
  template <typename T>
  void bottom_solve(int l) {
    if (inner() && l == nout() - 1) {
      inner_solve<T>(l);
      if (round_ref()) round3(lev<T>(l), lev<T>(l).u.p);
      return;
    }
    bottom_dense<T>(l, round_ref());
  }

  // u = M^-1 b on the deepest level (nodes without unknowns keep b)
  template <typename T>
  void bottom_dense(int l, bool round) {
    Level<T>& d = lev<T>(l);
    // nodes without unknowns keep b (the reference copies b in and out)
    SGS_CUDA(cudaMemcpyAsync(d.u.p, d.b.p, 3 * d.N * sizeof(T), cudaMemcpyDeviceToDevice, stream));
    if (bottom.ndof_nodes > 0) {
      launch(bottom_gather_kernel<T>, blocks_for(bottom.ndof_nodes, 128), 128, 0, bottom.ndof_nodes, bottom.dof_node.p,
                                                                                     d.b.p, d.N, bottom.xb.p);
      if (sizeof(T) == 4 && bottom.Minv32.p)  // the FP32 V-cycle applies the FP32 copy
        launch(gemv32_kernel, blocks_for(bottom.ld, GEMV32_ROWS), 1024, size_t(bottom.ld) * sizeof(float),
               bottom.Minv32.p, bottom.ld, bottom.ld, bottom.xb.p, bottom.xs.p);
      else
        launch(gemv_kernel, blocks_for(bottom.ld * 32, 256), 256, 0, bottom.Minv.p, bottom.ld, bottom.ld, bottom.xb.p,
               bottom.xs.p);
      launch(bottom_scatter_kernel<T>, blocks_for(bottom.ndof_nodes, 128), 128, 0, bottom.ndof_nodes,
                                                                                      bottom.dof_node.p, bottom.xs.p,
                                                                                      d.u.p, d.N);
      launch_counter += 3;
    }
    if (round) round3(d, d.u.p);
  }

  // ---- exact solve of a bottom level too large for the dense inverse.  The
  // reference factors the bottom's Galerkin operator with PARDISO
  // (Elasticity_Matrix.cpp:169-269); here it is solved in FP64 by CG on the
  // unknowns of the dense path (nodes with an active spoke), preconditioned by
  // V-cycles over the levels that follow it (Gauss-Seidel on every level with
  // the stencil operators, the dense inverse at the deepest), until the
  // residual's 2-norm is below 1e-13 of the right-hand side's or stops
  // decreasing.  Nodes without unknowns keep b, as with PARDISO_Solve.
  struct InnerSolve {
    DevBuf<double> b, x, r, p, z, q, scal;
  } ib;

  void inner_alloc(int l) {
    const long n3 = 3 * L64[l]->N;
    for (DevBuf<double>* v : {&ib.b, &ib.x, &ib.r, &ib.p, &ib.z, &ib.q})
      if (long(v->n) != n3) v->alloc(size_t(n3));
    if (!ib.scal.p) ib.scal.alloc(16);
  }

  // V-cycle of the inner solve on levels top..nlev()-1 in FP64, no rounding:
  // right-hand side in L64[top]->b, result in L64[top]->u
  void inner_vcycle(int top) {
    const int n = nlev();
    Level<double>& t = *L64[top];
    SGS_CUDA(cudaMemsetAsync(t.u.p, 0, 3 * t.N * sizeof(double), stream));
    for (int l = top; l < n - 1; ++l) {
      Level<double>& d = *L64[l];
      inner_sweeps(l, true);
      Level<double>& c = *L64[l + 1];
      SGS_CUDA(cudaMemsetAsync(c.u.p, 0, 3 * c.N * sizeof(double), stream));
      SGS_CUDA(cudaMemsetAsync(c.b.p, 0, 3 * c.N * sizeof(double), stream));
      stencil<double, SOP_RES>(l, nullptr, d.nb, d.u.p, nullptr, d.b.p, d.r.p, 0);
      restrict_to<double>(l + 1, d.r.p);
    }
    bottom_dense<double>(n - 1, false);
    for (int l = n - 2; l >= top; --l) {
      prolongate_to<double>(l, L64[l]->u.p, 0);
      inner_sweeps(l, false);
    }
  }

  void inner_sweeps(int l, bool forward) {
    Level<double>& d = *L64[l];
    for (int t = 0; t < P.inner_boundary_smoothing; ++t) sweep<double>(l, d.u.p, d.b.p, forward, true, false);
    for (int t = 0; t < std::max(1, P.inner_smoothing); ++t) sweep<double>(l, d.u.p, d.b.p, forward, false, false);
    for (int t = 0; t < P.inner_boundary_smoothing; ++t) sweep<double>(l, d.u.p, d.b.p, forward, true, false);
  }

  template <typename T>
  void inner_solve(int l) {
    Level<T>& d = lev<T>(l);
    Level<double>& D = *L64[l];
    const long N = D.N, n3 = 3 * N;
    inner_alloc(l);
    if constexpr (sizeof(T) == 4)
      launch(convert_kernel<double, float>, blocks_for(n3, 256), 256, 0, ib.b.p, d.b.p, n3);
    else
      SGS_CUDA(cudaMemcpyAsync(ib.b.p, d.b.p, n3 * sizeof(double), cudaMemcpyDeviceToDevice, stream));
    inner_pcg(l);
    launch(inner_select_kernel<T>, blocks_for(N, 256), 256, 0, d.u.p, ib.x.p, ib.b.p, D.spokes.p, N);
    launch_counter += 2;
  }

  void inner_pcg(int l);

  // a tensor-core kernel whose MMA wait gave up reports it here (after a sync)
  void check_tensor_core_waits() {
    int bad = 0;
    SGS_CUDA(cudaMemcpyAsync(&bad, tc_err.p, sizeof(int), cudaMemcpyDeviceToHost, stream));
    SGS_CUDA(cudaStreamSynchronize(stream));
    if (bad) throw CudaError("a tensor-core MMA wait timed out", SGS_ERR_CUDA);
  }

  // K u (OP_KU) or b - K u (OP_RES) on the packed level-0 iterate: the tensor-core
  // kernel in single precision, the shared-memory CUDA-core kernel otherwise
  template <typename T, int OP>
  void level0_packed(const T* b, T* out) {
    Level<T>& d = lev<T>(0);
    if (d.nb <= 0) return;
    if constexpr (sizeof(T) == 4) {
      if (tensor_cores) {
        launch(level0_tc_kernel<OP>, std::min(d.nb, tc_grid), TC_THREADS, size_t(TC_SMEM_BYTES), d.nb, d.nbrz.p,
               reinterpret_cast<const float4*>(d.u4.p), b, out, d.N, float(P.dx), float(P.mu0 / 72.0),
               float(P.lambda0 / 72.0), tc_err.p);
        ++launch_counter;
        return;
      }
    }
    if (OP != OP_RES) throw CudaError("K u on the packed iterate runs on the tensor-core kernel only", SGS_ERR_INPUT);
    launch(level0_res4_kernel<T>, d.nb, 128, 0, d.nb, d.nbrz.p, d.u4.p, b, out, d.N, T(P.dx));
    ++launch_counter;
  }

  // V-cycle (Run_VCycle): level-0 right-hand side b0, correction written to u0.
  template <typename T>
  void vcycle(const T* b0, T* u0) {
    const int n = nout();
    const int ex = P.explicit_level;
    const bool rr = round_ref();
    Level<T>& l0 = lev<T>(0);
    // u0 == nullptr: the packed level-0 iterate l0.u4
    const bool packed = u0 == nullptr;
    if (packed) {
      launch(reset_u4_kernel<T>, blocks_for(l0.N, 256), 256, 0, l0.u4.p, Edev<T>(), l0.N);
      ++launch_counter;
    } else {
      SGS_CUDA(cudaMemsetAsync(u0, 0, 3 * l0.N * sizeof(T), stream));
    }
    if (n == 1) {
      // single level: exact solve on level 0 (its b is the given right-hand side)
      SGS_CUDA(cudaMemcpyAsync(l0.b.p, b0, 3 * l0.N * sizeof(T), cudaMemcpyDeviceToDevice, stream));
      bottom_solve<T>(0);
      SGS_CUDA(cudaMemcpyAsync(u0, l0.u.p, 3 * l0.N * sizeof(T), cudaMemcpyDeviceToDevice, stream));
      return;
    }
    auto U = [&](int l) -> T* { return l == 0 ? u0 : lev<T>(l).u.p; };
    auto B = [&](int l) -> const T* { return l == 0 ? b0 : lev<T>(l).b.p; };
    for (int l = 0; l < n - 1; ++l) {
      const bool smooth = l == 0 || l >= ex;
      if (smooth) sweeps<T>(l, U(l), B(l), true);
      Level<T>& c = lev<T>(l + 1);
      SGS_CUDA(cudaMemsetAsync(c.u.p, 0, 3 * c.N * sizeof(T), stream));
      SGS_CUDA(cudaMemsetAsync(c.b.p, 0, 3 * c.N * sizeof(T), stream));
      Level<T>& d = lev<T>(l);
      if (smooth) {
        if (l == 0) {
          if (packed) {
            level0_packed<T, OP_RES>(B(0), d.r.p);
          } else {
            level0<T, OP_RES>(U(0), B(0), d.r.p);
          }
          if (rr) round3(d, d.r.p);
        } else {
          stencil<T, SOP_RES>(l, nullptr, d.nb, U(l), nullptr, B(l), d.r.p, rr ? 1 : 0);
        }
        restrict_to<T>(l + 1, d.r.p);
      } else {
        restrict_to<T>(l + 1, B(l));
      }
    }
    bottom_solve<T>(n - 1);
    for (int l = n - 2; l >= 0; --l) {
      prolongate_to<T>(l, U(l));
      if (l == 0 || l >= ex) sweeps<T>(l, U(l), B(l), false);
    }
  }

  // ------------------------------------------------------------------ PCG
  void dot(const double* a, const double* b, double* out);
  void linf(const double* a, double* out);
  bool build_loop_graph();
  cudaGraphExec_t while_graph(const std::function<void(cudaGraphConditionalHandle)>& head,
                              const std::function<void(cudaGraphConditionalHandle)>& body, std::string* why);
  void drop_graphs() {
    if (iter_graph) SGS_CUDA(cudaGraphExecDestroy(iter_graph));
    if (loop_graph) SGS_CUDA(cudaGraphExecDestroy(loop_graph));
    iter_graph = loop_graph = nullptr;
  }
  void axpy(double* dst, double sign, int coef_slot, const double* xv, const double* yv);
  int precondition();  // returns the number of rho partials it wrote
  void stage_residual();
  void record_iteration();
  void solve();
  // displacements [nblocks][64][4] to host memory, records `pitch` bytes apart (0: packed)
  void pack_outputs(void* disp, size_t pitch = 0);
  double sensitivity(const double* rho, double penalty, double emin, double* dc, double* se);
  void filter_sensitivity(const double* rho, const double* dc0, double* dc1, double filter_size);
  double oc_update(double* rho, const double* dc0, const uint8_t* fixed, double volume_fraction, double step_limit,
                   double minimum_density, double fixed_density, int smart_oc, int exclude_fixed, double* change);
  // the same on device arrays (rho updated in place)
  void filter_dev(const double* rho, const double* dc0, double* dc1, double filter_size, double scale);
  double oc_dev(double* rho, const double* dc0, const uint8_t* fixed, double volume_fraction, double step_limit,
                double minimum_density, double fixed_density, int smart_oc, int exclude_fixed, int keep_inside,
                double* change);
  // device-resident design: densities, sensitivities and fixed-cell mask kept on the GPU
  DevBuf<double> design_rho, design_dc, design_dc1, design_scratch, design_part;
  DevBuf<uint8_t> design_fixed;
  void design_set(const double* rho, const uint8_t* fixed);
  void design_step(const sgs_design_params& prm, sgs_design_result* out);
  // the same iteration on a narrow band whose fatter blocks this session holds
  void band_attach(Band& B, const int64_t* container_block);
  void band_step(Band& B, const sgs_design_params& prm, sgs_design_result* out);
  // new stiffness scales from the design densities (session layout, rho_s):
  // E, the coarse operators and the bottom inverse are rebuilt on the device
  void design_refresh(const double* rho_s);
  // dense grid of the input 4x4x4 blocks (built on first use by the filter)
  DevBuf<int> in_grid, in_base_d;
  int in_gdim[3] = {0, 0, 0};

  // New densities for the same material pattern: E, the Galerkin operators and
  // the bottom inverse are rebuilt, the hierarchy and flags are kept.
  std::string update_density(const double* rho) {
    const size_t nin = P.in_block.size();
    auto E = P.E;
    for (size_t b = 0; b < nin; ++b) {
      const int blk = P.in_block[b];
      if (blk < 0) continue;
      for (int e = 0; e < 64; ++e) {
        const double d = rho[b * 64 + e];
        double val = 0;
        if (d > 0)
          val = P.penalty ? (1 - P.minimum_stiffness) * std::pow(std::max(P.minimum_density, d), P.penalty) +
                                P.minimum_stiffness
                          : d;
        if (!std::isfinite(val)) return "non-finite density";
        const size_t slot = size_t(blk) * NODES_PER_BLOCK + (e >> 4) * 32 + ((e >> 2) & 3) * 8 + (e & 3) + P.in_zoff[b];
        if ((val * P.mu0 != 0) != (P.E[slot] * P.mu0 != 0))
          return "the set of material cells changed; create a new session";
        E[slot] = val;
      }
    }
    P.E.swap(E);
    SGS_CUDA(cudaMemcpyAsync(E64.p, P.E.data(), P.E.size() * sizeof(double), cudaMemcpyHostToDevice, stream));
    g_h2d_bytes += P.E.size() * sizeof(double);
    if (mixed())
      launch(convert_kernel<float, double>, blocks_for(long(P.E.size()), 256), 256, 0, E32.p, E64.p, long(P.E.size()));
    drop_graphs();  // the captured iteration refers to the old operator buffers
    build_operators();
    build_bottom();
    SGS_CUDA(cudaStreamSynchronize(stream));
    return std::string();
  }
};

template <>
Level<double>& Solver::lev<double>(int l) { return *L64[l]; }
template <>
Level<float>& Solver::lev<float>(int l) { return *L32[l]; }
template <>
const double* Solver::Edev<double>() { return E64.p; }
template <>
const float* Solver::Edev<float>() { return E32.p; }

// ---------------------------------------------------------------------------
// CG vector kernels
// ---------------------------------------------------------------------------
constexpr int RED_BLOCKS = 592, RED_THREADS = 256;  // 4 CTAs per SM on 148 SMs
// the PCG's streaming kernels over node pairs (16-byte loads): 8 CTAs per SM
constexpr int PAIR_BLOCKS = 1184;

__global__ void dot_partial_kernel(const double* __restrict__ a, const double* __restrict__ b, long n,
                                   double* __restrict__ part) {
  pdl_wait();
  __shared__ double sm[RED_THREADS / 32];
  double s = 0;
  for (long i = long(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += long(gridDim.x) * blockDim.x) s += a[i] * b[i];
  for (int o = 16; o; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
  if ((threadIdx.x & 31) == 0) sm[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0;
    for (int w = 0; w < RED_THREADS / 32; ++w) t += sm[w];
    part[blockIdx.x] = t;
  }
}

__global__ void linf_partial_kernel(const double* __restrict__ a, long n, double* __restrict__ part) {
  pdl_wait();
  __shared__ double sm[RED_THREADS / 32];
  double s = 0;
  for (long i = long(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += long(gridDim.x) * blockDim.x) s = fmax(s, fabs(a[i]));
  for (int o = 16; o; o >>= 1) s = fmax(s, __shfl_down_sync(0xffffffffu, s, o));
  if ((threadIdx.x & 31) == 0) sm[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0;
    for (int w = 0; w < RED_THREADS / 32; ++w) t = fmax(t, sm[w]);
    part[blockIdx.x] = t;
  }
}

// Fixed-order final reduction by one CTA of FIN_THREADS; op 0 = sum, 1 = max.
// Also derives the PCG scalars: what = 0: rho -> beta = rho/rho_old;
// what = 1: sq -> alpha, -alpha, breakdown flag; what = 2: norm; what = 4: norm
// and rho_old = rho (the end of an iteration).
constexpr int FIN_THREADS = 256;
__global__ void finish_reduce_kernel(const double* __restrict__ part, int np, int op, double* scal, int what) {
  pdl_wait();
  __shared__ double sm[FIN_THREADS];
  double s = 0;
  for (int i = threadIdx.x; i < np; i += FIN_THREADS) s = op ? fmax(s, part[i]) : s + part[i];
  sm[threadIdx.x] = s;
  __syncthreads();
  for (int w = FIN_THREADS / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w) sm[threadIdx.x] = op ? fmax(sm[threadIdx.x], sm[threadIdx.x + w]) : sm[threadIdx.x] + sm[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    const double t = sm[0];
    if (what == 0) {
      scal[0] = t;               // rho
      scal[4] = t / scal[1];     // beta = rho / rho_old
    } else if (what == 1) {
      scal[2] = t;               // s.q
      if (!(t > 0)) scal[7] = 1;  // indefinite or singular (CONJUGATE_GRADIENT.cpp:49-52)
      scal[5] = scal[0] / t;     // alpha
      scal[6] = -scal[5];
    } else if (what == 2) {
      scal[3] = t;
    } else if (what == 4) {
      scal[3] = t;
      scal[1] = scal[0];
    } else {
      scal[8] = t;
    }
  }
}

// The V-cycle's z into q with Project and Project_Nullspace (KRYLOV_SYSTEM_BASE.cpp:25-31),
// and per-CTA partials of rho = q.r (CONJUGATE_GRADIENT.cpp:41); z may alias q.
template <typename TS>
__global__ void precond_out_kernel(const TS* z, double* q, const double* __restrict__ f,
                                   const uint32_t* __restrict__ flags, long N, double* __restrict__ part) {
  pdl_wait();
  __shared__ double sm[RED_THREADS / 32];
  double s = 0;
  for (long i = long(blockIdx.x) * blockDim.x + threadIdx.x; i < N; i += long(gridDim.x) * blockDim.x) {
    const uint32_t fl = flags[i];
#pragma unroll
    for (int v = 0; v < 3; ++v) {
      const long k = i + v * N;
      const double val = ((fl & ACTIVE_NODE) && !(fl & (DIR_X << v))) ? double(z[k]) : 0.0;
      q[k] = val;
      s += val * f[k];
    }
  }
  for (int o = 16; o; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
  if ((threadIdx.x & 31) == 0) sm[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0;
    for (int w = 0; w < RED_THREADS / 32; ++w) t += sm[w];
    part[blockIdx.x] = t;
  }
}

// precond_out_kernel for the packed single-precision level-0 iterate
template <typename T>
__global__ void precond_out4_kernel(const typename Pack4<T>::type* __restrict__ z4, double* q, const double* __restrict__ f,
                                    const uint32_t* __restrict__ flags, long N, double* __restrict__ part) {
  pdl_wait();
  __shared__ double sm[RED_THREADS / 32];
  double s = 0;
  for (long i = long(blockIdx.x) * blockDim.x + threadIdx.x; i < N; i += long(gridDim.x) * blockDim.x) {
    const uint32_t fl = flags[i];
    const auto z = z4[i];
    const double zc[3] = {double(z.x), double(z.y), double(z.z)};
#pragma unroll
    for (int v = 0; v < 3; ++v) {
      const long k = i + v * N;
      const double val = ((fl & ACTIVE_NODE) && !(fl & (DIR_X << v))) ? double(zc[v]) : 0.0;
      q[k] = val;
      s += val * f[k];
    }
  }
  for (int o = 16; o; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
  if ((threadIdx.x & 31) == 0) sm[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0;
    for (int w = 0; w < RED_THREADS / 32; ++w) t += sm[w];
    part[blockIdx.x] = t;
  }
}

// End of a PCG iteration (CONJUGATE_GRADIENT.cpp:54-57, 32-33): x += alpha s,
// r -= alpha q (float-rounded like CG_VECTOR in the reference mode), then
// Project_Nullspace(r), per-CTA partials of |r|_inf and, when b32 is given, the
// single-precision copy of r that the next V-cycle starts from.
__global__ void cg_update_kernel(double* x, const double* __restrict__ s, double* f, const double* __restrict__ q,
                                 const double* __restrict__ scal, const uint32_t* __restrict__ flags, long N,
                                 int float_round, float* __restrict__ b32, double* __restrict__ part) {
  pdl_wait();
  __shared__ double sm[RED_THREADS / 32];
  const double a = scal[5], na = scal[6];
  double m = 0;
  for (long i = long(blockIdx.x) * blockDim.x + threadIdx.x; i < N; i += long(gridDim.x) * blockDim.x) {
    const bool act = flags[i] & ACTIVE_NODE;
#pragma unroll
    for (int v = 0; v < 3; ++v) {
      const long k = i + v * N;
      double xv, fv;
      if (float_round) {
        xv = double(__fadd_rn(__fmul_rn(float(a), float(s[k])), float(x[k])));
        fv = double(__fadd_rn(__fmul_rn(float(na), float(q[k])), float(f[k])));
      } else {
        xv = a * s[k] + x[k];
        fv = na * q[k] + f[k];
      }
      if (!act) fv = 0;
      x[k] = xv;
      f[k] = fv;
      if (b32) b32[k] = float(fv);
      m = fmax(m, fabs(fv));
    }
  }
  for (int o = 16; o; o >>= 1) m = fmax(m, __shfl_down_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0) sm[threadIdx.x >> 5] = m;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0;
    for (int w = 0; w < RED_THREADS / 32; ++w) t = fmax(t, sm[w]);
    part[blockIdx.x] = t;
  }
}

// precond_out4_kernel over node pairs: two nodes per thread with 16-byte loads and
// stores (N is a multiple of 128), the same arithmetic per node.  The pair
// kernels skip pairs of inactive nodes: there every PCG vector is zero for the
// whole solve (Project_Nullspace zeroes them, K u vanishes where no active cell
// touches a node, x starts at zero), so only the flags are read for them and
// the sectors that hold no active node are never fetched.
template <typename T>
__global__ void __launch_bounds__(RED_THREADS, 4) precond_out4_pair_kernel(const typename Pack4<T>::type* __restrict__ z4,
                                                                       double* __restrict__ q,
                                                                       const double* __restrict__ f,
                                                                       const uint32_t* __restrict__ flags, long N,
                                                                       double* __restrict__ part) {
  pdl_wait();
  __shared__ double sm[RED_THREADS / 32];
  double s = 0;
  const long P = N >> 1;
  for (long p = long(blockIdx.x) * blockDim.x + threadIdx.x; p < P; p += long(gridDim.x) * blockDim.x) {
    const uint2 fl = reinterpret_cast<const uint2*>(flags)[p];
    if (!((fl.x | fl.y) & ACTIVE_NODE)) continue;
    const auto za = z4[2 * p], zb = z4[2 * p + 1];
    const double zc[2][3] = {{double(za.x), double(za.y), double(za.z)}, {double(zb.x), double(zb.y), double(zb.z)}};
    const uint32_t fls[2] = {fl.x, fl.y};
#pragma unroll
    for (int v = 0; v < 3; ++v) {
      double2 out;
      const double2 fv = reinterpret_cast<const double2*>(f + v * N)[p];
      out.x = ((fls[0] & ACTIVE_NODE) && !(fls[0] & (DIR_X << v))) ? zc[0][v] : 0.0;
      out.y = ((fls[1] & ACTIVE_NODE) && !(fls[1] & (DIR_X << v))) ? zc[1][v] : 0.0;
      reinterpret_cast<double2*>(q + v * N)[p] = out;
      s += out.x * fv.x;
      s += out.y * fv.y;
    }
  }
  for (int o = 16; o; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
  if ((threadIdx.x & 31) == 0) sm[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0;
    for (int w = 0; w < RED_THREADS / 32; ++w) t += sm[w];
    part[blockIdx.x] = t;
  }
}

// cg_update_kernel over node pairs (16-byte loads and stores), the same arithmetic per node.
__global__ void __launch_bounds__(RED_THREADS, 4) cg_update_pair_kernel(double* __restrict__ x, const double* __restrict__ s,
                                                                    double* __restrict__ f, const double* __restrict__ q,
                                                                    const double* __restrict__ scal,
                                                                    const uint32_t* __restrict__ flags, long N,
                                                                    int float_round, float* __restrict__ b32,
                                                                    double* __restrict__ part) {
  pdl_wait();
  __shared__ double sm[RED_THREADS / 32];
  const double a = scal[5], na = scal[6];
  double m = 0;
  const long P = N >> 1;
  for (long p = long(blockIdx.x) * blockDim.x + threadIdx.x; p < P; p += long(gridDim.x) * blockDim.x) {
    const uint2 fl = reinterpret_cast<const uint2*>(flags)[p];
    const bool act[2] = {(fl.x & ACTIVE_NODE) != 0, (fl.y & ACTIVE_NODE) != 0};
    if (!(act[0] || act[1])) continue;
#pragma unroll
    for (int v = 0; v < 3; ++v) {
      const long o = v * (N >> 1) + p;
      const double2 xv = reinterpret_cast<const double2*>(x)[o], sv = reinterpret_cast<const double2*>(s)[o];
      const double2 fv = reinterpret_cast<const double2*>(f)[o], qv = reinterpret_cast<const double2*>(q)[o];
      double2 xo, fo;
      if (float_round) {
        xo.x = double(__fadd_rn(__fmul_rn(float(a), float(sv.x)), float(xv.x)));
        xo.y = double(__fadd_rn(__fmul_rn(float(a), float(sv.y)), float(xv.y)));
        fo.x = double(__fadd_rn(__fmul_rn(float(na), float(qv.x)), float(fv.x)));
        fo.y = double(__fadd_rn(__fmul_rn(float(na), float(qv.y)), float(fv.y)));
      } else {
        xo.x = a * sv.x + xv.x;
        xo.y = a * sv.y + xv.y;
        fo.x = na * qv.x + fv.x;
        fo.y = na * qv.y + fv.y;
      }
      if (!act[0]) fo.x = 0;
      if (!act[1]) fo.y = 0;
      reinterpret_cast<double2*>(x)[o] = xo;
      reinterpret_cast<double2*>(f)[o] = fo;
      if (b32) reinterpret_cast<float2*>(b32)[o] = make_float2(float(fo.x), float(fo.y));
      m = fmax(m, fmax(fabs(fo.x), fabs(fo.y)));
    }
  }
  for (int o = 16; o; o >>= 1) m = fmax(m, __shfl_down_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0) sm[threadIdx.x >> 5] = m;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0;
    for (int w = 0; w < RED_THREADS / 32; ++w) t = fmax(t, sm[w]);
    part[blockIdx.x] = t;
  }
}

// dst = c*x + y over node pairs of three-component fields [3][N] (16-byte loads
// and stores), grid-stride; pairs of inactive nodes are skipped (both operands
// are zero there)
__global__ void __launch_bounds__(RED_THREADS, 4) axpy_pair_kernel(double* dst, const double* __restrict__ scal, int slot,
                                                               const double* xv, const double* yv, long N,
                                                               int float_round, const uint32_t* __restrict__ flags) {
  pdl_wait();
  const double c = scal[slot];
  const long P = N >> 1;
  for (long p = long(blockIdx.x) * blockDim.x + threadIdx.x; p < P; p += long(gridDim.x) * blockDim.x) {
    const uint2 fl = reinterpret_cast<const uint2*>(flags)[p];
    if (!((fl.x | fl.y) & ACTIVE_NODE)) continue;
#pragma unroll
    for (int v = 0; v < 3; ++v) {
      const long o = v * P + p;
      const double2 a = reinterpret_cast<const double2*>(xv)[o], b = reinterpret_cast<const double2*>(yv)[o];
      double2 r;
      if (float_round) {
        r.x = double(__fadd_rn(__fmul_rn(float(c), float(a.x)), float(b.x)));
        r.y = double(__fadd_rn(__fmul_rn(float(c), float(a.y)), float(b.y)));
      } else {
        r.x = c * a.x + b.x;
        r.y = c * a.y + b.y;
      }
      reinterpret_cast<double2*>(dst)[o] = r;
    }
  }
}

__global__ void rho_shift_kernel(double* scal) {
  pdl_wait(); scal[1] = scal[0]; }

// dst = c*x + y, c = scal[slot]; optionally in single precision like the
// reference's float-rounded CG_VECTOR::Copy (CG_VECTOR.cpp:96-114)
__global__ void axpy_kernel(double* dst, const double* __restrict__ scal, int slot, const double* xv, const double* yv,
                            long n, int float_round) {
  pdl_wait();
  long i = long(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double c = scal[slot];
  if (float_round) dst[i] = double(__fadd_rn(__fmul_rn(float(c), float(xv[i])), float(yv[i])));
  else dst[i] = c * xv[i] + yv[i];
}

// r = r - q with optional float rounding (CG_VECTOR::operator-=, CG_VECTOR.cpp:35-52)
__global__ void sub_kernel(double* r, const double* __restrict__ q, long n, int float_round) {
  pdl_wait();
  long i = long(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= n) return;
  if (float_round) r[i] = double(__fsub_rn(float(r[i]), float(q[i])));
  else r[i] -= q[i];
}

__global__ void scatter_lift_kernel(double* u, const int* __restrict__ node, const int* __restrict__ axis,
                                    const double* __restrict__ val, int n, long N) {
  pdl_wait();
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) u[node[i] + axis[i] * N] = val[i];
}

__global__ void scatter_force_kernel(double* s, const int* __restrict__ node, const double* __restrict__ val, int n, long N) {
  pdl_wait();
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  for (int v = 0; v < 3; ++v) s[node[i] + v * N] = val[3 * i + v];
}

__global__ void add_kernel(double* a, const double* __restrict__ b, long n) {
  pdl_wait();
  long i = long(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i < n) a[i] += b[i];
}

// Output packing (SPGrid_CPU_Solver.cpp:343-364): per input block node
// (u_x, u_y, u_z, max_v |r_v|)
__global__ void pack_kernel(int nin, const int* __restrict__ in_block, const int* __restrict__ in_zoff,
                            const double* __restrict__ u, const double* __restrict__ r, long N, double* __restrict__ out) {
  pdl_wait();
  long t = long(blockIdx.x) * blockDim.x + threadIdx.x;
  if (t >= long(nin) * 64) return;
  int b = int(t >> 6), e = int(t & 63);
  int blk = in_block[b];
  double* o = out + t * 4;
  if (blk < 0) {
    o[0] = o[1] = o[2] = o[3] = 0;
    return;
  }
  int ii = e >> 4, jj = (e >> 2) & 3, kk = e & 3;
  long n = long(blk) * 128 + ii * 32 + jj * 8 + (kk + in_zoff[b]);
  double m = 0;
  for (int v = 0; v < 3; ++v) {
    o[v] = u[n + v * N];
    m = fmax(m, fabs(r[n + v * N]));
  }
  o[3] = m;
}

// SIMP sensitivity per input-block cell (topo_opt/objective/minimal_compliance.cpp:86-146):
// s_e = u_e^T (mu0 K_mu + lambda0 K_la) u_e (no dx), dc = p rho^(p-1) (1-Emin) s_e,
// objective term s_e (Emin + rho^p (1-Emin)).
__global__ void sensitivity_kernel(int nin, const int* __restrict__ in_block, const int* __restrict__ in_zoff,
                                   const int* __restrict__ nbr, const double* __restrict__ u, long N,
                                   const double* __restrict__ rho, double penalty, double emin, double* __restrict__ dc,
                                   double* __restrict__ se, double* __restrict__ obj_part) {
  long t = long(blockIdx.x) * blockDim.x + threadIdx.x;
  double objv = 0;
  if (t < long(nin) * 64) {
    int b = int(t >> 6), e = int(t & 63);
    int blk = in_block[b];
    double r = rho[t], s = 0;
    if (blk >= 0 && r > 0) {
      int x = e >> 4, y = (e >> 2) & 3, z = (e & 3) + in_zoff[b];
      double ue[8][3];
      for (int a = 0; a < 8; ++a) {
        int nx = x + (a >> 2), ny = y + ((a >> 1) & 1), nz = z + (a & 1);
        int d = (nx > 3 ? 2 : 1) * 9 + (ny > 3 ? 2 : 1) * 3 + (nz > 7 ? 2 : 1);
        int nb = nbr[long(blk) * 27 + d];
        for (int v = 0; v < 3; ++v)
          ue[a][v] = nb < 0 ? 0.0 : u[long(nb) * 128 + ((nx & 3) << 5) + ((ny & 3) << 3) + (nz & 7) + v * N];
      }
      for (int a = 0; a < 8; ++a)
        for (int bb = 0; bb < 8; ++bb) {
          const int k = (a * 8 + bb) * 9;
          for (int i = 0; i < 3; ++i)
            s += ue[a][i] * (c_Kc64[k + i * 3] * ue[bb][0] + c_Kc64[k + i * 3 + 1] * ue[bb][1] + c_Kc64[k + i * 3 + 2] * ue[bb][2]);
        }
      dc[t] = s * pow(r, penalty - 1.0) * penalty * (1 - emin);
      objv = s * (emin + pow(r, penalty) * (1 - emin));
    } else {
      dc[t] = 0;
    }
    se[t] = s;
  }
  // block partial of the objective (fixed order)
  __shared__ double sm[256];
  sm[threadIdx.x] = objv;
  __syncthreads();
  for (int o = 128; o; o >>= 1) {
    if (threadIdx.x < o) sm[threadIdx.x] += sm[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) obj_part[blockIdx.x] = sm[0];
}

// Gradient of the compliance per input-block cell for the PyTorch layer:
// grad = factor * (*scale) * p rho^(p-1) (1-Emin) u_e^T K0 u_e (0 for empty cells),
// u in the level-0 layout [3][N] (a saved solution).
__global__ void sensitivity_grad_kernel(int nin, const int* __restrict__ in_block, const int* __restrict__ in_zoff,
                                        const int* __restrict__ nbr, const double* __restrict__ u, long N,
                                        const double* __restrict__ rho, double penalty, double emin, double factor,
                                        const double* __restrict__ scale, double* __restrict__ grad) {
  const long t = long(blockIdx.x) * blockDim.x + threadIdx.x;
  if (t >= long(nin) * 64) return;
  const int b = int(t >> 6), e = int(t & 63);
  const int blk = in_block[b];
  const double r = rho[t];
  if (blk < 0 || !(r > 0)) {
    grad[t] = 0;
    return;
  }
  const int x = e >> 4, y = (e >> 2) & 3, z = (e & 3) + in_zoff[b];
  double ue[8][3];
  for (int a = 0; a < 8; ++a) {
    const int nx = x + (a >> 2), ny = y + ((a >> 1) & 1), nz = z + (a & 1);
    const int d = (nx > 3 ? 2 : 1) * 9 + (ny > 3 ? 2 : 1) * 3 + (nz > 7 ? 2 : 1);
    const int nb = nbr[long(blk) * 27 + d];
    for (int v = 0; v < 3; ++v)
      ue[a][v] = nb < 0 ? 0.0 : u[long(nb) * 128 + ((nx & 3) << 5) + ((ny & 3) << 3) + (nz & 7) + v * N];
  }
  double s = 0;
  for (int a = 0; a < 8; ++a)
    for (int bb = 0; bb < 8; ++bb) {
      const int k = (a * 8 + bb) * 9;
      for (int i = 0; i < 3; ++i)
        s += ue[a][i] * (c_Kc64[k + i * 3] * ue[bb][0] + c_Kc64[k + i * 3 + 1] * ue[bb][1] + c_Kc64[k + i * 3 + 2] * ue[bb][2]);
    }
  grad[t] = factor * (scale ? *scale : 1.0) * s * pow(r, penalty - 1.0) * penalty * (1 - emin);
}

// f.u over the loaded nodes (one value per node, the last force entry of a node,
// as the solve assembles them), summed in a fixed order by one CTA.
__global__ void compliance_kernel(const int* __restrict__ node, const double* __restrict__ val, int n,
                                  const double* __restrict__ x, long N, double* __restrict__ out) {
  __shared__ double sm[256];
  double s = 0;
  for (int k = threadIdx.x; k < n; k += 256)
    for (int v = 0; v < 3; ++v) s += val[3 * k + v] * x[node[k] + v * N];
  sm[threadIdx.x] = s;
  __syncthreads();
  for (int o = 128; o; o >>= 1) {
    if (threadIdx.x < o) sm[threadIdx.x] += sm[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) *out = sm[0];
}

// New densities on the device: bit 0 of *bad for a non-finite stiffness, bit 1
// for a cell whose material status (E != 0) would change.
__global__ void simp_E_check_kernel(int nin, const int* __restrict__ in_block, const int* __restrict__ in_zoff,
                                    const double* __restrict__ rho, double penalty, double emin, double rho_min,
                                    double mu0, const double* __restrict__ E, int* bad) {
  const long t = long(blockIdx.x) * blockDim.x + threadIdx.x;
  if (t >= long(nin) * 64) return;
  const int b = int(t >> 6), e = int(t & 63);
  const int blk = in_block[b];
  if (blk < 0) return;
  const double d = rho[t];
  double val = 0;
  if (d > 0) val = penalty != 0 ? (1 - emin) * pow(fmax(rho_min, d), penalty) + emin : d;
  const double old = E[long(blk) * 128 + (e >> 4) * 32 + ((e >> 2) & 3) * 8 + (e & 3) + in_zoff[b]];
  if (!isfinite(val)) atomicOr(bad, 1);
  if ((val * mu0 != 0) != (old * mu0 != 0)) atomicOr(bad, 2);
}

void Solver::dot(const double* a, const double* b, double* out_unused) {
  (void)out_unused;
  launch(dot_partial_kernel, RED_BLOCKS, RED_THREADS, 0, a, b, 3 * N0(), red.p);
  launch_counter += 1;
}

void Solver::linf(const double* a, double*) {
  launch(linf_partial_kernel, RED_BLOCKS, RED_THREADS, 0, a, 3 * N0(), red.p);
  launch(finish_reduce_kernel, 1, FIN_THREADS, 0, red.p, RED_BLOCKS, 1, scal.p, 2);
  launch_counter += 2;
}

void Solver::axpy(double* dst, double, int slot, const double* xv, const double* yv) {
  launch(axpy_kernel, blocks_for(3 * N0(), 256), 256, 0, dst, scal.p, slot, xv, yv, 3 * N0(), round_ref() ? 1 : 0);
  ++launch_counter;
}

// z = M^-1 r into q (z and q share storage, SPGrid_CPU_Solver.cpp:91-92), then
// Project and Project_Nullspace (KRYLOV_SYSTEM_BASE.cpp:25-31), fused with the
// partial sums of rho = q.r.  In mixed precision the V-cycle starts from the
// FP32 copy of r in level 0's b, written by stage_residual() or by the previous
// iteration's update.
int Solver::precondition() {
  Level<double>& l0 = *L64[0];
  const long N = l0.N;
  int parts = RED_BLOCKS;
  if (P.disable_mg) {
    SGS_CUDA(cudaMemcpyAsync(q.p, f.p, 3 * N * sizeof(double), cudaMemcpyDeviceToDevice, stream));
    launch(precond_out_kernel<double>, RED_BLOCKS, RED_THREADS, 0, q.p, q.p, f.p, l0.flags.p, N, red.p);
  } else if (mixed()) {
    Level<float>& m0 = *L32[0];
    if (packed0()) {
      vcycle<float>(m0.b.p, nullptr);
      launch(precond_out4_pair_kernel<float>, PAIR_BLOCKS, RED_THREADS, 0, m0.u4.p, q.p, f.p, l0.flags.p, N, red.p);
      parts = PAIR_BLOCKS;
    } else {
      vcycle<float>(m0.b.p, m0.u.p);
      launch(precond_out_kernel<float>, RED_BLOCKS, RED_THREADS, 0, m0.u.p, q.p, f.p, l0.flags.p, N, red.p);
    }
  } else if (packed0()) {
    vcycle<double>(f.p, nullptr);
    launch(precond_out4_pair_kernel<double>, PAIR_BLOCKS, RED_THREADS, 0, l0.u4.p, q.p, f.p, l0.flags.p, N, red.p);
    parts = PAIR_BLOCKS;
  } else {
    vcycle<double>(f.p, q.p);
    launch(precond_out_kernel<double>, RED_BLOCKS, RED_THREADS, 0, q.p, q.p, f.p, l0.flags.p, N, red.p);
  }
  ++launch_counter;
  return parts;
}

// Inner solve of a large bottom level: CG on its unknowns (see InnerSolve).
void Solver::inner_pcg(int l) {
  Level<double>& D = *L64[l];
  const long N = D.N, n3 = 3 * N;
  const int rb = int(std::min<long>(RED_BLOCKS, std::max<long>(1, (n3 + RED_THREADS - 1) / RED_THREADS)));
  auto dotp = [&](const double* a, const double* b, int what) {
    launch(dot_partial_kernel, rb, RED_THREADS, 0, a, b, n3, red.p);
    launch(finish_reduce_kernel, 1, FIN_THREADS, 0, red.p, rb, 0, ib.scal.p, what);
    launch_counter += 2;
  };
  double init[16] = {0};
  init[1] = 1e300;  // rho_old: beta = 0 in the first iteration
  SGS_CUDA(cudaMemcpyAsync(ib.scal.p, init, sizeof(init), cudaMemcpyHostToDevice, stream));
  ib.x.zero(stream);
  ib.p.zero(stream);
  launch(inner_mask_kernel, blocks_for(N, 256), 256, 0, ib.r.p, ib.b.p, D.spokes.p, N);
  dotp(ib.r.p, ib.r.p, 3);
  double h[16];
  SGS_CUDA(cudaMemcpyAsync(h, ib.scal.p, sizeof(h), cudaMemcpyDeviceToHost, stream));
  SGS_CUDA(cudaStreamSynchronize(stream));
  const double b2 = h[8];
  if (!(b2 > 0)) return;  // x = 0
  const double tol2 = 1e-26 * b2;
  double best = b2;
  int since_best = 0;
  for (int it = 1; it <= 300; ++it) {
    // z = V(r) on the unknowns
    SGS_CUDA(cudaMemcpyAsync(D.b.p, ib.r.p, n3 * sizeof(double), cudaMemcpyDeviceToDevice, stream));
    inner_vcycle(l);
    launch(inner_mask_kernel, blocks_for(N, 256), 256, 0, ib.z.p, D.u.p, D.spokes.p, N);
    dotp(ib.r.p, ib.z.p, 0);                                     // rho, beta = rho / rho_old
    launch(axpy_kernel, blocks_for(n3, 256), 256, 0, ib.p.p, ib.scal.p, 4, ib.p.p, ib.z.p, n3, 0);  // p = beta p + z
    launch(rho_shift_kernel, 1, 1, 0, ib.scal.p);
    stencil<double, SOP_MUL>(l, nullptr, D.nb, ib.p.p, nullptr, nullptr, ib.q.p, 0);
    launch(inner_mask_kernel, blocks_for(N, 256), 256, 0, ib.q.p, ib.q.p, D.spokes.p, N);
    dotp(ib.p.p, ib.q.p, 1);                                     // alpha, breakdown flag
    launch(axpy_kernel, blocks_for(n3, 256), 256, 0, ib.x.p, ib.scal.p, 5, ib.p.p, ib.x.p, n3, 0);  // x += alpha p
    launch(axpy_kernel, blocks_for(n3, 256), 256, 0, ib.r.p, ib.scal.p, 6, ib.q.p, ib.r.p, n3, 0);  // r -= alpha q
    dotp(ib.r.p, ib.r.p, 3);
    launch_counter += 6;
    SGS_CUDA(cudaMemcpyAsync(h, ib.scal.p, sizeof(h), cudaMemcpyDeviceToHost, stream));
    SGS_CUDA(cudaStreamSynchronize(stream));
    if (h[7] != 0 || !std::isfinite(h[8]))
      throw CudaError("the bottom level's operator is not positive definite", SGS_ERR_BREAKDOWN);
    if (h[8] <= tol2) break;
    if (h[8] < 0.5 * best) {
      best = h[8];
      since_best = 0;
    } else if (++since_best >= 8) {
      break;  // round-off floor reached
    }
  }
}

// the FP32 copy of the residual for the mixed V-cycle
void Solver::stage_residual() {
  if (!mixed() || P.disable_mg) return;
  const long n3 = 3 * N0();
  launch(convert_kernel<float, double>, blocks_for(n3, 256), 256, 0, L32[0]->b.p, f.p, n3);
  ++launch_counter;
}

// One PCG iteration after the convergence test (CONJUGATE_GRADIENT.cpp:41-57) plus
// the next iteration's Project_Nullspace and norm (:32-33).
void Solver::record_iteration() {
  Level<double>& l0 = *L64[0];
  const int parts = precondition();                                      // q = z, rho partials
  launch(finish_reduce_kernel, 1, FIN_THREADS, 0, red.p, parts, 0, scal.p, 0);  // rho, beta
  launch(axpy_pair_kernel, PAIR_BLOCKS, RED_THREADS, 0, s.p, scal.p, 4, s.p, q.p, N0(),
         round_ref() ? 1 : 0, l0.flags.p);                               // s = beta*s + z
  level0<double, OP_KUP>(s.p, nullptr, q.p);                             // q = K s, Project, s.q partials
  launch(finish_reduce_kernel, 1, FIN_THREADS, 0, red.p, l0.nb, 0, scal.p, 1);       // alpha
  launch(cg_update_pair_kernel, PAIR_BLOCKS, RED_THREADS, 0, x.p, s.p, f.p, q.p, scal.p, l0.flags.p, l0.N,
         round_ref() ? 1 : 0, (mixed() && !P.disable_mg) ? L32[0]->b.p : (float*)nullptr, red.p);
  launch(finish_reduce_kernel, 1, FIN_THREADS, 0, red.p, PAIR_BLOCKS, 1, scal.p, 4);  // |r|_inf, rho_old
  launch_counter += 4;
}

// The device-side PCG loop's record, at the head of Solver::loop_buf, followed
// by LOOP_HIST residual norms (the history of iterations base .. limit).
constexpr int LOOP_REC = 6, LOOP_HIST = 1024;  // in doubles
struct PcgLoop {
  double tol, norm;
  int it, maxit, limit, base, stopped, breakdown;
};
static_assert(sizeof(PcgLoop) <= LOOP_REC * sizeof(double), "loop record size");

// The convergence test of the device-side PCG loop (CONJUGATE_GRADIENT.cpp:32-40),
// run before the first iteration and at the end of every iteration: records
// |r|_inf of iteration `it`; stops on convergence, at the iteration cap, on a
// breakdown (a non-positive s.q, CONJUGATE_GRADIENT.cpp:49-52) or on a
// non-finite norm; otherwise counts the iteration and keeps the WHILE node
// running, up to `limit`, where the host takes the history out and relaunches.
// The loop therefore ends after at most limit - base iterations.
__global__ void pcg_check_kernel(const double* __restrict__ scal, double* loop, cudaGraphConditionalHandle h) {
  pdl_wait();
  PcgLoop* st = reinterpret_cast<PcgLoop*>(loop);
  const int it = st->it;
  const double norm = scal[3];
  loop[LOOP_REC + (it - st->base)] = norm;
  const bool breakdown = scal[7] != 0;
  const bool stop = breakdown || !isfinite(norm) || norm <= st->tol || it >= st->maxit;
  const bool more = !stop && it < st->limit;
  if (more) st->it = it + 1;
  st->norm = norm;
  st->stopped = stop;
  st->breakdown = breakdown;
  cudaGraphSetConditional(h, more ? 1u : 0u);
}

// A graph [head] -> WHILE([body]) whose condition the kernels that head and
// body launch set: head(h) and body(h) are captured from the solver stream.
// Returns the instantiated graph, or nullptr with the reason in *why where the
// runtime refuses a step (conditional nodes need CUDA 12.4 or later).
cudaGraphExec_t Solver::while_graph(const std::function<void(cudaGraphConditionalHandle)>& head,
                                    const std::function<void(cudaGraphConditionalHandle)>& body, std::string* why) {
  cudaGraph_t g = nullptr;
  cudaGraphExec_t exec = nullptr;
  bool capturing = false;
  auto give_up = [&](const char* what, cudaError_t e) -> cudaGraphExec_t {
    if (capturing) {
      cudaGraph_t partial = nullptr;
      cudaStreamEndCapture(stream, &partial);
    }
    if (g) cudaGraphDestroy(g);
    cudaGetLastError();
    *why = std::string(what) + ": " + cudaGetErrorString(e);
    return nullptr;
  };
  cudaError_t e = cudaGraphCreate(&g, 0);
  if (e != cudaSuccess) return give_up("cudaGraphCreate", e);
  cudaGraphConditionalHandle h = 0;
  e = cudaGraphConditionalHandleCreate(&h, g, 0, cudaGraphCondAssignDefault);
  if (e != cudaSuccess) return give_up("cudaGraphConditionalHandleCreate", e);
  e = cudaStreamBeginCaptureToGraph(stream, g, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal);
  if (e != cudaSuccess) return give_up("cudaStreamBeginCaptureToGraph", e);
  capturing = true;
  head(h);
  e = cudaStreamEndCapture(stream, &g);
  capturing = false;
  if (e != cudaSuccess) return give_up("cudaStreamEndCapture", e);
  // the WHILE node follows the head's last nodes (those without dependents)
  size_t n = 0;
  SGS_CUDA(cudaGraphGetNodes(g, nullptr, &n));
  std::vector<cudaGraphNode_t> nodes(n), deps;
  SGS_CUDA(cudaGraphGetNodes(g, nodes.data(), &n));
  for (cudaGraphNode_t node : nodes) {
    size_t out = 0;
    SGS_CUDA(cudaGraphNodeGetDependentNodes(node, nullptr, &out));
    if (out == 0) deps.push_back(node);
  }
  cudaGraphNodeParams cp = {};
  cp.type = cudaGraphNodeTypeConditional;
  cp.conditional.handle = h;
  cp.conditional.type = cudaGraphCondTypeWhile;
  cp.conditional.size = 1;
  cudaGraphNode_t wnode;
  e = cudaGraphAddNode(&wnode, g, deps.data(), deps.size(), &cp);
  if (e != cudaSuccess) return give_up("cudaGraphAddNode (WHILE)", e);
  cudaGraph_t bg = cp.conditional.phGraph_out[0];
  e = cudaStreamBeginCaptureToGraph(stream, bg, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal);
  if (e != cudaSuccess) return give_up("cudaStreamBeginCaptureToGraph (body)", e);
  capturing = true;
  body(h);
  e = cudaStreamEndCapture(stream, &bg);
  capturing = false;
  if (e != cudaSuccess) return give_up("cudaStreamEndCapture (body)", e);
  e = cudaGraphInstantiate(&exec, g, 0);
  if (e != cudaSuccess) return give_up("cudaGraphInstantiate", e);
  SGS_CUDA(cudaGraphDestroy(g));
  return exec;
}

// Builds loop_graph once per operator set: [test] -> WHILE([iteration, test]).
// Returns false, and remembers why, where the runtime refuses conditional nodes.
bool Solver::build_loop_graph() {
  if (loop_graph) return true;
  if (loop_unavailable) return false;
  if (!loop_buf.p) loop_buf.alloc(LOOP_REC + LOOP_HIST);
  if (!h_loop) SGS_CUDA(cudaMallocHost(&h_loop, (LOOP_REC + LOOP_HIST) * sizeof(double)));
  loop_graph = while_graph(
      [&](cudaGraphConditionalHandle h) {  // the test before the first iteration
        launch(pcg_check_kernel, 1, 1, 0, (const double*)scal.p, loop_buf.p, h);
      },
      [&](cudaGraphConditionalHandle h) {
        const long before = launch_counter;
        record_iteration();
        launches_per_iteration = launch_counter - before;
        launch(pcg_check_kernel, 1, 1, 0, (const double*)scal.p, loop_buf.p, h);
        launch_counter += 2;  // the two tests
      },
      &loop_note);
  if (!loop_graph) loop_unavailable = true;
  return loop_graph != nullptr;
}

void Solver::solve() {
  Level<double>& l0 = *L64[0];
  const long N = l0.N, n3 = 3 * N;
  const int fr = round_ref() ? 1 : 0;
  history.clear();
  iterations = 0;
  solve_launches = 0;
  const long launches_before = launch_counter;
  if (!ev_start) {
    SGS_CUDA(cudaEventCreate(&ev_start));
    SGS_CUDA(cudaEventCreate(&ev_end));
  }
  SGS_CUDA(cudaEventRecord(ev_start, stream));
  // u = g on the listed Dirichlet nodes (SPGrid_CPU_Solver.cpp:241-285),
  // over the previous solution when warm starting
  auto lift = [&] {
    if (!P.lift_node.empty())
      launch(scatter_lift_kernel, blocks_for(long(P.lift_node.size()), 128), 128, 0, x.p, lift_node.p, lift_axis.p,
             lift_val.p, int(P.lift_node.size()), N);
  };
  // s = forces; Project; Project_Nullspace; f = s - K u; Project (:287-301)
  auto residual = [&] {
    s.zero(stream);
    if (!P.force_node.empty())
      launch(scatter_force_kernel, blocks_for(long(P.force_node.size()), 128), 128, 0, s.p, force_node.p,
             force_val.p, int(P.force_node.size()), N);
    project<double>(l0, s.p);
    project_null<double>(l0, s.p);
    level0<double, OP_RES>(x.p, s.p, f.p);
    project<double>(l0, f.p);
  };
  const bool warm = warm_u.p != nullptr;
  warm_reused = false;
  if (warm) {
    // keep the previous u only if forced or if it beats the zero guess (:247-277)
    SGS_CUDA(cudaMemcpyAsync(x.p, warm_u.p, n3 * sizeof(double), cudaMemcpyDeviceToDevice, stream));
    lift();
    residual();
    linf(f.p, nullptr);
    SGS_CUDA(cudaMemcpyAsync(h_scal, scal.p, 16 * sizeof(double), cudaMemcpyDeviceToHost, stream));
    SGS_CUDA(cudaStreamSynchronize(stream));
    warm_residual = h_scal[3];
    warm_reused = forced_reuse || warm_reference > warm_residual;
  }
  if (!warm_reused) {
    x.zero(stream);
    lift();
  }
  residual();
  SGS_CUDA(cudaMemcpyAsync(ubk.p, x.p, n3 * sizeof(double), cudaMemcpyDeviceToDevice, stream));
  q.zero(stream);
  s.zero(stream);
  linf(f.p, nullptr);
  SGS_CUDA(cudaMemcpyAsync(h_scal, scal.p, 16 * sizeof(double), cudaMemcpyDeviceToHost, stream));
  SGS_CUDA(cudaStreamSynchronize(stream));
  // the stopping rule is relative to the first call's zero-guess residual
  initial_residual = warm ? warm_reference : h_scal[3];
  const double tol = P.tolerance * initial_residual;
  auto t0 = std::chrono::steady_clock::now();
  x.zero(stream);
  // CONJUGATE_GRADIENT_4Ch::Solve: q = K x (= 0); r -= q; Project(r)
  level0<double, OP_KU>(x.p, nullptr, q.p);
  launch(sub_kernel, blocks_for(n3, 256), 256, 0, f.p, q.p, n3, fr);
  project<double>(l0, f.p);
  double init_scal[16] = {0};
  init_scal[1] = 3.40282346638528859811704183484516925440e+38;  // FLT_MAX (rho_old)
  SGS_CUDA(cudaMemcpyAsync(scal.p, init_scal, sizeof(init_scal), cudaMemcpyHostToDevice, stream));
  project_null<double>(l0, f.p);
  linf(f.p, nullptr);
  stage_residual();
  // The loop on the device: one graph launch runs iterations until the test
  // stops them (or pauses at the history buffer's end).  With an inner bottom
  // solve, whose iteration count is decided on the host, or without
  // conditional nodes: one graph launch per iteration after a host-side test.
  long capture_launches = 0;
  const bool use_graph = !inner();
  int it = 0;
  double norm = 0;
  bool breakdown = false;
  const int max_iterations = std::max(0, P.max_iterations);
  const long before_build = launch_counter;
  if (use_graph && build_loop_graph()) {
    capture_launches = launch_counter - before_build;
    PcgLoop* st = reinterpret_cast<PcgLoop*>(h_loop);
    for (;;) {
      const int hist = std::max(2, std::min(loop_history, LOOP_HIST));  // >= 2: every launch makes progress
      *st = PcgLoop{tol, 0.0, it, max_iterations, std::min(max_iterations, it + hist - 1), it, 0, 0};
      const int it0 = it, span = st->limit - it0 + 1;
      SGS_CUDA(cudaMemcpyAsync(loop_buf.p, h_loop, LOOP_REC * sizeof(double), cudaMemcpyHostToDevice, stream));
      SGS_CUDA(cudaGraphLaunch(loop_graph, stream));
      SGS_CUDA(cudaMemcpyAsync(h_loop, loop_buf.p, (LOOP_REC + span) * sizeof(double), cudaMemcpyDeviceToHost, stream));
      g_d2h_bytes += (LOOP_REC + span) * sizeof(double);
      SGS_CUDA(cudaStreamSynchronize(stream));
      it = st->it;
      solve_launches += 1 + long(it - it0) * (launches_per_iteration + 1);
      // a paused launch re-tests its last iteration at the next launch
      const int recorded = it - it0 + (st->stopped ? 1 : 0);
      for (int k = 0; k < recorded; ++k) history.push_back(h_loop[LOOP_REC + k]);
      if (st->stopped) {
        norm = st->norm;
        breakdown = st->breakdown != 0;
        break;
      }
    }
  } else {
    capture_launches = launch_counter - before_build;  // a refused loop graph's capture
    if (use_graph && !iter_graph) {
      cudaGraph_t g;
      long before = launch_counter;
      SGS_CUDA(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal));
      record_iteration();
      SGS_CUDA(cudaStreamEndCapture(stream, &g));
      SGS_CUDA(cudaGraphInstantiate(&iter_graph, g, 0));
      SGS_CUDA(cudaGraphDestroy(g));
      launches_per_iteration = launch_counter - before;
      capture_launches += launches_per_iteration;
    }
    for (;; ++it) {
      SGS_CUDA(cudaMemcpyAsync(h_scal, scal.p, 16 * sizeof(double), cudaMemcpyDeviceToHost, stream));
      g_d2h_bytes += 16 * sizeof(double);
      SGS_CUDA(cudaStreamSynchronize(stream));
      norm = h_scal[3];
      history.push_back(norm);
      breakdown = h_scal[7] != 0;
      if (breakdown || !std::isfinite(norm) || norm <= tol || it >= max_iterations) break;
      if (use_graph) {
        SGS_CUDA(cudaGraphLaunch(iter_graph, stream));
        solve_launches += launches_per_iteration;
      } else {
        record_iteration();
      }
    }
  }
  iterations = it;
  if (breakdown) {
    final_residual = norm;
    throw CudaError("CG detected an indefinite or singular operator", SGS_ERR_BREAKDOWN);
  }
  if (!std::isfinite(norm)) throw CudaError("non-finite residual", SGS_ERR_BREAKDOWN);
  final_residual = norm;
  launch(add_kernel, blocks_for(n3, 256), 256, 0, x.p, ubk.p, n3);
  ++launch_counter;
  SGS_CUDA(cudaEventRecord(ev_end, stream));
  SGS_CUDA(cudaGetLastError());
  SGS_CUDA(cudaStreamSynchronize(stream));
  solve_seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  check_tensor_core_waits();
  float ms = 0;
  SGS_CUDA(cudaEventElapsedTime(&ms, ev_start, ev_end));
  solve_device_seconds = ms * 1e-3;
  solve_launches += launch_counter - launches_before - (capture_launches);
}

// The output field, [input block][64 nodes][4] doubles, copied straight into
// the caller's buffer.
// Pinned staging for pitched read-backs, kept for the process: two halves of
// 32 MiB, so that the copy of one chunk overlaps the host scatter of the last.
static std::mutex g_staging_mutex;
static char* g_staging = nullptr;
constexpr size_t STAGING_HALF = size_t(32) << 20;

// Chunks of the source go into one half of the staging buffer (copied by the
// host threads) while the other half's copy to the device runs; the call ends
// when the last copy has left the buffer, so the next user finds it free.
void staged_h2d(void* dst, const void* src, size_t bytes, cudaStream_t s) {
  if (bytes == 0) return;
  std::lock_guard<std::mutex> lock(g_staging_mutex);
  if (!g_staging) SGS_CUDA(cudaMallocHost(reinterpret_cast<void**>(&g_staging), 2 * STAGING_HALF));
  cudaEvent_t done[2];
  SGS_CUDA(cudaEventCreateWithFlags(&done[0], cudaEventDisableTiming));
  SGS_CUDA(cudaEventCreateWithFlags(&done[1], cudaEventDisableTiming));
  const size_t nchunks = (bytes + STAGING_HALF - 1) / STAGING_HALF;
  cudaError_t err = cudaSuccess;
  for (size_t c = 0; c < nchunks && err == cudaSuccess; ++c) {
    const size_t off = c * STAGING_HALF, n = std::min(STAGING_HALF, bytes - off);
    char* half = g_staging + (c & 1) * STAGING_HALF;
    if (c >= 2) err = cudaEventSynchronize(done[c & 1]);  // that half's previous copy has left
    if (err != cudaSuccess) break;
    const char* from = static_cast<const char*>(src) + off;
    const long pieces = long((n + (size_t(1) << 20) - 1) >> 20);
#pragma omp parallel for schedule(static)
    for (long k = 0; k < pieces; ++k) {
      const size_t a = size_t(k) << 20;
      std::memcpy(half + a, from + a, std::min(size_t(1) << 20, n - a));
    }
    err = cudaMemcpyAsync(static_cast<char*>(dst) + off, half, n, cudaMemcpyHostToDevice, s);
    if (err == cudaSuccess) err = cudaEventRecord(done[c & 1], s);
  }
  const cudaError_t e0 = cudaEventSynchronize(done[0]), e1 = cudaEventSynchronize(done[1]);
  cudaEventDestroy(done[0]);
  cudaEventDestroy(done[1]);
  SGS_CUDA(err);
  SGS_CUDA(e0);
  SGS_CUDA(e1);
}

void Solver::pack_outputs(void* disp, size_t pitch) {
  const long nin = long(P.in_block.size());
  if (nin == 0) return;
  launch(pack_kernel, blocks_for(nin * 64, 256), 256, 0, int(nin), in_block.p, in_zoff.p, x.p, f.p, N0(), out_disp.p);
  const size_t row = 256 * sizeof(double), bytes = size_t(nin) * row;
  g_d2h_bytes += bytes;
  if (pitch == 0 || pitch == row) {
    SGS_CUDA(cudaMemcpyAsync(disp, out_disp.p, bytes, cudaMemcpyDeviceToHost, stream));
    SGS_CUDA(cudaStreamSynchronize(stream));
    return;
  }
  // records `pitch` bytes apart: chunks of rows through the pinned staging
  // buffer, each scattered by the host threads while the next one is copied
  std::lock_guard<std::mutex> lock(g_staging_mutex);
  if (!g_staging) SGS_CUDA(cudaMallocHost(reinterpret_cast<void**>(&g_staging), 2 * STAGING_HALF));
  const size_t rows_per = STAGING_HALF / row;
  const size_t nchunks = (size_t(nin) + rows_per - 1) / rows_per;
  cudaEvent_t done[2];
  SGS_CUDA(cudaEventCreateWithFlags(&done[0], cudaEventDisableTiming));
  SGS_CUDA(cudaEventCreateWithFlags(&done[1], cudaEventDisableTiming));
  auto issue = [&](size_t c) {
    const size_t r0 = c * rows_per, nr = std::min(rows_per, size_t(nin) - r0);
    SGS_CUDA(cudaMemcpyAsync(g_staging + (c & 1) * STAGING_HALF, reinterpret_cast<const char*>(out_disp.p) + r0 * row,
                             nr * row, cudaMemcpyDeviceToHost, stream));
    SGS_CUDA(cudaEventRecord(done[c & 1], stream));
  };
  issue(0);
  for (size_t c = 0; c < nchunks; ++c) {
    SGS_CUDA(cudaEventSynchronize(done[c & 1]));
    if (c + 1 < nchunks) issue(c + 1);
    const size_t r0 = c * rows_per, nr = std::min(rows_per, size_t(nin) - r0);
    const char* src = g_staging + (c & 1) * STAGING_HALF;
    char* dst = static_cast<char*>(disp) + r0 * pitch;
#pragma omp parallel for schedule(static)
    for (long r = 0; r < long(nr); ++r) std::memcpy(dst + size_t(r) * pitch, src + size_t(r) * row, row);
  }
  cudaEventDestroy(done[0]);
  cudaEventDestroy(done[1]);
}

double Solver::sensitivity(const double* rho_host, double penalty, double emin, double* dc_host, double* se_host) {
  const long nin = long(P.in_block.size());
  if (nin == 0) return 0;
  DevBuf<double> rho, dc, se, part;
  rho.upload(rho_host, size_t(nin) * 64, stream);
  dc.alloc(size_t(nin) * 64);
  se.alloc(size_t(nin) * 64);
  const unsigned nblk = blocks_for(nin * 64, 256);
  part.alloc(nblk);
  sensitivity_kernel<<<nblk, 256, 0, stream>>>(int(nin), in_block.p, in_zoff.p, L64[0]->nbr.p, x.p, N0(), rho.p, penalty,
                                               emin, dc.p, se.p, part.p);
  std::vector<double> hp(nblk);
  SGS_CUDA(cudaMemcpyAsync(dc_host, dc.p, nin * 64 * sizeof(double), cudaMemcpyDeviceToHost, stream));
  if (se_host) SGS_CUDA(cudaMemcpyAsync(se_host, se.p, nin * 64 * sizeof(double), cudaMemcpyDeviceToHost, stream));
  SGS_CUDA(cudaMemcpyAsync(hp.data(), part.p, nblk * sizeof(double), cudaMemcpyDeviceToHost, stream));
  SGS_CUDA(cudaStreamSynchronize(stream));
  double obj = 0;
  for (double v : hp) obj += v;
  return obj;
}

// Sensitivity filter of the driver (topo_opt/spgrid_topo_opt.cpp:527-579) on the
// input blocks; host arrays [input block][64].
void Solver::filter_dev(const double* rho, const double* dc0, double* dc1, double filter_size, double scale) {
  const long nin = long(P.in_block.size());
  if (nin == 0) return;
  if (!in_grid.p) {
    for (int v = 0; v < 3; ++v) in_gdim[v] = (P.resolution[v] + 3) / 4;
    std::vector<int32_t> g(size_t(in_gdim[0]) * in_gdim[1] * in_gdim[2], -1);
    for (long b = 0; b < nin; ++b)
      g[(size_t(P.in_base[3 * b] >> 2) * in_gdim[1] + (P.in_base[3 * b + 1] >> 2)) * in_gdim[2] +
        (P.in_base[3 * b + 2] >> 2)] = int32_t(b);
    in_grid.upload(g, stream);
    in_base_d.upload(P.in_base, stream);
  }
  filter_dc_kernel<<<blocks_for(nin * 64, 256), 256, 0, stream>>>(int(nin), in_base_d.p, in_grid.p, in_gdim[0],
                                                                  in_gdim[1], in_gdim[2], rho, dc0, dc1, filter_size,
                                                                  int(std::floor(filter_size)), scale);
  SGS_CUDA(cudaGetLastError());
}

void Solver::filter_sensitivity(const double* rho_h, const double* dc0_h, double* dc1_h, double filter_size) {
  const long nin = long(P.in_block.size());
  if (nin == 0) return;
  DevBuf<double> rho, dc0, dc1;
  rho.upload(rho_h, size_t(nin) * 64, stream);
  dc0.upload(dc0_h, size_t(nin) * 64, stream);
  dc1.alloc(size_t(nin) * 64);
  filter_dev(rho.p, dc0.p, dc1.p, filter_size, 1.0);
  SGS_CUDA(cudaMemcpyAsync(dc1_h, dc1.p, size_t(nin) * 64 * sizeof(double), cudaMemcpyDeviceToHost, stream));
  g_d2h_bytes += size_t(nin) * 64 * sizeof(double);
  SGS_CUDA(cudaStreamSynchronize(stream));
}

// One optimality-criteria update (topo_opt/optimizer/optimality_criterion.cpp:19-145):
// bisection on the Lagrange multiplier with the reference's bounds and stopping
// rule, each trial one pass over the cells on the GPU (sums reduced in a fixed
// order), then the densities of the final multiplier.  Returns the multiplier.
double Solver::oc_dev(double* rho, const double* dc0, const uint8_t* fx, double volume_fraction,
                      double step_limit, double minimum_density, double fixed_density, int smart_oc,
                      int exclude_fixed, int keep_inside, double* change) {
  const long n = long(P.in_block.size()) * 64;
  if (change) *change = 0;
  if (n == 0) return 0;
  DevBuf<double> part_s, part_c, part3;
  part_s.alloc(OC_BLOCKS);
  part_c.alloc(OC_BLOCKS);
  part3.alloc(3 * OC_BLOCKS);
  oc_stats_kernel<<<OC_BLOCKS, OC_THREADS, 0, stream>>>(n, rho, dc0, fx, part3.p);
  SGS_CUDA(cudaGetLastError());
  std::vector<double> h3(3 * OC_BLOCKS), hs(OC_BLOCKS), hc(OC_BLOCKS);
  SGS_CUDA(cudaMemcpyAsync(h3.data(), part3.p, h3.size() * sizeof(double), cudaMemcpyDeviceToHost, stream));
  SGS_CUDA(cudaStreamSynchronize(stream));
  double inside = 0, nfix = 0, neg_dc_min = 1e30;
  for (int k = 0; k < OC_BLOCKS; ++k) {
    inside += h3[3 * k];
    nfix += h3[3 * k + 1];
    neg_dc_min = std::min(neg_dc_min, h3[3 * k + 2]);
  }
  const double shift = smart_oc ? std::min(0.0, neg_dc_min) : 0.0;
  // Taichi's real is float64 in the driver (static_assert, spgrid_topo_opt.h:28-29):
  // the target, the bracket and the stopping factor are all double
  const double target = volume_fraction * (inside - (exclude_fixed ? nfix : 0));
  auto trial = [&](double mid, double* out, double* chg) {
    oc_trial_kernel<<<OC_BLOCKS, OC_THREADS, 0, stream>>>(n, rho, dc0, fx, mid, shift, step_limit, minimum_density,
                                                          fixed_density, exclude_fixed, out, part_s.p, part_c.p,
                                                          keep_inside);
    SGS_CUDA(cudaGetLastError());
    SGS_CUDA(cudaMemcpyAsync(hs.data(), part_s.p, OC_BLOCKS * sizeof(double), cudaMemcpyDeviceToHost, stream));
    if (chg) SGS_CUDA(cudaMemcpyAsync(hc.data(), part_c.p, OC_BLOCKS * sizeof(double), cudaMemcpyDeviceToHost, stream));
    SGS_CUDA(cudaStreamSynchronize(stream));
    double sum = 0;
    for (double v : hs) sum += v;
    if (chg) {
      *chg = 0;
      for (double v : hc) *chg = std::max(*chg, v);
    }
    return sum;
  };
  double mid = 0, lower = 1e-20, upper = 1e20;
  const double factor = 1 + 1e-7;
  while (lower * factor < upper) {
    mid = 0.5 * (lower + upper);
    const double sum = trial(mid, nullptr, nullptr);
    if (!(sum == sum)) throw CudaError("OC update produced a non-finite volume", SGS_ERR_BREAKDOWN);
    if (sum > target) lower = mid;
    else upper = mid;
  }
  double chg = 0;
  trial(mid, rho, &chg);
  if (change) *change = chg;
  return mid;
}

double Solver::oc_update(double* rho_h, const double* dc0_h, const uint8_t* fixed_h, double volume_fraction,
                         double step_limit, double minimum_density, double fixed_density, int smart_oc,
                         int exclude_fixed, double* change) {
  const long n = long(P.in_block.size()) * 64;
  if (change) *change = 0;
  if (n == 0) return 0;
  DevBuf<double> rho, dc0;
  DevBuf<uint8_t> fx;
  rho.upload(rho_h, size_t(n), stream);
  dc0.upload(dc0_h, size_t(n), stream);
  if (fixed_h) fx.upload(fixed_h, size_t(n), stream);
  const double mid = oc_dev(rho.p, dc0.p, fx.p, volume_fraction, step_limit, minimum_density, fixed_density, smart_oc,
                            exclude_fixed, 0, change);
  SGS_CUDA(cudaMemcpyAsync(rho_h, rho.p, size_t(n) * sizeof(double), cudaMemcpyDeviceToHost, stream));
  g_d2h_bytes += size_t(n) * sizeof(double);
  SGS_CUDA(cudaStreamSynchronize(stream));
  return mid;
}

// Device-resident design (the optimizer loop without host round trips).
void Solver::design_set(const double* rho_h, const uint8_t* fixed_h) {
  const size_t n = P.in_block.size() * 64;
  design_rho.upload(rho_h, n, stream);
  if (fixed_h) design_fixed.upload(fixed_h, n, stream);
  else design_fixed.release();
  design_dc.alloc(n);
  design_dc1.alloc(n);
  design_scratch.alloc(n);
  design_part.alloc(blocks_for(long(n), 256));
  SGS_CUDA(cudaStreamSynchronize(stream));
}

// One iteration of the driver's loop (Opt::iterate, spgrid_topo_opt.cpp:1289-1331,
// without page-map maintenance): solve, sensitivity, filter, OC update, and the
// new stiffness scales with rebuilt coarse operators and bottom inverse.
void Solver::design_step(const sgs_design_params& prm, sgs_design_result* out) {
  const long nin = long(P.in_block.size());
  if (!design_rho.p || nin == 0) throw CudaError("no design densities set", SGS_ERR_INPUT);
  const auto t0 = std::chrono::steady_clock::now();
  P.tolerance = prm.tolerance;
  solve();
  const auto t1 = std::chrono::steady_clock::now();
  const unsigned nblk = blocks_for(nin * 64, 256);
  sensitivity_kernel<<<nblk, 256, 0, stream>>>(int(nin), in_block.p, in_zoff.p, L64[0]->nbr.p, x.p, N0(),
                                               design_rho.p, P.penalty, P.minimum_stiffness, design_dc.p,
                                               design_scratch.p, design_part.p);
  SGS_CUDA(cudaGetLastError());
  std::vector<double> hp(nblk);
  SGS_CUDA(cudaMemcpyAsync(hp.data(), design_part.p, nblk * sizeof(double), cudaMemcpyDeviceToHost, stream));
  filter_dev(design_rho.p, design_dc.p, design_dc1.p, prm.filter_size, -1.0);
  double change = 0;
  const double mid = oc_dev(design_rho.p, design_dc1.p, design_fixed.p, prm.volume_fraction, prm.step_limit,
                            prm.minimum_density, prm.fixed_density, prm.smart_oc, prm.exclude_fixed, 1, &change);
  design_refresh(design_rho.p);
  double obj = 0;
  for (double v : hp) obj += v;
  if (out) {
    out->objective = obj;
    out->change = change;
    out->lagrange = mid;
    out->cg_iterations = iterations;
    out->solve_device_seconds = solve_device_seconds;
    out->solve_seconds = std::chrono::duration<double>(t1 - t0).count();
    out->step_seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t1).count();
  }
}

void Solver::design_refresh(const double* rho_s) {
  const long nin = long(P.in_block.size());
  simp_E_kernel<<<blocks_for(nin * 64, 256), 256, 0, stream>>>(int(nin), in_block.p, in_zoff.p, rho_s, P.penalty,
                                                               P.minimum_stiffness, P.minimum_density, E64.p);
  SGS_CUDA(cudaGetLastError());
  if (mixed())
    launch(convert_kernel<float, double>, blocks_for(long(P.E.size()), 256), 256, 0, E32.p, E64.p, long(P.E.size()));
  drop_graphs();
  build_operators();
  build_bottom();
  SGS_CUDA(cudaStreamSynchronize(stream));
}

// The session's input blocks must be the band's blocks container_block[i], in
// order, and its material cells exactly the container cells of fat blocks (the
// packing of spgrid_topo_opt.cpp:1068-1160).
void Solver::band_attach(Band& B, const int64_t* container_block) {
  const long nin = long(P.in_block.size());
  std::vector<int32_t> map(static_cast<size_t>(nin));
  std::vector<uint8_t> fat(static_cast<size_t>(B.n)), fl(static_cast<size_t>(B.n) * 64);
  SGS_CUDA(cudaMemcpyAsync(fat.data(), B.fat.p, fat.size(), cudaMemcpyDeviceToHost, B.stream));
  SGS_CUDA(cudaMemcpyAsync(fl.data(), B.flags.p, fl.size(), cudaMemcpyDeviceToHost, B.stream));
  SGS_CUDA(cudaStreamSynchronize(B.stream));
  for (long i = 0; i < nin; ++i) {
    const int64_t c = container_block[i];
    if (c < 0 || c >= B.n) throw CudaError("container block index out of range", SGS_ERR_INPUT);
    for (int v = 0; v < 3; ++v)
      if (B.base_h[size_t(3 * c + v)] != P.in_base[size_t(3 * i + v)])
        throw CudaError("session block " + std::to_string(i) + " is not container block " + std::to_string(c),
                        SGS_ERR_INPUT);
    const int blk = P.in_block[size_t(i)];
    for (int e = 0; e < 64; ++e) {
      const bool material = fat[size_t(c)] && (fl[size_t(c) * 64 + e] & SGS_CELL_INSIDE);
      const bool solid = blk >= 0 && P.E[size_t(blk) * 128 + (e >> 4) * 32 + ((e >> 2) & 3) * 8 + (e & 3) +
                                         P.in_zoff[size_t(i)]] > 0;
      if (material != solid)
        throw CudaError("session material differs from the band's fat container cells", SGS_ERR_INPUT);
    }
    map[size_t(i)] = int32_t(c);
  }
  B.sess_map.upload(map, stream);
  if (!B.dc0.p) {
    B.dc0.alloc(size_t(B.n) * 64);
    B.dc1.alloc(size_t(B.n) * 64);
    B.dc0.zero(stream);
    B.dc1.zero(stream);
  }
  design_scratch.alloc(size_t(nin) * 64);
  design_dc.alloc(size_t(nin) * 64);
  design_dc1.alloc(size_t(nin) * 64);  // element energies of the sensitivity pass
  design_part.alloc(blocks_for(nin * 64, 256));
  SGS_CUDA(cudaStreamSynchronize(stream));
  B.attached = this;
}

// One iteration of the driver (Opt::iterate after its page-map update,
// spgrid_topo_opt.cpp:1301-1330) with the design on the band: clear_gradients
// over the fat blocks, solve, the compliance sensitivity of the fat container
// cells, smooth_dc over the fat blocks, the OC update over the fat container
// cells against total_container_voxels, and the new stiffness scales.
void Solver::band_step(Band& B, const sgs_design_params& prm, sgs_design_result* out) {
  if (B.attached != this) throw CudaError("the band is not attached to this session", SGS_ERR_INPUT);
  const long nin = long(P.in_block.size()), ns = nin * 64, nc = B.n * 64;
  const auto t0 = std::chrono::steady_clock::now();
  // the band's updates ran on its own stream; the step runs on the solver's
  SGS_CUDA(cudaStreamSynchronize(B.stream));
  P.tolerance = prm.tolerance;
  solve();
  const auto t1 = std::chrono::steady_clock::now();
  const unsigned gs = blocks_for(ns, 256), gc = blocks_for(nc, 256);
  band_clear_kernel<<<gc, 256, 0, stream>>>(nc, B.fat.p, B.dc0.p);
  band_gather_kernel<<<gs, 256, 0, stream>>>(ns, B.sess_map.p, B.fat.p, B.flags.p, B.rho.p, design_scratch.p);
  sensitivity_kernel<<<gs, 256, 0, stream>>>(int(nin), in_block.p, in_zoff.p, L64[0]->nbr.p, x.p, N0(),
                                             design_scratch.p, P.penalty, P.minimum_stiffness, design_dc.p,
                                             design_dc1.p, design_part.p);
  band_scatter_dc_kernel<<<gs, 256, 0, stream>>>(ns, B.sess_map.p, design_scratch.p, design_dc.p, B.dc0.p);
  SGS_CUDA(cudaGetLastError());
  std::vector<double> hp(gs);
  SGS_CUDA(cudaMemcpyAsync(hp.data(), design_part.p, gs * sizeof(double), cudaMemcpyDeviceToHost, stream));
  band_filter_kernel<<<gc, 256, 0, stream>>>(nc, B.base.p, B.grid.p, B.gdim[0], B.gdim[1], B.gdim[2], B.fat.p,
                                             B.flags.p, B.rho.p, B.dc0.p, B.dc1.p, prm.filter_size,
                                             int(std::floor(prm.filter_size)));
  band_copy_kernel<<<gc, 256, 0, stream>>>(nc, B.fat.p, B.dc1.p, B.dc0.p);
  SGS_CUDA(cudaGetLastError());
  // OC (optimality_criterion.cpp:19-145)
  DevBuf<double> pa, pb;
  pa.alloc(OC_BLOCKS);
  pb.alloc(OC_BLOCKS);
  std::vector<double> ha(OC_BLOCKS), hb(OC_BLOCKS);
  auto read_parts = [&] {
    SGS_CUDA(cudaMemcpyAsync(ha.data(), pa.p, OC_BLOCKS * sizeof(double), cudaMemcpyDeviceToHost, stream));
    SGS_CUDA(cudaMemcpyAsync(hb.data(), pb.p, OC_BLOCKS * sizeof(double), cudaMemcpyDeviceToHost, stream));
    SGS_CUDA(cudaStreamSynchronize(stream));
  };
  band_oc_stats_kernel<<<OC_BLOCKS, OC_THREADS, 0, stream>>>(nc, B.fat.p, B.flags.p, B.dc0.p, pa.p, pb.p);
  SGS_CUDA(cudaGetLastError());
  read_parts();
  double nfix = 0, neg_dc_min = 1e30;
  for (int k = 0; k < OC_BLOCKS; ++k) {
    nfix += ha[size_t(k)];
    neg_dc_min = std::min(neg_dc_min, hb[size_t(k)]);
  }
  const double shift = prm.smart_oc ? std::min(0.0, neg_dc_min) : 0.0;
  const double target = prm.volume_fraction * double(B.total_inside - (prm.exclude_fixed ? long(nfix) : 0));
  auto trial = [&](double mid, double* rho_out, double* chg) {
    band_oc_trial_kernel<<<OC_BLOCKS, OC_THREADS, 0, stream>>>(nc, B.fat.p, B.flags.p, B.rho.p, B.dc0.p, mid, shift,
                                                               prm.step_limit, prm.minimum_density, prm.fixed_density,
                                                               prm.exclude_fixed, rho_out, pa.p, pb.p);
    SGS_CUDA(cudaGetLastError());
    read_parts();
    double sum = 0;
    for (double v : ha) sum += v;
    if (chg) {
      *chg = 0;
      for (double v : hb) *chg = std::max(*chg, v);
    }
    return sum;
  };
  double mid = 0, lower = 1e-20, upper = 1e20;
  const double factor = 1 + 1e-7;
  while (lower * factor < upper) {
    mid = 0.5 * (lower + upper);
    const double sum = trial(mid, nullptr, nullptr);
    if (!(sum == sum)) throw CudaError("OC update produced a non-finite volume", SGS_ERR_BREAKDOWN);
    if (sum > target) lower = mid;
    else upper = mid;
  }
  double change = 0;
  trial(mid, B.rho.p, &change);
  band_gather_kernel<<<gs, 256, 0, stream>>>(ns, B.sess_map.p, B.fat.p, B.flags.p, B.rho.p, design_scratch.p);
  SGS_CUDA(cudaGetLastError());
  design_refresh(design_scratch.p);
  double obj = 0;
  for (double v : hp) obj += v;
  if (out) {
    out->objective = obj;
    out->change = change;
    out->lagrange = mid;
    out->cg_iterations = iterations;
    out->solve_device_seconds = solve_device_seconds;
    out->solve_seconds = std::chrono::duration<double>(t1 - t0).count();
    out->step_seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t1).count();
  }
}

// ---------------------------------------------------------------------------
// The solver state kept between fem_solve calls with keep_state
// (SPGrid_CPU_Solver.cpp:17-26, 56-73, 389-408): the zero-guess residual of the
// call that created it and the last solution on every level-0 page solved on
// (the reference keeps both in its SPGrid allocation), to warm-start later calls.
// ---------------------------------------------------------------------------
struct KeptState {
  static constexpr uint64_t MAGIC = 0x5347535354415445ull;
  uint64_t magic = MAGIC;
  double initial_residual_linf = 0;
  std::unordered_map<uint64_t, int32_t> slot;  // page -> slot of the store
  DevBuf<double> store;                         // [slot][3][128]
  long nslots = 0;
};

static uint64_t page_id(int x, int y, int z) {
  return (uint64_t(uint32_t(x >> 2)) << 42) | (uint64_t(uint32_t(y >> 2)) << 21) | uint64_t(uint32_t(z >> 3));
}

// x[v][b*128 + e] <- store[slot[b]][v][e] (0 where the page has no slot)
__global__ void warm_gather_kernel(long nb, const int* __restrict__ slot, const double* __restrict__ store,
                                   double* __restrict__ x, long N) {
  const long t = long(blockIdx.x) * blockDim.x + threadIdx.x;
  if (t >= nb * 128) return;
  const long b = t >> 7;
  const int e = int(t & 127), sl = slot[b];
  for (int v = 0; v < 3; ++v) x[v * N + t] = sl >= 0 ? store[(long(sl) * 3 + v) * 128 + e] : 0.0;
}

__global__ void warm_scatter_kernel(long nb, const int* __restrict__ slot, const double* __restrict__ x, long N,
                                    double* __restrict__ store) {
  const long t = long(blockIdx.x) * blockDim.x + threadIdx.x;
  if (t >= nb * 128) return;
  const long b = t >> 7;
  const int e = int(t & 127), sl = slot[b];
  for (int v = 0; v < 3; ++v) store[(long(sl) * 3 + v) * 128 + e] = x[v * N + t];
}

// The previous solution on this call's pages becomes the warm-start candidate.
static void warm_start_from(Solver& S, const KeptState& K) {
  const HostLevel& h = S.P.levels[0];
  std::vector<int32_t> sl(static_cast<size_t>(h.nb));
  for (int b = 0; b < h.nb; ++b) {
    auto it = K.slot.find(page_id(h.coords[3 * b], h.coords[3 * b + 1], h.coords[3 * b + 2]));
    sl[size_t(b)] = it == K.slot.end() ? -1 : it->second;
  }
  DevBuf<int32_t> d;
  d.upload(sl, S.stream);
  S.warm_u.alloc(size_t(3) * S.N0());
  const long nb = h.nb;
  if (nb)
    warm_gather_kernel<<<blocks_for(nb * 128, 256), 256, 0, S.stream>>>(nb, d.p, K.store.p, S.warm_u.p, S.N0());
  SGS_CUDA(cudaGetLastError());
  SGS_CUDA(cudaStreamSynchronize(S.stream));
  S.warm_reference = K.initial_residual_linf;
}

// The solution of this call into the kept state (new pages get new slots).
static void keep_solution(Solver& S, KeptState& K) {
  const HostLevel& h = S.P.levels[0];
  std::vector<int32_t> sl(static_cast<size_t>(h.nb));
  for (int b = 0; b < h.nb; ++b) {
    const uint64_t id = page_id(h.coords[3 * b], h.coords[3 * b + 1], h.coords[3 * b + 2]);
    auto it = K.slot.find(id);
    if (it == K.slot.end()) it = K.slot.emplace(id, int32_t(K.nslots++)).first;
    sl[size_t(b)] = it->second;
  }
  const size_t need = size_t(K.nslots) * 3 * 128;
  if (K.store.n < need) {  // grow, keeping the stored pages
    DevBuf<double> grown;
    grown.alloc(std::max(need, 2 * K.store.n));
    if (K.store.n)
      SGS_CUDA(cudaMemcpyAsync(grown.p, K.store.p, K.store.n * sizeof(double), cudaMemcpyDeviceToDevice, S.stream));
    std::swap(grown.p, K.store.p);
    std::swap(grown.n, K.store.n);
  }
  DevBuf<int32_t> d;
  d.upload(sl, S.stream);
  const long nb = h.nb;
  if (nb) warm_scatter_kernel<<<blocks_for(nb * 128, 256), 256, 0, S.stream>>>(nb, d.p, S.x.p, S.N0(), K.store.p);
  SGS_CUDA(cudaGetLastError());
  SGS_CUDA(cudaStreamSynchronize(S.stream));
}

}  // namespace sgs

// ===========================================================================
// C ABI
// ===========================================================================
using namespace sgs;

struct sgs_session {
  std::unique_ptr<Solver> solver;
  std::string error;
};

static void set_err(char* buf, int len, const std::string& m) {
  if (buf && len > 0) std::snprintf(buf, size_t(len), "%s", m.c_str());
}

static int session_from_inputs(const FEMInputs& in, int precision, sgs_session** out, std::string* err) {
  std::unique_ptr<sgs_session> h(new sgs_session());
  h->solver.reset(new Solver());
  int code = 0;
  const auto th = std::chrono::steady_clock::now();
  std::string m = build_problem(in, h->solver->P, &code);
  h->solver->host_setup_seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - th).count();
  if (!m.empty()) {
    *err = m;
    return code ? code : SGS_ERR_INPUT;
  }
  h->solver->P.max_iterations = 500;  // the reference hard-codes 500 (SPGrid_CPU_Solver.cpp:326)
  if (in.get_int("sgs_honor_max_iterations", 0)) h->solver->P.max_iterations = in.krylov.max_iterations;
  h->solver->tensor_cores = in.get_int("sgs_tensor_cores", 0) != 0;
  h->solver->loop_unavailable = in.get_int("sgs_device_loop", 1) == 0;
  if (h->solver->loop_unavailable) h->solver->loop_note = "sgs_device_loop = 0";
  h->solver->loop_history = in.get_int("sgs_loop_history", 1024);
  if (precision == SGS_HOST_SETUP_ONLY) {  // inspection of the host-side hierarchy, no device work
    h->solver->precision = precision;
    *out = h.release();
    return 0;
  }
  try {
    h->solver->init(precision);
  } catch (const CudaError& e) {
    *err = e.what();
    return e.code;
  } catch (const std::exception& e) {
    *err = e.what();
    return SGS_ERR_INTERNAL;
  }
  *out = h.release();
  return 0;
}

// host compact [3][N] <-> device level field
template <typename T>
static void put_field(Solver& S, T* dst, const double* src, long N) {
  std::vector<T> tmp(size_t(3 * N));
  for (long i = 0; i < 3 * N; ++i) tmp[i] = T(src[i]);
  SGS_CUDA(cudaMemcpyAsync(dst, tmp.data(), tmp.size() * sizeof(T), cudaMemcpyHostToDevice, S.stream));
  SGS_CUDA(cudaStreamSynchronize(S.stream));
}
template <typename T>
static void get_field(Solver& S, double* dst, const T* src, long N) {
  std::vector<T> tmp(size_t(3 * N));
  SGS_CUDA(cudaMemcpyAsync(tmp.data(), src, tmp.size() * sizeof(T), cudaMemcpyDeviceToHost, S.stream));
  SGS_CUDA(cudaStreamSynchronize(S.stream));
  for (long i = 0; i < 3 * N; ++i) dst[i] = double(tmp[i]);
}

template <typename T>
static int apply_op(Solver& S, int op, int level, int arg, const double* in, const double* in2, double* out) {
  const int n = S.nlev();
  if (level < 0 || level >= n) return SGS_ERR_INPUT;
  Level<T>& d = S.lev<T>(level);
  const long N = d.N;
  switch (op) {
    case 0:
    case 1:
      if (level != 0) return SGS_ERR_INPUT;
      put_field<T>(S, d.u.p, in, N);
      if (op == 1) put_field<T>(S, d.b.p, in2, N);
      if (op == 0) S.level0<T, OP_KU>(d.u.p, nullptr, d.r.p);
      else S.level0<T, OP_RES>(d.u.p, d.b.p, d.r.p);
      get_field<T>(S, out, d.r.p, N);
      return 0;
    case 2:
      if (level != 0 && !d.has_matrix) return SGS_ERR_INPUT;
      put_field<T>(S, d.u.p, in, N);
      put_field<T>(S, d.b.p, in2, N);
      S.sweep<T>(level, d.u.p, d.b.p, arg & 1, (arg >> 1) & 1);
      get_field<T>(S, out, d.u.p, N);
      return 0;
    case 3:
      if (level + 1 >= n) return SGS_ERR_INPUT;
      put_field<T>(S, d.r.p, in, N);
      S.restrict_to<T>(level + 1, d.r.p);
      get_field<T>(S, out, S.lev<T>(level + 1).b.p, S.lev<T>(level + 1).N);
      return 0;
    case 4:
      if (level + 1 >= n) return SGS_ERR_INPUT;
      put_field<T>(S, S.lev<T>(level + 1).u.p, in, S.lev<T>(level + 1).N);
      put_field<T>(S, d.r.p, in2, N);
      S.prolongate_to<T>(level, d.r.p);
      get_field<T>(S, out, d.r.p, N);
      return 0;
    case 5:
      if (!d.has_matrix) return SGS_ERR_INPUT;
      put_field<T>(S, d.u.p, in, N);
      S.stencil<T, SOP_MUL>(level, nullptr, d.nb, d.u.p, nullptr, nullptr, d.r.p, 0);
      get_field<T>(S, out, d.r.p, N);
      return 0;
    case 6:
      if (level != S.nout() - 1 || S.P.disable_mg) return SGS_ERR_INPUT;
      put_field<T>(S, d.b.p, in, N);
      S.bottom_solve<T>(level);
      get_field<T>(S, out, d.u.p, N);
      return 0;
    case 8:  // the V-cycle's level-0 residual on the packed iterate (tensor cores in mixed sessions)
      if (level != 0 || !S.packed0()) return SGS_ERR_INPUT;
      put_field<T>(S, d.u.p, in, N);
      put_field<T>(S, d.b.p, in2, N);
      S.launch(pack_u4_kernel<T>, blocks_for(N, 256), 256, 0, d.u4.p, d.u.p, S.Edev<T>(), N);
      S.level0_packed<T, OP_RES>(d.b.p, d.r.p);
      S.check_tensor_core_waits();
      get_field<T>(S, out, d.r.p, N);
      return 0;
    case 7: {
      if (level != 0) return SGS_ERR_INPUT;
      std::vector<double> tmp(in, in + 3 * N);
      SGS_CUDA(cudaMemcpyAsync(S.f.p, tmp.data(), 3 * N * sizeof(double), cudaMemcpyHostToDevice, S.stream));
      S.stage_residual();
      S.precondition();
      SGS_CUDA(cudaMemcpyAsync(out, S.q.p, 3 * N * sizeof(double), cudaMemcpyDeviceToHost, S.stream));
      SGS_CUDA(cudaStreamSynchronize(S.stream));
      return 0;
    }
  }
  return SGS_ERR_INPUT;
}

template <typename T>
static double time_op(Solver& S, int op, int reps) {
  Level<T>& d = S.lev<T>(0);
  cudaEvent_t a, b;
  SGS_CUDA(cudaEventCreate(&a));
  SGS_CUDA(cudaEventCreate(&b));
  // with a packed level 0 the residual and the sweep run on the packed iterate, as in the V-cycle
  const bool packed = S.packed0();
  auto run = [&]() {
    if (op == 0) {
      S.level0<double, OP_KUP>(S.s.p, nullptr, S.q.p);  // the PCG matvec, FP64 in every mode
    } else if (op == 1) {
      if (packed) {
        S.level0_packed<T, OP_RES>(d.b.p, d.r.p);
        return;
      }
      S.level0<T, OP_RES>(d.u.p, d.b.p, d.r.p);
    } else if (op == 2) {
      S.sweep<T>(0, packed ? nullptr : d.u.p, d.b.p, true, false);
    } else if (op == 3) {
      S.precondition();
    } else if (op == 5) {  // the V-cycle residual on the tensor cores, whatever the session uses
      if (!(packed && sizeof(T) == 4)) throw CudaError("op 5 needs a mixed-precision session", SGS_ERR_INPUT);
      const bool keep = S.tensor_cores;
      S.tensor_cores = true;
      S.level0_packed<T, OP_RES>(d.b.p, d.r.p);
      S.tensor_cores = keep;
    } else if (op == 4) {  // K u in the V-cycle's precision, on the tensor cores where the V-cycle uses them
      if (packed && sizeof(T) == 4 && S.tensor_cores) S.level0_packed<T, OP_KU>(nullptr, d.r.p);
      else S.level0<T, OP_KU>(d.u.p, nullptr, d.r.p);
    }
  };
  run();
  SGS_CUDA(cudaEventRecord(a, S.stream));
  for (int i = 0; i < reps; ++i) run();
  SGS_CUDA(cudaEventRecord(b, S.stream));
  SGS_CUDA(cudaEventSynchronize(b));
  S.check_tensor_core_waits();
  float ms = 0;
  SGS_CUDA(cudaEventElapsedTime(&ms, a, b));
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  return double(ms) / reps;
}

extern "C" {

SGS_API int sgs_create(const void* input_blob, int precision, sgs_session** out, char* err, int errlen) {
  if (!input_blob || !out) return SGS_ERR_INPUT;
  *out = nullptr;
  if (precision < 0 || precision > SGS_HOST_SETUP_ONLY) {
    set_err(err, errlen, "precision must be 0 (reference), 1 (fp64), 2 (mixed) or 3 (host set-up only)");
    return SGS_ERR_INPUT;
  }
  try {
    FEMInputs in = decode_inputs(input_blob);
    std::string m;
    int rc = session_from_inputs(in, precision, out, &m);
    if (rc) set_err(err, errlen, m);
    return rc;
  } catch (const WireError& e) {
    set_err(err, errlen, std::string("malformed input blob: ") + e.what());
    return SGS_ERR_WIRE;
  } catch (const std::exception& e) {
    set_err(err, errlen, e.what());
    return SGS_ERR_INTERNAL;
  }
}

SGS_API void sgs_destroy(sgs_session* h) { delete h; }

SGS_API const char* sgs_last_error(sgs_session* h) { return h ? h->error.c_str() : ""; }

static bool host_only(sgs_session* h) { return h->solver->precision == SGS_HOST_SETUP_ONLY; }

SGS_API int sgs_solve(sgs_session* h, double tolerance, int max_iterations, sgs_stats* stats) {
  if (!h || host_only(h)) return SGS_ERR_INPUT;
  Solver& S = *h->solver;
  if (tolerance > 0) S.P.tolerance = tolerance;
  if (max_iterations > 0) S.P.max_iterations = max_iterations;
  int rc = 0;
  try {
    S.solve();
  } catch (const CudaError& e) {
    h->error = e.what();
    rc = e.code;
  } catch (const std::exception& e) {
    h->error = e.what();
    rc = SGS_ERR_INTERNAL;
  }
  if (stats) {
    stats->iterations = S.iterations;
    stats->levels = S.nlev();
    stats->initial_residual = S.initial_residual;
    stats->final_residual = S.final_residual;
    stats->setup_seconds = S.setup_seconds;
    stats->solve_seconds = S.solve_seconds;
    stats->launches_per_iteration = S.launches_per_iteration;
    stats->dof = 3 * S.active_nodes0;
    stats->bottom_unknowns = S.bottom.n;
    stats->solve_device_seconds = S.solve_device_seconds;
    stats->kernel_launches = S.solve_launches;
    stats->h2d_bytes = double(g_h2d_bytes.load());
    stats->d2h_bytes = double(g_d2h_bytes.load());
  }
  return rc;
}

SGS_API int sgs_residual_history(sgs_session* h, double* out, int cap) {
  if (!h) return 0;
  int n = int(h->solver->history.size());
  for (int i = 0; i < n && i < cap; ++i) out[i] = h->solver->history[i];
  return n;
}

SGS_API int sgs_displacements(sgs_session* h, double* out) {
  if (!h || !out || host_only(h)) return SGS_ERR_INPUT;
  try {
    h->solver->pack_outputs(out);
  } catch (const CudaError& e) {
    h->error = e.what();
    return e.code;
  }
  return 0;
}

SGS_API double sgs_sensitivity(sgs_session* h, const double* density, double* dc, double* element_energy) {
  if (!h || !density || !dc || host_only(h)) return std::nan("");
  try {
    return h->solver->sensitivity(density, h->solver->P.penalty, h->solver->P.minimum_stiffness, dc, element_energy);
  } catch (const CudaError& e) {
    h->error = e.what();
    return std::nan("");
  }
}

SGS_API int sgs_filter_sensitivity(sgs_session* h, const double* density, const double* dc0, double* dc1,
                                   double filter_size) {
  if (!h || !density || !dc0 || !dc1 || host_only(h) || !(filter_size >= 0)) return SGS_ERR_INPUT;
  try {
    h->solver->filter_sensitivity(density, dc0, dc1, filter_size);
  } catch (const CudaError& e) {
    h->error = e.what();
    return e.code;
  }
  return 0;
}

SGS_API int sgs_oc_update(sgs_session* h, double* density, const double* dc0, const uint8_t* fixed,
                          double volume_fraction, double step_limit, double minimum_density, double fixed_density,
                          int smart_oc, int exclude_fixed, double* lagrange, double* max_change) {
  if (!h || !density || !dc0 || host_only(h)) return SGS_ERR_INPUT;
  try {
    const double mid = h->solver->oc_update(density, dc0, fixed, volume_fraction, step_limit, minimum_density,
                                            fixed_density, smart_oc, exclude_fixed, max_change);
    if (lagrange) *lagrange = mid;
  } catch (const CudaError& e) {
    h->error = e.what();
    return e.code;
  }
  return 0;
}

SGS_API int sgs_design_set(sgs_session* h, const double* density, const uint8_t* fixed) {
  if (!h || !density || host_only(h)) return SGS_ERR_INPUT;
  try {
    h->solver->design_set(density, fixed);
  } catch (const CudaError& e) {
    h->error = e.what();
    return e.code;
  }
  return 0;
}

SGS_API int sgs_design_step(sgs_session* h, const sgs_design_params* p, sgs_design_result* r) {
  if (!h || !p || host_only(h)) return SGS_ERR_INPUT;
  try {
    h->solver->design_step(*p, r);
  } catch (const CudaError& e) {
    h->error = e.what();
    return e.code;
  }
  return 0;
}

SGS_API int sgs_band_attach(sgs_band* b, sgs_session* h, const int64_t* container_block) {
  if (!b || !b->band || !h || !container_block || host_only(h)) return SGS_ERR_INPUT;
  try {
    h->solver->band_attach(*b->band, container_block);
  } catch (const CudaError& e) {
    h->error = e.what();
    b->error = e.what();
    return e.code;
  }
  return 0;
}

// The driver's packing of FEMInputs from its maps (spgrid_topo_opt.cpp:1068-1160):
// the fatter blocks in container order, max(density, DBL_MIN) in the container
// cells of fat blocks, 0 elsewhere; everything else from the template.
SGS_API int sgs_band_session(sgs_band* b, const void* template_blob, int precision, sgs_session** out, char* err,
                             int errlen) {
  if (!b || !b->band || !template_blob || !out || precision == SGS_HOST_SETUP_ONLY) return SGS_ERR_INPUT;
  *out = nullptr;
  Band& B = *b->band;
  std::string msg;
  int code = 0;
  try {
    FEMInputs in = decode_inputs(template_blob);
    std::vector<uint8_t> fat(static_cast<size_t>(B.n)), fatter(static_cast<size_t>(B.n));
    std::vector<double> rho(static_cast<size_t>(B.n) * 64);
    SGS_CUDA(cudaMemcpyAsync(fat.data(), B.fat.p, fat.size(), cudaMemcpyDeviceToHost, B.stream));
    SGS_CUDA(cudaMemcpyAsync(fatter.data(), B.fatter.p, fatter.size(), cudaMemcpyDeviceToHost, B.stream));
    SGS_CUDA(cudaMemcpyAsync(rho.data(), B.rho.p, rho.size() * sizeof(double), cudaMemcpyDeviceToHost, B.stream));
    SGS_CUDA(cudaStreamSynchronize(B.stream));
    g_d2h_bytes += 2 * fat.size() + rho.size() * sizeof(double);
    std::vector<int64_t> idx;
    for (long c = 0; c < B.n; ++c)
      if (fatter[size_t(c)]) idx.push_back(c);
    const size_t m = idx.size();
    in.density.base.resize(3 * m);
    in.density.data.resize(64 * m);
#pragma omp parallel for schedule(static)
    for (long i = 0; i < long(m); ++i) {
      const size_t c = size_t(idx[size_t(i)]);
      for (int v = 0; v < 3; ++v) in.density.base[3 * size_t(i) + v] = B.base_h[3 * c + v];
      for (int e = 0; e < 64; ++e) {
        const bool material = fat[c] && (B.flags_h[c * 64 + e] & SGS_CELL_INSIDE);
        in.density.data[64 * size_t(i) + e] = material ? std::max(rho[c * 64 + e], DBL_MIN_D) : 0.0;
      }
    }
    // FEMInputs::preserve_output (fem_interface.h:445-454)
    in.preserved_buffer_size = (uint64_t(1) << 20) + m * (3 * 4 + 64 * 4 * 8);
    sgs_session* h = nullptr;
    code = session_from_inputs(in, precision, &h, &msg);
    if (code == 0) {
      try {
        h->solver->band_attach(B, idx.data());
      } catch (const CudaError& e) {
        delete h;
        throw;
      }
      *out = h;
    }
  } catch (const CudaError& e) {
    msg = e.what();
    code = e.code;
  } catch (const WireError& e) {
    msg = e.what();
    code = SGS_ERR_WIRE;
  } catch (const std::exception& e) {
    msg = e.what();
    code = SGS_ERR_INTERNAL;
  }
  if (code) {
    set_err(err, errlen, msg);
    b->error = msg;
  }
  return code;
}

SGS_API int sgs_band_step(sgs_band* b, sgs_session* h, const sgs_design_params* p, sgs_design_result* r) {
  if (!b || !b->band || !h || !p || host_only(h)) return SGS_ERR_INPUT;
  try {
    h->solver->band_step(*b->band, *p, r);
  } catch (const CudaError& e) {
    h->error = e.what();
    b->error = e.what();
    return e.code;
  }
  return 0;
}

SGS_API int sgs_design_get(sgs_session* h, double* density) {
  if (!h || !density || host_only(h) || !h->solver->design_rho.p) return SGS_ERR_INPUT;
  try {
    Solver& S = *h->solver;
    SGS_CUDA(cudaMemcpyAsync(density, S.design_rho.p, S.design_rho.n * sizeof(double), cudaMemcpyDeviceToHost,
                             S.stream));
    SGS_CUDA(cudaStreamSynchronize(S.stream));
  } catch (const CudaError& e) {
    h->error = e.what();
    return e.code;
  }
  return 0;
}

// ---------------------------------------------------------------------------
// Allocation-free sensitivity.  Some callers cannot allocate device memory
// while they run (an allocator locked down by a framework, a region that must
// not call cudaMalloc/cudaFree, a memory budget that is fixed after start-up).
// This variant takes caller-owned device buffers and keeps the only scratch it
// needs, the per-CTA partial sums of the objective, in a fixed static device
// array of SGS_SENSITIVITY_STATIC_MAX_PARTIALS doubles (128 KiB, held by every
// GPU that loads the library until the process exits).
// ---------------------------------------------------------------------------
// The array itself is declared before the Solver class, whose set-up resolves
// its device address on the session's device.

// Sum the partials in index order, the order sgs_sensitivity uses on the host.
__global__ void sum_in_order_kernel(const double* __restrict__ part, int n, double* __restrict__ out) {
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    double s = 0;
    for (int i = 0; i < n; ++i) s += part[i];
    *out = s;
  }
}

SGS_API int sgs_sensitivity_static(sgs_session* h, const double* density_dev, double* dc_dev,
                                   double* element_energy_dev, double* objective_dev) {
  if (!h || host_only(h) || !density_dev || !dc_dev || !element_energy_dev || !objective_dev) return SGS_ERR_INPUT;
  Solver& S = *h->solver;
  const long nin = long(S.P.in_block.size());
  const long ncta = (nin * 64 + 255) / 256;
  if (ncta > SGS_SENSITIVITY_STATIC_MAX_PARTIALS) {
    char m[200];
    std::snprintf(m, sizeof m, "sgs_sensitivity_static handles at most %d x 256 cells (%ld input blocks given)",
                  SGS_SENSITIVITY_STATIC_MAX_PARTIALS, nin);
    h->error = m;
    return SGS_ERR_INPUT;
  }
  try {
    // the buffers, the stream and the scratch address all belong to the session's device
    int dev = -1;
    SGS_CUDA(cudaGetDevice(&dev));
    if (dev != S.device) {
      char m[160];
      std::snprintf(m, sizeof m, "sgs_sensitivity_static called with device %d current; the session lives on device %d",
                    dev, S.device);
      h->error = m;
      return SGS_ERR_INPUT;
    }
    double* part = S.static_partials;
    if (nin == 0) {
      SGS_CUDA(cudaMemsetAsync(objective_dev, 0, sizeof(double), S.stream));
    } else {
      sensitivity_kernel<<<unsigned(ncta), 256, 0, S.stream>>>(int(nin), S.in_block.p, S.in_zoff.p, S.L64[0]->nbr.p, S.x.p,
                                                              S.N0(), density_dev, S.P.penalty, S.P.minimum_stiffness,
                                                              dc_dev, element_energy_dev, part);
      sum_in_order_kernel<<<1, 32, 0, S.stream>>>(part, int(ncta), objective_dev);
    }
    SGS_CUDA(cudaGetLastError());
    SGS_CUDA(cudaStreamSynchronize(S.stream));
  } catch (const CudaError& e) {
    h->error = e.what();
    return e.code;
  }
  return 0;
}

SGS_API int sgs_set_density(sgs_session* h, const double* density) {
  if (!h || !density || host_only(h)) return SGS_ERR_INPUT;
  try {
    std::string m = h->solver->update_density(density);
    if (!m.empty()) {
      h->error = m;
      return SGS_ERR_INPUT;
    }
  } catch (const CudaError& e) {
    h->error = e.what();
    return e.code;
  }
  return 0;
}

// ---- device-resident calls for the PyTorch layer ---------------------------
// The session's stream waits for the caller's stream (an event, no host wait)
// before it reads the caller's buffers; the calls return once the session's
// stream has finished, so the caller may use the results on any stream.
static void wait_for_caller(Solver& S, void* caller_stream) {
  if (!caller_stream) {
    SGS_CUDA(cudaDeviceSynchronize());
    return;
  }
  cudaEvent_t ev;
  SGS_CUDA(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
  SGS_CUDA(cudaEventRecord(ev, static_cast<cudaStream_t>(caller_stream)));
  SGS_CUDA(cudaStreamWaitEvent(S.stream, ev, 0));
  SGS_CUDA(cudaEventDestroy(ev));
}

static int device_call(sgs_session* h, void* caller_stream, const std::function<void(Solver&)>& body) {
  if (!h || host_only(h)) return SGS_ERR_INPUT;
  Solver& S = *h->solver;
  try {
    int dev = -1;
    SGS_CUDA(cudaGetDevice(&dev));
    if (dev != S.device) {
      h->error = "a device-resident call needs the session's device to be current";
      return SGS_ERR_INPUT;
    }
    wait_for_caller(S, caller_stream);
    body(S);
    SGS_CUDA(cudaGetLastError());
    SGS_CUDA(cudaStreamSynchronize(S.stream));
  } catch (const CudaError& e) {
    h->error = e.what();
    return e.code;
  }
  return 0;
}

SGS_API int64_t sgs_solution_size(sgs_session* h) { return h && !host_only(h) ? 3 * h->solver->N0() : 0; }

SGS_API int sgs_set_density_device(sgs_session* h, const double* density_dev, void* caller_stream) {
  if (!density_dev) return SGS_ERR_INPUT;
  std::string msg;
  const int rc = device_call(h, caller_stream, [&](Solver& S) {
    const long nin = long(S.P.in_block.size());
    if (nin == 0) return;
    DevBuf<int> bad;
    bad.alloc(1);
    bad.zero(S.stream);
    simp_E_check_kernel<<<blocks_for(nin * 64, 256), 256, 0, S.stream>>>(
        int(nin), S.in_block.p, S.in_zoff.p, density_dev, S.P.penalty, S.P.minimum_stiffness, S.P.minimum_density,
        S.P.mu0, S.E64.p, bad.p);
    SGS_CUDA(cudaGetLastError());
    int hbad = 0;
    SGS_CUDA(cudaMemcpyAsync(&hbad, bad.p, sizeof(int), cudaMemcpyDeviceToHost, S.stream));
    SGS_CUDA(cudaStreamSynchronize(S.stream));
    if (hbad & 1) msg = "non-finite density";
    else if (hbad & 2) msg = "the set of material cells changed; create a new session";
    else S.design_refresh(density_dev);
  });
  if (rc) return rc;
  if (!msg.empty()) {
    h->error = msg;
    return SGS_ERR_INPUT;
  }
  return 0;
}

SGS_API int sgs_solution_device(sgs_session* h, double* u_dev, void* caller_stream) {
  if (!u_dev) return SGS_ERR_INPUT;
  return device_call(h, caller_stream, [&](Solver& S) {
    SGS_CUDA(cudaMemcpyAsync(u_dev, S.x.p, 3 * S.N0() * sizeof(double), cudaMemcpyDeviceToDevice, S.stream));
  });
}

SGS_API int sgs_compliance_device(sgs_session* h, double* out_dev, void* caller_stream) {
  if (!out_dev) return SGS_ERR_INPUT;
  return device_call(h, caller_stream, [&](Solver& S) {
    compliance_kernel<<<1, 256, 0, S.stream>>>(S.load_node.p, S.load_val.p, int(S.load_node.n), S.x.p, S.N0(), out_dev);
  });
}

SGS_API int sgs_sensitivity_device(sgs_session* h, const double* u_dev, const double* density_dev, double factor,
                                   const double* scale_dev, double* grad_dev, void* caller_stream) {
  if (!density_dev || !grad_dev) return SGS_ERR_INPUT;
  return device_call(h, caller_stream, [&](Solver& S) {
    const long nin = long(S.P.in_block.size());
    if (nin == 0) return;
    sensitivity_grad_kernel<<<blocks_for(nin * 64, 256), 256, 0, S.stream>>>(
        int(nin), S.in_block.p, S.in_zoff.p, S.L64[0]->nbr.p, u_dev ? u_dev : S.x.p, S.N0(), density_dev,
        S.P.penalty, S.P.minimum_stiffness, factor, scale_dev, grad_dev);
  });
}

SGS_API int sgs_level_count(sgs_session* h) { return h ? h->solver->nlev() : 0; }

SGS_API int sgs_level_blocks(sgs_session* h, int level, int32_t* coords) {
  if (!h || level < 0 || level >= h->solver->nlev()) return -1;
  const HostLevel& L = h->solver->P.levels[level];
  if (coords) std::memcpy(coords, L.coords.data(), size_t(L.nb) * 3 * sizeof(int32_t));
  return L.nb;
}

SGS_API int sgs_level_flags(sgs_session* h, int level, uint32_t* flags) {
  if (!h || level < 0 || level >= h->solver->nlev()) return -1;
  const HostLevel& L = h->solver->P.levels[level];
  std::memcpy(flags, L.flags.data(), size_t(L.nb) * NODES_PER_BLOCK * sizeof(uint32_t));
  return 0;
}

SGS_API int sgs_boundary_blocks(sgs_session* h, int level, int32_t* ordinals) {
  if (!h || level < 0 || level >= h->solver->nlev()) return -1;
  const HostLevel& L = h->solver->P.levels[level];
  if (ordinals) std::memcpy(ordinals, L.boundary.data(), L.boundary.size() * sizeof(int32_t));
  return int(L.boundary.size());
}

SGS_API int sgs_apply(sgs_session* h, int op, int level, int arg, const double* in, const double* in2, double* out) {
  if (!h || !in || !out || host_only(h)) return SGS_ERR_INPUT;
  try {
    if (op == 7) return apply_op<double>(*h->solver, op, level, arg, in, in2, out);
    return h->solver->mixed() ? apply_op<float>(*h->solver, op, level, arg, in, in2, out)
                              : apply_op<double>(*h->solver, op, level, arg, in, in2, out);
  } catch (const CudaError& e) {
    h->error = e.what();
    return e.code;
  }
}

SGS_API int sgs_level_stencils(sgs_session* h, int level, double* out, uint32_t* spokes) {
  if (!h || host_only(h) || level < 0 || level >= h->solver->nlev()) return SGS_ERR_INPUT;
  Level<double>& d = *h->solver->L64[level];
  if (!d.has_matrix) return SGS_ERR_INPUT;
  try {
    SGS_CUDA(cudaMemcpyAsync(out, d.A.p, size_t(243) * d.N * sizeof(double), cudaMemcpyDeviceToHost, h->solver->stream));
    if (spokes) SGS_CUDA(cudaMemcpyAsync(spokes, d.spokes.p, d.N * 4, cudaMemcpyDeviceToHost, h->solver->stream));
    SGS_CUDA(cudaStreamSynchronize(h->solver->stream));
  } catch (const CudaError& e) {
    h->error = e.what();
    return e.code;
  }
  return 0;
}

// Drop-in entry (see include/spgrid_fem.h).
// The output blob of a large fem_solve, allocated before the solve with its
// pages touched by a helper thread while the GPU solves (the host only waits
// then): the displacement records are later copied into resident memory
// instead of faulting it in page by page.  Blobs under 64 MiB are allocated
// when they are encoded, as before.
class OutputBlob {
 public:
  explicit OutputBlob(size_t bytes) : capacity_(bytes) {
    if (bytes < (size_t(64) << 20)) return;
    worker_ = std::thread([this] {
      char* p = new (std::nothrow) char[capacity_];
      if (p) {
        const uintptr_t lo = reinterpret_cast<uintptr_t>(p), hi = lo + capacity_, huge = uintptr_t(2) << 20;
        const uintptr_t a = (lo + huge - 1) & ~(huge - 1);
        if (a < hi) madvise(reinterpret_cast<void*>(a), hi - a, MADV_HUGEPAGE);  // advice only
        const long pages = long((capacity_ + 4095) / 4096);
#pragma omp parallel for schedule(static)
        for (long i = 0; i < pages; ++i) p[size_t(i) * 4096] = 0;
      }
      buffer_ = p;
    });
  }
  OutputBlob(const OutputBlob&) = delete;
  OutputBlob& operator=(const OutputBlob&) = delete;
  ~OutputBlob() { delete[] take(); }
  // the buffer (nullptr if none), owned by the caller from here on
  char* take() {
    if (worker_.joinable()) worker_.join();
    char* p = buffer_;
    buffer_ = nullptr;
    return p;
  }
  size_t capacity() const { return capacity_; }

 private:
  size_t capacity_;
  char* buffer_ = nullptr;
  std::thread worker_;
};

SGS_API void fem_solve(void* input, void* output) {
  if (!output) return;
  void** out_ptr = reinterpret_cast<void**>(output);
  *out_ptr = nullptr;
  FEMOutputs outs;
  outs.success = false;
  using clk = std::chrono::steady_clock;
  auto secs = [](clk::time_point a, clk::time_point b) { return std::chrono::duration<double>(b - a).count(); };
  try {
    const auto t0 = clk::now();
    FEMInputs in = decode_inputs(input);
    for (int v = 0; v < 3; ++v) outs.displacements.resolution[v] = in.resolution[v];
    const int precision = in.get_int("sgs_precision", PREC_REFERENCE);
    const unsigned long long h2d0 = g_h2d_bytes.load(), d2h0 = g_d2h_bytes.load();
    sgs_session* h = nullptr;
    std::string err;
    const auto t1 = clk::now();
    int rc = (precision < 0 || precision > 2) ? SGS_ERR_INPUT : session_from_inputs(in, precision, &h, &err);
    outs.extra_doubles["decode_seconds"] = secs(t0, t1);
    outs.extra_doubles["session_seconds"] = secs(t1, clk::now());
    if (rc) {
      outs.error_code = rc;
      outs.info = err.empty() ? "invalid sgs_precision" : err;
    } else {
      std::unique_ptr<sgs_session> guard(h);
      // a kept state passed back by the caller (fem_interface.h:200-214): warm start
      KeptState* state = nullptr;
      if (in.extra_ints.count("state_ptr_lower")) {
        const uint64_t addr = (uint64_t(uint32_t(in.get_int("state_ptr_higher", 0))) << 32) |
                              uint64_t(uint32_t(in.get_int("state_ptr_lower", 0)));
        state = reinterpret_cast<KeptState*>(addr);
        if (state && state->magic != KeptState::MAGIC)
          throw CudaError("the solver state pointer does not name a state of this library", SGS_ERR_INPUT);
      }
      const bool keep = in.get_int("keep_state", 0) != 0;
      if (state) {
        warm_start_from(*h->solver, *state);
        h->solver->forced_reuse = in.get_int("forced_reuse", 0) != 0;
      }
      sgs_stats st{};
      // an upper bound of the output blob: the displacement grid (payload and
      // block bases), the residual history and 1 MiB for the rest
      OutputBlob blob_memory(in.density.num_blocks() * (256 * sizeof(double) + 3 * sizeof(int32_t)) +
                             size_t(std::max(0, h->solver->P.max_iterations) + 2) * sizeof(double) + (size_t(1) << 20));
      rc = sgs_solve(h, 0, 0, &st);
      if (state) {
        outs.extra_ints["warm_start_reused"] = h->solver->warm_reused ? 1 : 0;
        outs.extra_doubles["warm_start_residual"] = h->solver->warm_residual;
      }
      // keep (or create) the state, or release a state passed in (:389-408)
      if (keep) {
        if (!state) {
          state = new KeptState();
          state->initial_residual_linf = h->solver->initial_residual;
        }
        if (rc == 0) keep_solution(*h->solver, *state);
        const uint64_t addr = reinterpret_cast<uint64_t>(state);
        outs.extra_ints["state_ptr_lower"] = int32_t(uint32_t(addr & 0xffffffffu));
        outs.extra_ints["state_ptr_higher"] = int32_t(uint32_t(addr >> 32));
      } else if (state) {
        delete state;
      }
      outs.residuals = h->solver->history;
      outs.extra_ints["iterations"] = st.iterations;
      outs.extra_ints["device_loop"] = h->solver->loop_graph ? 1 : 0;
      outs.extra_doubles["initial_residual"] = st.initial_residual;
      outs.extra_doubles["final_residual"] = st.final_residual;
      outs.extra_doubles["setup_seconds"] = st.setup_seconds;
      outs.extra_doubles["host_setup_seconds"] = h->solver->host_setup_seconds;
      outs.extra_doubles["host_level0_seconds"] = h->solver->P.host_phase[0];
      outs.extra_doubles["host_coarsen_seconds"] = h->solver->P.host_phase[1];
      outs.extra_doubles["host_flags_seconds"] = h->solver->P.host_phase[2];
      outs.extra_doubles["host_rest_seconds"] = h->solver->P.host_phase[3];
      outs.extra_doubles["device_levels_seconds"] = h->solver->setup_phase[0];
      outs.extra_doubles["device_operators_seconds"] = h->solver->setup_phase[1];
      outs.extra_doubles["device_bottom_seconds"] = h->solver->setup_phase[2];
      outs.extra_doubles["device_vectors_seconds"] = h->solver->setup_phase[3];
      outs.extra_doubles["solve_seconds"] = st.solve_seconds;
      if (rc) {
        outs.error_code = rc;
        outs.info = h->error;
      } else {
        // The displacements go from the device straight into the output blob
        // (a pitched copy into its records); the phase times that follow are
        // patched into the encoded blob.
        const size_t nin = in.density.num_blocks();
        outs.displacements.base.assign(in.density.base.begin(), in.density.base.end());
        outs.extra_doubles["h2d_bytes"] = double(g_h2d_bytes.load() - h2d0);
        outs.extra_doubles["d2h_bytes"] = double(g_d2h_bytes.load() - d2h0 + nin * 256 * sizeof(double));
        outs.extra_doubles["solve_device_seconds"] = st.solve_device_seconds;
        outs.extra_doubles["output_seconds"] = 0;
        outs.extra_doubles["teardown_seconds"] = 0;
        outs.extra_ints["kernel_launches"] = int(st.kernel_launches);
        // as the reference, a solve that reaches the iteration cap still
        // returns its displacements with success set (SPGrid_CPU_Solver.cpp:326-341);
        // "converged" and the message say whether the stopping rule was met
        const bool converged = st.final_residual <= h->solver->P.tolerance * st.initial_residual;
        outs.extra_ints["converged"] = converged ? 1 : 0;
        outs.success = true;
        char m[200];
        std::snprintf(m, sizeof m,
                      converged ? "converged in %d iterations, L-inf residual %.6g of %.6g"
                                : "stopped at the iteration cap after %d iterations without converging, L-inf residual "
                                  "%.6g of %.6g",
                      st.iterations, st.final_residual, st.initial_residual);
        outs.info = m;
        const auto t2 = clk::now();
        char* blob = nullptr;
        try {
          Solver* S = h->solver.get();
          blob = encode_outputs(outs, nullptr, [S](uint8_t* p, size_t pitch, size_t) { S->pack_outputs(p, pitch); },
                                blob_memory.take(), blob_memory.capacity());
        } catch (const CudaError& e) {
          outs.displacements.base.clear();
          outs.success = false;
          outs.error_code = e.code;
          outs.info = e.what();
        } catch (const std::exception& e) {
          outs.displacements.base.clear();
          outs.success = false;
          outs.error_code = SGS_ERR_INTERNAL;
          outs.info = e.what();
        }
        if (blob) {
          patch_output_double(blob, outs, "output_seconds", secs(t2, clk::now()));
          const auto t3 = clk::now();
          guard.reset();
          patch_output_double(blob, outs, "teardown_seconds", secs(t3, clk::now()));
          *out_ptr = blob;
          return;
        }
      }
      const auto t3 = clk::now();
      guard.reset();
      outs.extra_doubles["teardown_seconds"] = secs(t3, clk::now());
    }
  } catch (const WireError& e) {
    outs.error_code = SGS_ERR_WIRE;
    outs.info = std::string("malformed input blob: ") + e.what();
  } catch (const CudaError& e) {
    outs.error_code = e.code;
    outs.info = e.what();
  } catch (const std::exception& e) {
    outs.error_code = SGS_ERR_INTERNAL;
    outs.info = e.what();
  }
  // a failure after the displacement grid was named leaves it without payload
  if (outs.displacements.data.size() != outs.displacements.num_blocks() * 256) {
    outs.displacements.base.clear();
    outs.displacements.data.clear();
  }
  try {
    *out_ptr = encode_outputs(outs, nullptr);
  } catch (...) {
    *out_ptr = nullptr;
  }
}

SGS_API void fem_solve_free(void* blob) { delete[] static_cast<char*>(blob); }

SGS_API int sgs_time_op(sgs_session* h, int op, int reps, double* ms) {
  if (!h || !ms || host_only(h) || reps <= 0 || op < 0 || op > 5) return SGS_ERR_INPUT;
  try {
    *ms = h->solver->mixed() && op != 0 && op != 3 ? time_op<float>(*h->solver, op, reps)
                                                   : time_op<double>(*h->solver, op, reps);
  } catch (const CudaError& e) {
    h->error = e.what();
    return e.code;
  }
  return 0;
}

SGS_API int sgs_codec_roundtrip(const void* blob, int which, void** out) {
  if (!blob || !out) return SGS_ERR_INPUT;
  *out = nullptr;
  try {
    if (which == 0) {
      std::vector<uint8_t> b = encode_inputs(decode_inputs(blob));
      char* o = new char[b.size()];
      std::memcpy(o, b.data(), b.size());
      *out = o;
    } else {
      *out = encode_outputs(decode_outputs(blob), nullptr);
    }
  } catch (const WireError&) {
    return SGS_ERR_WIRE;
  }
  return 0;
}

}  // extern "C"
