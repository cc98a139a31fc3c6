// Byte-compatible codec for the solver's FEMInputs / FEMOutputs records.
//
// Layout (topo_opt/serialization.h:234-530, topo_opt/fem_interface.h:165-390):
// a size_t total length, then every field of the record's io() method in order;
// PODs little-endian at their C++ size, vectors and strings as a size_t count
// followed by the elements, maps as a count followed by key/value pairs in key
// order.  The structs here keep the reference's field names.
#pragma once
#include <cstdint>
#include <cstdlib>
#include <functional>
#include <map>
#include <memory>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include <sys/mman.h>

namespace sgs {

struct ForceOnNode {
  int32_t coord[3];
  double f[3];
};
struct DirichletOnNode {
  int32_t coord[3];
  int32_t axis;
  double value;
};
struct KrylovSolverParameters {
  double tolerance = 1e-4;
  int32_t max_iterations = 50;
  int32_t restart_iterations = 0;
  bool print_residuals = false;
};

// Host buffers of 8 MiB and more: 2 MiB aligned with transparent huge pages
// advised (the first touch faults a 2 MiB page at a time where the kernel
// allows it).  A released buffer goes to a process-wide cache (up to 4 GiB in
// all), from which the next request of at least four fifths of its size takes
// it back (the smallest such buffer): the buffers of repeated solves are then
// neither mapped nor faulted in again.  A buffer taken from the cache holds
// the contents it was released with.
void* host_large_alloc(size_t bytes);
void host_large_free(void* p);

// A host vector whose resize leaves new elements uninitialised, so that a large
// buffer can be zeroed and filled by parallel loops (first touch spread over
// the threads) instead of one serial value-initialisation.  Buffers of 8 MiB
// and more come from host_large_alloc.
template <typename T>
struct UninitAlloc : std::allocator<T> {
  template <typename U>
  struct rebind {
    using other = UninitAlloc<U>;
  };
  static constexpr size_t LARGE = size_t(8) << 20;
  UninitAlloc() = default;
  template <typename U>
  UninitAlloc(const UninitAlloc<U>&) {}
  T* allocate(size_t n) {
    if (n * sizeof(T) < LARGE) return std::allocator<T>::allocate(n);
    return static_cast<T*>(host_large_alloc(n * sizeof(T)));
  }
  void deallocate(T* p, size_t n) {
    if (n * sizeof(T) < LARGE)
      std::allocator<T>::deallocate(p, n);
    else
      host_large_free(p);
  }
  template <typename U>
  void construct(U* p) noexcept {
    ::new (static_cast<void*>(p)) U;
  }
  template <typename U, typename... Args>
  void construct(U* p, Args&&... args) {
    ::new (static_cast<void*>(p)) U(std::forward<Args>(args)...);
  }
};
template <typename T>
using HostBuf = std::vector<T, UninitAlloc<T>>;

// BlockedGrid with 4x4x4 blocks (fem_interface.h:109-160); payload per block is
// `width` doubles per node, in-block index i*16 + j*4 + k.

struct BlockedGrid {
  int32_t resolution[3] = {0, 0, 0};
  std::vector<int32_t> base;   // [n*3]
  HostBuf<double> data;        // [n*64*width], filled in parallel by the codec
  size_t num_blocks() const { return base.size() / 3; }
};

struct FEMBase {
  int32_t version_major = 3;
  int32_t version_minor = 1;
  std::map<std::string, std::string> extra_strings;
  std::map<std::string, int32_t> extra_ints;
  std::map<std::string, double> extra_doubles;

  int32_t get_int(const std::string& k, int32_t d) const {
    auto it = extra_ints.find(k);
    return it == extra_ints.end() ? d : it->second;
  }
  double get_double(const std::string& k, double d) const {
    auto it = extra_doubles.find(k);
    return it == extra_doubles.end() ? d : it->second;
  }
  // Solver-state pointer split in two ints (fem_interface.h:193-209).
  void set_state_ptr(void* p) {
    uint64_t a = reinterpret_cast<uint64_t>(p);
    extra_ints["state_ptr_lower"] = int32_t(uint32_t(a & 0xffffffffu));
    extra_ints["state_ptr_higher"] = int32_t(uint32_t(a >> 32));
  }
  void* get_state_ptr() const {
    auto lo = extra_ints.find("state_ptr_lower");
    if (lo == extra_ints.end()) return nullptr;
    auto hi = extra_ints.find("state_ptr_higher");
    uint64_t a = uint64_t(uint32_t(lo->second)) | (uint64_t(uint32_t(hi == extra_ints.end() ? 0 : hi->second)) << 32);
    return reinterpret_cast<void*>(a);
  }
};

struct FEMInputs : FEMBase {
  int32_t resolution[3] = {0, 0, 0};
  double dx = 1.0;
  KrylovSolverParameters krylov;
  uint64_t preserved_buffer_size = 0;
  bool use_density_only = true;
  BlockedGrid density, mu, lambda;
  double global_mu = 0, global_lambda = 0;
  int32_t mg_level = 3, explicit_mg_level = 0, pre_and_post_smoothing_iter = 1, bottom_smoothing_iter = 600;
  double jacobi_damping = 0.4;
  std::string caller_method;
  std::vector<DirichletOnNode> dirichlet_nodes, dirichlet_cells;
  std::vector<ForceOnNode> forces;
};

struct FEMOutputs : FEMBase {
  BlockedGrid displacements;   // width 4: (u_x, u_y, u_z, |r|_inf)
  BlockedGrid residual_field;  // width 1
  std::string info;
  std::vector<double> residuals;
  int32_t error_code = 0;
  bool success = false;
};

class WireError : public std::runtime_error {
 public:
  using std::runtime_error::runtime_error;
};

// Decode an input blob (its first 8 bytes hold the total length).
FEMInputs decode_inputs(const void* blob);
// Encode outputs; the returned buffer is allocated with new char[] so that the
// reference caller can release it with delete[] (fem_interface.h:438-441, 477).
char* encode_outputs(const FEMOutputs& o, size_t* length);
// The same, with the displacement payload written straight into the blob by
// `fill` (o.displacements.base set, o.displacements.data empty):
// fill(first record's payload, record pitch in bytes, record count).
using GridFill = std::function<void(uint8_t*, size_t, size_t)>;
char* encode_outputs(const FEMOutputs& o, size_t* length, const GridFill& fill);
// The same into `buffer` (allocated with new char[] by the caller, ownership
// passes to the result) when its `capacity` holds the blob, else into a new one
// (and `buffer` is released).
char* encode_outputs(const FEMOutputs& o, size_t* length, const GridFill& fill, char* buffer, size_t capacity);
// Overwrite extra_doubles[key] (present in o when it was encoded) in the blob.
void patch_output_double(char* blob, const FEMOutputs& o, const std::string& key, double value);
// Encode inputs (used by tests and tools that drive the library from C++).
std::vector<uint8_t> encode_inputs(const FEMInputs& p);
FEMOutputs decode_outputs(const void* blob);

}  // namespace sgs
