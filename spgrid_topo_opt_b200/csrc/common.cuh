// Host utilities shared by the library's translation units: CUDA error
// checking, device buffers from the stream-ordered pool, host<->device byte
// counters.
#pragma once
#include <cuda_runtime.h>

#include <atomic>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/spgrid_fem.h"

namespace sgs {

struct CudaError : std::runtime_error {
  int code;
  CudaError(const std::string& m, int c) : std::runtime_error(m), code(c) {}
};

#define SGS_CUDA(x)                                                                                     \
  do {                                                                                                  \
    cudaError_t e_ = (x);                                                                               \
    if (e_ != cudaSuccess)                                                                              \
      throw CudaError(std::string(#x) + ": " + cudaGetErrorString(e_), SGS_ERR_CUDA);                   \
  } while (0)

// Host<->device bytes moved by this library (uploads, read-backs); sessions and
// fem_solve report the difference across a call.
inline std::atomic<unsigned long long> g_h2d_bytes{0}, g_d2h_bytes{0};

// Device buffers come from the device's default stream-ordered memory pool,
// whose release threshold is raised once per device so that freed memory stays
// with the process: a later session or fem_solve call of similar size then
// allocates without going to the driver.  Allocation is ordered on the legacy
// default stream and waited for, and release first waits for the device (as
// cudaFree does), so a buffer is ready when alloc returns and idle when freed.
inline void keep_pool_memory() {
  static bool done[64] = {false};
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64 || done[dev]) return;
  cudaMemPool_t pool;
  if (cudaDeviceGetDefaultMemPool(&pool, dev) == cudaSuccess) {
    uint64_t keep = ~uint64_t(0);
    cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
  }
  cudaGetLastError();
  done[dev] = true;
}

// Host-to-device copy of pageable memory through the library's pinned staging
// buffer (defined with it); returns when the source may be reused.
void staged_h2d(void* dst, const void* src, size_t bytes, cudaStream_t s);

template <typename T>
struct DevBuf {
  T* p = nullptr;
  size_t n = 0;
  DevBuf() = default;
  DevBuf(const DevBuf&) = delete;
  DevBuf& operator=(const DevBuf&) = delete;
  ~DevBuf() { release(); }
  void release() {
    if (p) {
      cudaDeviceSynchronize();
      cudaFreeAsync(p, 0);
    }
    p = nullptr;
    n = 0;
  }
  void alloc(size_t count) {
    release();
    n = count;
    if (count) {
      keep_pool_memory();
      SGS_CUDA(cudaMallocAsync(reinterpret_cast<void**>(&p), count * sizeof(T), 0));
      SGS_CUDA(cudaStreamSynchronize(0));
    }
  }
  void upload(const T* h, size_t count, cudaStream_t s) {
    alloc(count);
    // large arrays through the pinned staging buffer (about twice the
    // bandwidth of a pageable copy), small ones directly
    if (count * sizeof(T) >= (size_t(8) << 20))
      staged_h2d(p, h, count * sizeof(T), s);
    else if (count)
      SGS_CUDA(cudaMemcpyAsync(p, h, count * sizeof(T), cudaMemcpyHostToDevice, s));
    g_h2d_bytes += count * sizeof(T);
  }
  template <typename Alloc>
  void upload(const std::vector<T, Alloc>& v, cudaStream_t s) {
    upload(v.data(), v.size(), s);
  }
  void zero(cudaStream_t s) {
    if (n) SGS_CUDA(cudaMemsetAsync(p, 0, n * sizeof(T), s));
  }
};

inline unsigned blocks_for(long n, int t) { return unsigned((n + t - 1) / t); }

}  // namespace sgs
