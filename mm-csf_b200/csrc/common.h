// Internal definitions shared by the library's translation units.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <cstdarg>
#include <string>
#include <vector>

#include <nvtx3/nvToolsExt.h>

#include "../../include/mmcsf.h"

namespace mmcsf {

// An NVTX range over a scope, so that a profiler's timeline shows the
// library's entry points and CP-ALS phases by name (header-only NVTX 3: with
// no tool attached a push/pop is a call through a no-op pointer).
struct Range {
  explicit Range(const char* name) { nvtxRangePushA(name); }
  ~Range() { nvtxRangePop(); }
  Range(const Range&) = delete;
  Range& operator=(const Range&) = delete;
};

// Record a message for mmcsf_last_error() and return the status.
int set_error(int status, const char* fmt, ...);
void clear_error();

// Device buffer owned by a handle (cudaFree on destruction).
struct DevBuf {
  void* p = nullptr;
  size_t bytes = 0;
  DevBuf() = default;
  DevBuf(const DevBuf&) = delete;
  DevBuf& operator=(const DevBuf&) = delete;
  DevBuf(DevBuf&& o) noexcept : p(o.p), bytes(o.bytes) { o.p = nullptr; o.bytes = 0; }
  DevBuf& operator=(DevBuf&& o) noexcept {
    if (this != &o) { release(); p = o.p; bytes = o.bytes; o.p = nullptr; o.bytes = 0; }
    return *this;
  }
  ~DevBuf() { release(); }
  void release() {
    if (p) cudaFree(p);
    p = nullptr;
    bytes = 0;
  }
  // Returns cudaSuccess or the allocation error.
  cudaError_t alloc(size_t n) {
    release();
    if (n == 0) n = 16;
    cudaError_t e = cudaMalloc(&p, n);
    if (e != cudaSuccess) { p = nullptr; return e; }
    bytes = n;
    return cudaSuccess;
  }
  template <class T> T* as() const { return static_cast<T*>(p); }
};

// Stream from the ABI's void*.
inline cudaStream_t S(void* s) { return static_cast<cudaStream_t>(s); }

}  // namespace mmcsf

#define MMCSF_RANGE(name) ::mmcsf::Range mmcsf_range_(name)

// Evaluate a CUDA call; on failure record and return MMCSF_ERR_CUDA (or NOMEM).
#define MMCSF_CUDA(call)                                                                        \
  do {                                                                                          \
    cudaError_t e_ = (call);                                                                    \
    if (e_ != cudaSuccess) {                                                                    \
      return ::mmcsf::set_error(e_ == cudaErrorMemoryAllocation ? MMCSF_ERR_NOMEM : MMCSF_ERR_CUDA, \
                                "%s failed: %s (%s:%d)", #call, cudaGetErrorString(e_), __FILE__, __LINE__); \
    }                                                                                           \
  } while (0)

// Propagate a non-OK mmcsf status.
#define MMCSF_TRY(expr)            \
  do {                             \
    int s_ = (expr);               \
    if (s_ != MMCSF_OK) return s_; \
  } while (0)

// Check the last kernel launch.
#define MMCSF_LAUNCH_CHECK() MMCSF_CUDA(cudaGetLastError())

// mmcsf_coo internals.
struct mmcsf_coo {
  int nd = 0;
  uint64_t dims[4] = {0, 0, 0, 0};
  uint64_t nnz = 0;
  bool host_valid = false, dev_valid = false;
  std::vector<uint32_t> h_inds[4];
  std::vector<float> h_vals;
  mmcsf::DevBuf d_inds[4];
  mmcsf::DevBuf d_vals;
};
