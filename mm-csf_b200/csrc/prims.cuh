// Device primitives used by format construction and the generator:
// exclusive scans and a stable LSD radix sort, written for sm_100a.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace mmcsf {

// Stream-ordered temporary device allocation (cudaMallocAsync).
struct Tmp {
  void* p = nullptr;
  cudaStream_t s = nullptr;
  Tmp() = default;
  Tmp(const Tmp&) = delete;
  Tmp& operator=(const Tmp&) = delete;
  ~Tmp() { if (p) cudaFreeAsync(p, s); }
  cudaError_t alloc(size_t bytes, cudaStream_t st) {
    if (p) cudaFreeAsync(p, s);
    s = st;
    p = nullptr;
    return cudaMallocAsync(&p, bytes ? bytes : 16, st);
  }
  template <class T> T* as() const { return static_cast<T*>(p); }
};

// out[i] = sum(in[0..i-1]) for i in [0, n]; out has n+1 entries (out[n] =
// total). in and out may alias. Returns cudaSuccess or the first error.
cudaError_t exclusive_scan_u32(const uint32_t* in, uint32_t* out, uint64_t n, cudaStream_t s);

// Stable sort of (keys, vals) pairs by key bits [0, key_bits). On return the
// sorted data is in (keys, vals) — alt buffers are scratch of the same size.
cudaError_t radix_sort_pairs(uint64_t* keys, uint32_t* vals, uint64_t* keys_alt, uint32_t* vals_alt,
                             uint64_t n, int key_bits, cudaStream_t s);

// vals[i] = i
cudaError_t iota_u32(uint32_t* v, uint64_t n, cudaStream_t s);
// out[i] = in[perm[i]] for 4-byte elements
cudaError_t gather_u32(const uint32_t* in, const uint32_t* perm, uint32_t* out, uint64_t n, cudaStream_t s);

// The composite sort key of a format's construction (build.cu).
int sort_key_plan(int impl, int nd, const uint64_t* dims, int mode, int* keys);
void order_modes(int nd, const uint64_t* dims, int mode, int* order);

// Grid size for a grid-stride kernel: a multiple of the SM count.
int grid_for(uint64_t n, int threads);
int sm_count();

}  // namespace mmcsf
