// MTTKRP kernel arguments and the per-rank launchers shared by the host code
// (mttkrp.cu, sampled.cu) and the kernel translation units (mttkrp_r<R>.cu).
#pragma once
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "format.h"

namespace mmcsf {

template <class T>
struct Args {
  const float* vals;
  const uint32_t* leaf;
  const uint32_t* fptr;   // leaf fibers -> nonzeros [F+1]
  const uint32_t* fidx;   // leaf-fiber index (o1 in 3-D, o2 in 4-D)
  const uint32_t* fpar;   // 4-D: fiber -> fbrS
  const uint32_t* sidx1;  // 4-D: fbrS index (o1)
  const uint32_t* like;   // o0 per level-1 entry (3-D: fiber, 4-D: fbrS)
  const uint32_t* cfib;   // first fiber of every team's chunk, or null (binary search)
  const uint32_t* mid;    // per-nonzero walk: o_{nd-2} of every nonzero
  const uint32_t* mid2;   // ... 4-D: o1 of every nonzero
  const uint32_t* snz;    // ... first nonzero of every slice [nslc + 1]
  const uint32_t* sidx;   // ... slice index (o0) of every slice
  const uint32_t* cslc;   // ... slice of every team's chunk start, or null (binary search)
  uint32_t nslc;
  uint64_t nnz;
  uint32_t nfib;
  uint32_t chunk;
  uint32_t R;
  const T* U[4];  // factor of mode order[l], by level l
  float* out;
  float* out2;    // two-output walk: the middle mode's output
  double* out64;  // leaf-level outputs: per-nonzero scatters accumulate here in FP64 (converted by the host code)
};

template <class T, int R>
cudaError_t launch_fixed(const Args<T>& a, int nd, int lvl, int kern, int threads, int mb, cudaStream_t s);
template <class T, int R>
cudaError_t launch_pair_fixed(const Args<T>& a, int nd, int threads, int mb, int kern, cudaStream_t s);

// One mode's kernel for rank a.R (4, 8, ..., 256) at level `lvl`.
template <class T>
cudaError_t launch_R(const Args<T>& a, int nd, int lvl, int kern, int threads, int mb, cudaStream_t s) {
  switch (a.R) {
    case 4: return launch_fixed<T, 4>(a, nd, lvl, kern, threads, mb, s);
    case 8: return launch_fixed<T, 8>(a, nd, lvl, kern, threads, mb, s);
    case 16: return launch_fixed<T, 16>(a, nd, lvl, kern, threads, mb, s);
    case 32: return launch_fixed<T, 32>(a, nd, lvl, kern, threads, mb, s);
    case 64: return launch_fixed<T, 64>(a, nd, lvl, kern, threads, mb, s);
    case 128: return launch_fixed<T, 128>(a, nd, lvl, kern, threads, mb, s);
    case 256: return launch_fixed<T, 256>(a, nd, lvl, kern, threads, mb, s);
    default: return cudaErrorInvalidValue;
  }
}

// The two-output walk for rank a.R (4 .. 128).
template <class T>
cudaError_t launch_pair_R(const Args<T>& a, int nd, int threads, int mb, int kern, cudaStream_t s) {
  switch (a.R) {
    case 4: return launch_pair_fixed<T, 4>(a, nd, threads, mb, kern, s);
    case 8: return launch_pair_fixed<T, 8>(a, nd, threads, mb, kern, s);
    case 16: return launch_pair_fixed<T, 16>(a, nd, threads, mb, kern, s);
    case 32: return launch_pair_fixed<T, 32>(a, nd, threads, mb, kern, s);
    case 64: return launch_pair_fixed<T, 64>(a, nd, threads, mb, kern, s);
    case 128: return launch_pair_fixed<T, 128>(a, nd, threads, mb, kern, s);
    default: return cudaErrorInvalidValue;
  }
}

}  // namespace mmcsf
