// Sparse tensor-times-matrix along the leaf mode of a 3-D CSF (TTM).
//
// Replaces TTM_GPU / TTM_CPU (src/ttm_gpu.cu:83-143, src/ttm_cpu.cpp:60-86):
// for every leaf fiber f (slice a, fiber index b; the rows of the reference's
// semi-sparse Y, src/util.h:182-187, 3175-3180)
//   Y[f, :] = sum over the fiber's nonzeros x of vals[x] * U[leaf(x), :].
// The reference runs a warp (or 16) per slice/fiber with scalar loads; here a
// team of G lanes (R = 4*G*V) walks a contiguous, nonzero-balanced chunk,
// numbers fibers from the fiber-start flags in bit 31 of the leaf index (one
// ballot and popcount per block of G nonzeros, from the chunk's precomputed
// first fiber) and accumulates in registers. Y is written with plain stores,
// never zeroed or read: the team that holds a fiber's first nonzero stores the
// fiber's row; a team whose chunk begins inside a fiber leaves that partial
// row in a per-chunk side buffer, and a second small kernel adds the side rows
// into Y once every owner has stored.
#include <cuda_bf16.h>

#include "format.h"
#include "prims.cuh"

using mmcsf::set_error;

namespace mmcsf {
namespace {

constexpr unsigned FULL = 0xffffffffu;
constexpr uint32_t FLAG = 0x80000000u;

template <class T> __device__ __forceinline__ float4 ldrow(const T* p);
template <> __device__ __forceinline__ float4 ldrow<float>(const float* p) {
  return __ldg(reinterpret_cast<const float4*>(p));
}
template <> __device__ __forceinline__ float4 ldrow<__nv_bfloat16>(const __nv_bfloat16* p) {
  const uint2 u = __ldg(reinterpret_cast<const uint2*>(p));
  return make_float4(__uint_as_float(u.x << 16), __uint_as_float(u.x & 0xffff0000u), __uint_as_float(u.y << 16),
                     __uint_as_float(u.y & 0xffff0000u));
}
__device__ __forceinline__ void red4(float* p, float4 v) {
  asm volatile("red.global.add.v4.f32 [%0], {%1, %2, %3, %4};" ::"l"(p), "f"(v.x), "f"(v.y), "f"(v.z), "f"(v.w)
               : "memory");
}

template <class T>
struct TArgs {
  const float* vals;
  const uint32_t* leaf;  // leaf index, bit 31 on each fiber's first nonzero
  const uint32_t* fptr;  // fiber -> first nonzero [F+1]
  const uint32_t* cfib;  // first fiber of every chunk, or null
  uint64_t nnz;
  uint32_t nfib, chunk;
  const T* U;            // leaf-mode factor, rows of R
  float* Y;              // F x R
  float* side;           // per chunk: R floats, the partial of a fiber begun in an earlier chunk
  uint32_t* side_fib;    // per chunk: that fiber, or NO_FIB
};

constexpr uint32_t NO_FIB = 0xffffffffu;

template <int G, int V, class T>
__global__ void __launch_bounds__(256) k_ttm(const TArgs<T> a) {
  constexpr uint32_t R = 4 * G * V;
  constexpr uint32_t GMASK = G == 32 ? FULL : ((1u << G) - 1u);
  const int lane = threadIdx.x & 31, tl = lane & (G - 1), tb = lane - tl;
  const uint64_t team = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) / G;
  const bool active = team * a.chunk < a.nnz;
  const uint64_t x0 = active ? team * a.chunk : a.nnz - 1;
  const uint64_t x1 = active ? min(x0 + a.chunk, a.nnz) : x0;
  auto col = [&](int v) { return (uint32_t)(tl + v * G) * 4; };
  uint32_t f;
  if (a.cfib) {
    f = active ? __ldg(a.cfib + team) : a.nfib - 1;
  } else {
    uint32_t lo = 0, hi = a.nfib - 1;
    while (lo < hi) {
      const uint32_t m = (lo + hi + 1) >> 1;
      if ((uint64_t)__ldg(a.fptr + m) <= x0) lo = m; else hi = m - 1;
    }
    f = lo;
  }
  float4 acc[V];
#pragma unroll
  for (int v = 0; v < V; ++v) acc[v] = make_float4(0.f, 0.f, 0.f, 0.f);
  // the open fiber began in an earlier chunk: its partial goes to the side buffer
  bool cont = active && (uint64_t)__ldg(a.fptr + f) < x0;
  auto emit = [&]() {
    float* dst = cont ? a.side + team * R : a.Y + (uint64_t)f * R;
#pragma unroll
    for (int v = 0; v < V; ++v) *reinterpret_cast<float4*>(dst + col(v)) = acc[v];
    if (cont && tl == 0) a.side_fib[team] = f;
    cont = false;
  };
  if (active && !cont && tl == 0) a.side_fib[team] = NO_FIB;
  for (uint32_t it = 0; it < a.chunk; it += G) {
    const uint64_t xl = x0 + it + tl;
    uint32_t kv = 0;
    float vv = 0.f;
    if (xl < x1) { kv = __ldg(a.leaf + xl); vv = __ldg(a.vals + xl); }
    const uint32_t fm = (__ballot_sync(FULL, (kv & FLAG) && xl != x0) >> tb) & GMASK;
    const uint32_t k = kv & ~FLAG;
    float4 rows[G][V];
#pragma unroll
    for (int j = 0; j < G; ++j) {
      const uint32_t kj = __shfl_sync(FULL, k, tb + j);
#pragma unroll
      for (int v = 0; v < V; ++v) rows[j][v] = ldrow(a.U + (uint64_t)kj * R + col(v));
    }
#pragma unroll
    for (int j = 0; j < G; ++j) {
      const float val = __shfl_sync(FULL, vv, tb + j);
      if ((fm >> j) & 1u) {  // nonzero j opens the next fiber: the open one is complete here
        emit();
#pragma unroll
        for (int v = 0; v < V; ++v) acc[v] = make_float4(0.f, 0.f, 0.f, 0.f);
        ++f;
      }
#pragma unroll
      for (int v = 0; v < V; ++v) {
        acc[v].x = fmaf(val, rows[j][v].x, acc[v].x);
        acc[v].y = fmaf(val, rows[j][v].y, acc[v].y);
        acc[v].z = fmaf(val, rows[j][v].z, acc[v].z);
        acc[v].w = fmaf(val, rows[j][v].w, acc[v].w);
      }
    }
  }
  if (active) emit();
}

// Y[side_fib[c]] += side[c] for every chunk c that began inside a fiber.
template <int G>
__global__ void __launch_bounds__(256) k_ttm_side(const float* __restrict__ side,
                                                   const uint32_t* __restrict__ side_fib, uint64_t nchunks,
                                                   uint32_t R, float* __restrict__ Y) {
  const uint64_t t = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) / G;
  const int tl = threadIdx.x & (G - 1);
  if (t >= nchunks) return;
  const uint32_t f = side_fib[t];
  if (f == NO_FIB) return;
  for (uint32_t c = tl * 4; c < R; c += G * 4)
    red4(Y + (uint64_t)f * R + c, *reinterpret_cast<const float4*>(side + t * R + c));
}

template <class T>
cudaError_t launch_ttm(const TArgs<T>& a, int R, cudaStream_t s) {
  auto go = [&](auto kern, int G) {
    const uint64_t teams = (a.nnz + a.chunk - 1) / a.chunk;
    kern<<<(unsigned)((teams * G + 255) / 256), 256, 0, s>>>(a);
    return cudaGetLastError();
  };
  switch (R) {
    case 4: return go(k_ttm<1, 1, T>, 1);
    case 8: return go(k_ttm<2, 1, T>, 2);
    case 16: return go(k_ttm<4, 1, T>, 4);
    case 32: return go(k_ttm<8, 1, T>, 8);
    case 64: return go(k_ttm<16, 1, T>, 16);
    case 128: return go(k_ttm<32, 1, T>, 32);
    default: return cudaErrorInvalidValue;
  }
}

}  // namespace
}  // namespace mmcsf

using namespace mmcsf;

extern "C" int mmcsf_ttm(const mmcsf_format* F, int R, int factor_dtype, const void* d_factor, float* d_Y,
                         uint64_t* n_fibers, void* stream) {
  MMCSF_RANGE("mmcsf_ttm");
  if (!F) return set_error(MMCSF_ERR_INVALID, "null format");
  MMCSF_TRY(bounds_gate(F, stream));
  if (F->impl != MMCSF_IMPL_BCSF) return set_error(MMCSF_ERR_INVALID, "TTM runs on a B-CSF format (-t 8) of the mode");
  const CsfPart& P = F->parts[0];
  if (P.nd != 3) return set_error(MMCSF_ERR_UNSUPPORTED, "TTM is 3-D (as the reference's)");
  if (n_fibers) *n_fibers = P.present ? P.n_fibers() : 0;
  if (!d_factor || !d_Y) return n_fibers ? MMCSF_OK : set_error(MMCSF_ERR_INVALID, "null pointer");
  if (R != 4 && R != 8 && R != 16 && R != 32 && R != 64 && R != 128)
    return set_error(MMCSF_ERR_UNSUPPORTED, "TTM runs ranks 4, 8, ..., 128");
  if (factor_dtype != MMCSF_DTYPE_F32 && factor_dtype != MMCSF_DTYPE_BF16)
    return set_error(MMCSF_ERR_INVALID, "bad dtype");
  if (!P.present || P.nnz == 0) return MMCSF_OK;
  cudaStream_t s = S(stream);
  const int slot = CsfPart::cfib_slot(512);
  const uint64_t nchunks = (P.nnz + 511) / 512;
  // the per-chunk side rows live with the format, sized for the largest R used
  mmcsf_format* Fm = const_cast<mmcsf_format*>(F);
  const uint64_t side_bytes = nchunks * ((uint64_t)R * 4 + 4);
  if (Fm->ttm_side.bytes < side_bytes) MMCSF_CUDA(Fm->ttm_side.alloc(side_bytes));
  float* side = Fm->ttm_side.as<float>();
  uint32_t* side_fib = reinterpret_cast<uint32_t*>(side + nchunks * (uint64_t)R);
  cudaError_t e;
  auto fill = [&](auto& a, auto tag) {
    using T = decltype(tag);
    a.vals = P.vals.as<float>();
    a.leaf = P.leaf.as<uint32_t>();
    a.fptr = P.ptr[1].as<uint32_t>();
    a.cfib = P.cfib[slot].p ? P.cfib[slot].as<uint32_t>() : nullptr;
    a.nnz = P.nnz;
    a.nfib = (uint32_t)P.n_fibers();
    a.chunk = 512;
    a.U = static_cast<const T*>(d_factor);
    a.Y = d_Y;
    a.side = side;
    a.side_fib = side_fib;
  };
  if (factor_dtype == MMCSF_DTYPE_F32) {
    TArgs<float> a{};
    fill(a, float{});
    e = launch_ttm<float>(a, R, s);
  } else {
    TArgs<__nv_bfloat16> a{};
    fill(a, __nv_bfloat16{});
    e = launch_ttm<__nv_bfloat16>(a, R, s);
  }
  if (e != cudaSuccess) return set_error(MMCSF_ERR_CUDA, "TTM launch: %s", cudaGetErrorString(e));
  k_ttm_side<8><<<(unsigned)((nchunks * 8 + 255) / 256), 256, 0, s>>>(side, side_fib, nchunks, (uint32_t)R, d_Y);
  e = cudaGetLastError();
  if (e != cudaSuccess) return set_error(MMCSF_ERR_CUDA, "TTM side launch: %s", cudaGetErrorString(e));
  Fm->last_launches = 2;
  return MMCSF_OK;
}
