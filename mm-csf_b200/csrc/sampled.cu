// Sampled CP model: xhat[x] = sum_r lambda_r prod_m A_m[i_m(x), r] at every
// nonzero x of a format, in the format's nonzero order (no counterpart in the
// reference). Its adjoint with respect to A_n is an MTTKRP of the tensor with
// the same sparsity and the upstream gradients as values
// (mmcsf_cp_adjoint), which is how gradient-based CP uses it.
//
// Traversal: a team of G lanes per row of R = 4*G*V values walks a contiguous
// range of nonzeros. k_sampled_rows (parts that carry per-nonzero middle
// indices, i.e. every MM-CSF and B-CSF part) gathers per nonzero the middle
// rows and the leaf row and reduces a block's partial dot products with one
// transposed butterfly; k_sampled (fallback) forms w = lambda (.) the rows
// above the leaf once per fiber and reduces each nonzero's dot product with
// shuffles inside the team.
#include <cuda_bf16.h>

#include "format.h"
#include "prims.cuh"

using mmcsf::set_error;

namespace mmcsf {
namespace {

constexpr unsigned FULL = 0xffffffffu;
constexpr uint32_t FLAG = 0x80000000u;

template <class T> __device__ __forceinline__ float4 ld4(const T* p);
template <> __device__ __forceinline__ float4 ld4<float>(const float* p) {
  return __ldg(reinterpret_cast<const float4*>(p));
}
template <> __device__ __forceinline__ float4 ld4<__nv_bfloat16>(const __nv_bfloat16* p) {
  const uint2 u = __ldg(reinterpret_cast<const uint2*>(p));
  return make_float4(__uint_as_float(u.x << 16), __uint_as_float(u.x & 0xffff0000u), __uint_as_float(u.y << 16),
                     __uint_as_float(u.y & 0xffff0000u));
}
__device__ __forceinline__ float4 mul4(float4 a, float4 b) {
  return make_float4(a.x * b.x, a.y * b.y, a.z * b.z, a.w * b.w);
}

template <class T>
struct SArgs {
  const uint32_t *leaf, *fptr, *fidx, *fpar, *sidx1, *like;
  const uint32_t* cfib;  // first fiber of every chunk, or null (binary search)
  const uint32_t *mid, *mid2, *snz, *sidx, *cslc;  // per-nonzero walk (see k_sampled_rows)
  uint32_t nslc;
  uint64_t nnz;
  uint32_t nfib, chunk;
  const T* U[4];      // by level
  const float* lam;   // R entries or null
  float* out;
};

__device__ __forceinline__ uint32_t find_fiber(const uint32_t* __restrict__ fptr, uint32_t nfib, uint64_t x) {
  uint32_t lo = 0, hi = nfib - 1;
  while (lo < hi) {
    const uint32_t mid = (lo + hi + 1) >> 1;
    if ((uint64_t)__ldg(fptr + mid) <= x) lo = mid; else hi = mid - 1;
  }
  return lo;
}

template <int ND, int G, int V, class T>
__global__ void __launch_bounds__(256) k_sampled(const SArgs<T> a) {
  constexpr uint32_t R = 4 * G * V;
  constexpr int LEAF = ND - 1;
  const int lane = threadIdx.x & 31, tl = lane & (G - 1), tb = lane - tl;
  const uint64_t team = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) / G;
  const bool active = team * a.chunk < a.nnz;
  const uint64_t x0 = active ? team * a.chunk : a.nnz - 1;
  const uint64_t x1 = active ? min(x0 + a.chunk, a.nnz) : x0;
  auto col = [&](int v) { return (uint32_t)(tl + v * G) * 4; };
  uint32_t f = a.cfib ? (active ? __ldg(a.cfib + team) : a.nfib - 1) : find_fiber(a.fptr, a.nfib, x0);
  float4 w[V];
  auto weights = [&]() {
    const uint32_t c = __ldg(a.fidx + f);
    uint32_t pa, pb;
    if (ND == 3) {
      pa = __ldg(a.like + f);
      pb = c;
    } else {
      const uint32_t fs = __ldg(a.fpar + f);
      pa = __ldg(a.like + fs);
      pb = __ldg(a.sidx1 + fs);
    }
#pragma unroll
    for (int v = 0; v < V; ++v) {
      float4 x = mul4(ld4(a.U[0] + (uint64_t)pa * R + col(v)), ld4(a.U[1] + (uint64_t)pb * R + col(v)));
      if (ND == 4) x = mul4(x, ld4(a.U[2] + (uint64_t)c * R + col(v)));
      if (a.lam) x = mul4(x, __ldg(reinterpret_cast<const float4*>(a.lam + col(v))));
      w[v] = x;
    }
  };
  weights();
  for (uint32_t it = 0; it < a.chunk; it += G) {
    const uint64_t xi = x0 + it + tl;
    const uint32_t kv = xi < x1 ? __ldg(a.leaf + xi) : 0u;
    const bool fl = xi < x1 && (kv & FLAG) && xi != x0;
    const uint32_t fm = __ballot_sync(FULL, fl) >> tb;
#pragma unroll
    for (int j = 0; j < G; ++j) {
      const uint32_t k = __shfl_sync(FULL, kv & ~FLAG, tb + j);
      const uint64_t x = x0 + it + j;
      if ((fm >> j) & 1u) {
        ++f;
        weights();
      }
      float p = 0.f;
#pragma unroll
      for (int v = 0; v < V; ++v) {
        const float4 r = ld4(a.U[LEAF] + (uint64_t)k * R + col(v));
        p += w[v].x * r.x + w[v].y * r.y + w[v].z * r.z + w[v].w * r.w;
      }
#pragma unroll
      for (int o = G / 2; o > 0; o >>= 1) p += __shfl_xor_sync(FULL, p, o);
      if (tl == 0 && x < x1) a.out[x] = p;
    }
  }
}


// Per-nonzero form: every nonzero carries its middle-level indices (`mid`,
// and `mid2` in 4-D), so per nonzero a team gathers the middle rows and the
// leaf row and forms the partial dot product of (lambda (.) slice row (.)
// middle rows) with the leaf row over its lane's columns. The G partial sums
// of a block (one per nonzero) are reduced across the team by a transposed
// butterfly -- G-1 shuffles per block instead of log2(G) per nonzero -- after
// which lane j holds the value of the block's nonzero j and the team stores
// the block with one coalesced write.
template <int ND, int G, int V, class T>
__global__ void __launch_bounds__(256) k_sampled_rows(const SArgs<T> a) {
  constexpr uint32_t R = 4 * G * V;
  constexpr int LEAF = ND - 1;
  const int lane = threadIdx.x & 31, tl = lane & (G - 1), tb = lane - tl;
  const uint64_t team = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) / G;
  const bool active = team * a.chunk < a.nnz;
  const uint64_t x0 = active ? team * a.chunk : a.nnz - 1;
  const uint64_t x1 = active ? min(x0 + a.chunk, a.nnz) : x0;
  auto col = [&](int v) { return (uint32_t)(tl + v * G) * 4; };
  uint32_t sl;
  if (a.cslc) {
    sl = active ? __ldg(a.cslc + team) : a.nslc - 1;
  } else {
    uint32_t lo = 0, hi = a.nslc - 1;
    while (lo < hi) {
      const uint32_t m = (lo + hi + 1) >> 1;
      if ((uint64_t)__ldg(a.snz + m) <= x0) lo = m; else hi = m - 1;
    }
    sl = lo;
  }
  uint64_t nxt = __ldg(a.snz + sl + 1);
  float4 wa[V];  // lambda (.) slice row
  auto slice_row = [&]() {
    const uint32_t ca = __ldg(a.sidx + sl);
#pragma unroll
    for (int v = 0; v < V; ++v) {
      float4 x = ld4(a.U[0] + (uint64_t)ca * R + col(v));
      if (a.lam) x = mul4(x, __ldg(reinterpret_cast<const float4*>(a.lam + col(v))));
      wa[v] = x;
    }
  };
  slice_row();
  for (uint32_t it = 0; it < a.chunk; it += G) {
    const uint64_t xb = x0 + it;
    const uint64_t xl = xb + tl;
    uint32_t k = 0, b = 0, q = 0;
    if (xl < x1) {
      k = __ldg(a.leaf + xl) & ~FLAG;
      b = __ldg(a.mid + xl);
      if constexpr (ND == 4) q = __ldg(a.mid2 + xl);
    }
    const bool slow = __any_sync(FULL, xb < x1 && xb + G > nxt);
    float p[G];
#pragma unroll
    for (int j = 0; j < G; ++j) {
      const uint32_t kj = __shfl_sync(FULL, k, tb + j);
      const uint32_t bj = __shfl_sync(FULL, b, tb + j);
      uint32_t qj = 0;
      if constexpr (ND == 4) qj = __shfl_sync(FULL, q, tb + j);
      if (slow) {
        if (xb + j < x1 && xb + j == nxt) {  // slice change (slices are never empty)
          ++sl;
          nxt = __ldg(a.snz + sl + 1);
          slice_row();
        }
      }
      float acc = 0.f;
#pragma unroll
      for (int v = 0; v < V; ++v) {
        float4 w = mul4(wa[v], ld4(a.U[ND - 2] + (uint64_t)bj * R + col(v)));
        if constexpr (ND == 4) w = mul4(w, ld4(a.U[1] + (uint64_t)qj * R + col(v)));
        const float4 c = ld4(a.U[LEAF] + (uint64_t)kj * R + col(v));
        acc += w.x * c.x + w.y * c.y + w.z * c.z + w.w * c.w;
      }
      p[j] = acc;
    }
    // transposed butterfly: lane tl ends with the sum of p[tl] over the team
#pragma unroll
    for (int st = G / 2; st >= 1; st >>= 1) {
      const bool up = (tl & st) != 0;
#pragma unroll
      for (int i = 0; i < st; ++i) {
        const float send = up ? p[i] : p[i + st];
        const float keep = up ? p[i + st] : p[i];
        p[i] = keep + __shfl_xor_sync(FULL, send, st);
      }
    }
    if (xl < x1) a.out[xl] = p[0];
  }
}

template <int ND, int G, int V, class T>
cudaError_t launch_s(const SArgs<T>& a, cudaStream_t s) {
  const uint64_t teams = (a.nnz + a.chunk - 1) / a.chunk;
  const uint64_t blocks = (teams * G + 255) / 256;
  if (a.mid) k_sampled_rows<ND, G, V, T><<<(unsigned)blocks, 256, 0, s>>>(a);
  else k_sampled<ND, G, V, T><<<(unsigned)blocks, 256, 0, s>>>(a);
  return cudaGetLastError();
}

template <class T>
cudaError_t launch_sR(const SArgs<T>& a, int nd, int R, cudaStream_t s) {
#define MMCSF_SCASE(RR, GG, VV) \
  case RR: return nd == 3 ? launch_s<3, GG, VV, T>(a, s) : launch_s<4, GG, VV, T>(a, s);
  switch (R) {
    MMCSF_SCASE(4, 1, 1)
    MMCSF_SCASE(8, 2, 1)
    MMCSF_SCASE(16, 4, 1)
    MMCSF_SCASE(32, 8, 1)
    MMCSF_SCASE(64, 16, 1)
    MMCSF_SCASE(128, 32, 1)
    MMCSF_SCASE(256, 32, 2)
    default: return cudaErrorInvalidValue;
  }
#undef MMCSF_SCASE
}

const CsfPart* main_part(const mmcsf_format* F) {
  if (F->impl == MMCSF_IMPL_MMCSF) {
    for (int p = 0; p < F->nd; ++p)
      if (F->parts[p].present) return &F->parts[p];
    return nullptr;
  }
  return F->parts[0].present ? &F->parts[0] : nullptr;
}

}  // namespace
}  // namespace mmcsf

using namespace mmcsf;

extern "C" int mmcsf_sampled_model(const mmcsf_format* F, int R, int factor_dtype, const void* const* d_factors,
                                   const float* d_lambda, float* d_out, void* stream) {
  if (!F || !d_factors || !d_out) return set_error(MMCSF_ERR_INVALID, "null argument");
  if (F->impl == MMCSF_IMPL_HBCSF) return set_error(MMCSF_ERR_UNSUPPORTED, "not available for HB-CSF formats");
  if (R != 4 && R != 8 && R != 16 && R != 32 && R != 64 && R != 128 && R != 256)
    return set_error(MMCSF_ERR_UNSUPPORTED, "sampled model runs ranks 4, 8, ..., 256");
  if (factor_dtype != MMCSF_DTYPE_F32 && factor_dtype != MMCSF_DTYPE_BF16)
    return set_error(MMCSF_ERR_INVALID, "bad dtype");
  const CsfPart* P = main_part(F);
  if (!P || !P->nnz) return MMCSF_OK;
  const int lf = P->nd - 2;
  cudaError_t e;
  auto fill = [&](auto& a, auto tag) {
    using T = decltype(tag);
    a.leaf = P->leaf.as<uint32_t>();
    a.fptr = P->ptr[lf].as<uint32_t>();
    a.fidx = P->idx[lf].as<uint32_t>();
    a.fpar = P->fpar.as<uint32_t>();
    a.sidx1 = P->nd == 4 ? P->idx[1].as<uint32_t>() : nullptr;
    a.like = P->fbr_like.as<uint32_t>();
    a.nnz = P->nnz;
    a.nfib = (uint32_t)P->n_fibers();
    a.chunk = 256;
    a.cfib = P->cfib[CsfPart::cfib_slot(256)].p ? P->cfib[CsfPart::cfib_slot(256)].as<uint32_t>() : nullptr;
    a.mid = P->mid.as<uint32_t>();
    a.mid2 = P->mid2.as<uint32_t>();
    a.snz = P->snz.as<uint32_t>();
    a.sidx = P->idx[0].as<uint32_t>();
    a.cslc = P->cslc[CsfPart::cfib_slot(256)].p ? P->cslc[CsfPart::cfib_slot(256)].as<uint32_t>() : nullptr;
    a.nslc = (uint32_t)P->n[0];
    for (int l = 0; l < P->nd; ++l) a.U[l] = static_cast<const T*>(d_factors[P->order[l]]);
    a.lam = d_lambda;
    a.out = d_out;
  };
  if (factor_dtype == MMCSF_DTYPE_F32) {
    SArgs<float> a{};
    fill(a, float{});
    e = launch_sR<float>(a, P->nd, R, S(stream));
  } else {
    SArgs<__nv_bfloat16> a{};
    fill(a, __nv_bfloat16{});
    e = launch_sR<__nv_bfloat16>(a, P->nd, R, S(stream));
  }
  if (e != cudaSuccess) return set_error(MMCSF_ERR_CUDA, "sampled model launch: %s", cudaGetErrorString(e));
  const_cast<mmcsf_format*>(F)->last_launches = 1;
  return MMCSF_OK;
}

extern "C" int mmcsf_format_values(const mmcsf_format* F, const float** d_vals, uint64_t* nnz) {
  if (!F) return set_error(MMCSF_ERR_INVALID, "null argument");
  if (F->impl == MMCSF_IMPL_HBCSF) return set_error(MMCSF_ERR_UNSUPPORTED, "not available for HB-CSF formats");
  const CsfPart* P = main_part(F);
  if (d_vals) *d_vals = P ? P->vals.as<float>() : nullptr;
  if (nnz) *nnz = P ? P->nnz : 0;
  return MMCSF_OK;
}
