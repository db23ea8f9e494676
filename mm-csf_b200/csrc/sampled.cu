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
  // fused Poisson step (k_poisson_rows)
  const float* y;      // tensor values, format order
  float* grad_root;    // dims[order[0]] x R, zeroed by the caller
  double* loss;        // one double, zeroed by the caller
  float eps;
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


__device__ __forceinline__ void red4(float* p, float4 v) {
  asm volatile("red.global.add.v4.f32 [%0], {%1, %2, %3, %4};" ::"l"(p), "f"(v.x), "f"(v.y), "f"(v.z), "f"(v.w)
               : "memory");
}

// Fused Poisson step on a 3-D part (gradient CP; no counterpart in the
// reference). One per-nonzero walk computes, for every nonzero x,
//   xhat[x] = sum_r A[a,r] B[b,r] C[k,r]       (A, B, C: the part's levels)
//   w[x]    = y[x] / (xhat[x] + eps)           (stored, format order)
// and accumulates
//   loss    = sum_x y[x] log(xhat[x] + eps)
//   G[a,:] += w[x] B[b,:] (.) C[k,:]           (the slice mode's gradient of loss)
// so the sampled model, the loss's elementwise work and the slice mode's
// adjoint share one gather of B and C per nonzero. Per block of G nonzeros a
// lane keeps B (.) C of every nonzero, the partial dot products with the slice
// row are reduced by one transposed butterfly (lane j ends with xhat of
// nonzero j), w goes back to the team by shuffles and G accumulates per slice
// run with one vector reduction per run. A slice change inside a block is
// followed by two trackers: one for the slice row (before the reduction), one
// for the accumulator (after it).
template <int G, int V, class T>
__global__ void __launch_bounds__(256) k_poisson_rows(const SArgs<T> a) {
  constexpr uint32_t R = 4 * G * V;
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
  uint32_t sl2 = sl;                         // accumulator's slice
  uint64_t nxt = __ldg(a.snz + sl + 1), nxt2 = nxt;
  uint32_t ca2 = __ldg(a.sidx + sl);
  float4 ra[V], acc[V];
  auto slice_row = [&]() {
    const uint32_t ca = __ldg(a.sidx + sl);
#pragma unroll
    for (int v = 0; v < V; ++v) ra[v] = ld4(a.U[0] + (uint64_t)ca * R + col(v));
  };
  slice_row();
#pragma unroll
  for (int v = 0; v < V; ++v) acc[v] = make_float4(0.f, 0.f, 0.f, 0.f);
  double lsum = 0.0;
  for (uint32_t it = 0; it < a.chunk; it += G) {
    const uint64_t xb = x0 + it;
    const uint64_t xl = xb + tl;
    uint32_t k = 0, b = 0;
    float yv = 0.f;
    if (xl < x1) {
      k = __ldg(a.leaf + xl) & ~FLAG;
      b = __ldg(a.mid + xl);
      yv = __ldg(a.y + xl);
    }
    const bool slow = __any_sync(FULL, xb < x1 && xb + G > nxt);
    float4 bc[G][V];
    float p[G];
#pragma unroll
    for (int j = 0; j < G; ++j) {
      const uint32_t kj = __shfl_sync(FULL, k, tb + j);
      const uint32_t bj = __shfl_sync(FULL, b, tb + j);
      if (slow) {
        if (xb + j < x1 && xb + j == nxt) {
          ++sl;
          nxt = __ldg(a.snz + sl + 1);
          slice_row();
        }
      }
      float d = 0.f;
#pragma unroll
      for (int v = 0; v < V; ++v) {
        bc[j][v] = mul4(ld4(a.U[1] + (uint64_t)bj * R + col(v)), ld4(a.U[2] + (uint64_t)kj * R + col(v)));
        d += ra[v].x * bc[j][v].x + ra[v].y * bc[j][v].y + ra[v].z * bc[j][v].z + ra[v].w * bc[j][v].w;
      }
      p[j] = d;
    }
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
    float wv = 0.f;
    if (xl < x1) {
      const float m = p[0] + a.eps;
      wv = yv / m;
      a.out[xl] = wv;
      lsum += (double)yv * (double)logf(m);
    }
#pragma unroll
    for (int j = 0; j < G; ++j) {
      const float wj = __shfl_sync(FULL, wv, tb + j);
      if (slow) {
        if (xb + j < x1 && xb + j == nxt2) {
#pragma unroll
          for (int v = 0; v < V; ++v) {
            red4(a.grad_root + (uint64_t)ca2 * R + col(v), acc[v]);
            acc[v] = make_float4(0.f, 0.f, 0.f, 0.f);
          }
          ++sl2;
          nxt2 = __ldg(a.snz + sl2 + 1);
          ca2 = __ldg(a.sidx + sl2);
        }
      }
#pragma unroll
      for (int v = 0; v < V; ++v) {
        acc[v].x = fmaf(wj, bc[j][v].x, acc[v].x);
        acc[v].y = fmaf(wj, bc[j][v].y, acc[v].y);
        acc[v].z = fmaf(wj, bc[j][v].z, acc[v].z);
        acc[v].w = fmaf(wj, bc[j][v].w, acc[v].w);
      }
    }
  }
  if (active) {
#pragma unroll
    for (int v = 0; v < V; ++v) red4(a.grad_root + (uint64_t)ca2 * R + col(v), acc[v]);
  }
  // loss: lanes of a team hold partial sums of their own nonzeros
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) lsum += __shfl_xor_sync(FULL, lsum, o);
  if (lane == 0) atomicAdd(a.loss, lsum);
}

template <class T>
cudaError_t launch_poisson(const SArgs<T>& a, int R, cudaStream_t s) {
  auto go = [&](auto kern, int G) {
    const uint64_t teams = (a.nnz + a.chunk - 1) / a.chunk;
    const uint64_t blocks = (teams * G + 255) / 256;
    kern<<<(unsigned)blocks, 256, 0, s>>>(a);
    return cudaGetLastError();
  };
  switch (R) {
    case 4: return go(k_poisson_rows<1, 1, T>, 1);
    case 8: return go(k_poisson_rows<2, 1, T>, 2);
    case 16: return go(k_poisson_rows<4, 1, T>, 4);
    case 32: return go(k_poisson_rows<8, 1, T>, 8);
    case 64: return go(k_poisson_rows<16, 1, T>, 16);
    default: return cudaErrorInvalidValue;
  }
}

int n_parts(const mmcsf_format* F) {
  int k = 0;
  for (int p = 0; p < 4; ++p) k += F->parts[p].present ? 1 : 0;
  return k;
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
  MMCSF_RANGE("mmcsf_sampled_model");
  if (!F || !d_factors || !d_out) return set_error(MMCSF_ERR_INVALID, "null argument");
  MMCSF_TRY(bounds_gate(F, stream));
  if (F->impl == MMCSF_IMPL_HBCSF) return set_error(MMCSF_ERR_UNSUPPORTED, "not available for HB-CSF formats");
  if (R != 4 && R != 8 && R != 16 && R != 32 && R != 64 && R != 128 && R != 256)
    return set_error(MMCSF_ERR_UNSUPPORTED, "sampled model runs ranks 4, 8, ..., 256");
  if (factor_dtype != MMCSF_DTYPE_F32 && factor_dtype != MMCSF_DTYPE_BF16)
    return set_error(MMCSF_ERR_INVALID, "bad dtype");
  // every part in the format's nonzero order (MM-CSF partitions 0..nd-1)
  uint64_t off = 0;
  int launched = 0;
  for (int p = 0; p < 4; ++p) {
  const CsfPart* P = F->impl == MMCSF_IMPL_MMCSF ? &F->parts[p] : (p == 0 ? &F->parts[0] : nullptr);
  if (!P || !P->present || !P->nnz) continue;
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
    a.out = d_out + off;
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
  off += P->nnz;
  ++launched;
  }
  const_cast<mmcsf_format*>(F)->last_launches = launched;
  return MMCSF_OK;
}

extern "C" int mmcsf_poisson_step(const mmcsf_format* F, int R, int factor_dtype, const void* const* d_factors,
                                  float eps, float* d_w, float* d_grad_root, double* d_loss, int* root_mode,
                                  void* stream) {
  MMCSF_RANGE("mmcsf_poisson_step");
  if (!F || !d_factors || !d_w || !d_grad_root || !d_loss) return set_error(MMCSF_ERR_INVALID, "null argument");
  MMCSF_TRY(bounds_gate(F, stream));
  if (F->impl == MMCSF_IMPL_HBCSF) return set_error(MMCSF_ERR_UNSUPPORTED, "not available for HB-CSF formats");
  if (R != 4 && R != 8 && R != 16 && R != 32 && R != 64)
    return set_error(MMCSF_ERR_UNSUPPORTED, "the fused Poisson step runs ranks 4, 8, 16, 32, 64");
  if (factor_dtype != MMCSF_DTYPE_F32 && factor_dtype != MMCSF_DTYPE_BF16)
    return set_error(MMCSF_ERR_INVALID, "bad dtype");
  if (n_parts(F) > 1)
    return set_error(MMCSF_ERR_UNSUPPORTED, "the fused Poisson step needs a single-partition format");
  const CsfPart* P = main_part(F);
  if (!P || P->nd != 3 || !P->mid.p) return set_error(MMCSF_ERR_UNSUPPORTED, "the fused Poisson step needs a 3-D part");
  if (root_mode) *root_mode = P->order[0];
  cudaStream_t s = S(stream);
  MMCSF_CUDA(cudaMemsetAsync(d_grad_root, 0, F->dims[P->order[0]] * (uint64_t)R * sizeof(float), s));
  MMCSF_CUDA(cudaMemsetAsync(d_loss, 0, sizeof(double), s));
  if (!P->nnz) return MMCSF_OK;
  cudaError_t e;
  auto fill = [&](auto& a, auto tag) {
    using T = decltype(tag);
    a.leaf = P->leaf.as<uint32_t>();
    a.mid = P->mid.as<uint32_t>();
    a.snz = P->snz.as<uint32_t>();
    a.sidx = P->idx[0].as<uint32_t>();
    a.cslc = P->cslc[CsfPart::cfib_slot(256)].p ? P->cslc[CsfPart::cfib_slot(256)].as<uint32_t>() : nullptr;
    a.nslc = (uint32_t)P->n[0];
    a.nnz = P->nnz;
    a.chunk = 256;
    for (int l = 0; l < 3; ++l) a.U[l] = static_cast<const T*>(d_factors[P->order[l]]);
    a.y = P->vals.as<float>();
    a.out = d_w;
    a.grad_root = d_grad_root;
    a.loss = d_loss;
    a.eps = eps;
  };
  if (factor_dtype == MMCSF_DTYPE_F32) {
    SArgs<float> a{};
    fill(a, float{});
    e = launch_poisson<float>(a, R, s);
  } else {
    SArgs<__nv_bfloat16> a{};
    fill(a, __nv_bfloat16{});
    e = launch_poisson<__nv_bfloat16>(a, R, s);
  }
  if (e != cudaSuccess) return set_error(MMCSF_ERR_CUDA, "Poisson step launch: %s", cudaGetErrorString(e));
  const_cast<mmcsf_format*>(F)->last_launches = 1;
  return MMCSF_OK;
}

extern "C" int mmcsf_format_values(const mmcsf_format* F, const float** d_vals, uint64_t* nnz) {
  if (!F) return set_error(MMCSF_ERR_INVALID, "null argument");
  if (F->impl == MMCSF_IMPL_HBCSF) return set_error(MMCSF_ERR_UNSUPPORTED, "not available for HB-CSF formats");
  if (n_parts(F) > 1) {  // several partitions: their values concatenated at construction
    if (d_vals) *d_vals = F->all_vals.as<float>();
    if (nnz) *nnz = F->nnz;
    return MMCSF_OK;
  }
  const CsfPart* P = main_part(F);
  if (d_vals) *d_vals = P ? P->vals.as<float>() : nullptr;
  if (nnz) *nnz = P ? P->nnz : 0;
  return MMCSF_OK;
}
