// MTTKRP kernels for MM-CSF / B-CSF / HB-CSF parts on sm_100a.
//
// The reference launches one warp (or -w warps) per fiber, strides lanes over
// the rank with scalar 4-byte loads, and issues atomicAdd per fiber (slice and
// fiber modes) or per nonzero (leaf mode) (src/mttkrp_gpu.cu:716-1509).
// Here every mode uses the same nonzero-balanced traversal:
//   * a TEAM of G lanes owns one factor row (R = 4*G*V floats, each lane V
//     float4 = 16 B vectors), so one warp works on 32/G nonzeros at once;
//   * a team walks a fixed, contiguous range of `chunk` nonzeros — skewed
//     fibers and slices cost the same as uniform ones — locating its first
//     fiber by binary search over the fiber pointers;
//   * the team loads G leaf indices and values with one coalesced access,
//     broadcasts them by shuffle, and issues all G row gathers before using
//     any, so G independent 16-byte loads per lane are in flight;
//   * products are accumulated in registers along the fiber / fbrS / slice
//     hierarchy and flushed with ONE vector atomic (red.global.add.v4.f32) per
//     output row segment: per slice run for the slice mode, per fiber or fbrS
//     for the middle modes, per nonzero for the leaf mode (which scatters).
// Correct for every R (the reference's kernels keep one scalar accumulator per
// lane across the rank loop and are wrong for R > 32).
#include <algorithm>
#include <cuda_bf16.h>

#include <cstring>
#include <type_traits>

#include "format.h"
#include "prims.cuh"

using mmcsf::set_error;

namespace mmcsf {
namespace {

constexpr unsigned FULL = 0xffffffffu;

template <class T> struct Row;
template <> struct Row<float> {
  static __device__ __forceinline__ float4 load(const float* base, uint64_t off) {
    return __ldg(reinterpret_cast<const float4*>(base + off));
  }
};
template <> struct Row<__nv_bfloat16> {
  static __device__ __forceinline__ float4 load(const __nv_bfloat16* base, uint64_t off) {
    uint2 u = __ldg(reinterpret_cast<const uint2*>(base + off));
    float4 r;
    r.x = __uint_as_float(u.x << 16);
    r.y = __uint_as_float(u.x & 0xffff0000u);
    r.z = __uint_as_float(u.y << 16);
    r.w = __uint_as_float(u.y & 0xffff0000u);
    return r;
  }
};

__device__ __forceinline__ float4 f4(float a) { return make_float4(a, a, a, a); }
__device__ __forceinline__ float4 operator*(float4 a, float4 b) {
  return make_float4(a.x * b.x, a.y * b.y, a.z * b.z, a.w * b.w);
}
__device__ __forceinline__ float4 fma4(float s, float4 a, float4 c) {
  return make_float4(fmaf(s, a.x, c.x), fmaf(s, a.y, c.y), fmaf(s, a.z, c.z), fmaf(s, a.w, c.w));
}
__device__ __forceinline__ float4 fma4v(float4 a, float4 b, float4 c) {
  return make_float4(fmaf(a.x, b.x, c.x), fmaf(a.y, b.y, c.y), fmaf(a.z, b.z, c.z), fmaf(a.w, b.w, c.w));
}
// One vector reduction (PTX ISA 8.1+, sm_90+): four floats added at p (16 B aligned).
__device__ __forceinline__ void red4(float* p, float4 v) {
  asm volatile("red.global.add.v4.f32 [%0], {%1, %2, %3, %4};" ::"l"(p), "f"(v.x), "f"(v.y), "f"(v.z), "f"(v.w)
               : "memory");
}

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
  float* out2;  // two-output walk: the middle mode's output
};

// largest f with fptr[f] <= x
__device__ __forceinline__ uint32_t find_fiber(const uint32_t* __restrict__ fptr, uint32_t nfib, uint64_t x) {
  uint32_t lo = 0, hi = nfib - 1;
  while (lo < hi) {
    uint32_t mid = (lo + hi + 1) >> 1;
    if ((uint64_t)__ldg(fptr + mid) <= x) lo = mid; else hi = mid - 1;
  }
  return lo;
}

// ND: 3 or 4. OUT: output level (0 = slice ... ND-1 = leaf). G lanes per row,
// V float4 per lane, R = 4*G*V (a compile-time constant: row offsets are
// shifts, not 64-bit multiplies).
//
// Per team the only dependent-load chain left per block of G nonzeros is the
// factor-row gather: leaf indices and values for the next block are loaded
// while the current block is processed; fiber starts are flagged in bit 31 of
// the leaf index (no fiber-pointer reads after the initial search); the
// fibers' metadata (index, slice map) sits in a G-wide register window
// refilled with one coalesced load every G fibers; and the factor row a fiber
// needs when it closes is requested as soon as the fiber opens.
// MB: minimum resident 256-thread CTAs per SM the register allocation must
// allow; PFX: row gathers in flight per lane. The occupancy level picks the
// pair (1: 8 rows / 3 CTAs = 80 registers, 2: 8 rows / 4 CTAs = 64,
// 3: 4 rows / 5 CTAs = 48, 4: 4 rows / 6 CTAs = 40); the tuner picks per mode.
template <int ND, int OUT, int G, int V, class T, int MB, int PFX>
__global__ void __launch_bounds__(256, MB) k_mttkrp(const Args<T> a) {
  constexpr uint32_t R = 4 * G * V;
  constexpr int LEAF = ND - 1;
  constexpr uint32_t FLAG = 0x80000000u;
  constexpr int PF = G > PFX ? PFX : G;  // row gathers in flight per lane per batch
  const int lane = threadIdx.x & 31;
  const int tl = lane & (G - 1);
  const int tb = lane - tl;
  // kernel parameters in registers
  const float* __restrict__ vals = a.vals;
  const uint32_t* __restrict__ leaf = a.leaf;
  const uint32_t* __restrict__ fidx = a.fidx;
  const uint32_t* __restrict__ fpar = a.fpar;
  const uint32_t* __restrict__ sidx1 = a.sidx1;
  const uint32_t* __restrict__ like = a.like;
  const uint32_t nfib = a.nfib, chunk = a.chunk;
  const T* __restrict__ U0 = a.U[0];
  const T* __restrict__ U1 = a.U[1];
  const T* __restrict__ U2 = a.U[2];
  const T* __restrict__ UL = a.U[LEAF];
  float* __restrict__ out = a.out;
  const uint32_t c0 = (uint32_t)tl * 4;  // this lane's first column
  auto ld = [&](const T* U, uint32_t row, int v) -> float4 {
    return Row<T>::load(U + (uint64_t)row * R, c0 + (uint32_t)(v * G * 4));
  };
  auto rd = [&](uint32_t row, int v, float4 x) { red4(out + (uint64_t)row * R + c0 + v * G * 4, x); };

  const uint64_t team = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) / G;
  // Teams past the end stay in the loop (empty range) so every full-warp
  // shuffle sees all lanes; all teams run the same number of iterations.
  const bool active = team * chunk < a.nnz;
  const uint64_t x0 = active ? team * chunk : a.nnz - 1;
  const uint64_t x1 = active ? min(x0 + chunk, a.nnz) : x0;

  uint32_t f = a.cfib ? (active ? __ldg(a.cfib + team) : nfib - 1) : find_fiber(a.fptr, nfib, x0);
  // metadata of the open fiber (ci: b in 3-D, c in 4-D; cp: a in 3-D, fbrS
  // in 4-D) and of the next one, loaded a fiber ahead
  auto meta_i = [&](uint32_t q) { return __ldg(fidx + min(q, nfib - 1)); };
  auto meta_p = [&](uint32_t q) { return (ND == 3) ? __ldg(like + min(q, nfib - 1)) : __ldg(fpar + min(q, nfib - 1)); };
  uint32_t ci = meta_i(f), cp = meta_p(f);
  uint32_t nci = meta_i(f + 1), ncp = meta_p(f + 1);
  uint32_t sb = 0, sa = 0;                   // 4-D: current fbrS's b and a
  if (ND == 4) { sb = __ldg(sidx1 + cp); sa = __ldg(like + cp); }

  float4 acc[V], acc1[V], acc2[V], crow[V], srow[V];
#pragma unroll
  for (int v = 0; v < V; ++v) acc[v] = acc1[v] = acc2[v] = crow[v] = srow[v] = f4(0.f);
  uint32_t cur_a = (ND == 3) ? cp : sa;  // slice whose accumulation is open (OUT == 0)

  // rows needed per fbrS (4-D) and per fiber, requested when they open
  auto open_fbrs = [&]() {
    if constexpr (ND == 4) {
#pragma unroll
      for (int v = 0; v < V; ++v) {
        if constexpr (OUT == 0) srow[v] = ld(U1, sb, v);
        else if constexpr (OUT == 1) srow[v] = ld(U0, sa, v);
        else srow[v] = ld(U0, sa, v) * ld(U1, sb, v);
      }
    }
  };
  auto open_fiber = [&]() {
#pragma unroll
    for (int v = 0; v < V; ++v) {
      if constexpr (ND == 3) {
        if constexpr (OUT == 0) crow[v] = ld(U1, ci, v);
        else if constexpr (OUT == 1) crow[v] = ld(U0, cp, v);
        else crow[v] = ld(U0, cp, v) * ld(U1, ci, v);
      } else {
        if constexpr (OUT == 3) crow[v] = srow[v] * ld(U2, ci, v);
        else if constexpr (OUT != 2) crow[v] = ld(U2, ci, v);
      }
    }
  };
  open_fbrs();
  open_fiber();

  // Fold the open fiber's partial (acc) into the level above / the output.
  auto close_fiber = [&]() {
    if constexpr (OUT != LEAF) {
#pragma unroll
      for (int v = 0; v < V; ++v) {
        if constexpr (ND == 3 && OUT == 1) rd(ci, v, crow[v] * acc[v]);
        else if constexpr (ND == 4 && OUT == 2) rd(ci, v, srow[v] * acc[v]);
        else acc1[v] = fma4v(crow[v], acc[v], acc1[v]);
      }
    }
  };
  // 4-D: fold the open fbrS (acc1) upward (OUT 0) or out (OUT 1).
  auto close_fbrs = [&]() {
#pragma unroll
    for (int v = 0; v < V; ++v) {
      if constexpr (ND == 4 && OUT == 1) { rd(sb, v, srow[v] * acc1[v]); acc1[v] = f4(0.f); }
      else if constexpr (ND == 4 && OUT == 0) { acc2[v] = fma4v(srow[v], acc1[v], acc2[v]); acc1[v] = f4(0.f); }
    }
  };
  auto flush_slice = [&]() {
#pragma unroll
    for (int v = 0; v < V; ++v) {
      if constexpr (OUT == 0 && ND == 3) { rd(cur_a, v, acc1[v]); acc1[v] = f4(0.f); }
      else if constexpr (OUT == 0) { rd(cur_a, v, acc2[v]); acc2[v] = f4(0.f); }
    }
  };
  // nonzero x opens fiber f+1 (team-uniform branch; no shuffles inside)
  auto advance = [&]() {
    close_fiber();
    ++f;
    ci = nci;
    const uint32_t np = ncp;
    nci = meta_i(f + 1);
    ncp = meta_p(f + 1);
    if constexpr (ND == 3) {
      if (OUT == 0 && np != cur_a) { flush_slice(); cur_a = np; }
      cp = np;
    } else {
      if (np != cp) {  // new fbrS
        close_fbrs();
        cp = np;
        sb = __ldg(sidx1 + cp);
        sa = __ldg(like + cp);
        if (OUT == 0 && sa != cur_a) { flush_slice(); cur_a = sa; }
        open_fbrs();
      }
    }
    open_fiber();
  };

  uint32_t nk = 0;
  float nv = 0.f;
  if (x0 + tl < x1) { nk = __ldg(leaf + x0 + tl); nv = __ldg(vals + x0 + tl); }
  for (uint32_t it = 0; it < chunk; it += G) {
    const uint64_t xb = x0 + it;
    const uint32_t kv = nk;
    const float vv = nv;
    {  // next block's indices and values, while this block is processed
      const uint64_t xn = xb + G + tl;
      nk = 0;
      nv = 0.f;
      if (it + G < chunk && xn < x1) { nk = __ldg(leaf + xn); nv = __ldg(vals + xn); }
    }
    // a lane past the range holds val 0 and no flag, and gathers row 0
    const bool fl = (kv & FLAG) && (xb + tl != x0);
    const uint32_t fm = (__ballot_sync(FULL, fl) >> tb);
    const uint32_t k = kv & ~FLAG;
#pragma unroll
    for (int jb = 0; jb < G; jb += PF) {
      float4 rows[PF][V];
      uint32_t kj[PF];
#pragma unroll
      for (int j = 0; j < PF; ++j) {
        kj[j] = __shfl_sync(FULL, k, tb + jb + j);
        if constexpr (OUT != LEAF) {
#pragma unroll
          for (int v = 0; v < V; ++v) rows[j][v] = ld(UL, kj[j], v);
        }
      }
#pragma unroll
      for (int j = 0; j < PF; ++j) {
        const float val = __shfl_sync(FULL, vv, tb + jb + j);
        if ((fm >> (jb + j)) & 1u) {
          advance();
#pragma unroll
          for (int v = 0; v < V; ++v) acc[v] = f4(0.f);
        }
        if constexpr (OUT != LEAF) {
#pragma unroll
          for (int v = 0; v < V; ++v) acc[v] = fma4(val, rows[j][v], acc[v]);
        } else {
          if (xb + jb + j < x1) {
#pragma unroll
            for (int v = 0; v < V; ++v) rd(kj[j], v, f4(val) * crow[v]);
          }
        }
      }
    }
  }
  if (active) {
    close_fiber();
    close_fbrs();
    flush_slice();
  }
}

// ---------------------------------------------------------------------------
// Branch-free 3-D traversal ("flat" kernel). Same teams and nonzero ranges as
// k_mttkrp, but a fiber start no longer sends its team down a separate code
// path: every lane locates the fiber of its own nonzero from the block's
// fiber-start ballot (popcount of the flags at or below it), loads that
// fiber's metadata only if its nonzero opens the fiber, and the per-nonzero
// step is the same straight-line code for every team of the warp, with the
// fiber-open work predicated. Slice changes (rare: one per slice run) take a
// slower variant of the block, chosen per warp. Arithmetic uses the packed
// FP32x2 FMA of sm_100 (two fused multiply-adds per instruction).
__device__ __forceinline__ float4 pfma(float4 a, float4 b, float4 c) {
  const float2 lo = __ffma2_rn(make_float2(a.x, a.y), make_float2(b.x, b.y), make_float2(c.x, c.y));
  const float2 hi = __ffma2_rn(make_float2(a.z, a.w), make_float2(b.z, b.w), make_float2(c.z, c.w));
  return make_float4(lo.x, lo.y, hi.x, hi.y);
}
__device__ __forceinline__ float4 pfma_s(float s, float4 b, float4 c) {
  const float2 ss = make_float2(s, s);
  const float2 lo = __ffma2_rn(ss, make_float2(b.x, b.y), make_float2(c.x, c.y));
  const float2 hi = __ffma2_rn(ss, make_float2(b.z, b.w), make_float2(c.z, c.w));
  return make_float4(lo.x, lo.y, hi.x, hi.y);
}
__device__ __forceinline__ float4 pmul(float4 a, float4 b) {
  const float2 lo = __fmul2_rn(make_float2(a.x, a.y), make_float2(b.x, b.y));
  const float2 hi = __fmul2_rn(make_float2(a.z, a.w), make_float2(b.z, b.w));
  return make_float4(lo.x, lo.y, hi.x, hi.y);
}
__device__ __forceinline__ float4 pmul_s(float s, float4 b) {
  const float2 ss = make_float2(s, s);
  const float2 lo = __fmul2_rn(ss, make_float2(b.x, b.y));
  const float2 hi = __fmul2_rn(ss, make_float2(b.z, b.w));
  return make_float4(lo.x, lo.y, hi.x, hi.y);
}

// OUT 0 (slice rows): acc_s[a] += U1[b] (.) sum_fiber v U2[k]; the fiber's
//   U1 row is requested when the fiber opens and used when it closes.
// OUT 1 (fiber rows): out[b] += U0[a] (.) sum_fiber v U2[k], one vector
//   reduction per fiber.
// OUT 2 (leaf rows): out[k] += v U0[a] (.) U1[b], one reduction per nonzero;
//   the fiber's U1 rows for a batch are requested before the batch.
template <int OUT, int G, int V, class T, int MB, int PFX>
__global__ void __launch_bounds__(256, MB) k_mttkrp_flat(const Args<T> a) {
  constexpr uint32_t R = 4 * G * V;
  constexpr uint32_t FLAG = 0x80000000u;
  constexpr int PF = G > PFX ? PFX : G;
  constexpr uint32_t GMASK = G == 32 ? FULL : ((1u << G) - 1u);
  const int lane = threadIdx.x & 31;
  const int tl = lane & (G - 1);
  const int tb = lane - tl;
  const uint32_t le_mask = tl == 31 ? FULL : ((2u << tl) - 1u);  // lanes 0..tl of the team
  const float* __restrict__ vals = a.vals;
  const uint32_t* __restrict__ leaf = a.leaf;
  const uint32_t* __restrict__ fidx = a.fidx;
  const uint32_t* __restrict__ like = a.like;
  const uint32_t chunk = a.chunk;
  const T* __restrict__ U0 = a.U[0];
  const T* __restrict__ U1 = a.U[1];
  const T* __restrict__ U2 = a.U[2];
  float* __restrict__ out = a.out;
  float* __restrict__ out2 = a.out2;
  const uint32_t c0 = (uint32_t)tl * 4;
  auto ld = [&](const T* U, uint32_t row, int v) -> float4 {
    return Row<T>::load(U + (uint64_t)row * R, c0 + (uint32_t)(v * G * 4));
  };
  auto rd = [&](uint32_t row, int v, float4 x) { red4(out + (uint64_t)row * R + c0 + v * G * 4, x); };
  auto rd2 = [&](uint32_t row, int v, float4 x) { red4(out2 + (uint64_t)row * R + c0 + v * G * 4, x); };

  const uint64_t team = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) / G;
  const bool active = team * chunk < a.nnz;
  const uint64_t x0 = active ? team * chunk : a.nnz - 1;
  const uint64_t x1 = active ? min(x0 + chunk, a.nnz) : x0;

  uint32_t f = a.cfib ? (active ? __ldg(a.cfib + team) : a.nfib - 1) : find_fiber(a.fptr, a.nfib, x0);
  uint32_t cb = __ldg(fidx + f);  // open fiber's o1
  uint32_t ca = __ldg(like + f);  // open slice's o0
  float4 accf[V], accs[V], rowB[V], rowA[V];
#pragma unroll
  for (int v = 0; v < V; ++v) {
    accf[v] = accs[v] = f4(0.f);
    if constexpr (OUT == 0) rowB[v] = ld(U1, cb, v);
    if constexpr (OUT == 1) rowA[v] = ld(U0, ca, v);
    if constexpr (OUT == 2) { rowA[v] = ld(U0, ca, v); rowB[v] = rowA[v] * ld(U1, cb, v); }
    if constexpr (OUT == 3) { rowA[v] = ld(U0, ca, v); rowB[v] = ld(U1, cb, v); }
  }

  // Block pipeline: when block i (G nonzeros) is processed, its indices,
  // values and fiber metadata are in registers; block i+1's indices are in
  // flight or ready (their fiber flags decide which metadata to request) and
  // block i+2's are requested.
  auto load_kv = [&](uint32_t itb, uint32_t& kk, float& vq) {
    const uint64_t xx = x0 + itb + tl;
    kk = 0;
    vq = 0.f;
    if (itb < chunk && xx < x1) { kk = __ldg(leaf + xx); vq = __ldg(vals + xx); }
  };
  auto load_meta = [&](uint32_t itb, uint32_t kk, uint32_t& fm_, uint32_t& mb_, uint32_t& ma_) {
    const bool fl_ = (kk & FLAG) && (itb + tl != 0);
    fm_ = (__ballot_sync(FULL, fl_) >> tb) & GMASK;
    mb_ = 0;
    ma_ = 0;
    if (fl_) {
      const uint32_t fib = f + __popc(fm_ & le_mask);
      mb_ = __ldg(fidx + fib);
      ma_ = __ldg(like + fib);
    }
    f += __popc(fm_);
  };
  uint32_t kc, kn, fmc, mbc, mac;
  float vc, vn;
  load_kv(0, kc, vc);
  load_kv(G, kn, vn);
  load_meta(0, kc, fmc, mbc, mac);
  for (uint32_t it = 0; it < chunk; it += G) {
    const uint64_t xb = x0 + it;
    uint32_t kf;
    float vf;
    load_kv(it + 2 * G, kf, vf);
    uint32_t fmn, mbn, man;
    load_meta(it + G, kn, fmn, mbn, man);
    const uint32_t kv = kc, fm = fmc, mb = mbc, ma = mac;
    const float vv = vc;
    kc = kn; vc = vn; fmc = fmn; mbc = mbn; mac = man;
    kn = kf; vn = vf;
    const bool slow = __ballot_sync(FULL, ((fm >> tl) & 1u) && ma != ca) != 0u;  // a slice changes in this block
    const uint32_t k = kv & ~FLAG;

    auto block = [&](auto slow_tag) {
      constexpr bool SLOW = decltype(slow_tag)::value;
#pragma unroll
      for (int jb = 0; jb < G; jb += PF) {
        float4 rows[PF][V];
        uint32_t kj[PF], bj[PF];
#pragma unroll
        for (int j = 0; j < PF; ++j) {
          kj[j] = __shfl_sync(FULL, k, tb + jb + j);
          if constexpr (OUT == 2) bj[j] = __shfl_sync(FULL, mb, tb + jb + j);
          if constexpr (OUT != 2) {
#pragma unroll
            for (int v = 0; v < V; ++v) rows[j][v] = ld(U2, kj[j], v);
          } else {
            if ((fm >> (jb + j)) & 1u) {
#pragma unroll
              for (int v = 0; v < V; ++v) rows[j][v] = ld(U1, bj[j], v);
            }
          }
        }
#pragma unroll
        for (int j = 0; j < PF; ++j) {
          const float val = __shfl_sync(FULL, vv, tb + jb + j);
          if constexpr (OUT != 2) bj[j] = __shfl_sync(FULL, mb, tb + jb + j);
          uint32_t aj = 0;
          if constexpr (SLOW) aj = __shfl_sync(FULL, ma, tb + jb + j);
          if ((fm >> (jb + j)) & 1u) {
            if constexpr (OUT == 0) {
#pragma unroll
              for (int v = 0; v < V; ++v) { accs[v] = pfma(rowB[v], accf[v], accs[v]); accf[v] = f4(0.f); }
              if constexpr (SLOW) {
                if (aj != ca) {
#pragma unroll
                  for (int v = 0; v < V; ++v) { rd(ca, v, accs[v]); accs[v] = f4(0.f); }
                  ca = aj;
                }
              }
#pragma unroll
              for (int v = 0; v < V; ++v) rowB[v] = ld(U1, bj[j], v);
            } else if constexpr (OUT == 1) {
#pragma unroll
              for (int v = 0; v < V; ++v) { rd(cb, v, pmul(rowA[v], accf[v])); accf[v] = f4(0.f); }
              cb = bj[j];
              if constexpr (SLOW) {
                if (aj != ca) {
                  ca = aj;
#pragma unroll
                  for (int v = 0; v < V; ++v) rowA[v] = ld(U0, ca, v);
                }
              }
            } else if constexpr (OUT == 3) {
              // both outputs: the closing fiber's sum goes to the middle
              // mode's row and, through its middle row, into the slice sum
#pragma unroll
              for (int v = 0; v < V; ++v) {
                rd2(cb, v, pmul(rowA[v], accf[v]));
                accs[v] = pfma(rowB[v], accf[v], accs[v]);
                accf[v] = f4(0.f);
              }
              cb = bj[j];
              if constexpr (SLOW) {
                if (aj != ca) {
#pragma unroll
                  for (int v = 0; v < V; ++v) { rd(ca, v, accs[v]); accs[v] = f4(0.f); }
                  ca = aj;
#pragma unroll
                  for (int v = 0; v < V; ++v) rowA[v] = ld(U0, ca, v);
                }
              }
#pragma unroll
              for (int v = 0; v < V; ++v) rowB[v] = ld(U1, cb, v);
            } else {
              if constexpr (SLOW) {
                if (aj != ca) {
                  ca = aj;
#pragma unroll
                  for (int v = 0; v < V; ++v) rowA[v] = ld(U0, ca, v);
                }
              }
#pragma unroll
              for (int v = 0; v < V; ++v) rowB[v] = pmul(rowA[v], rows[j][v]);
            }
          }
          if constexpr (OUT != 2) {
#pragma unroll
            for (int v = 0; v < V; ++v) accf[v] = pfma_s(val, rows[j][v], accf[v]);
          } else {
            if (xb + jb + j < x1) {
#pragma unroll
              for (int v = 0; v < V; ++v) rd(kj[j], v, pmul_s(val, rowB[v]));
            }
          }
        }
      }
    };
    if (slow) block(std::true_type{});
    else block(std::false_type{});
  }
  if (active) {
#pragma unroll
    for (int v = 0; v < V; ++v) {
      if constexpr (OUT == 0) rd(ca, v, pfma(rowB[v], accf[v], accs[v]));
      if constexpr (OUT == 1) rd(cb, v, pmul(rowA[v], accf[v]));
      if constexpr (OUT == 3) {
        rd(ca, v, pfma(rowB[v], accf[v], accs[v]));
        rd2(cb, v, pmul(rowA[v], accf[v]));
      }
    }
  }
}

// ---------------------------------------------------------------------------
// Per-nonzero traversal ("rows" kernel), 3-D and 4-D, for the slice-level
// (OUT 0) and leaf-level (OUT ND-1) outputs. Every nonzero carries the
// indices of its middle levels (`mid` = o_{ND-2}, and `mid2` = o1 in 4-D), so
// a team needs no fiber bookkeeping: per nonzero it combines the middle rows
// and the leaf row, adding v * U1[b] (.) U2[k] (4-D: v * U1[b] (.) U2[c] (.)
// U3[k]) to the open slice's accumulator (OUT 0), or scattering
// v * U0[a] (.) U1[b] [(.) U2[c]] to the leaf row. The middle rows repeat along
// fibers, so most of their gathers hit L1 (gathering them unconditionally
// measured faster than predicating the repeats away). Slice changes come from the slices' first nonzero positions
// (`snz`), not from flags, and a block with a slice change takes a slower
// variant.
template <int ND, int OUT, int G, int V, class T, int MB, int PFX>
__global__ void __launch_bounds__(256, MB) k_mttkrp_rows(const Args<T> a) {
  static_assert(OUT == 0 || OUT == ND - 1 || (ND == 3 && OUT == 1), "slice, leaf or 3-D middle level");
  constexpr int LEAF = ND - 1;
  constexpr bool MIDL = ND == 3 && OUT == 1;  // fiber-row output: sum v U2[k] per fiber, times U0[a], one reduction
  constexpr uint32_t R = 4 * G * V;
  constexpr uint32_t FLAG = 0x80000000u;
  constexpr uint32_t GMASK = G == 32 ? FULL : ((1u << G) - 1u);
  constexpr int PF = G > PFX ? PFX : G;
  const int lane = threadIdx.x & 31;
  const int tl = lane & (G - 1);
  const int tb = lane - tl;
  const float* __restrict__ vals = a.vals;
  const uint32_t* __restrict__ leaf = a.leaf;
  const uint32_t* __restrict__ mid = a.mid;
  const uint32_t* __restrict__ mid2 = a.mid2;
  const uint32_t* __restrict__ snz = a.snz;
  const uint32_t* __restrict__ sidx = a.sidx;
  const uint32_t chunk = a.chunk, nslc = a.nslc;
  const T* __restrict__ U0 = a.U[0];
  const T* __restrict__ U1 = a.U[1];
  const T* __restrict__ U2 = a.U[2];
  const T* __restrict__ UL = a.U[LEAF];
  float* __restrict__ out = a.out;
  const uint32_t c0 = (uint32_t)tl * 4;
  auto ld = [&](const T* U, uint32_t row, int v) -> float4 {
    return Row<T>::load(U + (uint64_t)row * R, c0 + (uint32_t)(v * G * 4));
  };
  auto rd = [&](uint32_t row, int v, float4 x) { red4(out + (uint64_t)row * R + c0 + v * G * 4, x); };

  const uint64_t team = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) / G;
  const bool active = team * chunk < a.nnz;
  const uint64_t x0 = active ? team * chunk : a.nnz - 1;
  const uint64_t x1 = active ? min(x0 + chunk, a.nnz) : x0;

  // open slice: number sl, index ca, first nonzero of the next slice nxt
  uint32_t sl;
  if (a.cslc) {
    sl = active ? __ldg(a.cslc + team) : nslc - 1;
  } else {
    uint32_t lo = 0, hi = nslc - 1;
    while (lo < hi) {
      const uint32_t m = (lo + hi + 1) >> 1;
      if ((uint64_t)__ldg(snz + m) <= x0) lo = m; else hi = m - 1;
    }
    sl = lo;
  }
  uint32_t ca = __ldg(sidx + sl);
  uint64_t nxt = __ldg(snz + sl + 1);
  float4 acc[V], rowA[V];
#pragma unroll
  for (int v = 0; v < V; ++v) {
    acc[v] = f4(0.f);
    if constexpr (OUT == LEAF || MIDL) rowA[v] = ld(U0, ca, v);
  }
  [[maybe_unused]] uint32_t bopen = 0;  // middle level: the open fiber's row
  if constexpr (MIDL) bopen = __ldg(mid + x0);

  auto load_blk = [&](uint32_t itb, uint32_t& kk, uint32_t& bb, uint32_t& qq, float& vq) {
    const uint64_t xx = x0 + itb + tl;
    kk = 0;
    bb = 0;
    qq = 0;
    vq = 0.f;
    if (itb < chunk && xx < x1) {
      kk = __ldg(leaf + xx);
      bb = __ldg(mid + xx);
      if constexpr (ND == 4) qq = __ldg(mid2 + xx);
      vq = __ldg(vals + xx);
    }
  };
  uint32_t kc, bc, qc, kn, bn, qn;
  float vc, vn;
  load_blk(0, kc, bc, qc, vc);
  load_blk(G, kn, bn, qn, vn);
  for (uint32_t it = 0; it < chunk; it += G) {
    const uint64_t xb = x0 + it;
    const uint32_t k = kc & ~FLAG, b = bc, q = qc;
    const float vv = vc;
    [[maybe_unused]] uint32_t fm = 0;  // middle level: nonzero j of the block opens a fiber
    if constexpr (MIDL) fm = (__ballot_sync(FULL, (kc & FLAG) && (xb + tl != x0)) >> tb) & GMASK;
    kc = kn; bc = bn; qc = qn; vc = vn;
    load_blk(it + 2 * G, kn, bn, qn, vn);
    // a slice starts inside this block for some team of the warp
    const bool slow = __any_sync(FULL, xb < x1 && xb + G > nxt);

    auto block = [&](auto slow_tag) {
      constexpr bool SLOW = decltype(slow_tag)::value;
#pragma unroll
      for (int jb = 0; jb < G; jb += PF) {
        [[maybe_unused]] float4 rc[(OUT == 0 || MIDL) ? PF : 1][V];
        [[maybe_unused]] float4 rb[MIDL ? 1 : PF][V];
        [[maybe_unused]] float4 rq[ND == 4 ? PF : 1][V];
        [[maybe_unused]] uint32_t bjs[MIDL ? PF : 1];
        uint32_t kj[PF];
#pragma unroll
        for (int j = 0; j < PF; ++j) {
          kj[j] = __shfl_sync(FULL, k, tb + jb + j);
          const uint32_t bj = __shfl_sync(FULL, b, tb + jb + j);
          [[maybe_unused]] uint32_t qj = 0;
          if constexpr (ND == 4) qj = __shfl_sync(FULL, q, tb + jb + j);
          if constexpr (MIDL) bjs[j] = bj;
#pragma unroll
          for (int v = 0; v < V; ++v) {
            if constexpr (MIDL) {
              rc[j][v] = ld(UL, kj[j], v);
            } else if constexpr (ND == 3) {
              rb[j][v] = ld(U1, bj, v);
            } else {
              rb[j][v] = ld(U2, bj, v);  // level 2 (fiber index c)
              rq[j][v] = ld(U1, qj, v);  // level 1 (fbrS index b)
            }
            if constexpr (OUT == 0) rc[j][v] = ld(UL, kj[j], v);
          }
        }
#pragma unroll
        for (int j = 0; j < PF; ++j) {
          const float val = __shfl_sync(FULL, vv, tb + jb + j);
          const uint64_t x = xb + jb + j;
          if constexpr (MIDL) {
            if ((fm >> (jb + j)) & 1u) {  // the open fiber ends before nonzero j (it is in the old slice)
#pragma unroll
              for (int v = 0; v < V; ++v) { rd(bopen, v, pmul(rowA[v], acc[v])); acc[v] = f4(0.f); }
              bopen = bjs[j];
            }
          }
          if constexpr (SLOW) {
            if (x < x1 && x == nxt) {  // slice change (slices are never empty)
              if constexpr (OUT == 0) {
#pragma unroll
                for (int v = 0; v < V; ++v) { rd(ca, v, acc[v]); acc[v] = f4(0.f); }
              }
              ++sl;
              ca = __ldg(sidx + sl);
              nxt = __ldg(snz + sl + 1);
              if constexpr (OUT == LEAF || MIDL) {
#pragma unroll
                for (int v = 0; v < V; ++v) rowA[v] = ld(U0, ca, v);
              }
            }
          }
          if constexpr (MIDL) {
#pragma unroll
            for (int v = 0; v < V; ++v) acc[v] = pfma_s(val, rc[j][v], acc[v]);
          } else if constexpr (OUT == 0) {
#pragma unroll
            for (int v = 0; v < V; ++v) {
              float4 m = pmul_s(val, rb[j][v]);
              if constexpr (ND == 4) m = pmul(m, rq[j][v]);
              acc[v] = pfma(m, rc[j][v], acc[v]);
            }
          } else {
            if (x < x1) {
#pragma unroll
              for (int v = 0; v < V; ++v) {
                float4 m = pmul(rowA[v], rb[j][v]);
                if constexpr (ND == 4) m = pmul(m, rq[j][v]);
                rd(kj[j], v, pmul_s(val, m));
              }
            }
          }
        }
      }
    };
    if (slow) block(std::true_type{});
    else block(std::false_type{});
  }
  if constexpr (OUT == 0) {
    if (active) {
#pragma unroll
      for (int v = 0; v < V; ++v) rd(ca, v, acc[v]);
    }
  }
  if constexpr (MIDL) {
    if (active) {
#pragma unroll
      for (int v = 0; v < V; ++v) rd(bopen, v, pmul(rowA[v], acc[v]));
    }
  }
}

// ---------------------------------------------------------------------------
// Two outputs from one walk of a 3-D part (MM-CSF's reuse across modes): the
// slice mode's MTTKRP, out[a] += v U1[b] (.) U2[k], and the middle mode's,
// out2[b] += U0[a] (.) sum over the fiber (a, b) of v U2[k], share every
// nonzero's gathers of U1[b] and U2[k]. Slice accumulation as in the
// per-nonzero walk, fiber sums closed at the leaf-index flags with one vector
// reduction per fiber; both outputs zeroed by the caller.
template <int G, int V, class T, int MB, int PFX>
__global__ void __launch_bounds__(256, MB) k_mttkrp_pair(const Args<T> a) {
  constexpr uint32_t R = 4 * G * V;
  constexpr uint32_t FLAG = 0x80000000u;
  constexpr int PF = G > PFX ? PFX : G;
  constexpr uint32_t GMASK = G == 32 ? FULL : ((1u << G) - 1u);
  const int lane = threadIdx.x & 31;
  const int tl = lane & (G - 1);
  const int tb = lane - tl;
  const float* __restrict__ vals = a.vals;
  const uint32_t* __restrict__ leaf = a.leaf;
  const uint32_t* __restrict__ mid = a.mid;
  const uint32_t* __restrict__ snz = a.snz;
  const uint32_t* __restrict__ sidx = a.sidx;
  const uint32_t chunk = a.chunk, nslc = a.nslc;
  const T* __restrict__ U0 = a.U[0];
  const T* __restrict__ U1 = a.U[1];
  const T* __restrict__ U2 = a.U[2];
  float* __restrict__ out = a.out;
  float* __restrict__ out2 = a.out2;
  const uint32_t c0 = (uint32_t)tl * 4;
  auto ld = [&](const T* U, uint32_t row, int v) -> float4 {
    return Row<T>::load(U + (uint64_t)row * R, c0 + (uint32_t)(v * G * 4));
  };
  auto rd = [&](float* o, uint32_t row, int v, float4 x) { red4(o + (uint64_t)row * R + c0 + v * G * 4, x); };

  const uint64_t team = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) / G;
  const bool active = team * chunk < a.nnz;
  const uint64_t x0 = active ? team * chunk : a.nnz - 1;
  const uint64_t x1 = active ? min(x0 + chunk, a.nnz) : x0;
  uint32_t sl;
  if (a.cslc) {
    sl = active ? __ldg(a.cslc + team) : nslc - 1;
  } else {
    uint32_t lo = 0, hi = nslc - 1;
    while (lo < hi) {
      const uint32_t m = (lo + hi + 1) >> 1;
      if ((uint64_t)__ldg(snz + m) <= x0) lo = m; else hi = m - 1;
    }
    sl = lo;
  }
  uint32_t ca = __ldg(sidx + sl);
  uint64_t nxt = __ldg(snz + sl + 1);
  uint32_t bopen = __ldg(mid + x0);
  float4 acc[V], accf[V], rowA[V];
#pragma unroll
  for (int v = 0; v < V; ++v) {
    acc[v] = accf[v] = f4(0.f);
    rowA[v] = ld(U0, ca, v);
  }
  auto load_blk = [&](uint32_t itb, uint32_t& kk, uint32_t& bb, float& vq) {
    const uint64_t xx = x0 + itb + tl;
    kk = 0;
    bb = 0;
    vq = 0.f;
    if (itb < chunk && xx < x1) { kk = __ldg(leaf + xx); bb = __ldg(mid + xx); vq = __ldg(vals + xx); }
  };
  uint32_t kc, bc, kn, bn;
  float vc, vn;
  load_blk(0, kc, bc, vc);
  load_blk(G, kn, bn, vn);
  for (uint32_t it = 0; it < chunk; it += G) {
    const uint64_t xb = x0 + it;
    const uint32_t k = kc & ~FLAG, b = bc;
    const float vv = vc;
    const uint32_t fm = (__ballot_sync(FULL, (kc & FLAG) && (xb + tl != x0)) >> tb) & GMASK;
    kc = kn; bc = bn; vc = vn;
    load_blk(it + 2 * G, kn, bn, vn);
    const bool slow = __any_sync(FULL, xb < x1 && xb + G > nxt);
    auto block = [&](auto slow_tag) {
      constexpr bool SLOW = decltype(slow_tag)::value;
#pragma unroll
      for (int jb = 0; jb < G; jb += PF) {
        float4 rb[PF][V], rc[PF][V];
        uint32_t bjs[PF];
#pragma unroll
        for (int j = 0; j < PF; ++j) {
          const uint32_t kj = __shfl_sync(FULL, k, tb + jb + j);
          bjs[j] = __shfl_sync(FULL, b, tb + jb + j);
#pragma unroll
          for (int v = 0; v < V; ++v) {
            rb[j][v] = ld(U1, bjs[j], v);
            rc[j][v] = ld(U2, kj, v);
          }
        }
#pragma unroll
        for (int j = 0; j < PF; ++j) {
          const float val = __shfl_sync(FULL, vv, tb + jb + j);
          const uint64_t x = xb + jb + j;
          if ((fm >> (jb + j)) & 1u) {  // the open fiber ends before nonzero j (in the open slice)
#pragma unroll
            for (int v = 0; v < V; ++v) { rd(out2, bopen, v, pmul(rowA[v], accf[v])); accf[v] = f4(0.f); }
            bopen = bjs[j];
          }
          if constexpr (SLOW) {
            if (x < x1 && x == nxt) {
#pragma unroll
              for (int v = 0; v < V; ++v) { rd(out, ca, v, acc[v]); acc[v] = f4(0.f); }
              ++sl;
              ca = __ldg(sidx + sl);
              nxt = __ldg(snz + sl + 1);
#pragma unroll
              for (int v = 0; v < V; ++v) rowA[v] = ld(U0, ca, v);
            }
          }
#pragma unroll
          for (int v = 0; v < V; ++v) {
            acc[v] = pfma(pmul_s(val, rb[j][v]), rc[j][v], acc[v]);
            accf[v] = pfma_s(val, rc[j][v], accf[v]);
          }
        }
      }
    };
    if (slow) block(std::true_type{});
    else block(std::false_type{});
  }
  if (active) {
#pragma unroll
    for (int v = 0; v < V; ++v) {
      rd(out, ca, v, acc[v]);
      rd(out2, bopen, v, pmul(rowA[v], accf[v]));
    }
  }
}

// The 4-D two-output walk: the slice mode's MTTKRP, out[a] += v U1[b] (.)
// U2[c] (.) U3[k], and the level-1 mode's, out2[b] += U0[a] (.) sum over the
// (a, b) group of v U2[c] (.) U3[k], from one walk that gathers each
// nonzero's three rows once (b = mid2, c = mid, k = leaf). A group closes at a
// leaf-fiber start whose b differs from the open one, or where a slice
// starts; splits of one (a, b) group (the fbrS split) only add reductions.
// Both outputs zeroed by the caller.
template <int G, int V, class T, int MB, int PFX>
__global__ void __launch_bounds__(256, MB) k_mttkrp_pair4(const Args<T> a) {
  constexpr uint32_t R = 4 * G * V;
  constexpr uint32_t FLAG = 0x80000000u;
  constexpr int PF = G > PFX ? PFX : G;
  constexpr uint32_t GMASK = G == 32 ? FULL : ((1u << G) - 1u);
  const int lane = threadIdx.x & 31;
  const int tl = lane & (G - 1);
  const int tb = lane - tl;
  const float* __restrict__ vals = a.vals;
  const uint32_t* __restrict__ leaf = a.leaf;
  const uint32_t* __restrict__ mid = a.mid;
  const uint32_t* __restrict__ mid2 = a.mid2;
  const uint32_t* __restrict__ snz = a.snz;
  const uint32_t* __restrict__ sidx = a.sidx;
  const uint32_t chunk = a.chunk, nslc = a.nslc;
  const T* __restrict__ U0 = a.U[0];
  const T* __restrict__ U1 = a.U[1];
  const T* __restrict__ U2 = a.U[2];
  const T* __restrict__ U3 = a.U[3];
  float* __restrict__ out = a.out;
  float* __restrict__ out2 = a.out2;
  const uint32_t c0 = (uint32_t)tl * 4;
  auto ld = [&](const T* U, uint32_t row, int v) -> float4 {
    return Row<T>::load(U + (uint64_t)row * R, c0 + (uint32_t)(v * G * 4));
  };
  auto rd = [&](float* o, uint32_t row, int v, float4 x) { red4(o + (uint64_t)row * R + c0 + v * G * 4, x); };

  const uint64_t team = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) / G;
  const bool active = team * chunk < a.nnz;
  const uint64_t x0 = active ? team * chunk : a.nnz - 1;
  const uint64_t x1 = active ? min(x0 + chunk, a.nnz) : x0;
  uint32_t sl;
  if (a.cslc) {
    sl = active ? __ldg(a.cslc + team) : nslc - 1;
  } else {
    uint32_t lo = 0, hi = nslc - 1;
    while (lo < hi) {
      const uint32_t m = (lo + hi + 1) >> 1;
      if ((uint64_t)__ldg(snz + m) <= x0) lo = m; else hi = m - 1;
    }
    sl = lo;
  }
  uint32_t ca = __ldg(sidx + sl);
  uint64_t nxt = __ldg(snz + sl + 1);
  uint32_t bopen = __ldg(mid2 + x0);
  float4 acc[V], accf[V], rowA[V];
#pragma unroll
  for (int v = 0; v < V; ++v) {
    acc[v] = accf[v] = f4(0.f);
    rowA[v] = ld(U0, ca, v);
  }
  auto load_blk = [&](uint32_t itb, uint32_t& kk, uint32_t& bb, uint32_t& cc, float& vq) {
    const uint64_t xx = x0 + itb + tl;
    kk = 0;
    bb = 0;
    cc = 0;
    vq = 0.f;
    if (itb < chunk && xx < x1) {
      kk = __ldg(leaf + xx);
      bb = __ldg(mid2 + xx);
      cc = __ldg(mid + xx);
      vq = __ldg(vals + xx);
    }
  };
  uint32_t kc, bc, cc, kn, bn, cn;
  float vc, vn;
  load_blk(0, kc, bc, cc, vc);
  load_blk(G, kn, bn, cn, vn);
  for (uint32_t it = 0; it < chunk; it += G) {
    const uint64_t xb = x0 + it;
    const uint32_t k = kc & ~FLAG, b = bc, c = cc;
    const float vv = vc;
    const uint32_t fm = (__ballot_sync(FULL, (kc & FLAG) && (xb + tl != x0)) >> tb) & GMASK;
    kc = kn; bc = bn; cc = cn; vc = vn;
    load_blk(it + 2 * G, kn, bn, cn, vn);
    const bool slow = __any_sync(FULL, xb < x1 && xb + G > nxt);
    auto block = [&](auto slow_tag) {
      constexpr bool SLOW = decltype(slow_tag)::value;
#pragma unroll
      for (int jb = 0; jb < G; jb += PF) {
        float4 rb[PF][V], rc[PF][V], rk[PF][V];
        uint32_t bjs[PF];
#pragma unroll
        for (int j = 0; j < PF; ++j) {
          const uint32_t kj = __shfl_sync(FULL, k, tb + jb + j);
          const uint32_t cj = __shfl_sync(FULL, c, tb + jb + j);
          bjs[j] = __shfl_sync(FULL, b, tb + jb + j);
#pragma unroll
          for (int v = 0; v < V; ++v) {
            rb[j][v] = ld(U1, bjs[j], v);
            rc[j][v] = ld(U2, cj, v);
            rk[j][v] = ld(U3, kj, v);
          }
        }
#pragma unroll
        for (int j = 0; j < PF; ++j) {
          const float val = __shfl_sync(FULL, vv, tb + jb + j);
          const uint64_t x = xb + jb + j;
          if ((fm >> (jb + j)) & 1u) {
            bool close = bjs[j] != bopen;
            if constexpr (SLOW) close = close || (x < x1 && x == nxt);
            if (close) {  // the open (a, b) group ends before nonzero j
#pragma unroll
              for (int v = 0; v < V; ++v) { rd(out2, bopen, v, pmul(rowA[v], accf[v])); accf[v] = f4(0.f); }
              bopen = bjs[j];
            }
          }
          if constexpr (SLOW) {
            if (x < x1 && x == nxt) {
#pragma unroll
              for (int v = 0; v < V; ++v) { rd(out, ca, v, acc[v]); acc[v] = f4(0.f); }
              ++sl;
              ca = __ldg(sidx + sl);
              nxt = __ldg(snz + sl + 1);
#pragma unroll
              for (int v = 0; v < V; ++v) rowA[v] = ld(U0, ca, v);
            }
          }
#pragma unroll
          for (int v = 0; v < V; ++v) {
            const float4 u = pmul(rc[j][v], rk[j][v]);
            acc[v] = pfma(pmul_s(val, rb[j][v]), u, acc[v]);
            accf[v] = pfma_s(val, u, accf[v]);
          }
        }
      }
    };
    if (slow) block(std::true_type{});
    else block(std::false_type{});
  }
  if (active) {
#pragma unroll
    for (int v = 0; v < V; ++v) {
      rd(out, ca, v, acc[v]);
      rd(out2, bopen, v, pmul(rowA[v], accf[v]));
    }
  }
}

template <int G, int V, class T>
cudaError_t launch_pair4(const Args<T>& a, int threads, int mb, cudaStream_t s) {
  const uint64_t teams = (a.nnz + a.chunk - 1) / a.chunk;
  const uint64_t blocks = (teams * G + threads - 1) / threads;
  switch (mb) {
    case 1: k_mttkrp_pair4<G, V, T, 1, 8><<<(unsigned)blocks, threads, 0, s>>>(a); break;
    case 3: k_mttkrp_pair4<G, V, T, 2, 2><<<(unsigned)blocks, threads, 0, s>>>(a); break;
    case 4: k_mttkrp_pair4<G, V, T, 3, 2><<<(unsigned)blocks, threads, 0, s>>>(a); break;
    default: k_mttkrp_pair4<G, V, T, 2, 4><<<(unsigned)blocks, threads, 0, s>>>(a); break;
  }
  return cudaGetLastError();
}

template <int G, int V, class T>
cudaError_t launch_pair(const Args<T>& a, int threads, int mb, cudaStream_t s) {
  const uint64_t teams = (a.nnz + a.chunk - 1) / a.chunk;
  const uint64_t blocks = (teams * G + threads - 1) / threads;
  switch (mb) {
    case 1: k_mttkrp_pair<G, V, T, 2, 8><<<(unsigned)blocks, threads, 0, s>>>(a); break;
    case 3: k_mttkrp_pair<G, V, T, 4, 4><<<(unsigned)blocks, threads, 0, s>>>(a); break;
    case 4: k_mttkrp_pair<G, V, T, 5, 4><<<(unsigned)blocks, threads, 0, s>>>(a); break;
    default: k_mttkrp_pair<G, V, T, 3, 8><<<(unsigned)blocks, threads, 0, s>>>(a); break;
  }
  return cudaGetLastError();
}

template <int OUT, int G, int V, class T>
cudaError_t launch_flat(const Args<T>& a, int threads, int mb, cudaStream_t s);

// kern 2: the branch-free fiber walk with both outputs; otherwise the
// per-nonzero form
template <class T>
cudaError_t launch_pair_R(const Args<T>& a, int nd, int threads, int mb, int kern, cudaStream_t s) {
  if (nd == 4) {
    switch (a.R) {
      case 4: return launch_pair4<1, 1, T>(a, threads, mb, s);
      case 8: return launch_pair4<2, 1, T>(a, threads, mb, s);
      case 16: return launch_pair4<4, 1, T>(a, threads, mb, s);
      case 32: return launch_pair4<8, 1, T>(a, threads, mb, s);
      case 64: return launch_pair4<16, 1, T>(a, threads, mb, s);
      case 128: return launch_pair4<32, 1, T>(a, threads, mb, s);
      default: return cudaErrorInvalidValue;
    }
  }
  if (kern == 2) {
    switch (a.R) {
      case 4: return launch_flat<3, 1, 1, T>(a, threads, mb, s);
      case 8: return launch_flat<3, 2, 1, T>(a, threads, mb, s);
      case 16: return launch_flat<3, 4, 1, T>(a, threads, mb, s);
      case 32: return launch_flat<3, 8, 1, T>(a, threads, mb, s);
      case 64: return launch_flat<3, 16, 1, T>(a, threads, mb, s);
      case 128: return launch_flat<3, 32, 1, T>(a, threads, mb, s);
      default: return cudaErrorInvalidValue;
    }
  }
  switch (a.R) {
    case 4: return launch_pair<1, 1, T>(a, threads, mb, s);
    case 8: return launch_pair<2, 1, T>(a, threads, mb, s);
    case 16: return launch_pair<4, 1, T>(a, threads, mb, s);
    case 32: return launch_pair<8, 1, T>(a, threads, mb, s);
    case 64: return launch_pair<16, 1, T>(a, threads, mb, s);
    case 128: return launch_pair<32, 1, T>(a, threads, mb, s);
    default: return cudaErrorInvalidValue;
  }
}

template <int ND, int OUT, int G, int V, class T>
cudaError_t launch_one(const Args<T>& a, int threads, int mb, cudaStream_t s) {
  const uint64_t teams = (a.nnz + a.chunk - 1) / a.chunk;
  const uint64_t thr = teams * G;
  const uint64_t blocks = (thr + threads - 1) / threads;
  switch (mb) {
    case 1: k_mttkrp<ND, OUT, G, V, T, 3, 8><<<(unsigned)blocks, threads, 0, s>>>(a); break;
    case 3: k_mttkrp<ND, OUT, G, V, T, 5, 4><<<(unsigned)blocks, threads, 0, s>>>(a); break;
    case 4: k_mttkrp<ND, OUT, G, V, T, 6, 4><<<(unsigned)blocks, threads, 0, s>>>(a); break;
    default: k_mttkrp<ND, OUT, G, V, T, 4, 8><<<(unsigned)blocks, threads, 0, s>>>(a); break;
  }
  return cudaGetLastError();
}

template <int OUT, int G, int V, class T>
cudaError_t launch_flat(const Args<T>& a, int threads, int mb, cudaStream_t s) {
  const uint64_t teams = (a.nnz + a.chunk - 1) / a.chunk;
  const uint64_t thr = teams * G;
  const uint64_t blocks = (thr + threads - 1) / threads;
  switch (mb) {
    case 1: k_mttkrp_flat<OUT, G, V, T, 2, 8><<<(unsigned)blocks, threads, 0, s>>>(a); break;
    case 3: k_mttkrp_flat<OUT, G, V, T, 4, 4><<<(unsigned)blocks, threads, 0, s>>>(a); break;
    case 4: k_mttkrp_flat<OUT, G, V, T, 5, 4><<<(unsigned)blocks, threads, 0, s>>>(a); break;
    default: k_mttkrp_flat<OUT, G, V, T, 3, 8><<<(unsigned)blocks, threads, 0, s>>>(a); break;
  }
  return cudaGetLastError();
}

template <int ND, int OUT, int G, int V, class T>
cudaError_t launch_rows(const Args<T>& a, int threads, int mb, cudaStream_t s) {
  const uint64_t teams = (a.nnz + a.chunk - 1) / a.chunk;
  const uint64_t thr = teams * G;
  const uint64_t blocks = (thr + threads - 1) / threads;
  switch (mb) {
    case 1: k_mttkrp_rows<ND, OUT, G, V, T, 2, 8><<<(unsigned)blocks, threads, 0, s>>>(a); break;
    case 3: k_mttkrp_rows<ND, OUT, G, V, T, 4, 4><<<(unsigned)blocks, threads, 0, s>>>(a); break;
    case 4: k_mttkrp_rows<ND, OUT, G, V, T, 5, 4><<<(unsigned)blocks, threads, 0, s>>>(a); break;
    default: k_mttkrp_rows<ND, OUT, G, V, T, 3, 8><<<(unsigned)blocks, threads, 0, s>>>(a); break;
  }
  return cudaGetLastError();
}

// kern: 1 = per-team fiber walk (k_mttkrp), 2 = branch-free walk (3-D only),
// 3 = per-nonzero walk (slice and leaf levels of parts that carry `mid`)
template <int ND, int G, int V, class T>
cudaError_t launch_lvl(const Args<T>& a, int lvl, int kern, int threads, int mb, cudaStream_t s) {
  if (kern == 3 && lvl == 0) return launch_rows<ND, 0, G, V, T>(a, threads, mb, s);
  if (kern == 3 && lvl == ND - 1) return launch_rows<ND, ND - 1, G, V, T>(a, threads, mb, s);
  if constexpr (ND == 3)
    if (kern == 3 && lvl == 1) return launch_rows<3, 1, G, V, T>(a, threads, mb, s);
  if constexpr (ND == 3) {
    if (kern >= 2) {
      switch (lvl) {
        case 0: return launch_flat<0, G, V, T>(a, threads, mb, s);
        case 1: return launch_flat<1, G, V, T>(a, threads, mb, s);
        case 2: return launch_flat<2, G, V, T>(a, threads, mb, s);
        default: return cudaErrorInvalidValue;
      }
    }
  }
  switch (lvl) {
    case 0: return launch_one<ND, 0, G, V, T>(a, threads, mb, s);
    case 1: return launch_one<ND, 1, G, V, T>(a, threads, mb, s);
    case 2: return launch_one<ND, 2, G, V, T>(a, threads, mb, s);
    default:
      if constexpr (ND == 4) return launch_one<ND, 3, G, V, T>(a, threads, mb, s);
      return cudaErrorInvalidValue;
  }
}

template <class T>
cudaError_t launch_R(const Args<T>& a, int nd, int lvl, int kern, int threads, int mb, cudaStream_t s) {
#define MMCSF_RCASE(RR, GG, VV)                                                        \
  case RR:                                                                            \
    return nd == 3 ? launch_lvl<3, GG, VV, T>(a, lvl, kern, threads, mb, s)           \
                   : launch_lvl<4, GG, VV, T>(a, lvl, kern, threads, mb, s);
  switch (a.R) {
    MMCSF_RCASE(4, 1, 1)
    MMCSF_RCASE(8, 2, 1)
    MMCSF_RCASE(16, 4, 1)
    MMCSF_RCASE(32, 8, 1)
    MMCSF_RCASE(64, 16, 1)
    MMCSF_RCASE(128, 32, 1)
    MMCSF_RCASE(256, 32, 2)
    default: return cudaErrorInvalidValue;
  }
#undef MMCSF_RCASE
}

bool native_R(int R) { return R == 4 || R == 8 || R == 16 || R == 32 || R == 64 || R == 128 || R == 256; }
int padded_R(int R) {
  const int opts[] = {4, 8, 16, 32, 64, 128, 256};
  for (int r : opts)
    if (r >= R) return r;
  return -1;
}

__global__ void k_pad_rows(const void* in, int esz, uint64_t rows, int R, int Rp, void* out) {
  const uint64_t n = rows * (uint64_t)Rp;
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
    uint64_t r = i / Rp, c = i % Rp;
    if (esz == 4) static_cast<float*>(out)[i] = c < (uint64_t)R ? static_cast<const float*>(in)[r * R + c] : 0.f;
    else static_cast<uint16_t*>(out)[i] = c < (uint64_t)R ? static_cast<const uint16_t*>(in)[r * R + c] : 0;
  }
}
__global__ void k_unpad_rows(const float* in, uint64_t rows, int R, int Rp, float* out) {
  const uint64_t n = rows * (uint64_t)R;
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
    out[i] = in[(i / R) * Rp + i % R];
}

int default_chunk(int R) {
  (void)R;
  return 512;
}

// Kernel arguments for part P (factors U by tensor mode, reordered by level).
template <class T>
void fill_args(Args<T>& a, const CsfPart& P, const float* vals_override, int slot, int chunk, int R,
               const void* const* U, float* out) {
  a.vals = vals_override ? vals_override : P.vals.as<float>();
  a.leaf = P.leaf.as<uint32_t>();
  const int lf = P.nd - 2;
  a.fptr = P.ptr[lf].as<uint32_t>();
  a.fidx = P.idx[lf].as<uint32_t>();
  a.fpar = P.fpar.as<uint32_t>();
  a.sidx1 = P.nd == 4 ? P.idx[1].as<uint32_t>() : nullptr;
  a.like = P.fbr_like.as<uint32_t>();
  a.cfib = slot >= 0 && P.cfib[slot].p ? P.cfib[slot].as<uint32_t>() : nullptr;
  a.mid = P.mid.as<uint32_t>();
  a.mid2 = P.mid2.as<uint32_t>();
  a.snz = P.snz.as<uint32_t>();
  a.sidx = P.idx[0].as<uint32_t>();
  a.cslc = slot >= 0 && P.cslc[slot].p ? P.cslc[slot].as<uint32_t>() : nullptr;
  a.nslc = (uint32_t)P.n[0];
  a.nnz = P.nnz;
  a.nfib = (uint32_t)P.n_fibers();
  a.chunk = (uint32_t)chunk;
  a.R = (uint32_t)R;
  for (int l = 0; l < P.nd; ++l) a.U[l] = static_cast<const T*>(U[P.order[l]]);
  a.out = out;
}

// MTTKRP on one part for tensor mode `mode`; out must be zeroed by the caller.
int part_mttkrp(const mmcsf_format* F, const CsfPart& P, int mode, int R, int dtype, const void* const* U,
                float* out, const mmcsf_kernel_cfg* cfg, cudaStream_t s, int* launches,
                const float* vals_override = nullptr) {
  if (!P.present || P.nnz == 0) return MMCSF_OK;
  int lvl = -1;
  for (int l = 0; l < P.nd; ++l)
    if (P.order[l] == mode) lvl = l;
  if (lvl < 0) return set_error(MMCSF_ERR_INVALID, "mode %d not in part", mode);
  int chunk = cfg && cfg->chunk > 0 ? cfg->chunk : default_chunk(R);
  int threads = cfg && cfg->block_threads > 0 ? cfg->block_threads : 256;
  const int mb = cfg && cfg->min_blocks > 0 ? cfg->min_blocks : 2;
  int kern = cfg && cfg->kernel > 0 ? cfg->kernel : (P.nd == 3 ? 2 : 1);
  if (kern < 1 || kern > 3) return set_error(MMCSF_ERR_INVALID, "kernel must be 0, 1, 2 or 3");
  if (kern == 3 && (!P.mid.p || (P.nd == 4 && lvl != 0 && lvl != 3))) kern = 2;  // per-nonzero walk not applicable
  if (kern == 2 && P.nd == 4) kern = 1;                                         // no 4-D branch-free fiber walk
  const int slot = CsfPart::cfib_slot((uint64_t)chunk);
  if (threads % 32 || threads > 256) return set_error(MMCSF_ERR_INVALID, "block_threads must be a multiple of 32, <= 256");
  cudaError_t e;
  if (dtype == MMCSF_DTYPE_F32) {
    Args<float> a{};
    fill_args(a, P, vals_override, slot, chunk, R, U, out);
    e = launch_R<float>(a, P.nd, lvl, kern, threads, mb, s);
  } else {
    Args<__nv_bfloat16> a{};
    fill_args(a, P, vals_override, slot, chunk, R, U, out);
    e = launch_R<__nv_bfloat16>(a, P.nd, lvl, kern, threads, mb, s);
  }
  if (e != cudaSuccess) return set_error(MMCSF_ERR_CUDA, "MTTKRP launch failed: %s", cudaGetErrorString(e));
  if (launches) ++*launches;
  return MMCSF_OK;
}

}  // namespace

int hyb_extra_mttkrp(const mmcsf_format* F, int R, int dtype, const void* const* U, float* out, cudaStream_t s,
                     int* launches);  // hyb.cu

__global__ void k_reorder_vals(const float* __restrict__ in, const uint32_t* __restrict__ from, uint64_t n,
                               float* __restrict__ out) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
    out[i] = in[from[i]];
}

// One mode over every part that holds nonzeros (the reference's per-mode loop
// over partitions, src/mttkrp_gpu.cu:3578-3724). vals: optional values in the
// format's nonzero order replacing the tensor's (the sampled model's adjoint).
int mttkrp_mode_vals(const mmcsf_format* F, int mode, int R, int dtype, const void* const* U, const float* vals,
                     float* out, const mmcsf_kernel_cfg* cfg, cudaStream_t s, int* launches) {
  MMCSF_CUDA(cudaMemsetAsync(out, 0, F->dims[mode] * (uint64_t)R * sizeof(float), s));
  int trav = cfg ? cfg->traversal : 0;
  if (trav == 0) trav = F->plan_traversal[mode] ? F->plan_traversal[mode] : (F->views[mode].present ? 2 : 1);
  mmcsf_kernel_cfg c{};
  if (cfg) c = *cfg;
  if (c.chunk == 0) c.chunk = F->plan_chunk[mode];
  if (c.min_blocks == 0) c.min_blocks = F->plan_mb[mode];
  if (c.kernel == 0) c.kernel = F->plan_kernel[mode];
  if (trav == 2) {
    const CsfPart& V = F->views[mode];
    if (!V.present) return set_error(MMCSF_ERR_INVALID, "no view for mode %d (build with views)", mode);
    const float* vv = nullptr;
    if (vals) {
      mmcsf_format* Fm = const_cast<mmcsf_format*>(F);
      if (Fm->vals_scratch.bytes < V.nnz * 4) MMCSF_CUDA(Fm->vals_scratch.alloc(V.nnz * 4));
      k_reorder_vals<<<grid_for(V.nnz, 256), 256, 0, s>>>(vals, V.from_part.as<uint32_t>(), V.nnz,
                                                          Fm->vals_scratch.as<float>());
      MMCSF_LAUNCH_CHECK();
      if (launches) ++*launches;
      vv = Fm->vals_scratch.as<float>();
    }
    return part_mttkrp(F, V, mode, R, dtype, U, out, &c, s, launches, vv);
  }
  uint64_t off = 0;  // caller values are in the format's order: partitions 0..nd-1
  for (int p = 0; p < F->nd; ++p) {
    MMCSF_TRY(part_mttkrp(F, F->parts[p], mode, R, dtype, U, out, &c, s, launches, vals ? vals + off : nullptr));
    if (F->parts[p].present) off += F->parts[p].nnz;
  }
  if (F->impl == MMCSF_IMPL_HBCSF) {
    if (vals) return set_error(MMCSF_ERR_UNSUPPORTED, "MTTKRP on other values is not available for HB-CSF");
    MMCSF_TRY(hyb_extra_mttkrp(F, R, dtype, U, out, s, launches));
  }
  return MMCSF_OK;
}

int mttkrp_mode(const mmcsf_format* F, int mode, int R, int dtype, const void* const* U, float* out,
                const mmcsf_kernel_cfg* cfg, cudaStream_t s, int* launches) {
  return mttkrp_mode_vals(F, mode, R, dtype, U, nullptr, out, cfg, s, launches);
}

}  // namespace mmcsf

using namespace mmcsf;

namespace {
int check_call(const mmcsf_format* F, int R, int dtype) {
  if (!F) return set_error(MMCSF_ERR_INVALID, "null format");
  if (R < 1) return set_error(MMCSF_ERR_INVALID, "rank must be >= 1");
  if (dtype != MMCSF_DTYPE_F32 && dtype != MMCSF_DTYPE_BF16) return set_error(MMCSF_ERR_INVALID, "bad dtype");
  if (R > 256) return set_error(MMCSF_ERR_UNSUPPORTED, "rank %d > 256", R);
  return MMCSF_OK;
}

// Run `fn(U, out_for_mode)` with rank padded to a native kernel width when R is
// not one (factors copied into zero-padded buffers, outputs copied back).
template <class Fn>
int with_padding(const mmcsf_format* F, int R, int dtype, const void* const* U, Fn fn, cudaStream_t s) {
  if (native_R(R)) return fn(R, U);
  const int Rp = padded_R(R);
  const int esz = dtype == MMCSF_DTYPE_F32 ? 4 : 2;
  DevBuf pu[4];
  const void* pp[4] = {nullptr, nullptr, nullptr, nullptr};
  for (int m = 0; m < F->nd; ++m) {
    MMCSF_CUDA(pu[m].alloc(F->dims[m] * (uint64_t)Rp * esz));
    k_pad_rows<<<grid_for(F->dims[m] * (uint64_t)Rp, 256), 256, 0, s>>>(U[m], esz, F->dims[m], R, Rp, pu[m].p);
    MMCSF_LAUNCH_CHECK();
    pp[m] = pu[m].p;
  }
  int st = fn(Rp, pp);
  MMCSF_CUDA(cudaStreamSynchronize(s));
  return st;
}
}  // namespace

extern "C" int mmcsf_mttkrp(const mmcsf_format* F, int mode, int R, int factor_dtype, const void* const* d_factors,
                            float* d_out, const mmcsf_kernel_cfg* cfg, void* stream) {
  MMCSF_TRY(check_call(F, R, factor_dtype));
  if (mode < 0 || mode >= F->nd) return set_error(MMCSF_ERR_INVALID, "Mode cannot be larger than tensor dimension.");
  if (!d_factors || !d_out) return set_error(MMCSF_ERR_INVALID, "null pointer");
  if (F->impl != MMCSF_IMPL_MMCSF && mode != F->mode)
    return set_error(MMCSF_ERR_INVALID, "this format was built for mode %d only", F->mode);
  cudaStream_t s = S(stream);
  mmcsf_format* Fm = const_cast<mmcsf_format*>(F);
  int launches = 0;
  int st = with_padding(F, R, factor_dtype, d_factors, [&](int Rk, const void* const* U) -> int {
    if (Rk == R) return mttkrp_mode(F, mode, R, factor_dtype, U, d_out, cfg, s, &launches);
    DevBuf tmp;
    MMCSF_CUDA(tmp.alloc(F->dims[mode] * (uint64_t)Rk * 4));
    MMCSF_TRY(mttkrp_mode(F, mode, Rk, factor_dtype, U, tmp.as<float>(), cfg, s, &launches));
    k_unpad_rows<<<grid_for(F->dims[mode] * (uint64_t)R, 256), 256, 0, s>>>(tmp.as<float>(), F->dims[mode], R, Rk,
                                                                           d_out);
    MMCSF_LAUNCH_CHECK();
    MMCSF_CUDA(cudaStreamSynchronize(s));
    return MMCSF_OK;
  }, s);
  Fm->last_launches = launches;
  return st;
}

__global__ void k_scale_cols(float* __restrict__ M, uint64_t rows, int R, const float* __restrict__ lam) {
  const uint64_t n = rows * (uint64_t)R;
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
    M[i] *= __ldg(lam + i % R);
}

extern "C" int mmcsf_cp_adjoint(const mmcsf_format* F, int mode, int R, int factor_dtype,
                                const void* const* d_factors, const float* d_lambda, const float* d_grad,
                                float* d_out, const mmcsf_kernel_cfg* cfg, void* stream) {
  MMCSF_TRY(check_call(F, R, factor_dtype));
  if (mode < 0 || mode >= F->nd) return set_error(MMCSF_ERR_INVALID, "Mode cannot be larger than tensor dimension.");
  if (!d_factors || !d_out || !d_grad) return set_error(MMCSF_ERR_INVALID, "null pointer");
  if (F->impl == MMCSF_IMPL_HBCSF) return set_error(MMCSF_ERR_UNSUPPORTED, "not available for HB-CSF formats");
  if (F->impl != MMCSF_IMPL_MMCSF && mode != F->mode)
    return set_error(MMCSF_ERR_INVALID, "this format was built for mode %d only", F->mode);
  cudaStream_t s = S(stream);
  mmcsf_format* Fm = const_cast<mmcsf_format*>(F);
  int launches = 0;
  int st = with_padding(F, R, factor_dtype, d_factors, [&](int Rk, const void* const* U) -> int {
    if (Rk == R) return mttkrp_mode_vals(F, mode, R, factor_dtype, U, d_grad, d_out, cfg, s, &launches);
    DevBuf tmp;
    MMCSF_CUDA(tmp.alloc(F->dims[mode] * (uint64_t)Rk * 4));
    MMCSF_TRY(mttkrp_mode_vals(F, mode, Rk, factor_dtype, U, d_grad, tmp.as<float>(), cfg, s, &launches));
    k_unpad_rows<<<grid_for(F->dims[mode] * (uint64_t)R, 256), 256, 0, s>>>(tmp.as<float>(), F->dims[mode], R, Rk,
                                                                           d_out);
    MMCSF_LAUNCH_CHECK();
    MMCSF_CUDA(cudaStreamSynchronize(s));
    return MMCSF_OK;
  }, s);
  if (st == MMCSF_OK && d_lambda) {
    k_scale_cols<<<grid_for(F->dims[mode] * (uint64_t)R, 256), 256, 0, s>>>(d_out, F->dims[mode], R, d_lambda);
    MMCSF_LAUNCH_CHECK();
    ++launches;
  }
  Fm->last_launches = launches;
  return st;
}

extern "C" int mmcsf_mttkrp_pair(const mmcsf_format* F, int R, int factor_dtype, const void* const* d_factors,
                                 float* d_out_slice, float* d_out_mid, int* modes, const mmcsf_kernel_cfg* cfg,
                                 void* stream) {
  MMCSF_TRY(check_call(F, R, factor_dtype));
  if (F->impl != MMCSF_IMPL_MMCSF) return set_error(MMCSF_ERR_INVALID, "the two-output walk needs an MM-CSF format");
  const CsfPart* P = nullptr;
  int np = 0;
  for (int p = 0; p < F->nd; ++p)
    if (F->parts[p].present) { P = &F->parts[p]; ++np; }
  if (np > 1) return set_error(MMCSF_ERR_UNSUPPORTED, "the two-output walk needs a single-partition format");
  if (!P || !P->mid.p || (P->nd == 4 && !P->mid2.p))
    return set_error(MMCSF_ERR_UNSUPPORTED, "the two-output walk needs the per-nonzero middle indices");
  if (modes) { modes[0] = P->order[0]; modes[1] = P->order[1]; }
  if (!d_factors || !d_out_slice || !d_out_mid) return modes ? MMCSF_OK : set_error(MMCSF_ERR_INVALID, "null pointer");
  if (!native_R(R) || R > 128) return set_error(MMCSF_ERR_UNSUPPORTED, "the two-output walk runs R in 4..128");
  cudaStream_t s = S(stream);
  MMCSF_CUDA(cudaMemsetAsync(d_out_slice, 0, F->dims[P->order[0]] * (uint64_t)R * sizeof(float), s));
  MMCSF_CUDA(cudaMemsetAsync(d_out_mid, 0, F->dims[P->order[1]] * (uint64_t)R * sizeof(float), s));
  const int chunk = cfg && cfg->chunk > 0 ? cfg->chunk : (F->pair_chunk ? F->pair_chunk : 256);
  const int threads = cfg && cfg->block_threads > 0 ? cfg->block_threads : 256;
  const int mb = cfg && cfg->min_blocks > 0 ? cfg->min_blocks : (F->pair_mb ? F->pair_mb : 3);
  const int kern = cfg && cfg->kernel > 0 ? cfg->kernel : F->pair_kernel;
  if (kern < 0 || kern > 3) return set_error(MMCSF_ERR_INVALID, "kernel must be 0, 1, 2 or 3");
  if (threads % 32 || threads > 256) return set_error(MMCSF_ERR_INVALID, "block_threads must be a multiple of 32, <= 256");
  const int slot = CsfPart::cfib_slot((uint64_t)chunk);
  cudaError_t e;
  if (factor_dtype == MMCSF_DTYPE_F32) {
    Args<float> a{};
    fill_args(a, *P, nullptr, slot, chunk, R, d_factors, d_out_slice);
    a.out2 = d_out_mid;
    e = launch_pair_R<float>(a, P->nd, threads, mb, kern, s);
  } else {
    Args<__nv_bfloat16> a{};
    fill_args(a, *P, nullptr, slot, chunk, R, d_factors, d_out_slice);
    a.out2 = d_out_mid;
    e = launch_pair_R<__nv_bfloat16>(a, P->nd, threads, mb, kern, s);
  }
  if (e != cudaSuccess) return set_error(MMCSF_ERR_CUDA, "two-output walk launch: %s", cudaGetErrorString(e));
  const_cast<mmcsf_format*>(F)->last_launches = 1;
  return MMCSF_OK;
}

namespace {
// The tuned plan runs the partition's two upper modes in one walk (only
// without a caller override of the traversal or kernel). modes[0..1] get
// them.
bool pair_active(const mmcsf_format* F, int R, const mmcsf_kernel_cfg* cfg, int* modes) {
  if (!F->pair_use || F->impl != MMCSF_IMPL_MMCSF || !native_R(R) || R > 128) return false;
  if (cfg && (cfg->traversal != 0 || cfg->kernel != 0)) return false;
  const CsfPart* P = nullptr;
  for (int p = 0; p < F->nd; ++p)
    if (F->parts[p].present) {
      if (P) return false;  // several partitions
      P = &F->parts[p];
    }
  if (!P || !P->mid.p) return false;
  modes[0] = P->order[0];
  modes[1] = P->order[1];
  return true;
}
}  // namespace

extern "C" int mmcsf_mttkrp_all(const mmcsf_format* F, int R, int factor_dtype, const void* const* d_factors,
                                float* const* d_outs, const mmcsf_kernel_cfg* cfg, void* stream) {
  MMCSF_TRY(check_call(F, R, factor_dtype));
  if (!d_factors || !d_outs) return set_error(MMCSF_ERR_INVALID, "null pointer");
  if (F->impl != MMCSF_IMPL_MMCSF)
    return set_error(MMCSF_ERR_INVALID, "all-mode MTTKRP needs an MM-CSF format (-t 12)");
  int total = 0;
  int pm[2] = {-1, -1};
  const bool pair = pair_active(F, R, cfg, pm);
  if (pair) {
    MMCSF_TRY(mmcsf_mttkrp_pair(F, R, factor_dtype, d_factors, d_outs[pm[0]], d_outs[pm[1]], nullptr, nullptr, stream));
    total += F->last_launches;
  }
  for (int m = 0; m < F->nd; ++m) {
    if (pair && (m == pm[0] || m == pm[1])) continue;
    MMCSF_TRY(mmcsf_mttkrp(F, m, R, factor_dtype, d_factors, d_outs[m], cfg, stream));
    total += F->last_launches;
  }
  const_cast<mmcsf_format*>(F)->last_launches = total;
  return MMCSF_OK;
}

// Host-buffer all-mode MTTKRP with the copies overlapped with the kernels:
// the mode whose inputs exclude the largest factor runs first, as soon as the
// other factors are on the device, while the largest factor is uploaded on a
// second stream; every output is downloaded on a third stream right after its
// mode finishes. With pinned host buffers the copies and kernels overlap.
extern "C" int mmcsf_mttkrp_all_host(mmcsf_format* F, int R, const float* const* h_factors, float* const* h_outs,
                                     const mmcsf_kernel_cfg* cfg, void* stream) {
  MMCSF_TRY(check_call(F, R, MMCSF_DTYPE_F32));
  if (!h_factors || !h_outs) return set_error(MMCSF_ERR_INVALID, "null pointer");
  if (F->impl != MMCSF_IMPL_MMCSF)
    return set_error(MMCSF_ERR_INVALID, "all-mode MTTKRP needs an MM-CSF format (-t 12)");
  cudaStream_t s = S(stream);
  const int nd = F->nd;
  if (F->stage_R != R) {
    for (int m = 0; m < nd; ++m) {
      MMCSF_CUDA(F->stage_in[m].alloc(F->dims[m] * (uint64_t)R * 4));
      MMCSF_CUDA(F->stage_out[m].alloc(F->dims[m] * (uint64_t)R * 4));
    }
    F->stage_R = R;
  }
  if (!F->copy_in) {
    MMCSF_CUDA(cudaStreamCreateWithFlags(&F->copy_in, cudaStreamNonBlocking));
    MMCSF_CUDA(cudaStreamCreateWithFlags(&F->copy_out, cudaStreamNonBlocking));
    for (int m = 0; m < 4; ++m) {
      MMCSF_CUDA(cudaEventCreateWithFlags(&F->ev_in[m], cudaEventDisableTiming));
      MMCSF_CUDA(cudaEventCreateWithFlags(&F->ev_done[m], cudaEventDisableTiming));
    }
    MMCSF_CUDA(cudaEventCreateWithFlags(&F->ev_start, cudaEventDisableTiming));
  }
  // order: the largest factor is uploaded last; its own mode (which does not
  // read it) runs first, and its output's download overlaps that upload. The
  // two-output walk is not used here: once the last factor has arrived, one
  // launch per mode lets the first output's download overlap the next launch
  // (measured 9.23 against 9.45 ms per call on the 100M-nonzero skewed 3-D
  // tensor, where the copies take ~6 ms each way).
  int big = 0;
  for (int m = 1; m < nd; ++m)
    if (F->dims[m] > F->dims[big]) big = m;
  int order[4], n = 0;
  order[n++] = big;
  for (int m = 0; m < nd; ++m)
    if (m != big) order[n++] = m;
  // then the larger outputs first, so that their downloads start earlier
  std::stable_sort(order + 1, order + nd, [&](int x, int y) { return F->dims[x] > F->dims[y]; });
  const void* din[4];
  MMCSF_CUDA(cudaEventRecord(F->ev_start, s));  // staging buffers are free once earlier work on s is done
  MMCSF_CUDA(cudaStreamWaitEvent(F->copy_in, F->ev_start, 0));
  for (int m = 0; m < nd; ++m) din[m] = F->stage_in[m].p;
  for (int q = 0; q < nd; ++q) {  // upload: all but the largest, then the largest
    const int m = q < nd - 1 ? order[q + 1] : big;
    MMCSF_CUDA(cudaMemcpyAsync(F->stage_in[m].p, h_factors[m], F->dims[m] * (uint64_t)R * 4,
                               cudaMemcpyHostToDevice, F->copy_in));
    MMCSF_CUDA(cudaEventRecord(F->ev_in[m], F->copy_in));
  }
  int total = 0;
  auto download = [&](int m) -> int {
    MMCSF_CUDA(cudaEventRecord(F->ev_done[m], s));
    MMCSF_CUDA(cudaStreamWaitEvent(F->copy_out, F->ev_done[m], 0));
    MMCSF_CUDA(cudaMemcpyAsync(h_outs[m], F->stage_out[m].p, F->dims[m] * (uint64_t)R * 4, cudaMemcpyDeviceToHost,
                               F->copy_out));
    return MMCSF_OK;
  };
  for (int q = 0; q < nd; ++q) {
    const int m = order[q];
    for (int p = 0; p < nd; ++p)
      if (p != m) MMCSF_CUDA(cudaStreamWaitEvent(s, F->ev_in[p], 0));
    MMCSF_TRY(mmcsf_mttkrp(F, m, R, MMCSF_DTYPE_F32, din, F->stage_out[m].as<float>(), cfg, stream));
    total += F->last_launches;
    MMCSF_TRY(download(m));
  }
  MMCSF_CUDA(cudaStreamSynchronize(F->copy_out));
  MMCSF_CUDA(cudaStreamSynchronize(s));
  F->last_launches = total;
  return MMCSF_OK;
}

extern "C" int mmcsf_tune(mmcsf_format* F, int R, int factor_dtype, const void* const* d_factors,
                          float* const* d_outs, void* stream, mmcsf_plan* plan) {
  MMCSF_TRY(check_call(F, R, factor_dtype));
  if (!d_factors || !d_outs) return set_error(MMCSF_ERR_INVALID, "null pointer");
  cudaStream_t s = S(stream);
  cudaEvent_t e0, e1;
  MMCSF_CUDA(cudaEventCreate(&e0));
  MMCSF_CUDA(cudaEventCreate(&e1));
  const int chunks[] = {128, 256, 512, 1024, 2048, 4096};
  const int nmodes = F->impl == MMCSF_IMPL_MMCSF ? F->nd : 1;
  float best_ms[4] = {0, 0, 0, 0};
  int st = MMCSF_OK;
  for (int i = 0; i < nmodes && st == MMCSF_OK; ++i) {
    const int m = F->impl == MMCSF_IMPL_MMCSF ? i : F->mode;
    float best = 1e30f;
    int bt = 1, bc = 512, bm = 2, bk = 1;
    const int nkern = 3;
    for (int trav = 1; trav <= 2 && st == MMCSF_OK; ++trav) {
      if (trav == 2 && !F->views[m].present) continue;
      for (int kern = 1; kern <= nkern && st == MMCSF_OK; ++kern) {
      if (kern == 2 && F->nd == 4) continue;  // 4-D has no branch-free fiber walk
      for (int mbv = 1; mbv <= 4; ++mbv) {
        for (int c : chunks) {
          mmcsf_kernel_cfg cfg{};
          cfg.chunk = c;
          cfg.traversal = trav;
          cfg.min_blocks = mbv;
          cfg.kernel = kern;
          float ms = 0;
          for (int rep = 0; rep < 2; ++rep) {  // the second run is timed
            if ((st = mmcsf_mttkrp(F, m, R, factor_dtype, d_factors, d_outs[m], &cfg, stream)) != MMCSF_OK) break;
            if (cudaEventRecord(e0, s) != cudaSuccess) { st = MMCSF_ERR_CUDA; break; }
            if ((st = mmcsf_mttkrp(F, m, R, factor_dtype, d_factors, d_outs[m], &cfg, stream)) != MMCSF_OK) break;
            if (cudaEventRecord(e1, s) != cudaSuccess || cudaEventSynchronize(e1) != cudaSuccess) {
              st = MMCSF_ERR_CUDA;
              break;
            }
            cudaEventElapsedTime(&ms, e0, e1);
          }
          if (st != MMCSF_OK) break;
          if (ms < best) { best = ms; bt = trav; bc = c; bm = mbv; bk = kern; }
        }
        if (st != MMCSF_OK) break;
      }
      }
    }
    F->plan_traversal[m] = bt;
    F->plan_chunk[m] = bc;
    F->plan_mb[m] = bm;
    F->plan_kernel[m] = bk;
    best_ms[m] = best;
    if (plan) {
      plan->traversal[m] = bt;
      plan->chunk[m] = bc;
      plan->min_blocks[m] = bm;
      plan->kernel[m] = bk;
      plan->ms[m] = best;
    }
  }
  // the two upper modes of the partition in one walk, kept when it beats the
  // two modes' best single-mode plans
  F->pair_use = false;
  int pm[2] = {-1, -1};
  if (st == MMCSF_OK && F->impl == MMCSF_IMPL_MMCSF &&
      mmcsf_mttkrp_pair(F, R, factor_dtype, nullptr, nullptr, nullptr, pm, nullptr, stream) == MMCSF_OK &&
      native_R(R) && R <= 128) {
    float bestp = 1e30f;
    int bpc = 0, bpm = 0, bpk = 0;
    for (int kern : {2, 3})
    for (int mbv = 1; mbv <= 3 && st == MMCSF_OK && (kern == 3 || F->nd == 3); ++mbv)
      for (int c : {256, 512, 1024}) {
        mmcsf_kernel_cfg cfg{};
        cfg.chunk = c;
        cfg.min_blocks = mbv;
        cfg.kernel = kern;
        float ms = 0;
        for (int rep = 0; rep < 2; ++rep) {
          if ((st = mmcsf_mttkrp_pair(F, R, factor_dtype, d_factors, d_outs[pm[0]], d_outs[pm[1]], nullptr, &cfg,
                                      stream)) != MMCSF_OK)
            break;
          if (cudaEventRecord(e0, s) != cudaSuccess) { st = MMCSF_ERR_CUDA; break; }
          if ((st = mmcsf_mttkrp_pair(F, R, factor_dtype, d_factors, d_outs[pm[0]], d_outs[pm[1]], nullptr, &cfg,
                                      stream)) != MMCSF_OK)
            break;
          if (cudaEventRecord(e1, s) != cudaSuccess || cudaEventSynchronize(e1) != cudaSuccess) {
            st = MMCSF_ERR_CUDA;
            break;
          }
          cudaEventElapsedTime(&ms, e0, e1);
        }
        if (st != MMCSF_OK) break;
        if (ms < bestp) { bestp = ms; bpc = c; bpm = mbv; bpk = kern; }
      }
    if (st == MMCSF_OK && bestp < best_ms[pm[0]] + best_ms[pm[1]]) {
      F->pair_use = true;
      F->pair_chunk = bpc;
      F->pair_mb = bpm;
      F->pair_kernel = bpk;
    }
    if (plan && st == MMCSF_OK) {
      plan->pair = F->pair_use ? 1 : 0;
      plan->pair_chunk = bpc;
      plan->pair_min_blocks = bpm;
      plan->pair_kernel = bpk;
      plan->pair_ms = bestp;
    }
  } else if (plan) {
    plan->pair = 0;
    plan->pair_chunk = plan->pair_min_blocks = plan->pair_kernel = 0;
    plan->pair_ms = 0.f;
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  return st;
}

extern "C" int mmcsf_set_plan(mmcsf_format* F, const mmcsf_plan* plan) {
  if (!F || !plan) return set_error(MMCSF_ERR_INVALID, "null argument");
  for (int m = 0; m < F->nd; ++m) {
    if (plan->traversal[m] == 2 && !F->views[m].present)
      return set_error(MMCSF_ERR_INVALID, "plan uses a view for mode %d that was not built", m);
    if (plan->traversal[m] < 0 || plan->traversal[m] > 2 || plan->chunk[m] < 0 || plan->kernel[m] < 0 ||
        plan->kernel[m] > 3)
      return set_error(MMCSF_ERR_INVALID, "bad plan entry for mode %d", m);
    F->plan_traversal[m] = plan->traversal[m];
    F->plan_chunk[m] = plan->chunk[m];
    F->plan_mb[m] = plan->min_blocks[m];
    F->plan_kernel[m] = plan->kernel[m];
  }
  if (plan->pair_chunk < 0 || plan->pair_min_blocks < 0 || plan->pair_kernel < 0 || plan->pair_kernel > 3)
    return set_error(MMCSF_ERR_INVALID, "bad pair entry");
  F->pair_use = plan->pair != 0;
  F->pair_chunk = plan->pair_chunk;
  F->pair_mb = plan->pair_min_blocks;
  F->pair_kernel = plan->pair_kernel;
  return MMCSF_OK;
}
