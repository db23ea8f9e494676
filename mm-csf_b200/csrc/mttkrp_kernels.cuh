#pragma once
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
#include <atomic>
#include <cuda_bf16.h>

#include <cstring>
#include <type_traits>

#include "mttkrp_args.h"
#include "prims.cuh"

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

// Columns a lane owns: lane tl of a team of G holds columns 4 tl + 4 G v,
// v < V, so one load instruction of the team covers a contiguous 16 G-byte
// (FP32) or 8 G-byte (BF16) piece of the row.
template <class T, int G, int V>
struct Cols {
  static __device__ __forceinline__ uint32_t of(int tl, int v) { return (uint32_t)(4 * tl + 4 * G * v); }
};
// 4 BF16 values (two 32-bit words) widened to FP32
__device__ __forceinline__ float4 bf16x4_to_f32(uint32_t lo, uint32_t hi) {
  return make_float4(__uint_as_float(lo << 16), __uint_as_float(lo & 0xffff0000u), __uint_as_float(hi << 16),
                     __uint_as_float(hi & 0xffff0000u));
}
// Row piece v of a lane (columns Cols::of(tl, v)) from row base `rb`.
template <class T, int G, int V>
__device__ __forceinline__ float4 load_piece(const T* rb, int tl, int v) {
  return Row<T>::load(rb, Cols<T, G, V>::of(tl, v));
}

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
// The leaf-level scatter's reduction: four FP64 additions. A leaf row of a
// skewed tensor receives up to ~10^6 per-nonzero terms, whose sequential FP32
// rounding reaches ~1e-4 relative; in FP64 it stays far below 1e-5.
__device__ __forceinline__ void red4_f64(double* p, float4 v) {
  asm volatile(
      "red.global.add.f64 [%0], %1;\n\tred.global.add.f64 [%0+8], %2;\n\t"
      "red.global.add.f64 [%0+16], %3;\n\tred.global.add.f64 [%0+24], %4;" ::"l"(p),
      "d"((double)v.x), "d"((double)v.y), "d"((double)v.z), "d"((double)v.w)
      : "memory");
}


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
  auto ld = [&](const T* U, uint32_t row, int v) -> float4 {
    return load_piece<T, G, V>(U + (uint64_t)row * R, tl, v);
  };
  auto rd = [&](uint32_t row, int v, float4 x) { red4(out + (uint64_t)row * R + Cols<T, G, V>::of(tl, v), x); };
  [[maybe_unused]] auto rd64 = [&](uint32_t row, int v, float4 x) { red4_f64(a.out64 + (uint64_t)row * R + Cols<T, G, V>::of(tl, v), x); };

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
            for (int v = 0; v < V; ++v) rd64(kj[j], v, f4(val) * crow[v]);
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
  auto ld = [&](const T* U, uint32_t row, int v) -> float4 {
    return load_piece<T, G, V>(U + (uint64_t)row * R, tl, v);
  };
  auto rd = [&](uint32_t row, int v, float4 x) { red4(out + (uint64_t)row * R + Cols<T, G, V>::of(tl, v), x); };
  [[maybe_unused]] auto rd64 = [&](uint32_t row, int v, float4 x) { red4_f64(a.out64 + (uint64_t)row * R + Cols<T, G, V>::of(tl, v), x); };
  auto rd2 = [&](uint32_t row, int v, float4 x) { red4(out2 + (uint64_t)row * R + Cols<T, G, V>::of(tl, v), x); };

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
              for (int v = 0; v < V; ++v) rd64(kj[j], v, pmul_s(val, rowB[v]));
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
  auto ld = [&](const T* U, uint32_t row, int v) -> float4 {
    return load_piece<T, G, V>(U + (uint64_t)row * R, tl, v);
  };
  auto rd = [&](uint32_t row, int v, float4 x) { red4(out + (uint64_t)row * R + Cols<T, G, V>::of(tl, v), x); };
  [[maybe_unused]] auto rd64 = [&](uint32_t row, int v, float4 x) { red4_f64(a.out64 + (uint64_t)row * R + Cols<T, G, V>::of(tl, v), x); };

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
                rd64(kj[j], v, pmul_s(val, m));
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
  auto ld = [&](const T* U, uint32_t row, int v) -> float4 {
    return load_piece<T, G, V>(U + (uint64_t)row * R, tl, v);
  };
  auto rd = [&](float* o, uint32_t row, int v, float4 x) { red4(o + (uint64_t)row * R + Cols<T, G, V>::of(tl, v), x); };

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

// ---------------------------------------------------------------------------
// Per-nonzero walk with the middle row gathered once per FIBER ("fib" kernel,
// kernel 4), 3-D parts with `mid`. The slice mode's MTTKRP is regrouped by
// fiber: out[a] += sum over fibers (a, b) of U1[b] (.) t, t = sum over the
// fiber of v U2[k]. Per nonzero a team gathers only the leaf row (U2[k]) and
// adds v U2[k] to the open fiber's sum t; the fiber's middle row U1[b] is
// requested by a predicated gather in the batch where the fiber opens (the
// fiber's first nonzero carries the leaf-index flag, its `mid` entry gives
// b) and used when the fiber closes: acc += U1[b] (.) t. With TWO the same
// walk also produces the middle mode, out2[b] += U0[a] (.) t, one vector
// reduction per fiber (the two-output walk). Compared with gathering the
// middle row at every nonzero this reads F instead of N middle rows (29.9M
// instead of 100M on the skewed 500,000 x 2,000,000 x 20,000 tensor): each
// gathered 128-byte row costs one L1 wavefront, the unit these walks keep
// busiest. Outputs zeroed by the caller.
template <bool TWO, int G, int V, class T, int MB, int PFX>
__global__ void __launch_bounds__(256, MB) k_mttkrp_fib(const Args<T> a) {
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
  auto ld = [&](const T* U, uint32_t row, int v) -> float4 {
    return load_piece<T, G, V>(U + (uint64_t)row * R, tl, v);
  };
  auto rd = [&](float* o, uint32_t row, int v, float4 x) { red4(o + (uint64_t)row * R + Cols<T, G, V>::of(tl, v), x); };

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
  // the open fiber: its middle index and row (a fiber the chunk starts inside
  // is opened here; its flag, if any, is ignored below)
  uint32_t bopen = __ldg(mid + x0);
  float4 acc[V], t[V], mopen[V];
  [[maybe_unused]] float4 rowA[V];
#pragma unroll
  for (int v = 0; v < V; ++v) {
    acc[v] = t[v] = f4(0.f);
    mopen[v] = ld(U1, bopen, v);
    if constexpr (TWO) rowA[v] = ld(U0, ca, v);
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
        float4 rc[PF][V], rm[PF][V];
        uint32_t bjs[PF];
#pragma unroll
        for (int j = 0; j < PF; ++j) {
          const uint32_t kj = __shfl_sync(FULL, k, tb + jb + j);
          bjs[j] = __shfl_sync(FULL, b, tb + jb + j);
          const bool opens = (fm >> (jb + j)) & 1u;
#pragma unroll
          for (int v = 0; v < V; ++v) {
            rc[j][v] = ld(U2, kj, v);
            rm[j][v] = opens ? ld(U1, bjs[j], v) : f4(0.f);
          }
        }
#pragma unroll
        for (int j = 0; j < PF; ++j) {
          const float val = __shfl_sync(FULL, vv, tb + jb + j);
          const uint64_t x = xb + jb + j;
          if ((fm >> (jb + j)) & 1u) {  // the open fiber ends before nonzero j (in the open slice)
#pragma unroll
            for (int v = 0; v < V; ++v) {
              if constexpr (TWO) rd(out2, bopen, v, pmul(rowA[v], t[v]));
              acc[v] = pfma(mopen[v], t[v], acc[v]);
              t[v] = f4(0.f);
              mopen[v] = rm[j][v];
            }
            bopen = bjs[j];
          }
          if constexpr (SLOW) {
            if (x < x1 && x == nxt) {
#pragma unroll
              for (int v = 0; v < V; ++v) { rd(out, ca, v, acc[v]); acc[v] = f4(0.f); }
              ++sl;
              ca = __ldg(sidx + sl);
              nxt = __ldg(snz + sl + 1);
              if constexpr (TWO) {
#pragma unroll
                for (int v = 0; v < V; ++v) rowA[v] = ld(U0, ca, v);
              }
            }
          }
#pragma unroll
          for (int v = 0; v < V; ++v) t[v] = pfma_s(val, rc[j][v], t[v]);
        }
      }
    };
    if (slow) block(std::true_type{});
    else block(std::false_type{});
  }
  if (active) {
#pragma unroll
    for (int v = 0; v < V; ++v) {
      if constexpr (TWO) rd(out2, bopen, v, pmul(rowA[v], t[v]));
      rd(out, ca, v, pfma(mopen[v], t[v], acc[v]));
    }
  }
}

// ---------------------------------------------------------------------------
// Per-nonzero walks with vector index loads ("rowsv" / "pairv", kernel 5),
// 3-D, G >= 4. The same walks as k_mttkrp_rows (slice, middle and leaf
// levels) and k_mttkrp_pair, but a team reads its nonzeros' leaf indices,
// middle indices and values four at a time: lane tl of a team holds nonzeros
// 4 tl .. 4 tl + 3 of a super-block of 4G, loaded as one 16-byte vector per
// array, and nonzero j of the super-block's sub-block sb (G nonzeros) comes
// to the team by one shuffle from lane tb + sb G/4 + j/4, component j % 4.
// Each of those loads touches one 64-byte (G = 4) to 512-byte (G = 32) span
// per team instead of a G x 4-byte span per G nonzeros: about a quarter of
// the L1 wavefronts the index loads cost. Needs chunk % 4 == 0 and 16-byte
// aligned index/value arrays (the host checks both).
template <class U4> __device__ __forceinline__ uint32_t comp4(const U4& u, int c) {
  return c == 0 ? u.x : (c == 1 ? u.y : (c == 2 ? u.z : u.w));
}
__device__ __forceinline__ float comp4f(const float4& u, int c) {
  return c == 0 ? u.x : (c == 1 ? u.y : (c == 2 ? u.z : u.w));
}

template <int OUT, int G, int V, class T, int MB, int PFX>
__global__ void __launch_bounds__(256, MB) k_mttkrp_rowsv(const Args<T> a) {
  static_assert(G >= 4 && G % 4 == 0, "vector index loads need teams of 4, 8, 16 or 32 lanes");
  constexpr int LEAF = 2;
  constexpr bool MIDL = OUT == 1;
  constexpr uint32_t R = 4 * G * V;
  constexpr uint32_t FLAG = 0x80000000u;
  constexpr int PF = G > PFX ? PFX : G;
  constexpr uint32_t SB = 4 * G;
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
  const T* __restrict__ UL = a.U[LEAF];
  float* __restrict__ out = a.out;
  auto ld = [&](const T* U, uint32_t row, int v) -> float4 {
    return load_piece<T, G, V>(U + (uint64_t)row * R, tl, v);
  };
  auto rd = [&](uint32_t row, int v, float4 x) { red4(out + (uint64_t)row * R + Cols<T, G, V>::of(tl, v), x); };
  [[maybe_unused]] auto rd64 = [&](uint32_t row, int v, float4 x) {
    red4_f64(a.out64 + (uint64_t)row * R + Cols<T, G, V>::of(tl, v), x);
  };

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
  float4 acc[V], rowA[V];
#pragma unroll
  for (int v = 0; v < V; ++v) {
    acc[v] = f4(0.f);
    if constexpr (OUT == LEAF || MIDL) rowA[v] = ld(U0, ca, v);
  }
  [[maybe_unused]] uint32_t bopen = 0;
  if constexpr (MIDL) bopen = __ldg(mid + x0);

  // this lane's four nonzeros of the super-block at offset its
  auto load_sb = [&](uint32_t its, uint4& K, uint4& B, float4& W) {
    const uint64_t xx = x0 + its + 4 * (uint32_t)tl;
    if (xx + 3 < x1) {
      K = __ldg(reinterpret_cast<const uint4*>(leaf + xx));
      B = __ldg(reinterpret_cast<const uint4*>(mid + xx));
      W = __ldg(reinterpret_cast<const float4*>(vals + xx));
    } else {
      K = make_uint4(0u, 0u, 0u, 0u);
      B = K;
      W = f4(0.f);
      if (xx < x1) { K.x = __ldg(leaf + xx); B.x = __ldg(mid + xx); W.x = __ldg(vals + xx); }
      if (xx + 1 < x1) { K.y = __ldg(leaf + xx + 1); B.y = __ldg(mid + xx + 1); W.y = __ldg(vals + xx + 1); }
      if (xx + 2 < x1) { K.z = __ldg(leaf + xx + 2); B.z = __ldg(mid + xx + 2); W.z = __ldg(vals + xx + 2); }
    }
  };
  uint4 Kc, Bc, Kn, Bn;
  float4 Wc, Wn;
  load_sb(0, Kc, Bc, Wc);
  for (uint32_t its = 0; its < chunk; its += SB) {
    load_sb(its + SB, Kn, Bn, Wn);  // the next super-block, while this one is processed
    [[maybe_unused]] uint32_t bal[4] = {0u, 0u, 0u, 0u};  // middle level: fiber starts, by component
    if constexpr (MIDL) {
#pragma unroll
      for (int c = 0; c < 4; ++c)
        bal[c] = __ballot_sync(FULL, (comp4(Kc, c) & FLAG) && (x0 + its + 4 * (uint32_t)tl + c != x0));
    }
    for (int sb = 0; sb < 4; ++sb) {
      const uint64_t xb = x0 + its + (uint32_t)sb * G;
      const int src0 = tb + sb * (G / 4);
      const bool slow = __any_sync(FULL, xb < x1 && xb + G > nxt);
      auto block = [&](auto slow_tag) {
        constexpr bool SLOW = decltype(slow_tag)::value;
#pragma unroll
        for (int jb = 0; jb < G; jb += PF) {
          [[maybe_unused]] float4 rc[(OUT == 0 || MIDL) ? PF : 1][V];
          [[maybe_unused]] float4 rb[MIDL ? 1 : PF][V];
          [[maybe_unused]] uint32_t bjs[MIDL ? PF : 1];
          uint32_t kj[PF];
#pragma unroll
          for (int j = 0; j < PF; ++j) {
            const int jj = jb + j, src = src0 + (jj >> 2);
            kj[j] = __shfl_sync(FULL, comp4(Kc, jj & 3), src) & ~FLAG;
            const uint32_t bj = __shfl_sync(FULL, comp4(Bc, jj & 3), src);
            if constexpr (MIDL) bjs[j] = bj;
#pragma unroll
            for (int v = 0; v < V; ++v) {
              if constexpr (MIDL) rc[j][v] = ld(UL, kj[j], v);
              else rb[j][v] = ld(U1, bj, v);
              if constexpr (OUT == 0) rc[j][v] = ld(UL, kj[j], v);
            }
          }
#pragma unroll
          for (int j = 0; j < PF; ++j) {
            const int jj = jb + j, src = src0 + (jj >> 2);
            const float val = __shfl_sync(FULL, comp4f(Wc, jj & 3), src);
            const uint64_t x = xb + jj;
            if constexpr (MIDL) {
              if ((bal[jj & 3] >> src) & 1u) {  // the open fiber ends before nonzero jj
#pragma unroll
                for (int v = 0; v < V; ++v) { rd(bopen, v, pmul(rowA[v], acc[v])); acc[v] = f4(0.f); }
                bopen = bjs[j];
              }
            }
            if constexpr (SLOW) {
              if (x < x1 && x == nxt) {
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
              for (int v = 0; v < V; ++v) acc[v] = pfma(pmul_s(val, rb[j][v]), rc[j][v], acc[v]);
            } else {
              if (x < x1) {
#pragma unroll
                for (int v = 0; v < V; ++v) rd64(kj[j], v, pmul_s(val, pmul(rowA[v], rb[j][v])));
              }
            }
          }
        }
      };
      if (slow) block(std::true_type{});
      else block(std::false_type{});
    }
    Kc = Kn; Bc = Bn; Wc = Wn;
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

template <int G, int V, class T, int MB, int PFX>
__global__ void __launch_bounds__(256, MB) k_mttkrp_pairv(const Args<T> a) {
  static_assert(G >= 4 && G % 4 == 0, "vector index loads need teams of 4, 8, 16 or 32 lanes");
  constexpr uint32_t R = 4 * G * V;
  constexpr uint32_t FLAG = 0x80000000u;
  constexpr int PF = G > PFX ? PFX : G;
  constexpr uint32_t SB = 4 * G;
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
  auto ld = [&](const T* U, uint32_t row, int v) -> float4 {
    return load_piece<T, G, V>(U + (uint64_t)row * R, tl, v);
  };
  auto rd = [&](float* o, uint32_t row, int v, float4 x) { red4(o + (uint64_t)row * R + Cols<T, G, V>::of(tl, v), x); };

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
  auto load_sb = [&](uint32_t its, uint4& K, uint4& B, float4& W) {
    const uint64_t xx = x0 + its + 4 * (uint32_t)tl;
    if (xx + 3 < x1) {
      K = __ldg(reinterpret_cast<const uint4*>(leaf + xx));
      B = __ldg(reinterpret_cast<const uint4*>(mid + xx));
      W = __ldg(reinterpret_cast<const float4*>(vals + xx));
    } else {
      K = make_uint4(0u, 0u, 0u, 0u);
      B = K;
      W = f4(0.f);
      if (xx < x1) { K.x = __ldg(leaf + xx); B.x = __ldg(mid + xx); W.x = __ldg(vals + xx); }
      if (xx + 1 < x1) { K.y = __ldg(leaf + xx + 1); B.y = __ldg(mid + xx + 1); W.y = __ldg(vals + xx + 1); }
      if (xx + 2 < x1) { K.z = __ldg(leaf + xx + 2); B.z = __ldg(mid + xx + 2); W.z = __ldg(vals + xx + 2); }
    }
  };
  uint4 Kc, Bc, Kn, Bn;
  float4 Wc, Wn;
  load_sb(0, Kc, Bc, Wc);
  for (uint32_t its = 0; its < chunk; its += SB) {
    load_sb(its + SB, Kn, Bn, Wn);
    uint32_t bal[4];
#pragma unroll
    for (int c = 0; c < 4; ++c)
      bal[c] = __ballot_sync(FULL, (comp4(Kc, c) & FLAG) && (x0 + its + 4 * (uint32_t)tl + c != x0));
    for (int sb = 0; sb < 4; ++sb) {
      const uint64_t xb = x0 + its + (uint32_t)sb * G;
      const int src0 = tb + sb * (G / 4);
      const bool slow = __any_sync(FULL, xb < x1 && xb + G > nxt);
      auto block = [&](auto slow_tag) {
        constexpr bool SLOW = decltype(slow_tag)::value;
#pragma unroll
        for (int jb = 0; jb < G; jb += PF) {
          float4 rb[PF][V], rc[PF][V];
          uint32_t bjs[PF];
#pragma unroll
          for (int j = 0; j < PF; ++j) {
            const int jj = jb + j, src = src0 + (jj >> 2);
            const uint32_t kj = __shfl_sync(FULL, comp4(Kc, jj & 3), src) & ~FLAG;
            bjs[j] = __shfl_sync(FULL, comp4(Bc, jj & 3), src);
#pragma unroll
            for (int v = 0; v < V; ++v) {
              rb[j][v] = ld(U1, bjs[j], v);
              rc[j][v] = ld(U2, kj, v);
            }
          }
#pragma unroll
          for (int j = 0; j < PF; ++j) {
            const int jj = jb + j, src = src0 + (jj >> 2);
            const float val = __shfl_sync(FULL, comp4f(Wc, jj & 3), src);
            const uint64_t x = xb + jj;
            if ((bal[jj & 3] >> src) & 1u) {  // the open fiber ends before nonzero jj (in the open slice)
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
    Kc = Kn; Bc = Bn; Wc = Wn;
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
  auto ld = [&](const T* U, uint32_t row, int v) -> float4 {
    return load_piece<T, G, V>(U + (uint64_t)row * R, tl, v);
  };
  auto rd = [&](float* o, uint32_t row, int v, float4 x) { red4(o + (uint64_t)row * R + Cols<T, G, V>::of(tl, v), x); };

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

// A lane's piece of one factor row as loaded (FP32: V float4; BF16: V 8-byte
// vectors), widened to FP32 only where it is used, so rows in flight hold
// half the registers at BF16.
template <class T, int G, int V>
struct RawPiece {
  static constexpr bool BF = std::is_same<T, __nv_bfloat16>::value;
  using W = std::conditional_t<BF, uint2, float4>;
  W w[V];
  __device__ __forceinline__ void load(const T* rb, int tl) {
#pragma unroll
    for (int i = 0; i < V; ++i) w[i] = __ldg(reinterpret_cast<const W*>(rb + Cols<T, G, V>::of(tl, i)));
  }
  __device__ __forceinline__ float4 get(int v) const {
    if constexpr (BF) return bf16x4_to_f32(w[v].x, w[v].y);
    else return w[v];
  }
};

// ---------------------------------------------------------------------------
// Per-nonzero walks of a 3-D part with `mid` whose teams are interleaved over
// one range of nonzeros per warp (kernel 6): the slice-level MTTKRP, out[a] +=
// v U1[b] (.) U2[k], and with PAIR also the middle mode's, out2[b] += U0[a]
// (.) sum over the fiber (a, b) of v U2[k] (the two-output walk).
//
// The warp owns the NT = 32 / G teams' chunks as one range [x0, x1). Team t
// takes the groups of 4Q consecutive nonzeros g = NT j + t (j = 0, 1, ...),
// and every lane of the team loads the group's leaf indices, middle indices
// and values itself, Q 16-byte vectors per array. One load instruction of
// the warp then reads the NT teams' adjacent vectors, one 128-byte line at
// most (G >= 4), so the index loads cost 3Q L1 wavefronts per 4Q NT nonzeros
// (0.19 per nonzero at G = 8, Q = 1) and nothing is broadcast; the shuffle
// broadcast of the contiguous-chunk walks costs ~1.1 wavefronts per nonzero
// at G = 8 (three shuffles per team per nonzero, four teams per shuffle, and
// the index loads). Each team keeps its own slice state; with PAIR also its
// own open fiber, which closes when the middle index or the slice changes, so
// a fiber spread over several teams' groups is reduced once per team. Needs
// chunk % 4 == 0 and 16-byte aligned index/value arrays; outputs zeroed by
// the caller.
template <bool PAIR, int Q, int G, int V, class T, int MB>
__global__ void __launch_bounds__(256, MB) k_mttkrp_il(const Args<T> a) {
  constexpr uint32_t NT = 32 / G;
  constexpr uint32_t R = 4 * G * V;
  constexpr uint32_t FLAG = 0x80000000u;
  constexpr uint32_t NONE = 0xffffffffu;
  constexpr uint32_t GS = 4 * Q;     // nonzeros per group
  constexpr uint32_t STEP = GS * NT;  // nonzeros per warp iteration
  using Piece = RawPiece<T, G, V>;
  const int lane = threadIdx.x & 31;
  const int tl = lane & (G - 1);
  const uint32_t t = (uint32_t)lane / G;
  const float* __restrict__ vals = a.vals;
  const uint32_t* __restrict__ leaf = a.leaf;
  const uint32_t* __restrict__ mid = a.mid;
  const uint32_t* __restrict__ snz = a.snz;
  const uint32_t* __restrict__ sidx = a.sidx;
  const T* __restrict__ U0 = a.U[0];
  const T* __restrict__ U1 = a.U[1];
  const T* __restrict__ U2 = a.U[2];
  float* __restrict__ out = a.out;
  [[maybe_unused]] float* __restrict__ out2 = a.out2;
  auto rd = [&](float* o, uint32_t row, int v, float4 x) { red4(o + (uint64_t)row * R + Cols<T, G, V>::of(tl, v), x); };

  // the warp's range (warp-uniform; the kernel has no warp-collective steps)
  const uint64_t warp = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
  const uint64_t span = (uint64_t)a.chunk * NT;
  const uint64_t x0 = warp * span;
  if (x0 >= a.nnz) return;
  const uint64_t x1 = min(x0 + span, a.nnz);
  uint32_t sl;
  if (a.cslc) {
    sl = __ldg(a.cslc + warp * NT);  // the slice of nonzero (warp NT) chunk = x0
  } else {
    uint32_t lo = 0, hi = a.nslc - 1;
    while (lo < hi) {
      const uint32_t m = (lo + hi + 1) >> 1;
      if ((uint64_t)__ldg(snz + m) <= x0) lo = m; else hi = m - 1;
    }
    sl = lo;
  }
  uint32_t ca = __ldg(sidx + sl);
  uint64_t nxt = __ldg(snz + sl + 1);
  float4 acc[V];
  [[maybe_unused]] float4 accf[V], rowA[V];
#pragma unroll
  for (int v = 0; v < V; ++v) {
    acc[v] = f4(0.f);
    if constexpr (PAIR) {
      accf[v] = f4(0.f);
      rowA[v] = load_piece<T, G, V>(U0 + (uint64_t)ca * R, tl, v);
    }
  }
  [[maybe_unused]] uint32_t bopen = NONE;

  // this team's group of the warp iteration starting at xs; positions at or
  // past x1 read as index 0, value 0 and are skipped
  auto load_grp = [&](uint64_t xs, uint4 (&K)[Q], uint4 (&B)[Q], float4 (&W)[Q]) {
#pragma unroll
    for (int q = 0; q < Q; ++q) {
      const uint64_t xx = xs + GS * t + 4 * q;
      if (xx + 3 < x1) {
        K[q] = __ldg(reinterpret_cast<const uint4*>(leaf + xx));
        B[q] = __ldg(reinterpret_cast<const uint4*>(mid + xx));
        W[q] = __ldg(reinterpret_cast<const float4*>(vals + xx));
      } else {
        K[q] = make_uint4(0u, 0u, 0u, 0u);
        B[q] = K[q];
        W[q] = f4(0.f);
        if (xx < x1) { K[q].x = __ldg(leaf + xx); B[q].x = __ldg(mid + xx); W[q].x = __ldg(vals + xx); }
        if (xx + 1 < x1) { K[q].y = __ldg(leaf + xx + 1); B[q].y = __ldg(mid + xx + 1); W[q].y = __ldg(vals + xx + 1); }
        if (xx + 2 < x1) { K[q].z = __ldg(leaf + xx + 2); B[q].z = __ldg(mid + xx + 2); W[q].z = __ldg(vals + xx + 2); }
      }
    }
  };
  uint4 Kc[Q], Bc[Q], Kn[Q], Bn[Q];
  float4 Wc[Q], Wn[Q];
  load_grp(x0, Kc, Bc, Wc);
  for (uint64_t xs = x0; xs < x1; xs += STEP) {
    load_grp(xs + STEP, Kn, Bn, Wn);  // the next group, while this one is processed
    const uint64_t xg = xs + GS * t;
    Piece rb[GS], rc[GS];
#pragma unroll
    for (int j = 0; j < (int)GS; ++j) {
      const uint32_t k = comp4(Kc[j >> 2], j & 3) & ~FLAG;
      const uint32_t b = comp4(Bc[j >> 2], j & 3);
      rb[j].load(U1 + (uint64_t)b * R, tl);
      rc[j].load(U2 + (uint64_t)k * R, tl);
    }
    // FAST: the whole group lies before x1 and in the team's open slice (the
    // common case), so no nonzero needs the end or slice tests
    auto body = [&](auto fast_tag) {
      constexpr bool FAST = decltype(fast_tag)::value;
#pragma unroll
      for (int j = 0; j < (int)GS; ++j) {
        const uint64_t x = xg + j;
        if (FAST || x < x1) {
          const float val = comp4f(Wc[j >> 2], j & 3);
          if constexpr (!FAST) {
            if (x >= nxt) {  // the team's slice ends before nonzero x
#pragma unroll
              for (int v = 0; v < V; ++v) { rd(out, ca, v, acc[v]); acc[v] = f4(0.f); }
              if constexpr (PAIR) {
                if (bopen != NONE) {
#pragma unroll
                  for (int v = 0; v < V; ++v) rd(out2, bopen, v, pmul(rowA[v], accf[v]));
                }
#pragma unroll
                for (int v = 0; v < V; ++v) accf[v] = f4(0.f);
                bopen = NONE;
              }
              do {
                ++sl;
                nxt = __ldg(snz + sl + 1);
              } while (x >= nxt);
              ca = __ldg(sidx + sl);
              if constexpr (PAIR) {
#pragma unroll
                for (int v = 0; v < V; ++v) rowA[v] = load_piece<T, G, V>(U0 + (uint64_t)ca * R, tl, v);
              }
            }
          }
          if constexpr (PAIR) {
            const uint32_t b = comp4(Bc[j >> 2], j & 3);
            if (b != bopen) {  // the team's open fiber ends before nonzero x
              if (bopen != NONE) {
#pragma unroll
                for (int v = 0; v < V; ++v) rd(out2, bopen, v, pmul(rowA[v], accf[v]));
              }
#pragma unroll
              for (int v = 0; v < V; ++v) accf[v] = f4(0.f);
              bopen = b;
            }
          }
#pragma unroll
          for (int v = 0; v < V; ++v) {
            const float4 c = rc[j].get(v);
            acc[v] = pfma(pmul_s(val, rb[j].get(v)), c, acc[v]);
            if constexpr (PAIR) accf[v] = pfma_s(val, c, accf[v]);
          }
        }
      }
    };
    if (xg + GS <= x1 && xg + GS <= nxt) body(std::true_type{});
    else body(std::false_type{});
#pragma unroll
    for (int q = 0; q < Q; ++q) { Kc[q] = Kn[q]; Bc[q] = Bn[q]; Wc[q] = Wn[q]; }
  }
#pragma unroll
  for (int v = 0; v < V; ++v) rd(out, ca, v, acc[v]);
  if constexpr (PAIR) {
    if (bopen != NONE) {
#pragma unroll
      for (int v = 0; v < V; ++v) rd(out2, bopen, v, pmul(rowA[v], accf[v]));
    }
  }
}

// occupancy levels of kernel 6: (CTAs per SM the registers must allow, groups
// of 4 nonzeros per team and iteration) = 1: (2, 2), 2: (2, 1), 3: (3, 1),
// 4: (4, 1)
template <bool PAIR, int G, int V, class T>
cudaError_t launch_il(const Args<T>& a, int threads, int mb, cudaStream_t s) {
  constexpr uint64_t NT = 32 / G;
  const uint64_t teams = (a.nnz + a.chunk - 1) / a.chunk;
  const uint64_t warps = (teams + NT - 1) / NT;
  const uint64_t blocks = (warps * 32 + threads - 1) / threads;
  switch (mb) {
    case 1: k_mttkrp_il<PAIR, 2, G, V, T, 2><<<(unsigned)blocks, threads, 0, s>>>(a); break;
    case 3: k_mttkrp_il<PAIR, 1, G, V, T, 3><<<(unsigned)blocks, threads, 0, s>>>(a); break;
    case 4: k_mttkrp_il<PAIR, 1, G, V, T, 4><<<(unsigned)blocks, threads, 0, s>>>(a); break;
    default: k_mttkrp_il<PAIR, 1, G, V, T, 2><<<(unsigned)blocks, threads, 0, s>>>(a); break;
  }
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Per-nonzero walk with the factor rows staged in shared memory (kernel 7),
// 3-D parts with `mid`: the slice-level MTTKRP, out[a] += sum over fibers
// (a, b) of U1[b] (.) t_f, t_f = sum over the fiber of v U2[k], and with PAIR
// also the middle mode's, out2[b] += U0[a] (.) t_f (the two-output walk).
//
// The walks above issue one batch of row gathers into registers and then
// wait a full memory latency before they can use any of it, so each warp
// keeps rows in flight only part of the time, and registers bound how many.
// Here the rows go to shared memory with cp.async (16-byte pieces, L2 only;
// 8-byte pieces for BF16 factors), D steps of GS nonzeros per team ahead of
// their use, and the indices and values another D steps ahead of that, so
// every warp keeps D steps of rows in flight continuously whatever the
// latency. A lane copies exactly the pieces of each row it later reads (its
// columns of the team's rows), so the row ring needs no synchronisation
// beyond the lane's own cp.async.wait_group; the index ring, copied by the
// warp together and read by every lane of a team, is guarded by __syncwarp.
//
// The middle row is fetched once per fiber (when the middle index changes
// along the team's nonzeros) and used when the fiber closes: acc += U1[b] (.)
// t_f. A team walks a contiguous range of nonzeros; the grid is one block per
// SM with as many warps as the rings allow in shared memory (at most 24), and
// the ranges split the nonzeros evenly over all teams. Positions are 32-bit
// (a format holds fewer than 2^32 nonzeros). Needs 16-byte aligned index and
// value arrays; outputs zeroed by the caller.
__device__ __forceinline__ uint32_t sm_addr(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
// 16 bytes global -> shared, bypassing L1; the first n bytes are copied and
// the rest of the 16 zero-filled (n = 0 reads nothing)
__device__ __forceinline__ void cpa16(uint32_t dst, const void* src, uint32_t n) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(dst), "l"(src), "r"(n) : "memory");
}
__device__ __forceinline__ void cpa_row16(uint32_t dst, const void* src) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(dst), "l"(src) : "memory");
}
__device__ __forceinline__ void cpa_row8(uint32_t dst, const void* src) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(dst), "l"(src) : "memory");
}
__device__ __forceinline__ void cpa_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cpa_wait() {
  asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

// Shared-memory layout of kernel 7, per warp: DI = 2 D index stages (three
// arrays x NT teams x GS / 4 16-byte vectors), then D row stages (leaf and
// middle slots x GS nonzeros x V pieces x 32 lanes).
template <int G, int V, class T, int GS, int D>
struct StgShape {
  static constexpr uint32_t NT = 32 / G;
  static constexpr uint32_t DI = 2 * D;
  static constexpr uint32_t PB = std::is_same<T, __nv_bfloat16>::value ? 8 : 16;
  static constexpr uint32_t NV = GS / 4;
  static constexpr uint32_t NIV = 3 * NT * NV;
  static constexpr uint32_t NR = (NIV + 31) / 32;  // copy rounds per index stage
  static constexpr uint32_t IDX_STAGE = NIV * 16;
  static constexpr uint32_t ROW_STAGE = 2 * GS * V * 32 * PB;
  static constexpr uint32_t WARP_BYTES = DI * IDX_STAGE + D * ROW_STAGE;
  static constexpr uint32_t MAX_SMEM = 227 * 1024;
  static constexpr uint32_t WPB = MAX_SMEM / WARP_BYTES > 24 ? 24 : MAX_SMEM / WARP_BYTES;
};

template <bool PAIR, int G, int V, class T, int GS, int D>
__global__ void __launch_bounds__(32 * StgShape<G, V, T, GS, D>::WPB, 1) k_mttkrp_stg(const Args<T> a) {
  using SS = StgShape<G, V, T, GS, D>;
  static_assert(GS == 4 || GS == 8, "steps of 4 or 8 nonzeros per team");
  constexpr uint32_t NT = SS::NT, DI = SS::DI, NV = SS::NV, NR = SS::NR;
  constexpr uint32_t R = 4 * G * V;
  constexpr uint32_t FLAG = 0x80000000u;
  constexpr uint32_t NONE = 0xffffffffu;
  constexpr bool BF = std::is_same<T, __nv_bfloat16>::value;
  using Piece = std::conditional_t<BF, uint2, float4>;
  extern __shared__ __align__(128) unsigned char stg_smem[];
  const int lane = threadIdx.x & 31;
  const int tl = lane & (G - 1);
  const uint32_t t = (uint32_t)lane / G;
  unsigned char* const wsm = stg_smem + (threadIdx.x >> 5) * SS::WARP_BYTES;
  unsigned char* const isc = wsm;                                   // index stages
  unsigned char* const rsc = wsm + DI * SS::IDX_STAGE + lane * SS::PB;  // this lane's row pieces
  const uint32_t* __restrict__ snz = a.snz;
  const uint32_t* __restrict__ sidx = a.sidx;
  const T* __restrict__ U0 = a.U[0];
  const T* __restrict__ U1 = a.U[1];
  const T* __restrict__ U2 = a.U[2];
  float* __restrict__ out = a.out;
  [[maybe_unused]] float* __restrict__ out2 = a.out2;
  const uint32_t chunk = a.chunk, nnz = (uint32_t)a.nnz;
  const uint32_t nsteps = chunk / GS;
  auto rd = [&](float* o, uint32_t row, int v, float4 x) { red4(o + (uint64_t)row * R + Cols<T, G, V>::of(tl, v), x); };

  // the warp's first team, and this team's range [x0, x1) (empty past nnz)
  const uint32_t team0 = (uint32_t)((blockIdx.x * (uint64_t)blockDim.x + (threadIdx.x & ~31u)) / G);
  const uint32_t x0 = (uint32_t)min((uint64_t)(team0 + t) * chunk, (uint64_t)nnz);
  const uint32_t x1 = (uint32_t)min((uint64_t)x0 + chunk, (uint64_t)nnz);

  // index copies: lane q of round r copies vector q = (array, team, vec) of
  // every index stage; its source advances GS nonzeros per stage
  const void* ibase_src[NR];
  uint32_t ip[NR], ie[NR];
  bool iq[NR];
#pragma unroll
  for (uint32_t r = 0; r < NR; ++r) {
    const uint32_t q = r * 32 + (uint32_t)lane;
    iq[r] = q < SS::NIV;
    const uint32_t arr = q / (NT * NV), tt = (q / NV) % NT, vec = q % NV;
    const uint32_t s0 = (uint32_t)min((uint64_t)(team0 + tt) * chunk, (uint64_t)nnz);
    ip[r] = s0 + 4 * vec;
    ie[r] = (uint32_t)min((uint64_t)s0 + chunk, (uint64_t)nnz);
    ibase_src[r] = arr == 0 ? (const void*)a.leaf : arr == 1 ? (const void*)a.mid : (const void*)a.vals;
  }
  auto issue_idx = [&](uint32_t slot) {
    const uint32_t dst = sm_addr(isc + slot * SS::IDX_STAGE) + (uint32_t)lane * 16;
#pragma unroll
    for (uint32_t r = 0; r < NR; ++r) {
      if (iq[r]) {
        const uint32_t n = ip[r] < ie[r] ? min(16u, (ie[r] - ip[r]) * 4) : 0u;
        cpa16(dst + r * 512, n ? (const void*)((const uint32_t*)ibase_src[r] + ip[r]) : ibase_src[r], n);
        ip[r] += GS;
      }
    }
  };
  // this team's vector vec of array arr in index stage `slot`
  auto ivec = [&](uint32_t slot, uint32_t arr, uint32_t vec) -> uint4 {
    return *reinterpret_cast<const uint4*>(isc + slot * SS::IDX_STAGE + ((arr * NT + t) * NV + vec) * 16);
  };
  auto piece_at = [&](uint32_t rslot, uint32_t kind, uint32_t j, int v) -> unsigned char* {
    return rsc + rslot * SS::ROW_STAGE + ((kind * GS + j) * V + v) * 32 * SS::PB;
  };
  auto copy_row = [&](unsigned char* dst, const T* U, uint32_t row, int v) {
    const T* src = U + (uint64_t)row * R + Cols<T, G, V>::of(tl, v);
    if constexpr (BF) cpa_row8(sm_addr(dst), src);
    else cpa_row16(sm_addr(dst), src);
  };
  auto widen = [&](const Piece& p) -> float4 {
    if constexpr (BF) return bf16x4_to_f32(p.x, p.y);
    else return p;
  };
  // row stage: this team's leaf rows, and the middle row wherever the middle
  // index changes along the team's nonzeros (bq: the last one seen)
  uint32_t bq = NONE, xr = x0;
  auto issue_rows = [&](uint32_t islot, uint32_t rslot) {
    uint32_t K[GS], B[GS];
#pragma unroll
    for (uint32_t c = 0; c < NV; ++c) {
      const uint4 k4 = ivec(islot, 0, c), b4 = ivec(islot, 1, c);
      K[4 * c] = k4.x; K[4 * c + 1] = k4.y; K[4 * c + 2] = k4.z; K[4 * c + 3] = k4.w;
      B[4 * c] = b4.x; B[4 * c + 1] = b4.y; B[4 * c + 2] = b4.z; B[4 * c + 3] = b4.w;
    }
    const bool full = xr + GS <= x1;
#pragma unroll
    for (uint32_t j = 0; j < GS; ++j) {
      if (full || xr + j < x1) {
#pragma unroll
        for (int v = 0; v < V; ++v) copy_row(piece_at(rslot, 0, j, v), U2, K[j] & ~FLAG, v);
        if (B[j] != bq) {
#pragma unroll
          for (int v = 0; v < V; ++v) copy_row(piece_at(rslot, 1, j, v), U1, B[j], v);
          bq = B[j];
        }
      }
    }
    xr += GS;
  };

  // open slice of this team
  uint32_t sl = 0;
  if (x0 < x1) {
    uint32_t lo = 0, hi = a.nslc - 1;
    while (lo < hi) {
      const uint32_t mm = (lo + hi + 1) >> 1;
      if (__ldg(snz + mm) <= x0) lo = mm; else hi = mm - 1;
    }
    sl = lo;
  }
  uint32_t ca = __ldg(sidx + sl);
  uint32_t nxt = __ldg(snz + sl + 1);
  float4 acc[V], accf[V], rowB[V];
  [[maybe_unused]] float4 rowA[V];
#pragma unroll
  for (int v = 0; v < V; ++v) {
    acc[v] = accf[v] = rowB[v] = f4(0.f);
    if constexpr (PAIR) rowA[v] = load_piece<T, G, V>(U0 + (uint64_t)ca * R, tl, v);
  }
  uint32_t bopen = NONE, blast = NONE;
  auto close_fiber = [&]() {
#pragma unroll
    for (int v = 0; v < V; ++v) {
      acc[v] = pfma(rowB[v], accf[v], acc[v]);
      if constexpr (PAIR) rd(out2, bopen, v, pmul(rowA[v], accf[v]));
      accf[v] = f4(0.f);
    }
  };

  // prologue: the first D index stages, then (once they have landed) the
  // first D row stages with index stages D .. 2D-1, one commit group each
#pragma unroll 1
  for (uint32_t m = 0; m < (uint32_t)D; ++m) issue_idx(m);
  cpa_commit();
  cpa_wait<0>();
  __syncwarp();
#pragma unroll 1
  for (uint32_t m = 0; m < (uint32_t)D; ++m) {
    if (m < nsteps) issue_rows(m, m);
    issue_idx(m + D);
    cpa_commit();
  }

  uint32_t is = 0, rs = 0;  // index and row slots of step n
  uint32_t xg = x0;
#pragma unroll 1
  for (uint32_t n = 0; n < nsteps; ++n) {
    // the commit group of step n - D (rows of step n, indices of step n + D)
    cpa_wait<D - 1>();
    __syncwarp();
    uint32_t B[GS];
    float Wv[GS];
    Piece lv[GS][V];
#pragma unroll
    for (uint32_t c = 0; c < NV; ++c) {
      const uint4 b4 = ivec(is, 1, c), w4 = ivec(is, 2, c);
      B[4 * c] = b4.x; B[4 * c + 1] = b4.y; B[4 * c + 2] = b4.z; B[4 * c + 3] = b4.w;
      Wv[4 * c] = __uint_as_float(w4.x); Wv[4 * c + 1] = __uint_as_float(w4.y);
      Wv[4 * c + 2] = __uint_as_float(w4.z); Wv[4 * c + 3] = __uint_as_float(w4.w);
    }
#pragma unroll
    for (uint32_t j = 0; j < GS; ++j)
#pragma unroll
      for (int v = 0; v < V; ++v) lv[j][v] = *reinterpret_cast<const Piece*>(piece_at(rs, 0, j, v));
    auto mid_row = [&](uint32_t j) {
#pragma unroll
      for (int v = 0; v < V; ++v) rowB[v] = widen(*reinterpret_cast<const Piece*>(piece_at(rs, 1, j, v)));
    };
    if (xg + GS <= x1 && xg + GS <= nxt && bopen != NONE) {
      // the common case: a fiber is open (so bopen == blast) and the whole
      // step lies in the open slice and the range
#pragma unroll
      for (uint32_t j = 0; j < GS; ++j) {
        if (B[j] != blast) {
          close_fiber();
          mid_row(j);
          blast = bopen = B[j];
        }
#pragma unroll
        for (int v = 0; v < V; ++v) accf[v] = pfma_s(Wv[j], widen(lv[j][v]), accf[v]);
      }
    } else {
#pragma unroll
      for (uint32_t j = 0; j < GS; ++j) {
        const uint32_t x = xg + j;
        if (x < x1) {
          if (x >= nxt) {  // the slice ends before nonzero x
            if (bopen != NONE) close_fiber();
#pragma unroll
            for (int v = 0; v < V; ++v) { rd(out, ca, v, acc[v]); acc[v] = f4(0.f); }
            do {
              ++sl;
              nxt = __ldg(snz + sl + 1);
            } while (x >= nxt);
            ca = __ldg(sidx + sl);
            if constexpr (PAIR) {
#pragma unroll
              for (int v = 0; v < V; ++v) rowA[v] = load_piece<T, G, V>(U0 + (uint64_t)ca * R, tl, v);
            }
            bopen = NONE;
          }
          const uint32_t b = B[j];
          if (b != bopen) {  // the open fiber ends before nonzero x
            if (bopen != NONE) close_fiber();
            bopen = b;
          }
          if (b != blast) {  // its middle row was staged with this nonzero
            mid_row(j);
            blast = b;
          }
#pragma unroll
          for (int v = 0; v < V; ++v) accf[v] = pfma_s(Wv[j], widen(lv[j][v]), accf[v]);
        }
      }
    }
    __syncwarp();  // every lane is done with index stage `is` before it is refilled
    const uint32_t is2 = is + D < DI ? is + D : is + D - DI;
    if (n + D < nsteps) issue_rows(is2, rs);
    issue_idx(is);
    cpa_commit();
    is = is + 1 == DI ? 0 : is + 1;
    rs = rs + 1 == (uint32_t)D ? 0 : rs + 1;
    xg += GS;
  }
  cpa_wait<0>();  // nothing of this warp's ring is left in flight at exit
  if (x0 < x1) {
    if (bopen != NONE) close_fiber();
#pragma unroll
    for (int v = 0; v < V; ++v) rd(out, ca, v, acc[v]);
  }
}

// Kernel 7's launch. Occupancy level -> (nonzeros per team and step, stages):
// 1: (4, 2), 2: (4, 3), 3: (8, 2), 4: (8, 3); warps per block as many as the
// rings fit in 227 KB of shared memory (at most 24); one block per SM; every
// team an equal range of nonzeros (a multiple of the step).
template <bool PAIR, int G, int V, class T, int GS, int D>
cudaError_t launch_stg_d(Args<T> a, cudaStream_t s) {
  using SS = StgShape<G, V, T, GS, D>;
  constexpr int wpb = (int)SS::WPB;
  static_assert(wpb >= 1, "rings exceed shared memory");
  const uint64_t per_block = (uint64_t)wpb * SS::NT * GS;  // nonzeros per block at the smallest range
  uint64_t blocks = (a.nnz + per_block - 1) / per_block;
  const uint64_t nsm = (uint64_t)sm_count();
  if (blocks > nsm) blocks = nsm;
  const uint64_t teams = blocks * wpb * SS::NT;
  uint64_t chunk = (a.nnz + teams - 1) / teams;
  chunk = (chunk + GS - 1) / GS * GS;
  if (a.nnz + chunk + 2 * GS >= 0xffffffffull) return cudaErrorInvalidValue;  // 32-bit positions
  a.chunk = (uint32_t)chunk;
  a.cslc = nullptr;
  const size_t smem = (size_t)wpb * SS::WARP_BYTES;
  auto k = k_mttkrp_stg<PAIR, G, V, T, GS, D>;
  // the shared-memory opt-in, once per device (the first launch on a device
  // sets it; later launches, captured ones included, only launch)
  static std::atomic<uint64_t> opted{0};
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  const uint64_t bit = 1ull << (dev & 63);
  if (!(opted.load() & bit)) {
    e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    opted.fetch_or(bit);
  }
  k<<<(unsigned)blocks, wpb * 32, smem, s>>>(a);
  return cudaGetLastError();
}

template <bool PAIR, int G, int V, class T>
cudaError_t launch_stg(const Args<T>& a, int mb, cudaStream_t s) {
  switch (mb) {
    case 1: return launch_stg_d<PAIR, G, V, T, 4, 2>(a, s);
    case 3: return launch_stg_d<PAIR, G, V, T, 8, 2>(a, s);
    case 4: return launch_stg_d<PAIR, G, V, T, 8, 3>(a, s);
    default: return launch_stg_d<PAIR, G, V, T, 4, 3>(a, s);
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

template <bool TWO, int G, int V, class T>
cudaError_t launch_fib(const Args<T>& a, int threads, int mb, cudaStream_t s) {
  const uint64_t teams = (a.nnz + a.chunk - 1) / a.chunk;
  const uint64_t blocks = (teams * G + threads - 1) / threads;
  switch (mb) {
    case 1: k_mttkrp_fib<TWO, G, V, T, 2, 8><<<(unsigned)blocks, threads, 0, s>>>(a); break;
    case 3: k_mttkrp_fib<TWO, G, V, T, 4, 4><<<(unsigned)blocks, threads, 0, s>>>(a); break;
    case 4: k_mttkrp_fib<TWO, G, V, T, 5, 4><<<(unsigned)blocks, threads, 0, s>>>(a); break;
    default: k_mttkrp_fib<TWO, G, V, T, 3, 8><<<(unsigned)blocks, threads, 0, s>>>(a); break;
  }
  return cudaGetLastError();
}

template <int OUT, int G, int V, class T>
cudaError_t launch_flat(const Args<T>& a, int threads, int mb, cudaStream_t s);

template <int OUT, int G, int V, class T>
cudaError_t launch_rowsv(const Args<T>& a, int threads, int mb, cudaStream_t s) {
  const uint64_t teams = (a.nnz + a.chunk - 1) / a.chunk;
  const uint64_t blocks = (teams * G + threads - 1) / threads;
  switch (mb) {
    case 1: k_mttkrp_rowsv<OUT, G, V, T, 2, 8><<<(unsigned)blocks, threads, 0, s>>>(a); break;
    case 3: k_mttkrp_rowsv<OUT, G, V, T, 4, 4><<<(unsigned)blocks, threads, 0, s>>>(a); break;
    case 4: k_mttkrp_rowsv<OUT, G, V, T, 5, 4><<<(unsigned)blocks, threads, 0, s>>>(a); break;
    default: k_mttkrp_rowsv<OUT, G, V, T, 3, 8><<<(unsigned)blocks, threads, 0, s>>>(a); break;
  }
  return cudaGetLastError();
}

template <int G, int V, class T>
cudaError_t launch_pairv(const Args<T>& a, int threads, int mb, cudaStream_t s) {
  const uint64_t teams = (a.nnz + a.chunk - 1) / a.chunk;
  const uint64_t blocks = (teams * G + threads - 1) / threads;
  switch (mb) {
    case 1: k_mttkrp_pairv<G, V, T, 2, 8><<<(unsigned)blocks, threads, 0, s>>>(a); break;
    case 3: k_mttkrp_pairv<G, V, T, 4, 4><<<(unsigned)blocks, threads, 0, s>>>(a); break;
    case 4: k_mttkrp_pairv<G, V, T, 5, 4><<<(unsigned)blocks, threads, 0, s>>>(a); break;
    default: k_mttkrp_pairv<G, V, T, 3, 8><<<(unsigned)blocks, threads, 0, s>>>(a); break;
  }
  return cudaGetLastError();
}

// The vector index loads need chunk % 4 == 0 and 16-byte aligned arrays.
template <class T>
bool vec_ok(const Args<T>& a) {
  auto al = [](const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15u) == 0; };
  return a.chunk % 4 == 0 && al(a.vals) && al(a.leaf) && al(a.mid);
}

// kern 2: the branch-free fiber walk with both outputs; otherwise the
// per-nonzero form

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
// 3 = per-nonzero walk (slice and leaf levels of parts that carry `mid`),
// 4 = per-nonzero walk with the middle row once per fiber (3-D slice level;
// elsewhere as 3), 5 = per-nonzero walk with vector index loads (3-D), 6 = the
// warp-interleaved per-nonzero walk (3-D slice level; elsewhere as 5), 7 = the
// walk with rows staged in shared memory (3-D slice level, R 16..128;
// elsewhere as 6)
template <int ND, int G, int V, class T>
cudaError_t launch_lvl(const Args<T>& a, int lvl, int kern, int threads, int mb, cudaStream_t s) {
  if constexpr (ND == 3 && G >= 4 && V == 1) {
    if (kern == 7 && lvl == 0 && vec_ok(a)) return launch_stg<false, G, V, T>(a, mb, s);
  }
  if (kern == 7) kern = 6;  // the staged walk covers the 3-D slice level at R 16..128; elsewhere kernel 6's rule
  if constexpr (ND == 3) {
    if (kern == 6) {
      if (lvl == 0 && vec_ok(a)) return launch_il<false, G, V, T>(a, threads, mb, s);
      kern = 5;  // the interleaved walk covers the slice level; elsewhere the vector-load walk
    }
  }
  if constexpr (ND == 3 && G >= 4) {
    if (kern == 5 && vec_ok(a)) {
      switch (lvl) {
        case 0: return launch_rowsv<0, G, V, T>(a, threads, mb, s);
        case 1: return launch_rowsv<1, G, V, T>(a, threads, mb, s);
        default: return launch_rowsv<2, G, V, T>(a, threads, mb, s);
      }
    }
  }
  if (kern == 5) kern = 3;  // 4-D, R < 16 or unaligned: the per-nonzero walk with scalar index loads
  if constexpr (ND == 3)
    if (kern == 4 && lvl == 0) return launch_fib<false, G, V, T>(a, threads, mb, s);
  if (kern == 4) kern = 3;  // the per-fiber middle row applies to the 3-D slice level; elsewhere the per-nonzero walk
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

}  // namespace

// Launch for one rank R (a compile-time constant: G lanes per row, V float4
// per lane, R = 4 G V). Each R is instantiated in its own translation unit
// (mttkrp_r<R>.cu) so the kernel variants compile in parallel.
// Lanes per factor row (G) and float4 per lane (V) for rank R: a 16-byte
// (FP32) or 8-byte (BF16) piece per lane, at most 32 lanes. (BF16 teams of
// R / 8 lanes, each reading 8 contiguous values with one 16-byte load, were
// slower at R = 32 and 64: 3.34 against 3.07 ms per all-mode step.)
template <class T, int R>
struct TeamShape {
  static constexpr int G = R >= 128 ? 32 : R / 4;
  static constexpr int V = R / (4 * G);
};

template <class T, int R>
cudaError_t launch_fixed(const Args<T>& a, int nd, int lvl, int kern, int threads, int mb, cudaStream_t s) {
  constexpr int G = TeamShape<T, R>::G;
  constexpr int V = TeamShape<T, R>::V;
  return nd == 3 ? launch_lvl<3, G, V, T>(a, lvl, kern, threads, mb, s)
                 : launch_lvl<4, G, V, T>(a, lvl, kern, threads, mb, s);
}

// The two-output walks (R <= 128). kern 2: the branch-free fiber walk with
// both outputs; 4: the per-nonzero walk with the middle row once per fiber;
// 5: the per-nonzero form with vector index loads; 6: the warp-interleaved
// per-nonzero form; 7: the form with rows staged in shared memory (R >= 16);
// otherwise the per-nonzero form. 4-D runs its own walk.
template <class T, int R>
cudaError_t launch_pair_fixed(const Args<T>& a, int nd, int threads, int mb, int kern, cudaStream_t s) {
  if constexpr (R > 128) {
    return cudaErrorInvalidValue;
  } else {
    constexpr int G = TeamShape<T, R>::G;
    constexpr int V = TeamShape<T, R>::V;
    if (nd == 4) return launch_pair4<G, V, T>(a, threads, mb, s);
    if constexpr (G >= 4 && V == 1)
      if (kern == 7 && vec_ok(a)) return launch_stg<true, G, V, T>(a, mb, s);
    if (kern == 7) kern = 6;
    if (kern == 6 && vec_ok(a)) return launch_il<true, G, V, T>(a, threads, mb, s);
    if (kern == 6) kern = 5;
    if constexpr (G >= 4)
      if (kern == 5 && vec_ok(a)) return launch_pairv<G, V, T>(a, threads, mb, s);
    if (kern == 4) return launch_fib<true, G, V, T>(a, threads, mb, s);
    if (kern == 2) return launch_flat<3, G, V, T>(a, threads, mb, s);
    return launch_pair<G, V, T>(a, threads, mb, s);
  }
}

}  // namespace mmcsf

#define MMCSF_INSTANTIATE_R(RR)                                                                                  \
  namespace mmcsf {                                                                                               \
  template cudaError_t launch_fixed<float, RR>(const Args<float>&, int, int, int, int, int, cudaStream_t);        \
  template cudaError_t launch_fixed<__nv_bfloat16, RR>(const Args<__nv_bfloat16>&, int, int, int, int, int,      \
                                                       cudaStream_t);                                             \
  template cudaError_t launch_pair_fixed<float, RR>(const Args<float>&, int, int, int, int, cudaStream_t);        \
  template cudaError_t launch_pair_fixed<__nv_bfloat16, RR>(const Args<__nv_bfloat16>&, int, int, int, int,      \
                                                            cudaStream_t);                                        \
  }

