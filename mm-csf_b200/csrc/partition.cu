// The MM-CSF partition heuristic on the device.
//
// mm_partition_reuseBased (src/util.h:2167-2516) assigns every nonzero to the
// partition of the mode whose fiber through it is longest, measured against
// per-fiber counters that earlier nonzeros decrement: a nonzero that picks
// partition p takes itself out of the fibers of the modes it did not pick.
// As shipped, the loop then overrides every choice with `mode = 2;` (:2517);
// partition_rule 1 keeps the choice. The loop is sequential by definition (the
// reference runs it under `omp for` on counters shared across threads, which
// makes its result depend on the schedule; one thread visits nonzeros in
// order, and that order is what is reproduced here).
//
// Sequential semantics, parallel evaluation. For nonzero x and mode m let
// t_m(x) be the counter x reads (its (o0, o1) group in mode m's CSF, with the
// reference's lookup quirks), c_m the group's initial size, and
// d_m(x) = #{y < x : t_m(y) = t_m(x) and y decrements mode m}. x's choice is
// a function of c_m(t_m(x)) - d_m(x) over the modes, and d_m(x) depends only
// on choices of earlier nonzeros. So the sequential result is the unique
// fixed point of
//     choice = decide(c - d(choice)),
// and Jacobi iteration from d = 0 reaches it: after k rounds every nonzero
// whose chain of dependencies is at most k long is final. Each round is one
// decision kernel over the nonzeros plus, per mode, a segmented exclusive
// count of decrements in (t_m, x) order (a gather, a scan and a scatter).
// Skewed and uniform tensors settle in 4-6 rounds; the count of changed
// choices is the stopping test, with a bound on the rounds.
#include <algorithm>
#include <climits>
#include <vector>

#include "format.h"
#include "prims.cuh"

namespace mmcsf {
namespace {

constexpr int HEUR_MAX_ROUNDS = 1000;

int bits_for_len(uint64_t d) {
  int b = 0;
  while (b < 64 && (d - 1) >> b) ++b;
  return d <= 1 ? 0 : b;
}

__global__ void k_group_key(const uint32_t* __restrict__ a, const uint32_t* __restrict__ b, int bb, uint64_t n,
                            uint64_t* __restrict__ key, uint32_t* __restrict__ pos) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
    key[i] = ((uint64_t)a[i] << bb) | b[i];
    pos[i] = (uint32_t)i;
  }
}

__global__ void k_head_flags(const uint64_t* __restrict__ key, int shift, uint64_t n, uint32_t* __restrict__ flag) {
  for (uint64_t j = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; j < n; j += (uint64_t)gridDim.x * blockDim.x)
    flag[j] = (j == 0 || (key[j] >> shift) != (key[j - 1] >> shift)) ? 1u : 0u;
}

// group starts (in sorted order) from the head flags and their exclusive scan
__global__ void k_group_starts(const uint32_t* __restrict__ flag, const uint32_t* __restrict__ excl, uint64_t n,
                               uint32_t* __restrict__ gst) {
  for (uint64_t j = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; j < n; j += (uint64_t)gridDim.x * blockDim.x)
    if (flag[j]) gst[excl[j]] = (uint32_t)j;
}

__global__ void k_group_sizes(const uint32_t* __restrict__ gst, uint64_t ng, uint64_t n, uint32_t* __restrict__ cnt) {
  for (uint64_t g = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; g < ng; g += (uint64_t)gridDim.x * blockDim.x)
    cnt[g] = (g + 1 < ng ? gst[g + 1] : (uint32_t)n) - gst[g];
}

// The counter a nonzero reads (src/util.h:2364-2383). denseSlcPtr gives the
// last slice an empty fiber range (:2203-2206), so its binary search finds
// only the slice's first group; any other group of the last slice reads (and
// later decrements) the counter just before the slice's first group.
__global__ void k_targets(const uint64_t* __restrict__ key, const uint32_t* __restrict__ pos,
                          const uint32_t* __restrict__ excl, int bb, uint64_t n, uint64_t last_slice,
                          uint32_t first_last, uint32_t* __restrict__ t) {
  for (uint64_t j = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; j < n; j += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t g = excl[j + 1] - 1;  // group of sorted position j
    const bool quirk = (key[j] >> bb) == last_slice && g != first_last;
    t[pos[j]] = quirk ? first_last - 1 : g;
  }
}

__global__ void k_t_key(const uint32_t* __restrict__ t, uint64_t n, uint64_t* __restrict__ key,
                        uint32_t* __restrict__ pos) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
    key[i] = t[i];
    pos[i] = (uint32_t)i;
  }
}

// hp[j] = sorted position of the first member of j's group (keys sorted by t)
__global__ void k_head_scatter(const uint64_t* __restrict__ key, uint64_t n, uint32_t* __restrict__ hs) {
  for (uint64_t j = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; j < n; j += (uint64_t)gridDim.x * blockDim.x)
    if (j == 0 || key[j] != key[j - 1]) hs[key[j]] = (uint32_t)j;
}
__global__ void k_head_gather(const uint64_t* __restrict__ key, const uint32_t* __restrict__ hs, uint64_t n,
                              uint32_t* __restrict__ hp) {
  for (uint64_t j = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; j < n; j += (uint64_t)gridDim.x * blockDim.x)
    hp[j] = hs[key[j]];
}

struct Decide {
  int nd, fbth, redun, partner, shortest;
  int has[4];            // the mode keeps its own counters
  int tgt[4];            // partition chosen when mode m's test passes
  uint32_t decmask[4];   // modes whose counters a choice of partition s decrements
  const uint32_t* t[4];
  const uint32_t* c0[4];
  const uint32_t* dec[4];
};

// One round of decisions (src/util.h:2386-2491 and the fallback at :2494-2495).
__global__ void k_decide(const Decide d, uint64_t n, uint8_t* __restrict__ part,
                         unsigned long long* __restrict__ changed) {
  unsigned long long local = 0;
  for (uint64_t x = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; x < n; x += (uint64_t)gridDim.x * blockDim.x) {
    uint64_t f[4] = {0, 0, 0, 0};
#pragma unroll
    for (int m = 0; m < 4; ++m)
      if (m < d.nd && d.has[m]) f[m] = (uint64_t)d.c0[m][d.t[m][x]] - (uint64_t)d.dec[m][x];
    if (d.redun >= 0) f[d.redun] = f[d.partner];
    int sel = -1;
    if (d.nd == 3) {
      // ITYPE counters against an int ratio promoted to ITYPE
      const uint64_t th = (uint64_t)(int64_t)d.fbth;
#pragma unroll
      for (int m = 0; m < 3; ++m) {
        const uint64_t a = f[m == 0 ? 1 : 0], b = f[m == 2 ? 1 : 2];
        if (sel < 0 && f[m] >= th * (a > b ? a : b)) sel = d.tgt[m];
      }
    } else {
      // maxOf3 takes ints (src/util.h:2142-2146): counters truncated to int,
      // their maximum times the int ratio, compared back as ITYPE
      int v[4];
#pragma unroll
      for (int m = 0; m < 4; ++m) v[m] = (int)(uint32_t)f[m];
#pragma unroll
      for (int m = 0; m < 4; ++m) {
        int mx = INT_MIN;
#pragma unroll
        for (int q = 0; q < 4; ++q)
          if (q != m) mx = v[q] > mx ? v[q] : mx;
        const int prod = (int)((uint32_t)d.fbth * (uint32_t)mx);
        if (sel < 0 && f[m] >= (uint64_t)(int64_t)prod) sel = d.tgt[m];
      }
    }
    if (sel < 0) sel = d.shortest;
    if (part[x] != (uint8_t)sel) {
      part[x] = (uint8_t)sel;
      ++local;
    }
  }
  // one atomic per warp
  for (int o = 16; o > 0; o >>= 1) local += __shfl_down_sync(0xffffffffu, local, o);
  if ((threadIdx.x & 31) == 0 && local) atomicAdd(changed, local);
}

__global__ void k_dec_flags(const uint32_t* __restrict__ P, const uint8_t* __restrict__ part, uint32_t mask_bit,
                            const uint32_t* __restrict__ decmask, uint64_t n, uint32_t* __restrict__ flag) {
  for (uint64_t j = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; j < n; j += (uint64_t)gridDim.x * blockDim.x)
    flag[j] = (decmask[part[P[j]]] >> mask_bit) & 1u;
}

__global__ void k_dec_counts(const uint32_t* __restrict__ P, const uint32_t* __restrict__ hp,
                             const uint32_t* __restrict__ pre, uint64_t n, uint32_t* __restrict__ dec) {
  for (uint64_t j = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; j < n; j += (uint64_t)gridDim.x * blockDim.x)
    dec[P[j]] = pre[j] - pre[hp[j]];
}

__global__ void k_fill_u8(uint8_t* p, uint64_t n, uint8_t v) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
    p[i] = v;
}

__global__ void k_find_first_last(const uint64_t* __restrict__ key, const uint32_t* __restrict__ excl, int bb,
                                  uint64_t n, uint64_t last_slice, uint32_t* __restrict__ out) {
  for (uint64_t j = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; j < n; j += (uint64_t)gridDim.x * blockDim.x)
    if ((key[j] >> bb) == last_slice && (j == 0 || (key[j - 1] >> bb) != last_slice)) *out = excl[j + 1] - 1;
}

__global__ void k_member_flags(const uint8_t* __restrict__ part, uint8_t p, uint64_t n, uint32_t* __restrict__ flag) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
    flag[i] = part[i] == p ? 1u : 0u;
}

__global__ void k_member_gather(const uint32_t* __restrict__ flag, const uint32_t* __restrict__ excl,
                                const uint32_t* __restrict__ perm, uint64_t n, uint32_t* __restrict__ out) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
    if (flag[i]) out[excl[i]] = perm[i];
}

}  // namespace

// populate_paritions (src/util.h:2088-2126): the COO indices (perm[i] for
// position i) of the positions whose partition is p, in position order.
int partition_members(const uint8_t* part, int p, const uint32_t* perm, uint64_t n, DevBuf& out, uint64_t* count,
                      int* launches, cudaStream_t s) {
  *count = 0;
  if (n == 0) return MMCSF_OK;
  DevBuf flag, excl;
  MMCSF_CUDA(flag.alloc(n * 4));
  MMCSF_CUDA(excl.alloc((n + 1) * 4));
  const int th = 256, gr = grid_for(n, th);
  k_member_flags<<<gr, th, 0, s>>>(part, (uint8_t)p, n, flag.as<uint32_t>());
  MMCSF_LAUNCH_CHECK();
  MMCSF_CUDA(exclusive_scan_u32(flag.as<uint32_t>(), excl.as<uint32_t>(), n, s));
  uint32_t c = 0;
  MMCSF_CUDA(cudaMemcpyAsync(&c, excl.as<uint32_t>() + n, 4, cudaMemcpyDeviceToHost, s));
  MMCSF_CUDA(cudaStreamSynchronize(s));
  *count = c;
  MMCSF_CUDA(out.alloc((uint64_t)std::max<uint32_t>(c, 1) * 4));
  k_member_gather<<<gr, th, 0, s>>>(flag.as<uint32_t>(), excl.as<uint32_t>(), perm, n, out.as<uint32_t>());
  MMCSF_LAUNCH_CHECK();
  *launches += 4;
  MMCSF_CUDA(cudaStreamSynchronize(s));
  return MMCSF_OK;
}

// sx: X's index arrays in the order the partition loop visits them (after
// the chain of per-mode sorts). orders[m]: arrX[m]'s mode order. Writes the
// chosen partition of every position into part (n bytes) and the number of
// rounds into *rounds.
int mm_partition_heuristic(int nd, const uint64_t* dims, const int (*orders)[4], const int* xorder, int redun,
                           int fbth, const uint32_t* const* sx, uint64_t n, uint8_t* part, int* rounds,
                           int* launches, cudaStream_t s) {
  *rounds = 0;
  if (n == 0) return MMCSF_OK;
  // same-fiber pairs, shortMode / longMode (src/util.h:2263-2308): mode m's
  // (slice, fiber) pair repeating an earlier mode's pair swapped
  auto same = [&](int a, int b) { return orders[a][1] == orders[b][0] && orders[a][0] == orders[b][1]; };
  bool s01 = false, s02 = false, s12 = false, s03 = false, s13 = false, s23 = false;
  int shortMode = 0, longMode = -1;
  auto setpair = [&](int a, int b) {
    shortMode = dims[a] <= dims[b] ? a : b;
    longMode = dims[a] <= dims[b] ? b : a;
  };
  if (nd > 1 && same(1, 0)) { s01 = true; setpair(0, 1); }
  if (nd > 2) {
    if (same(2, 0)) { s02 = true; setpair(0, 2); }
    else if (same(2, 1)) { s12 = true; setpair(1, 2); }
  }
  if (nd > 3) {
    if (same(3, 0)) { s03 = true; setpair(0, 3); }
    else if (same(3, 1)) { s13 = true; setpair(1, 3); }
    else if (same(3, 2)) { s23 = true; setpair(2, 3); }
  }
  // the counters of the redundant mode are copied from its pair partner
  // (:2343-2357); it never has counters of its own
  int partner = -1;
  if (redun >= 0) {
    if ((redun == 1 && s01) || (redun == 2 && s12) || (redun == 3 && s23)) partner = redun - 1;
    else if ((redun == 2 && s02) || (redun == 3 && s13)) partner = redun - 2;
    else if (redun == 3 && s03) partner = 0;
    if (partner < 0) return set_error(MMCSF_ERR_UNSUPPORTED, "partition heuristic: no pair for redundant mode %d", redun);
  }
  Decide d{};
  d.nd = nd;
  d.fbth = fbth;
  d.redun = redun;
  d.partner = partner;
  d.shortest = dims[xorder[0]] <= dims[xorder[1]] ? xorder[0] : xorder[1];  // :2261
  d.tgt[0] = (s01 || s02 || s03) ? shortMode : 0;
  d.tgt[1] = (s12 || s13) ? shortMode : 1;
  d.tgt[2] = s23 ? shortMode : 2;
  d.tgt[3] = 3;
  uint32_t decmask[4] = {0, 0, 0, 0};
  for (int sel = 0; sel < nd; ++sel)  // :2500-2513
    for (int i = 0; i < nd; ++i) {
      const bool dec = sel == shortMode ? (i != shortMode && i != longMode) : (i != redun && i != sel);
      if (dec) decmask[sel] |= 1u << i;
    }
  for (int sel = 0; sel < nd; ++sel)
    if (redun >= 0 && (decmask[sel] >> redun) & 1u)
      return set_error(MMCSF_ERR_UNSUPPORTED, "partition heuristic: the redundant mode has no counters");
  for (int i = 0; i < 4; ++i) d.decmask[i] = decmask[i];
  DevBuf dmask;
  MMCSF_CUDA(dmask.alloc(sizeof decmask));
  MMCSF_CUDA(cudaMemcpyAsync(dmask.p, decmask, sizeof decmask, cudaMemcpyHostToDevice, s));

  // per counted mode: targets, initial counts, (t, x) order and group heads
  DevBuf t[4], c0[4], P[4], hp[4], dec[4];
  const int th = 256, gr = grid_for(n, th);
  for (int m = 0; m < nd; ++m) {
    if (m == redun) continue;
    d.has[m] = 1;
    const int o0 = orders[m][0], o1 = orders[m][1];
    const int bb = bits_for_len(dims[o1]);
    const int kb = bb + bits_for_len(dims[o0]);
    DevBuf key, key2, pos, pos2, flag, excl;
    MMCSF_CUDA(key.alloc(n * 8));
    MMCSF_CUDA(key2.alloc(n * 8));
    MMCSF_CUDA(pos.alloc(n * 4));
    MMCSF_CUDA(pos2.alloc(n * 4));
    k_group_key<<<gr, th, 0, s>>>(sx[o0], sx[o1], bb, n, key.as<uint64_t>(), pos.as<uint32_t>());
    MMCSF_LAUNCH_CHECK();
    ++*launches;
    if (kb > 0) {
      MMCSF_CUDA(radix_sort_pairs(key.as<uint64_t>(), pos.as<uint32_t>(), key2.as<uint64_t>(), pos2.as<uint32_t>(), n,
                                  kb, s));
      *launches += 4 * ((kb + 7) / 8);
    }
    MMCSF_CUDA(flag.alloc(n * 4));
    MMCSF_CUDA(excl.alloc((n + 1) * 4));
    k_head_flags<<<gr, th, 0, s>>>(key.as<uint64_t>(), 0, n, flag.as<uint32_t>());
    MMCSF_LAUNCH_CHECK();
    MMCSF_CUDA(exclusive_scan_u32(flag.as<uint32_t>(), excl.as<uint32_t>(), n, s));
    *launches += 2;
    uint32_t ng = 0;
    MMCSF_CUDA(cudaMemcpyAsync(&ng, excl.as<uint32_t>() + n, 4, cudaMemcpyDeviceToHost, s));
    uint64_t last_key = 0;
    MMCSF_CUDA(cudaMemcpyAsync(&last_key, key.as<uint64_t>() + n - 1, 8, cudaMemcpyDeviceToHost, s));
    MMCSF_CUDA(cudaStreamSynchronize(s));
    const uint64_t last_slice = last_key >> bb;
    DevBuf gst, fl;
    MMCSF_CUDA(gst.alloc((uint64_t)ng * 4));
    MMCSF_CUDA(c0[m].alloc((uint64_t)ng * 4));
    MMCSF_CUDA(fl.alloc(4));
    k_group_starts<<<gr, th, 0, s>>>(flag.as<uint32_t>(), excl.as<uint32_t>(), n, gst.as<uint32_t>());
    MMCSF_LAUNCH_CHECK();
    k_group_sizes<<<grid_for(ng, th), th, 0, s>>>(gst.as<uint32_t>(), ng, n, c0[m].as<uint32_t>());
    MMCSF_LAUNCH_CHECK();
    k_find_first_last<<<gr, th, 0, s>>>(key.as<uint64_t>(), excl.as<uint32_t>(), bb, n, last_slice,
                                        fl.as<uint32_t>());
    MMCSF_LAUNCH_CHECK();
    *launches += 3;
    uint32_t first_last = 0;
    MMCSF_CUDA(cudaMemcpyAsync(&first_last, fl.p, 4, cudaMemcpyDeviceToHost, s));
    MMCSF_CUDA(cudaStreamSynchronize(s));
    if (first_last == 0 && ng > 1)  // one slice holding several groups: the reference reads before its arrays
      return set_error(MMCSF_ERR_UNSUPPORTED,
                       "partition heuristic: mode %d has a single slice with several fibers, where the reference "
                       "reads out of bounds", m);
    MMCSF_CUDA(t[m].alloc(n * 4));
    k_targets<<<gr, th, 0, s>>>(key.as<uint64_t>(), pos.as<uint32_t>(), excl.as<uint32_t>(), bb, n, last_slice,
                                first_last, t[m].as<uint32_t>());
    MMCSF_LAUNCH_CHECK();
    // (t, x) order: a stable sort of the positions by target
    k_t_key<<<gr, th, 0, s>>>(t[m].as<uint32_t>(), n, key.as<uint64_t>(), pos.as<uint32_t>());
    MMCSF_LAUNCH_CHECK();
    *launches += 2;
    const int tb = std::max(1, bits_for_len(ng));
    MMCSF_CUDA(radix_sort_pairs(key.as<uint64_t>(), pos.as<uint32_t>(), key2.as<uint64_t>(), pos2.as<uint32_t>(), n,
                                tb, s));
    *launches += 4 * ((tb + 7) / 8);
    DevBuf hs;
    MMCSF_CUDA(hs.alloc((uint64_t)std::max<uint32_t>(ng, 1) * 4));
    MMCSF_CUDA(hp[m].alloc(n * 4));
    k_head_scatter<<<gr, th, 0, s>>>(key.as<uint64_t>(), n, hs.as<uint32_t>());
    MMCSF_LAUNCH_CHECK();
    k_head_gather<<<gr, th, 0, s>>>(key.as<uint64_t>(), hs.as<uint32_t>(), n, hp[m].as<uint32_t>());
    MMCSF_LAUNCH_CHECK();
    *launches += 2;
    P[m] = std::move(pos);
    MMCSF_CUDA(dec[m].alloc(n * 4));
    MMCSF_CUDA(cudaMemsetAsync(dec[m].p, 0, n * 4, s));
    MMCSF_CUDA(cudaStreamSynchronize(s));  // the scratch above is freed on return from this scope
    d.t[m] = t[m].as<uint32_t>();
    d.c0[m] = c0[m].as<uint32_t>();
    d.dec[m] = dec[m].as<uint32_t>();
  }

  DevBuf flag, pre, changed;
  MMCSF_CUDA(flag.alloc(n * 4));
  MMCSF_CUDA(pre.alloc((n + 1) * 4));
  MMCSF_CUDA(changed.alloc(8));
  k_fill_u8<<<gr, th, 0, s>>>(part, n, 0xff);
  MMCSF_LAUNCH_CHECK();
  ++*launches;
  for (int round = 0; round < HEUR_MAX_ROUNDS; ++round) {
    MMCSF_CUDA(cudaMemsetAsync(changed.p, 0, 8, s));
    k_decide<<<gr, th, 0, s>>>(d, n, part, changed.as<unsigned long long>());
    MMCSF_LAUNCH_CHECK();
    ++*launches;
    unsigned long long nchg = 0;
    MMCSF_CUDA(cudaMemcpyAsync(&nchg, changed.p, 8, cudaMemcpyDeviceToHost, s));
    MMCSF_CUDA(cudaStreamSynchronize(s));
    *rounds = round + 1;
    if (nchg == 0) return MMCSF_OK;
    for (int m = 0; m < nd; ++m) {
      if (!d.has[m]) continue;
      k_dec_flags<<<gr, th, 0, s>>>(P[m].as<uint32_t>(), part, (uint32_t)m, dmask.as<uint32_t>(), n,
                                    flag.as<uint32_t>());
      MMCSF_LAUNCH_CHECK();
      MMCSF_CUDA(exclusive_scan_u32(flag.as<uint32_t>(), pre.as<uint32_t>(), n, s));
      k_dec_counts<<<gr, th, 0, s>>>(P[m].as<uint32_t>(), hp[m].as<uint32_t>(), pre.as<uint32_t>(), n,
                                     dec[m].as<uint32_t>());
      MMCSF_LAUNCH_CHECK();
      *launches += 4;
    }
  }
  return set_error(MMCSF_ERR_UNSUPPORTED, "partition heuristic did not settle in %d rounds", HEUR_MAX_ROUNDS);
}

}  // namespace mmcsf
