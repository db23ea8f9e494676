// Format construction on the device.
//
// The reference builds every format on the host (src/util.h:255-2526) with a
// chain of unstable sample sorts, pointer-chasing scans and push_backs. Here
// the same arrays come out of:
//   1. host planning that replays the reference's decisions (mode orders,
//      redundant mode, which sorts run in which order, partition rule);
//   2. ONE stable LSD radix sort on a composite key: a chain of stable sorts
//      equals a single stable sort keyed by the last sort's keys, then the
//      previous sort's, and so on (keys already present are dropped), with
//      ties left in file order;
//   3. boundary flags + exclusive scans + compactions for every CSF level,
//      fiber splitting at the -f threshold by position-in-run arithmetic, and
//      the 4-D fbrS split at 128 nonzeros by a warp-per-run greedy scan.
#include <algorithm>
#include <memory>
#include <cstring>
#include <vector>

#include "format.h"
#include "prims.cuh"

using mmcsf::set_error;

namespace mmcsf {
namespace {

constexpr uint64_t REF_DEFAULT_FBR_TH = 99999999ull;  // src/util.h:212
constexpr uint64_t FBRS_TH_MMCSF = 128;               // src/util.h:1325-1326
constexpr uint64_t FBRS_TH_OFF = 999999999ull;

struct Idx4 {
  const uint32_t* p[4];
};

// ---- kernels --------------------------------------------------------------

__global__ void k_pack(Idx4 in, const uint32_t* __restrict__ perm, int nk, Idx4 dummy, uint64_t n,
                       int4 modes, int4 shifts, uint64_t* __restrict__ keys) {
  (void)dummy;
  const int md[4] = {modes.x, modes.y, modes.z, modes.w};
  const int sh[4] = {shifts.x, shifts.y, shifts.z, shifts.w};
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
    uint32_t src = perm ? perm[i] : (uint32_t)i;
    uint64_t k = 0;
    for (int j = 0; j < nk; ++j) k |= (uint64_t)in.p[md[j]][src] << sh[j];
    keys[i] = k;
  }
}

// flag[x] = 1 where any of the first L level keys changes (x == 0 included)
__global__ void k_run_flags(Idx4 lev, int L, uint64_t n, uint32_t* __restrict__ flag) {
  for (uint64_t x = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; x < n; x += (uint64_t)gridDim.x * blockDim.x) {
    uint32_t f = (x == 0);
    if (!f)
      for (int l = 0; l < L; ++l) f |= (lev.p[l][x] != lev.p[l][x - 1]);
    flag[x] = f;
  }
}

// out[excl[i]] = i where flag[i]
__global__ void k_compact_pos(const uint32_t* __restrict__ flag, const uint32_t* __restrict__ excl, uint64_t n,
                              uint32_t* __restrict__ out) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
    if (flag[i]) out[excl[i]] = (uint32_t)i;
}

// new fiber at every th-th nonzero of a run (greedy chunks of th, src/util.h:1366-1374)
__global__ void k_split_flags(const uint32_t* __restrict__ excl_run, const uint32_t* __restrict__ run_start,
                              uint64_t n, uint64_t th, uint32_t* __restrict__ flag) {
  for (uint64_t x = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; x < n; x += (uint64_t)gridDim.x * blockDim.x) {
    uint32_t run = excl_run[x + 1] - 1;
    uint64_t pos = x - run_start[run];
    flag[x] = (pos % th) == 0;
  }
}

// flag[i] = 1 where a level key differs between nonzero starts[i] and starts[i]-1
__global__ void k_flags_at(Idx4 lev, int L, const uint32_t* __restrict__ starts, uint64_t n,
                           uint32_t* __restrict__ flag) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
    uint32_t x = starts[i];
    uint32_t f = (x == 0);
    if (!f)
      for (int l = 0; l < L; ++l) f |= (lev.p[l][x] != lev.p[l][x - 1]);
    flag[i] = f;
  }
}

// out[i] = a[b[i]] (double indirection helper when a needs an index from b)
__global__ void k_gather2(const uint32_t* __restrict__ a, const uint32_t* __restrict__ b,
                          const uint32_t* __restrict__ c, uint64_t n, uint32_t* __restrict__ out) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
    out[i] = a[b[c ? c[i] : i]];
}

__global__ void k_gather_f32(const float* __restrict__ in, const uint32_t* __restrict__ perm, uint64_t n,
                             float* __restrict__ out) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
    out[i] = in[perm[i]];
}

__global__ void k_set1(uint32_t* p, uint64_t i, uint32_t v) { p[i] = v; }

// parent id of every child: out[c] = (inclusive scan of flag)[c] - 1
__global__ void k_parent(const uint32_t* __restrict__ excl, uint64_t n, uint32_t* __restrict__ out) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
    out[i] = excl[i + 1] - 1;
}

// 4-D fbrS split (src/util.h:1388-1405): inside each (o0,o1) run of fibers a
// new fbrS starts at fiber g when fptr[g] > fptr[s] + th - off, s being the
// current fbrS's first fiber and off = 0 only for the fbrS that starts at
// nonzero 0 (the reference's counter starts one lower there). One warp per run.
__global__ void k_fbrs_split(const uint32_t* __restrict__ fptr, const uint32_t* __restrict__ run_first,
                             uint64_t nruns, uint64_t nfib, uint64_t th, uint32_t* __restrict__ fsflag) {
  const int lane = threadIdx.x & 31;
  const uint64_t warps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
  for (uint64_t r = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5; r < nruns; r += warps) {
    const uint64_t g0 = run_first[r], g1 = (r + 1 < nruns) ? run_first[r + 1] : nfib;
    uint64_t s = g0;
    uint64_t off = (fptr[g0] == 0) ? 0 : 1;
    for (;;) {
      const uint64_t limit = (uint64_t)fptr[s] + th - off;
      uint64_t found = g1;
      for (uint64_t base = s + 1; base < g1; base += 32) {
        uint64_t g = base + lane;
        bool pred = g < g1 && (uint64_t)fptr[g] > limit;
        unsigned b = __ballot_sync(0xffffffffu, pred);
        if (b) { found = base + (__ffs(b) - 1); break; }
      }
      if (found >= g1) break;
      if (lane == 0) fsflag[found] = 1;
      s = found;
      off = 1;
    }
  }
}

// bins of make_TiledBin (src/util.h:1887-1952) / make_HybBin (:1786-1885):
// count = (with_children ? #children : 0) + #nonzeros of the slice
__global__ void k_bins(const uint32_t* __restrict__ sptr, const uint32_t* __restrict__ nnz_start_of_child,
                       uint64_t nslc, uint64_t tot, int with_children, int32_t* __restrict__ bin_of) {
  const uint64_t TB = 512;
  for (uint64_t s = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; s < nslc; s += (uint64_t)gridDim.x * blockDim.x) {
    uint64_t c0 = sptr[s], c1 = sptr[s + 1];
    uint64_t n = (uint64_t)(nnz_start_of_child[c1] - nnz_start_of_child[c0]);
    if (with_children) n += c1 - c0;
    const uint64_t LB[10] = {0, 2, 4, 8, 16, 1024, 4 * TB, 8 * TB, 16 * TB, 32 * TB};
    const uint64_t UB[10] = {1025, 5, 9, 17, 1025, 4 * TB + 1, 8 * TB + 1, 16 * TB + 1, 32 * TB + 1, tot + 1};
    int b = -1;
    for (int i = 0; i < 10; ++i)
      if (n > LB[i] && n < UB[i]) { b = i; break; }
    bin_of[s] = b;
  }
}

// inv[perm[i]] = i
__global__ void k_invert(const uint32_t* __restrict__ perm, uint64_t n, uint32_t* __restrict__ inv) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
    inv[perm[i]] = (uint32_t)i;
}

// bit 31 of the leaf index marks the first nonzero of every leaf fiber
__global__ void k_flag_fibers(uint32_t* __restrict__ leaf, const uint32_t* __restrict__ fptr, uint64_t nfib) {
  for (uint64_t f = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; f < nfib; f += (uint64_t)gridDim.x * blockDim.x)
    leaf[fptr[f]] |= 0x80000000u;
}

// ---- host helpers ----------------------------------------------------------

int bits_for(uint64_t dim) {
  int b = 0;
  while (b < 64 && ((dim - 1) >> b)) ++b;
  return b;
}

struct Launches {
  int n = 0;
};

#define LCHECK(L) \
  do { ++(L).n; MMCSF_LAUNCH_CHECK(); } while (0)

// Excl scan with a fresh output buffer of n+1 entries; returns total via *tot.
int scan_total(const uint32_t* flag, uint64_t n, DevBuf& excl, uint32_t* tot, cudaStream_t s, Launches& L) {
  MMCSF_CUDA(excl.alloc((n + 1) * 4));
  MMCSF_CUDA(exclusive_scan_u32(flag, excl.as<uint32_t>(), n, s));
  L.n += 3;
  MMCSF_CUDA(cudaMemcpyAsync(tot, excl.as<uint32_t>() + n, 4, cudaMemcpyDeviceToHost, s));
  MMCSF_CUDA(cudaStreamSynchronize(s));
  return MMCSF_OK;
}

}  // namespace

// Reference mode ordering, src/util.h:255-311.
void order_modes(int nd, const uint64_t* dims, int mode, int* order) {
  uint64_t len[4];
  int taken[4] = {0, 0, 0, 0};
  for (int m = 0; m < nd; ++m) len[m] = dims[(m + mode) % nd];
  for (int i = 1; i < nd; i++)
    for (int j = i + 1; j < nd; j++)
      if (len[i] > len[j]) std::swap(len[i], len[j]);
  order[0] = mode;
  taken[mode] = 1;
  for (int i = 1; i < nd; i++)
    for (int j = 0; j < nd; j++)
      if (len[i] == dims[j] && !taken[j]) { order[i] = j; taken[j] = 1; break; }
}

// The composite sort key (most significant mode first) that reproduces the
// reference's chain of sorts for a format (the same plan mmcsf_build uses);
// returns the number of modes written to keys.
int sort_key_plan(int impl, int nd, const uint64_t* dims, int mode, int* keys) {
  const int K = nd == 3 ? 2 : 3;
  int xo[4];
  order_modes(nd, dims, mode, xo);
  std::vector<std::vector<int>> chain;
  chain.push_back(std::vector<int>(xo, xo + K));
  if (impl == MMCSF_IMPL_MMCSF) {
    int orders[4][4];
    int redun = -1;
    for (int m = 0; m < nd; ++m) {
      order_modes(nd, dims, m, orders[m]);
      for (int p = 0; p < m; ++p)
        if (orders[m][1] == orders[p][0] && orders[m][0] == orders[p][1]) redun = m;
      if (m != redun) chain.push_back(std::vector<int>(orders[m], orders[m] + K));
    }
    chain.push_back(std::vector<int>(orders[2], orders[2] + K));
  }
  int n = 0;
  for (int c = (int)chain.size() - 1; c >= 0; --c)
    for (int m : chain[c]) {
      bool seen = false;
      for (int i = 0; i < n; ++i) seen = seen || keys[i] == m;
      if (!seen) keys[n++] = m;
    }
  return n;
}

// Stable sort of the COO by the composite mode list `keys` (most significant
// first). Produces sorted copies of every mode's indices and the values.
// Stable sort of the nonzeros (or of the subset `subset[0..n_sub)` of COO
// indices, ties kept in subset order) by `keys`, most significant first.
static int sort_coo(const mmcsf_coo* X, const std::vector<int>& keys, DevBuf* sorted_inds, DevBuf& sorted_vals,
                    cudaStream_t s, Launches& L, DevBuf* perm_out = nullptr, const DevBuf* subset = nullptr,
                    uint64_t n_sub = 0) {
  const uint64_t n = subset ? n_sub : X->nnz;
  const int nd = X->nd;
  DevBuf perm, perm2, k1, k2;
  MMCSF_CUDA(perm.alloc(std::max<uint64_t>(n, 1) * 4));
  if (subset) {
    if (n) MMCSF_CUDA(cudaMemcpyAsync(perm.p, subset->p, n * 4, cudaMemcpyDeviceToDevice, s));
  } else {
    MMCSF_CUDA(iota_u32(perm.as<uint32_t>(), n, s));
    ++L.n;
  }
  if (n > 1 && !keys.empty()) {
    MMCSF_CUDA(perm2.alloc(n * 4));
    MMCSF_CUDA(k1.alloc(n * 8));
    MMCSF_CUDA(k2.alloc(n * 8));
    // split into <=64-bit groups from the least significant end
    std::vector<std::vector<int>> groups;
    std::vector<int> cur;
    int bits = 0;
    for (int i = (int)keys.size() - 1; i >= 0; --i) {
      int b = bits_for(X->dims[keys[i]]);
      if (bits + b > 64 || cur.size() == 4) {
        groups.push_back(cur);
        cur.clear();
        bits = 0;
      }
      cur.insert(cur.begin(), keys[i]);
      bits += b;
    }
    if (!cur.empty()) groups.push_back(cur);
    Idx4 in{};
    for (int m = 0; m < nd; ++m) in.p[m] = X->d_inds[m].as<uint32_t>();
    bool first = subset == nullptr;  // keys come through perm once it is not the identity
    for (auto& g : groups) {  // least significant group first
      int md[4] = {0, 0, 0, 0}, sh[4] = {0, 0, 0, 0};
      int tot = 0;
      for (int j = (int)g.size() - 1; j >= 0; --j) {
        md[j] = g[j];
        sh[j] = tot;
        tot += bits_for(X->dims[g[j]]);
      }
      if (tot == 0) continue;
      k_pack<<<grid_for(n, 256), 256, 0, s>>>(in, first ? nullptr : perm.as<uint32_t>(), (int)g.size(), in, n,
                                              make_int4(md[0], md[1], md[2], md[3]),
                                              make_int4(sh[0], sh[1], sh[2], sh[3]), k1.as<uint64_t>());
      LCHECK(L);
      MMCSF_CUDA(radix_sort_pairs(k1.as<uint64_t>(), perm.as<uint32_t>(), k2.as<uint64_t>(), perm2.as<uint32_t>(),
                                  n, tot, s));
      L.n += 4 * ((tot + 7) / 8);
      first = false;
    }
  }
  for (int m = 0; m < nd; ++m) {
    MMCSF_CUDA(sorted_inds[m].alloc(n * 4));
    MMCSF_CUDA(gather_u32(X->d_inds[m].as<uint32_t>(), perm.as<uint32_t>(), sorted_inds[m].as<uint32_t>(), n, s));
    ++L.n;
  }
  MMCSF_CUDA(sorted_vals.alloc(n * 4));
  if (n) {
    k_gather_f32<<<grid_for(n, 256), 256, 0, s>>>(X->d_vals.as<float>(), perm.as<uint32_t>(), n,
                                                  sorted_vals.as<float>());
    LCHECK(L);
  }
  if (perm_out) *perm_out = std::move(perm);  // COO index of every sorted position
  return MMCSF_OK;
}

// CSF levels over sorted arrays (src/util.h:1320-1436 create_TiledHCSR; with
// fbrs_th = "off" it is src/util.h:760-850 create_HCSR).
static int build_csf(int nd, const int* order, uint64_t n, DevBuf* sorted, DevBuf& vals, uint64_t fbr_th,
                     uint64_t fbrs_th, bool keep_coo, CsfPart& P, cudaStream_t s, Launches& L) {
  P.present = n > 0;
  P.nd = nd;
  for (int i = 0; i < nd; ++i) P.order[i] = order[i];
  P.nnz = n;
  const int Lv = nd - 1;  // index levels
  const uint32_t* o[4];
  for (int i = 0; i < nd; ++i) o[i] = sorted[order[i]].as<uint32_t>();
  if (n == 0) return MMCSF_OK;
  const int G = grid_for(n, 256);

  // --- leaf fibers: runs of equal (o0..o_{L-1}), split every fbr_th nonzeros
  DevBuf fl, exr;
  MMCSF_CUDA(fl.alloc(n * 4));
  Idx4 lev{};
  for (int i = 0; i < Lv; ++i) lev.p[i] = o[i];
  k_run_flags<<<G, 256, 0, s>>>(lev, Lv, n, fl.as<uint32_t>());
  LCHECK(L);
  if (fbr_th < n) {
    uint32_t nrun = 0;
    MMCSF_TRY(scan_total(fl.as<uint32_t>(), n, exr, &nrun, s, L));
    DevBuf rstart;
    MMCSF_CUDA(rstart.alloc((uint64_t)nrun * 4));
    k_compact_pos<<<G, 256, 0, s>>>(fl.as<uint32_t>(), exr.as<uint32_t>(), n, rstart.as<uint32_t>());
    LCHECK(L);
    k_split_flags<<<G, 256, 0, s>>>(exr.as<uint32_t>(), rstart.as<uint32_t>(), n, fbr_th, fl.as<uint32_t>());
    LCHECK(L);
  }
  uint32_t F = 0;
  DevBuf exf;
  MMCSF_TRY(scan_total(fl.as<uint32_t>(), n, exf, &F, s, L));
  const int lf = Lv - 1;  // level of leaf fibers: 1 (3-D) or 2 (4-D)
  MMCSF_CUDA(P.ptr[lf].alloc(((uint64_t)F + 1) * 4));
  k_compact_pos<<<G, 256, 0, s>>>(fl.as<uint32_t>(), exf.as<uint32_t>(), n, P.ptr[lf].as<uint32_t>());
  LCHECK(L);
  k_set1<<<1, 1, 0, s>>>(P.ptr[lf].as<uint32_t>(), F, (uint32_t)n);
  LCHECK(L);
  MMCSF_CUDA(P.idx[lf].alloc(((uint64_t)F + 1) * 4));
  MMCSF_CUDA(gather_u32(o[lf], P.ptr[lf].as<uint32_t>(), P.idx[lf].as<uint32_t>(), F, s));
  ++L.n;
  {  // sentinel: the last fiber's index (0 for a single nonzero, src/util.h:1416-1419)
    uint32_t last = 0;
    if (n > 1) MMCSF_CUDA(cudaMemcpyAsync(&last, o[lf] + (n - 1), 4, cudaMemcpyDeviceToHost, s));
    MMCSF_CUDA(cudaStreamSynchronize(s));
    k_set1<<<1, 1, 0, s>>>(P.idx[lf].as<uint32_t>(), F, last);
    LCHECK(L);
  }
  P.n[lf] = F;
  const int GF = grid_for(F, 256);

  // --- level 1 for 4-D: fbrS = runs of (o0,o1) over fibers, split at fbrs_th
  const uint32_t* lvl1_start = P.ptr[lf].as<uint32_t>();  // nonzero position where each fiber starts
  DevBuf fsstart;                                         // nonzero start of every fbrS (4-D)
  uint64_t n1 = F;                                        // entries at the level below slices
  if (nd == 4) {
    DevBuf rf, exrf;
    MMCSF_CUDA(rf.alloc((uint64_t)F * 4));
    Idx4 l2{};
    l2.p[0] = o[0];
    l2.p[1] = o[1];
    k_flags_at<<<GF, 256, 0, s>>>(l2, 2, P.ptr[2].as<uint32_t>(), F, rf.as<uint32_t>());
    LCHECK(L);
    if (fbrs_th < n) {
      uint32_t nruns = 0;
      MMCSF_TRY(scan_total(rf.as<uint32_t>(), F, exrf, &nruns, s, L));
      DevBuf rfirst;
      MMCSF_CUDA(rfirst.alloc((uint64_t)nruns * 4));
      k_compact_pos<<<GF, 256, 0, s>>>(rf.as<uint32_t>(), exrf.as<uint32_t>(), F, rfirst.as<uint32_t>());
      LCHECK(L);
      int gw = grid_for((uint64_t)nruns * 32, 256);
      k_fbrs_split<<<gw, 256, 0, s>>>(P.ptr[2].as<uint32_t>(), rfirst.as<uint32_t>(), nruns, F, fbrs_th,
                                      rf.as<uint32_t>());
      LCHECK(L);
    }
    uint32_t FS = 0;
    DevBuf exs;
    MMCSF_TRY(scan_total(rf.as<uint32_t>(), F, exs, &FS, s, L));
    MMCSF_CUDA(P.ptr[1].alloc(((uint64_t)FS + 1) * 4));
    k_compact_pos<<<GF, 256, 0, s>>>(rf.as<uint32_t>(), exs.as<uint32_t>(), F, P.ptr[1].as<uint32_t>());
    LCHECK(L);
    k_set1<<<1, 1, 0, s>>>(P.ptr[1].as<uint32_t>(), FS, F);
    LCHECK(L);
    MMCSF_CUDA(P.fpar.alloc((uint64_t)F * 4));
    k_parent<<<GF, 256, 0, s>>>(exs.as<uint32_t>(), F, P.fpar.as<uint32_t>());
    LCHECK(L);
    MMCSF_CUDA(fsstart.alloc(((uint64_t)FS + 1) * 4));
    k_gather2<<<grid_for(FS + 1, 256), 256, 0, s>>>(P.ptr[2].as<uint32_t>(), P.ptr[1].as<uint32_t>(), nullptr,
                                                    FS + 1, fsstart.as<uint32_t>());
    LCHECK(L);
    MMCSF_CUDA(P.idx[1].alloc(((uint64_t)FS + 1) * 4));
    MMCSF_CUDA(gather_u32(o[1], fsstart.as<uint32_t>(), P.idx[1].as<uint32_t>(), FS, s));
    ++L.n;
    P.n[1] = FS;
    n1 = FS;
    lvl1_start = fsstart.as<uint32_t>();
  }

  // --- slices: runs of o0 over level-1 entries
  const int G1 = grid_for(n1, 256);
  DevBuf sf, exsl;
  MMCSF_CUDA(sf.alloc(n1 * 4));
  Idx4 l1{};
  l1.p[0] = o[0];
  k_flags_at<<<G1, 256, 0, s>>>(l1, 1, lvl1_start, n1, sf.as<uint32_t>());
  LCHECK(L);
  uint32_t S_ = 0;
  MMCSF_TRY(scan_total(sf.as<uint32_t>(), n1, exsl, &S_, s, L));
  MMCSF_CUDA(P.ptr[0].alloc(((uint64_t)S_ + 1) * 4));
  k_compact_pos<<<G1, 256, 0, s>>>(sf.as<uint32_t>(), exsl.as<uint32_t>(), n1, P.ptr[0].as<uint32_t>());
  LCHECK(L);
  k_set1<<<1, 1, 0, s>>>(P.ptr[0].as<uint32_t>(), S_, (uint32_t)n1);
  LCHECK(L);
  MMCSF_CUDA(P.idx[0].alloc(((uint64_t)S_ + 1) * 4));
  k_gather2<<<grid_for(S_, 256), 256, 0, s>>>(o[0], lvl1_start, P.ptr[0].as<uint32_t>(), S_,
                                              P.idx[0].as<uint32_t>());
  LCHECK(L);
  P.n[0] = S_;
  // fbrLikeSlcInds: o0 of every level-1 entry (one spare entry for kernels)
  MMCSF_CUDA(P.fbr_like.alloc((n1 + 1) * 4));
  MMCSF_CUDA(gather_u32(o[0], lvl1_start, P.fbr_like.as<uint32_t>(), n1, s));
  ++L.n;
  MMCSF_CUDA(cudaMemcpyAsync(P.fbr_like.as<uint32_t>() + n1, o[0] + (n - 1), 4, cudaMemcpyDeviceToDevice, s));

  // --- per-nonzero arrays
  // middle-level indices of every nonzero, read by the per-nonzero traversal:
  // o_{nd-2} (and o1 in 4-D)
  MMCSF_CUDA(P.mid.alloc(n * 4));
  MMCSF_CUDA(cudaMemcpyAsync(P.mid.p, o[nd - 2], n * 4, cudaMemcpyDeviceToDevice, s));
  if (nd == 4) {
    MMCSF_CUDA(P.mid2.alloc(n * 4));
    MMCSF_CUDA(cudaMemcpyAsync(P.mid2.p, o[1], n * 4, cudaMemcpyDeviceToDevice, s));
  }
  P.leaf = std::move(sorted[order[nd - 1]]);
  P.vals = std::move(vals);
  if (keep_coo) {
    for (int m = 0; m < nd; ++m) {
      if (m == order[nd - 1]) {
        MMCSF_CUDA(P.coo[m].alloc(n * 4));
        MMCSF_CUDA(cudaMemcpyAsync(P.coo[m].p, P.leaf.p, n * 4, cudaMemcpyDeviceToDevice, s));
      } else {
        P.coo[m] = std::move(sorted[m]);
      }
    }
  }
  k_flag_fibers<<<GF, 256, 0, s>>>(P.leaf.as<uint32_t>(), P.ptr[lf].as<uint32_t>(), F);
  LCHECK(L);
  MMCSF_CUDA(cudaStreamSynchronize(s));
  return MMCSF_OK;
}

static int compute_bins(CsfPart& P, bool with_children, cudaStream_t s, Launches& L) {
  if (!P.present) return MMCSF_OK;
  const int lf = P.nd - 2;
  DevBuf nzstart;  // nonzero start of every level-1 entry (+ end)
  const uint64_t n1 = P.n[1];
  MMCSF_CUDA(nzstart.alloc((n1 + 1) * 4));
  if (P.nd == 3) {
    MMCSF_CUDA(cudaMemcpyAsync(nzstart.p, P.ptr[1].p, (n1 + 1) * 4, cudaMemcpyDeviceToDevice, s));
  } else {
    k_gather2<<<grid_for(n1 + 1, 256), 256, 0, s>>>(P.ptr[lf].as<uint32_t>(), P.ptr[1].as<uint32_t>(), nullptr,
                                                    n1 + 1, nzstart.as<uint32_t>());
    LCHECK(L);
  }
  MMCSF_CUDA(P.bin_of.alloc(P.n[0] * 4));
  k_bins<<<grid_for(P.n[0], 256), 256, 0, s>>>(P.ptr[0].as<uint32_t>(), nzstart.as<uint32_t>(), P.n[0], P.nnz,
                                               with_children ? 1 : 0, P.bin_of.as<int32_t>());
  LCHECK(L);
  MMCSF_CUDA(cudaStreamSynchronize(s));
  return MMCSF_OK;
}

int build_hyb(mmcsf_format* F, CsfPart& X, cudaStream_t s, int* launches);  // hyb.cu

// largest fiber f with fptr[f] <= x, for every chunk start x = c * chunk
__global__ void k_chunk_fibers(const uint32_t* __restrict__ fptr, uint32_t nfib, uint64_t chunk, uint64_t nchunks,
                               uint32_t* __restrict__ out) {
  const uint64_t c = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  if (c >= nchunks) return;
  const uint64_t x = c * chunk;
  uint32_t lo = 0, hi = nfib - 1;
  while (lo < hi) {
    const uint32_t mid = (lo + hi + 1) >> 1;
    if ((uint64_t)fptr[mid] <= x) lo = mid; else hi = mid - 1;
  }
  out[c] = lo;
}

// mid[x] = fiber index of nonzero x's leaf fiber (o_{nd-2}); 4-D: mid2[x] = its
// fbrS index (o1). One thread per nonzero, binary search over the fiber pointers.
__global__ void k_expand_mid(const uint32_t* __restrict__ fptr, const uint32_t* __restrict__ fidx,
                             const uint32_t* __restrict__ fpar, const uint32_t* __restrict__ sidx1, uint32_t nfib,
                             uint64_t nnz, uint32_t* __restrict__ mid, uint32_t* __restrict__ mid2) {
  for (uint64_t x = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; x < nnz; x += (uint64_t)gridDim.x * blockDim.x) {
    uint32_t lo = 0, hi = nfib - 1;
    while (lo < hi) {
      const uint32_t m = (lo + hi + 1) >> 1;
      if ((uint64_t)fptr[m] <= x) lo = m; else hi = m - 1;
    }
    mid[x] = fidx[lo];
    if (mid2) mid2[x] = sidx1[fpar[lo]];
  }
}

// Per-nonzero middle indices of a part built without them (the HB-CSF CSF part).
int expand_mid(CsfPart& P, cudaStream_t s, Launches& L) {
  if (!P.present || P.nnz == 0 || P.n_fibers() == 0) return MMCSF_OK;
  const int lf = P.nd - 2;
  MMCSF_CUDA(P.mid.alloc(P.nnz * 4));
  if (P.nd == 4) MMCSF_CUDA(P.mid2.alloc(P.nnz * 4));
  k_expand_mid<<<grid_for(P.nnz, 256), 256, 0, s>>>(P.ptr[lf].as<uint32_t>(), P.idx[lf].as<uint32_t>(),
                                                    P.nd == 4 ? P.fpar.as<uint32_t>() : nullptr,
                                                    P.nd == 4 ? P.idx[1].as<uint32_t>() : nullptr,
                                                    (uint32_t)P.n_fibers(), P.nnz, P.mid.as<uint32_t>(),
                                                    P.nd == 4 ? P.mid2.as<uint32_t>() : nullptr);
  LCHECK(L);
  return MMCSF_OK;
}

int chunk_fibers(CsfPart& P, cudaStream_t s, Launches& L) {
  if (!P.present || P.nnz == 0 || P.n_fibers() == 0) return MMCSF_OK;
  if (P.mid.p) {  // first nonzero of every slice: follow the slice's first entry down to the leaf
    MMCSF_CUDA(P.snz.alloc((P.n[0] + 1) * 4));
    MMCSF_CUDA(gather_u32(P.ptr[1].as<uint32_t>(), P.ptr[0].as<uint32_t>(), P.snz.as<uint32_t>(), P.n[0] + 1, s));
    ++L.n;
    if (P.nd == 4) {  // slice -> first fbrS -> first fiber -> first nonzero
      DevBuf t;
      MMCSF_CUDA(t.alloc((P.n[0] + 1) * 4));
      MMCSF_CUDA(gather_u32(P.ptr[2].as<uint32_t>(), P.snz.as<uint32_t>(), t.as<uint32_t>(), P.n[0] + 1, s));
      ++L.n;
      MMCSF_CUDA(cudaStreamSynchronize(s));
      P.snz = std::move(t);
    }
  }
  for (int i = 0; i < CsfPart::N_CHUNK_SIZES; ++i) {
    const uint64_t chunk = 128ull << i, nch = (P.nnz + chunk - 1) / chunk;
    MMCSF_CUDA(P.cfib[i].alloc(nch * 4));
    k_chunk_fibers<<<(unsigned)((nch + 255) / 256), 256, 0, s>>>(P.ptr[P.nd - 2].as<uint32_t>(),
                                                                 (uint32_t)P.n_fibers(), chunk, nch,
                                                                 P.cfib[i].as<uint32_t>());
    LCHECK(L);
    if (P.mid.p) {  // the same search over the slices' first nonzeros
      MMCSF_CUDA(P.cslc[i].alloc(nch * 4));
      k_chunk_fibers<<<(unsigned)((nch + 255) / 256), 256, 0, s>>>(P.snz.as<uint32_t>(), (uint32_t)P.n[0],
                                                                   chunk, nch, P.cslc[i].as<uint32_t>());
      LCHECK(L);
    }
  }
  return MMCSF_OK;
}

}  // namespace mmcsf

using namespace mmcsf;

extern "C" int mmcsf_build(mmcsf_coo* X, const mmcsf_build_opts* opts, void* stream, mmcsf_format** out) {
  MMCSF_RANGE("mmcsf_build");
  if (!X || !opts || !out) return set_error(MMCSF_ERR_INVALID, "null argument");
  const int nd = X->nd;
  if (opts->impl != MMCSF_IMPL_MMCSF && opts->impl != MMCSF_IMPL_BCSF && opts->impl != MMCSF_IMPL_HBCSF)
    return set_error(MMCSF_ERR_INVALID, "unknown implementation type -t %d", opts->impl);
  if (opts->mode < 0 || opts->mode > nd - 1)
    return set_error(MMCSF_ERR_INVALID, "Mode cannot be larger than tensor dimension.");
  if (opts->partition_rule != 0 && opts->partition_rule != 1)
    return set_error(MMCSF_ERR_UNSUPPORTED, "partition rule %d not implemented", opts->partition_rule);
  if (opts->partition_rule == 1 && opts->impl != MMCSF_IMPL_MMCSF)
    return set_error(MMCSF_ERR_INVALID, "the partition heuristic applies to MM-CSF formats (-t 12)");
  if (opts->partition_ratio < 0) return set_error(MMCSF_ERR_INVALID, "partition ratio must be >= 0");
  for (int m = 0; m < nd; ++m)
    if (X->dims[m] >= (1ull << 31))
      return set_error(MMCSF_ERR_UNSUPPORTED, "mode %d length %llu: formats need lengths below 2^31", m,
                       (unsigned long long)X->dims[m]);
  cudaStream_t s = S(stream);
  MMCSF_TRY(mmcsf_coo_to_device(X, stream));
  mmcsf_format* Fm = new (std::nothrow) mmcsf_format;
  if (!Fm) return set_error(MMCSF_ERR_NOMEM, "host allocation failed");
  std::unique_ptr<mmcsf_format> guard(Fm);
  Fm->impl = opts->impl;
  Fm->nd = nd;
  Fm->nnz = X->nnz;
  Fm->mode = opts->mode;
  for (int m = 0; m < nd; ++m) Fm->dims[m] = X->dims[m];
  const uint64_t fth = opts->fiber_threshold ? opts->fiber_threshold : REF_DEFAULT_FBR_TH;
  Fm->fbr_th = fth;
  const int K = nd == 3 ? 2 : 3;  // keys compared by the reference's sorts
  Launches L;
  order_modes(nd, X->dims, opts->mode, Fm->xorder);

  // the reference's chain of sorts, most recent last
  std::vector<std::vector<int>> chain;
  chain.push_back(std::vector<int>(Fm->xorder, Fm->xorder + K));
  int part_order[4] = {0, 1, 2, 3};
  bool heuristic = false;
  int orders_all[4][4] = {{0, 1, 2, 3}, {0, 1, 2, 3}, {0, 1, 2, 3}, {0, 1, 2, 3}};
  if (opts->impl == MMCSF_IMPL_MMCSF) {
    // src/mttkrp.cu:314-352: per-mode CSFs sorted in place on the shared arrays
    int orders[4][4];
    int redun = -1;
    for (int m = 0; m < nd; ++m) {
      order_modes(nd, X->dims, m, orders[m]);
      for (int p = 0; p < m; ++p)
        if (orders[m][1] == orders[p][0] && orders[m][0] == orders[p][1]) redun = m;
      if (m != redun) chain.push_back(std::vector<int>(orders[m], orders[m] + K));
    }
    Fm->redun = redun;
    Fm->partition_rule = opts->partition_rule;
    for (int m = 0; m < nd; ++m) {
      Fm->parts[m].nd = nd;
      for (int i = 0; i < nd; ++i) Fm->parts[m].order[i] = orders[m][i];
    }
    if (opts->partition_rule == 1) heuristic = true;
    // mm_partition_reuseBased ends with `mode = 2;` (src/util.h:2517): every
    // nonzero lands in partition 2, which sort_MI_CSF then sorts by its order.
    if (!heuristic) {
      chain.push_back(std::vector<int>(orders[2], orders[2] + K));
      for (int i = 0; i < nd; ++i) part_order[i] = orders[2][i];
    }
    for (int m = 0; m < nd; ++m)
      for (int i = 0; i < nd; ++i) orders_all[m][i] = orders[m][i];
  } else {
    for (int i = 0; i < nd; ++i) part_order[i] = Fm->xorder[i];
  }
  // composite key: latest sort first, then earlier ones, dropping repeats
  std::vector<int> keys;
  for (int c = (int)chain.size() - 1; c >= 0; --c)
    for (int m : chain[c])
      if (std::find(keys.begin(), keys.end(), m) == keys.end()) keys.push_back(m);

  DevBuf sorted[4], svals, part_perm;
  MMCSF_TRY(sort_coo(X, keys, sorted, svals, s, L, &part_perm));
  const int target = opts->impl == MMCSF_IMPL_MMCSF ? 2 : 0;
  const uint64_t fbrs_th = opts->impl == MMCSF_IMPL_MMCSF ? FBRS_TH_MMCSF : FBRS_TH_OFF;
  if (heuristic) {
    // X is now in the order the partition loop visits it (the chain of
    // per-mode sorts); the heuristic picks a partition per nonzero, and every
    // partition is filled in X order (populate_paritions) and sorted by its
    // own mode order (sort_MI_CSF, src/util.h:412-527)
    const uint32_t* sx[4] = {nullptr, nullptr, nullptr, nullptr};
    for (int m = 0; m < nd; ++m) sx[m] = sorted[m].as<uint32_t>();
    DevBuf part;
    MMCSF_CUDA(part.alloc(std::max<uint64_t>(X->nnz, 1)));
    const int ratio = opts->partition_ratio ? opts->partition_ratio : 1;
    MMCSF_TRY(mm_partition_heuristic(nd, X->dims, orders_all, Fm->xorder, Fm->redun, ratio, sx, X->nnz,
                                     part.as<uint8_t>(), &Fm->heur_rounds, &L.n, s));
    for (int m = 0; m < nd; ++m) sorted[m].release();
    svals.release();
    DevBuf gperm;  // the format's nonzero order: partitions 0..nd-1, each in its own sorted order
    MMCSF_CUDA(gperm.alloc(std::max<uint64_t>(X->nnz, 1) * 4));
    uint64_t off = 0;
    for (int p = 0; p < nd; ++p) {
      DevBuf members;
      uint64_t cnt = 0;
      MMCSF_TRY(partition_members(part.as<uint8_t>(), p, part_perm.as<uint32_t>(), X->nnz, members, &cnt, &L.n, s));
      if (cnt == 0) continue;
      std::vector<int> pkeys(orders_all[p], orders_all[p] + K);
      DevBuf ps[4], pv, pperm;
      MMCSF_TRY(sort_coo(X, pkeys, ps, pv, s, L, &pperm, &members, cnt));
      MMCSF_TRY(build_csf(nd, orders_all[p], cnt, ps, pv, fth, fbrs_th, opts->keep_coo != 0, Fm->parts[p], s, L));
      MMCSF_CUDA(cudaMemcpyAsync(gperm.as<uint32_t>() + off, pperm.p, cnt * 4, cudaMemcpyDeviceToDevice, s));
      if (cnt < X->nnz) {
        if (!Fm->all_vals.p) MMCSF_CUDA(Fm->all_vals.alloc(X->nnz * 4));
        MMCSF_CUDA(cudaMemcpyAsync(Fm->all_vals.as<float>() + off, Fm->parts[p].vals.p, cnt * 4,
                                   cudaMemcpyDeviceToDevice, s));
      }
      off += cnt;
      MMCSF_CUDA(cudaStreamSynchronize(s));
    }
    part_perm = std::move(gperm);
  } else {
    MMCSF_TRY(build_csf(nd, part_order, X->nnz, sorted, svals, fth, fbrs_th,
                        opts->keep_coo != 0 || opts->impl == MMCSF_IMPL_HBCSF, Fm->parts[target], s, L));
  }
  CsfPart& P = Fm->parts[target];
  if (opts->impl == MMCSF_IMPL_BCSF) MMCSF_TRY(compute_bins(P, true, s, L));
  if (opts->impl == MMCSF_IMPL_MMCSF && opts->views) {
    // Slice-major views: a CSF whose level 0 is mode m, in the reference's
    // order for a mode-m CSF (order_tensormode) or, with view_order 1, the
    // remaining modes longest first, fully sorted, no splits.
    for (int m = 0; m < nd; ++m) {
      bool at_leaf = false, root_everywhere = true;
      for (int p = 0; p < nd; ++p) {
        if (!Fm->parts[p].present) continue;
        if (Fm->parts[p].order[nd - 1] == m) at_leaf = true;
        if (Fm->parts[p].order[0] != m) root_everywhere = false;
      }
      if (opts->views == 1 && !at_leaf) continue;
      if (root_everywhere) continue;  // the partitions already serve m at level 0
      int vo[4];
      order_modes(nd, X->dims, m, vo);
      if (opts->view_order == 1) std::reverse(vo + 1, vo + nd);  // the shortest mode at the leaf level
      std::vector<int> vkeys(vo, vo + nd);
      DevBuf vs[4], vv, vperm;
      MMCSF_TRY(sort_coo(X, vkeys, vs, vv, s, L, &vperm));
      MMCSF_TRY(build_csf(nd, vo, X->nnz, vs, vv, REF_DEFAULT_FBR_TH, FBRS_TH_OFF, false, Fm->views[m], s, L));
      // view position -> partition position (to reorder caller values given in
      // the format's nonzero order, for MTTKRP on other values)
      DevBuf inv;
      MMCSF_CUDA(inv.alloc(X->nnz * 4));
      k_invert<<<grid_for(X->nnz, 256), 256, 0, s>>>(part_perm.as<uint32_t>(), X->nnz, inv.as<uint32_t>());
      LCHECK(L);
      MMCSF_CUDA(Fm->views[m].from_part.alloc(X->nnz * 4));
      MMCSF_CUDA(gather_u32(inv.as<uint32_t>(), vperm.as<uint32_t>(), Fm->views[m].from_part.as<uint32_t>(),
                            X->nnz, s));
      ++L.n;
      MMCSF_CUDA(cudaStreamSynchronize(s));
    }
  }
  if (opts->impl == MMCSF_IMPL_HBCSF) {
    MMCSF_TRY(build_hyb(Fm, P, s, &L.n));
    for (int p = 0; p < 4; ++p) {  // the CSF part now holds a subset: derive its middle indices again
      Fm->parts[p].mid.release();
      Fm->parts[p].mid2.release();
      MMCSF_TRY(expand_mid(Fm->parts[p], s, L));
    }
  }
  for (int p = 0; p < 4; ++p) MMCSF_TRY(chunk_fibers(Fm->parts[p], s, L));
  for (int m = 0; m < 4; ++m) MMCSF_TRY(chunk_fibers(Fm->views[m], s, L));
  MMCSF_CUDA(cudaStreamSynchronize(s));
  Fm->last_launches = L.n;
  *out = guard.release();
  return MMCSF_OK;
}

extern "C" void mmcsf_format_destroy(mmcsf_format* F) { delete F; }

extern "C" int mmcsf_format_info(const mmcsf_format* F, int part, mmcsf_part_info* info) {
  if (!F || !info) return set_error(MMCSF_ERR_INVALID, "null argument");
  if (part < 0 || part >= 8) return set_error(MMCSF_ERR_INVALID, "bad part %d", part);
  memset(info, 0, sizeof *info);
  const CsfPart& P = part < 4 ? F->parts[part] : F->views[part - 4];
  info->present = P.present ? 1 : 0;
  info->nd = F->nd;
  for (int i = 0; i < F->nd; ++i) info->mode_order[i] = P.present || (F->impl == MMCSF_IMPL_MMCSF && part < 4) ? P.order[i] : i;
  info->nnz = P.nnz;
  info->n_slices = P.n[0];
  info->n_fbrs = P.n[1];
  info->n_fibers = P.n_fibers();
  info->device_bytes = P.bytes();
  return MMCSF_OK;
}

extern "C" int mmcsf_format_partitioning(const mmcsf_format* F, int* partition_rule, int* rounds) {
  if (!F) return set_error(MMCSF_ERR_INVALID, "null argument");
  if (partition_rule) *partition_rule = F->partition_rule;
  if (rounds) *rounds = F->heur_rounds;
  return MMCSF_OK;
}

extern "C" int mmcsf_format_meta(const mmcsf_format* F, int* redun_mode, int* x_mode_order) {
  if (!F) return set_error(MMCSF_ERR_INVALID, "null argument");
  if (redun_mode) *redun_mode = F->redun;
  if (x_mode_order)
    for (int i = 0; i < F->nd; ++i) x_mode_order[i] = F->xorder[i];
  return MMCSF_OK;
}

extern "C" int mmcsf_format_last_launches(const mmcsf_format* F, int* launches) {
  if (!F || !launches) return set_error(MMCSF_ERR_INVALID, "null argument");
  *launches = F->last_launches;
  return MMCSF_OK;
}
