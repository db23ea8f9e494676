// Format consistency and bounds check (mmcsf_format_check): every index a
// kernel will dereference, validated on the device before it is used.
//
// For every present CSF part (partitions, views, the HB-CSF CSF part) and the
// HB-CSF COO/CSL parts: index arrays below the row counts of their modes'
// factors, pointer arrays starting at 0, strictly increasing and ending at
// the next level's count, the leaf-index fiber flags set exactly at fiber
// starts, the per-nonzero middle indices equal to their fibers' indices, the
// slice starts and the chunk-start tables consistent with the pointers.
// Every read is bounded by the buffer's allocated size, so a corrupt array is
// reported, never followed. The reference has no counterpart (it trusts its
// own builders); this is the library's bounds-checked mode: built with
// -DMMCSF_BOUNDS, every MTTKRP entry point runs it once per format first.
#include <algorithm>
#include <cstring>

#include "format.h"
#include "prims.cuh"

namespace mmcsf {
namespace {

constexpr uint32_t FLAG = 0x80000000u;
constexpr int NCHECK = 64;

struct Err {
  unsigned long long count[NCHECK];
  unsigned long long first[NCHECK];
};

__device__ __forceinline__ void bad(Err* e, int id, uint64_t pos) {
  atomicAdd(&e->count[id], 1ull);
  atomicMin(&e->first[id], (unsigned long long)pos);
}

#define GRID_LOOP(i, n) \
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < (n); i += (uint64_t)gridDim.x * blockDim.x)

// a[i] & mask < bound for i < n (n <= cap)
__global__ void k_bound(const uint32_t* __restrict__ a, uint64_t n, uint64_t cap, uint32_t mask, uint64_t bound,
                        Err* e, int id) {
  if (n > cap) {
    if (blockIdx.x == 0 && threadIdx.x == 0) bad(e, id, cap);
    n = cap;
  }
  GRID_LOOP(i, n) if ((uint64_t)(a[i] & mask) >= bound) bad(e, id, i);
}

// p[0] == 0, p[i] < p[i + 1], p[n] == end (n + 1 entries)
__global__ void k_ptr(const uint32_t* __restrict__ p, uint64_t n, uint64_t cap, uint64_t end, Err* e, int id) {
  if (n + 1 > cap) {
    if (blockIdx.x == 0 && threadIdx.x == 0) bad(e, id, cap);
    return;
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    if (p[0] != 0) bad(e, id, 0);
    if ((uint64_t)p[n] != end) bad(e, id, n);
  }
  GRID_LOOP(i, n) if (p[i] >= p[i + 1]) bad(e, id, i);
}

// the fiber flag of leaf[fptr[f]] for every fiber f; flags counted in *nflag
__global__ void k_flags(const uint32_t* __restrict__ leaf, uint64_t nnz, const uint32_t* __restrict__ fptr,
                        uint64_t nfib, unsigned long long* nflag, Err* e, int id) {
  GRID_LOOP(f, nfib) {
    const uint64_t x = fptr[f];
    if (x >= nnz || !(leaf[x] & FLAG)) bad(e, id, f);
  }
  unsigned long long c = 0;
  GRID_LOOP(x, nnz) c += (leaf[x] & FLAG) ? 1 : 0;
  if (c) atomicAdd(nflag, c);
}

// mid[x] == fidx[f] for every nonzero x of fiber f (and, 4-D, mid2[x] ==
// sidx1[fpar[f]])
__global__ void k_mid(const uint32_t* __restrict__ mid, const uint32_t* __restrict__ mid2, uint64_t nnz,
                      const uint32_t* __restrict__ fptr, const uint32_t* __restrict__ fidx,
                      const uint32_t* __restrict__ fpar, const uint32_t* __restrict__ sidx1, uint64_t n1,
                      uint64_t nfib, Err* e, int id) {
  GRID_LOOP(f, nfib) {
    const uint64_t x0 = fptr[f], x1 = std::min<uint64_t>(fptr[f + 1], nnz);
    uint32_t want2 = 0;
    if (mid2) {
      const uint32_t sp = fpar[f];
      if (sp >= n1) { bad(e, id, f); continue; }
      want2 = sidx1[sp];
    }
    for (uint64_t x = x0; x < x1; ++x)
      if (mid[x] != fidx[f] || (mid2 && mid2[x] != want2)) { bad(e, id, f); break; }
  }
}

// snz[s] == the first nonzero of slice s, following the pointers down
__global__ void k_snz(const uint32_t* __restrict__ snz, uint64_t ns, const uint32_t* __restrict__ p0,
                      const uint32_t* __restrict__ p1, uint64_t c1, const uint32_t* __restrict__ p2, uint64_t c2,
                      Err* e, int id) {
  GRID_LOOP(s, ns + 1) {
    uint64_t q = p0[s];
    if (q >= c1) { bad(e, id, s); continue; }
    q = p1[q];
    if (p2) {
      if (q >= c2) { bad(e, id, s); continue; }
      q = p2[q];
    }
    if ((uint64_t)snz[s] != q) bad(e, id, s);
  }
}

// tab[t] = c with starts[c] <= t chunk < starts[c + 1], c < nstarts
__global__ void k_table(const uint32_t* __restrict__ tab, uint64_t nt, uint64_t chunk,
                        const uint32_t* __restrict__ starts, uint64_t nstarts, Err* e, int id) {
  GRID_LOOP(t, nt) {
    const uint64_t c = tab[t], x = t * chunk;
    if (c >= nstarts || (uint64_t)starts[c] > x || (uint64_t)starts[c + 1] <= x) bad(e, id, t);
  }
}

// 4-D: fiber f lies in fbrS fpar[f]: p1[fpar[f]] <= f < p1[fpar[f] + 1]
__global__ void k_fpar(const uint32_t* __restrict__ fpar, uint64_t nfib, const uint32_t* __restrict__ p1,
                       uint64_t n1, Err* e, int id) {
  GRID_LOOP(f, nfib) {
    const uint64_t sp = fpar[f];
    if (sp >= n1 || (uint64_t)p1[sp] > f || (uint64_t)p1[sp + 1] <= f) bad(e, id, f);
  }
}

struct Checker {
  const mmcsf_format* F;
  const uint64_t* rows;
  cudaStream_t s;
  Err* e;
  int n = 0;
  char what[NCHECK][96];
  int next(const char* fmt, ...) {
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(what[n], sizeof what[n], fmt, ap);
    va_end(ap);
    return n++;
  }
  static unsigned grid(uint64_t n) { return (unsigned)std::max<uint64_t>(1, std::min<uint64_t>((n + 255) / 256, 4096)); }
  static uint64_t cap(const DevBuf& b) { return b.bytes / 4; }

  int part(const CsfPart& P, const char* name) {
    if (!P.present) return MMCSF_OK;
    const int nd = P.nd, L = nd - 1;
    if (n + 24 > NCHECK) return set_error(MMCSF_ERR_INVALID, "format check: too many parts");
    for (int l = 0; l < L; ++l) {
      const uint64_t cnt = P.n[l];
      const uint64_t end = l < L - 1 ? P.n[l + 1] : P.nnz;
      if (cnt == 0 && P.nnz == 0) continue;
      if (!P.ptr[l].p || !P.idx[l].p) return set_error(MMCSF_ERR_INVALID, "format check: %s level %d arrays missing", name, l);
      k_ptr<<<grid(cnt), 256, 0, s>>>(P.ptr[l].as<uint32_t>(), cnt, cap(P.ptr[l]), end, e,
                                      next("%s: level-%d pointers", name, l));
      k_bound<<<grid(cnt), 256, 0, s>>>(P.idx[l].as<uint32_t>(), cnt, cap(P.idx[l]), 0xffffffffu, rows[P.order[l]], e,
                                        next("%s: level-%d indices (mode %d)", name, l, P.order[l]));
    }
    if (P.nnz == 0) return MMCSF_OK;
    const uint64_t nfib = P.n_fibers();
    const DevBuf& fptr = P.ptr[nd - 2];
    const DevBuf& fidx = P.idx[nd - 2];
    if (cap(fptr) < nfib + 1 || cap(fidx) < nfib || cap(P.leaf) < P.nnz)
      return set_error(MMCSF_ERR_INVALID, "format check: %s: leaf-level arrays shorter than their counts", name);
    k_bound<<<grid(P.nnz), 256, 0, s>>>(P.leaf.as<uint32_t>(), P.nnz, cap(P.leaf), ~FLAG, rows[P.order[L]], e,
                                        next("%s: leaf indices (mode %d)", name, P.order[L]));
    const int idf = next("%s: leaf fiber flags", name);
    unsigned long long* nflag = reinterpret_cast<unsigned long long*>(&e->first[NCHECK - 1]);  // spare slot
    k_flags<<<grid(std::max(nfib, P.nnz)), 256, 0, s>>>(P.leaf.as<uint32_t>(), P.nnz, fptr.as<uint32_t>(), nfib,
                                                       nflag, e, idf);
    flag_id = idf;
    flag_want = nfib;
    if (P.fbr_like.p) {
      k_bound<<<grid(P.n[1]), 256, 0, s>>>(P.fbr_like.as<uint32_t>(), P.n[1], cap(P.fbr_like), 0xffffffffu,
                                           rows[P.order[0]], e, next("%s: fiber-to-slice indices", name));
    }
    if (nd == 4 && P.fpar.p) {
      if (cap(P.fpar) < nfib || cap(P.ptr[1]) < P.n[1] + 1)
        return set_error(MMCSF_ERR_INVALID, "format check: %s: fbrS arrays shorter than their counts", name);
      k_fpar<<<grid(nfib), 256, 0, s>>>(P.fpar.as<uint32_t>(), nfib, P.ptr[1].as<uint32_t>(), P.n[1], e,
                                        next("%s: fiber-to-fbrS map", name));
    }
    if (P.mid.p) {
      if (cap(P.mid) < P.nnz || (nd == 4 && (!P.mid2.p || cap(P.mid2) < P.nnz || !P.fpar.p)))
        return set_error(MMCSF_ERR_INVALID, "format check: %s: per-nonzero index arrays shorter than nnz", name);
      k_mid<<<grid(nfib), 256, 0, s>>>(P.mid.as<uint32_t>(), nd == 4 ? P.mid2.as<uint32_t>() : nullptr, P.nnz,
                                       fptr.as<uint32_t>(), fidx.as<uint32_t>(),
                                       nd == 4 ? P.fpar.as<uint32_t>() : nullptr,
                                       nd == 4 ? P.idx[1].as<uint32_t>() : nullptr, P.n[1], nfib, e,
                                       next("%s: per-nonzero middle indices", name));
    }
    if (P.snz.p) {
      if (cap(P.snz) < P.n[0] + 1 || cap(P.ptr[0]) < P.n[0] + 1)
        return set_error(MMCSF_ERR_INVALID, "format check: %s: slice starts shorter than the slices", name);
      k_ptr<<<grid(P.n[0]), 256, 0, s>>>(P.snz.as<uint32_t>(), P.n[0], cap(P.snz), P.nnz, e,
                                         next("%s: slice first nonzeros", name));
      k_snz<<<grid(P.n[0] + 1), 256, 0, s>>>(P.snz.as<uint32_t>(), P.n[0], P.ptr[0].as<uint32_t>(),
                                             P.ptr[1].as<uint32_t>(), cap(P.ptr[1]),
                                             nd == 4 ? P.ptr[2].as<uint32_t>() : nullptr,
                                             nd == 4 ? cap(P.ptr[2]) : 0, e, next("%s: slice starts vs pointers", name));
    }
    for (int i = 0; i < CsfPart::N_CHUNK_SIZES; ++i) {
      const uint64_t chunk = 128ull << i, nt = (P.nnz + chunk - 1) / chunk;
      if (P.cfib[i].p) {
        if (cap(P.cfib[i]) < nt) return set_error(MMCSF_ERR_INVALID, "format check: %s: chunk table %d short", name, i);
        k_table<<<grid(nt), 256, 0, s>>>(P.cfib[i].as<uint32_t>(), nt, chunk, fptr.as<uint32_t>(), nfib, e,
                                         next("%s: chunk-%llu fiber table", name, (unsigned long long)chunk));
      }
      if (P.cslc[i].p && P.snz.p) {
        if (cap(P.cslc[i]) < nt) return set_error(MMCSF_ERR_INVALID, "format check: %s: chunk table %d short", name, i);
        k_table<<<grid(nt), 256, 0, s>>>(P.cslc[i].as<uint32_t>(), nt, chunk, P.snz.as<uint32_t>(), P.n[0], e,
                                         next("%s: chunk-%llu slice table", name, (unsigned long long)chunk));
      }
    }
    return MMCSF_OK;
  }
  int flag_id = -1;
  uint64_t flag_want = 0;
};

}  // namespace
}  // namespace mmcsf

using namespace mmcsf;

extern "C" int mmcsf_format_check(const mmcsf_format* F, const uint64_t* rows, void* stream) {
  MMCSF_RANGE("mmcsf_format_check");
  if (!F) return set_error(MMCSF_ERR_INVALID, "null format");
  uint64_t r[4] = {0, 0, 0, 0};
  for (int m = 0; m < F->nd; ++m) {
    r[m] = rows ? rows[m] : F->dims[m];
    if (rows && r[m] > F->dims[m]) r[m] = F->dims[m];  // rows beyond the tensor's extent are never indexed
  }
  cudaStream_t s = S(stream);
  DevBuf eb;
  MMCSF_CUDA(eb.alloc(sizeof(Err)));
  Err h;
  for (int i = 0; i < NCHECK; ++i) { h.count[i] = 0; h.first[i] = ~0ull; }
  MMCSF_CUDA(cudaMemcpyAsync(eb.p, &h, sizeof h, cudaMemcpyHostToDevice, s));
  const char* pname[4] = {"partition 0", "partition 1", "partition 2", "partition 3"};
  const char* vname[4] = {"view of mode 0", "view of mode 1", "view of mode 2", "view of mode 3"};
  // one part at a time: each has its own flag counter in the spare slot
  auto run = [&](const CsfPart& P, const char* name) -> int {
    Checker c{F, r, s, eb.as<Err>()};
    MMCSF_CUDA(cudaMemsetAsync(&eb.as<Err>()->first[NCHECK - 1], 0, 8, s));
    MMCSF_CUDA(cudaMemsetAsync(eb.as<Err>()->count, 0, sizeof h.count, s));
    MMCSF_CUDA(cudaMemsetAsync(eb.as<Err>()->first, 0xff, sizeof(unsigned long long) * (NCHECK - 1), s));
    MMCSF_TRY(c.part(P, name));
    MMCSF_CUDA(cudaGetLastError());
    MMCSF_CUDA(cudaMemcpyAsync(&h, eb.p, sizeof h, cudaMemcpyDeviceToHost, s));
    MMCSF_CUDA(cudaStreamSynchronize(s));
    for (int i = 0; i < c.n; ++i)
      if (h.count[i])
        return set_error(MMCSF_ERR_INVALID, "format check: %s: %llu bad entries, first at %llu", c.what[i], h.count[i],
                         h.first[i]);
    if (c.flag_id >= 0 && h.first[NCHECK - 1] != c.flag_want)
      return set_error(MMCSF_ERR_INVALID, "format check: %s: %llu fiber flags for %llu fibers", c.what[c.flag_id],
                       h.first[NCHECK - 1], (unsigned long long)c.flag_want);
    return MMCSF_OK;
  };
  for (int p = 0; p < 4; ++p) MMCSF_TRY(run(F->parts[p], pname[p]));
  for (int m = 0; m < 4; ++m) MMCSF_TRY(run(F->views[m], vname[m]));
  // HB-CSF COO and CSL parts (levels in the CSF part's mode order)
  const mmcsf::HybExtra& H = F->hyb;
  if (F->impl == MMCSF_IMPL_HBCSF && (H.coo_nnz || H.csl_nnz)) {
    const CsfPart& P = F->parts[0];
    Checker c{F, r, s, eb.as<Err>()};
    MMCSF_CUDA(cudaMemsetAsync(eb.as<Err>()->count, 0, sizeof h.count, s));
    MMCSF_CUDA(cudaMemsetAsync(eb.as<Err>()->first, 0xff, sizeof h.first, s));
    for (int l = 0; l < F->nd && H.coo_nnz; ++l)
      k_bound<<<Checker::grid(H.coo_nnz), 256, 0, s>>>(H.coo_inds[l].as<uint32_t>(), H.coo_nnz, Checker::cap(H.coo_inds[l]),
                                                       0xffffffffu, r[P.order[l]], eb.as<Err>(),
                                                       c.next("HB-CSF COO part: level-%d indices", l));
    if (H.csl_nnz && F->nd == 3) {
      k_ptr<<<Checker::grid(H.n_csl_slices), 256, 0, s>>>(H.csl_ptr.as<uint32_t>(), H.n_csl_slices,
                                                          Checker::cap(H.csl_ptr), H.csl_nnz, eb.as<Err>(),
                                                          c.next("HB-CSF CSL part: slice pointers"));
      k_bound<<<Checker::grid(H.n_csl_slices), 256, 0, s>>>(H.csl_idx.as<uint32_t>(), H.n_csl_slices,
                                                            Checker::cap(H.csl_idx), 0xffffffffu, r[P.order[0]],
                                                            eb.as<Err>(), c.next("HB-CSF CSL part: slice indices"));
      k_bound<<<Checker::grid(H.csl_nnz), 256, 0, s>>>(H.csl_i1.as<uint32_t>(), H.csl_nnz, Checker::cap(H.csl_i1),
                                                       0xffffffffu, r[P.order[1]], eb.as<Err>(),
                                                       c.next("HB-CSF CSL part: middle indices"));
      k_bound<<<Checker::grid(H.csl_nnz), 256, 0, s>>>(H.csl_i2.as<uint32_t>(), H.csl_nnz, Checker::cap(H.csl_i2),
                                                       0xffffffffu, r[P.order[2]], eb.as<Err>(),
                                                       c.next("HB-CSF CSL part: leaf indices"));
    }
    MMCSF_CUDA(cudaGetLastError());
    MMCSF_CUDA(cudaMemcpyAsync(&h, eb.p, sizeof h, cudaMemcpyDeviceToHost, s));
    MMCSF_CUDA(cudaStreamSynchronize(s));
    for (int i = 0; i < c.n; ++i)
      if (h.count[i])
        return set_error(MMCSF_ERR_INVALID, "format check: %s: %llu bad entries, first at %llu", c.what[i], h.count[i],
                         h.first[i]);
  }
  return MMCSF_OK;
}
