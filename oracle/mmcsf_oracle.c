/*
 * Test infrastructure, not product code: a plain-C restatement of the
 * reference's (isratnisa/MM-CSF) host algorithms on the MTTKRP path. Only
 * tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg may load it,
 * and only as the checker. It is pinned against the reference itself (built by
 * oracle/build_ref.py) through the golden fixtures under tests/golden/.
 *
 * Conventions: indices are uint64 like the reference's ITYPE (size_t);
 * values are float like its DTYPE. Every function cites the reference code
 * it restates. Sorting is STABLE, matching the oracle build of the reference
 * whose Boost sample_sort is replaced by std::stable_sort.
 */
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

typedef uint64_t u64;

/* ---- mode ordering: src/util.h:255-311 (order_tensormode) ---------------- */
void orc_order_modes(int nd, const u64* dims, int mode, int natural, int* order) {
  int natMode[8], taken[8];
  u64 len[8];
  for (int m = 0; m < nd; ++m) {
    natMode[m] = (m + mode) % nd;
    len[m] = dims[natMode[m]];
    taken[m] = 0;
  }
  if (natural) {
    for (int i = 0; i < nd; ++i) order[i] = natMode[i];
    return;
  }
  /* the reference sorts positions 1..nd-1 of the length list ascending */
  for (int i = 1; i < nd; i++)
    for (int j = i + 1; j < nd; j++)
      if (len[i] > len[j]) { u64 t = len[i]; len[i] = len[j]; len[j] = t; }
  order[0] = mode;
  taken[mode] = 1;
  for (int i = 1; i < nd; i++)
    for (int j = 0; j < nd; j++)
      if (len[i] == dims[j] && !taken[j]) { order[i] = j; taken[j] = 1; break; }
}

/* ---- redundant-mode detection: src/mttkrp.cu:314-343 --------------------- */
static int same_pair(const int* a, const int* b) { return a[1] == b[0] && a[0] == b[1]; }

int orc_redundant_mode(int nd, const int orders[][8]) {
  int redun = -1; /* the reference leaves it uninitialised when none is found */
  for (int m = 1; m < nd; ++m) {
    int hit = 0;
    for (int p = 0; p < m; ++p)
      if (same_pair(orders[m], orders[p])) hit = 1;
    if (hit) redun = m;
  }
  return redun;
}

/* ---- stable sort on a key prefix: src/util.h:389-527 ---------------------- */
typedef struct {
  u64* const* inds;
  const int* keys;
  int nkeys;
} sort_ctx;

static int key_less(const sort_ctx* c, u64 a, u64 b) {
  for (int k = 0; k < c->nkeys; ++k) {
    u64 x = c->inds[c->keys[k]][a], y = c->inds[c->keys[k]][b];
    if (x != y) return x < y;
  }
  return 0;
}

static void merge_sort(const sort_ctx* c, u64* perm, u64* tmp, u64 n) {
  for (u64 w = 1; w < n; w *= 2) {
    for (u64 lo = 0; lo < n; lo += 2 * w) {
      u64 mid = lo + w < n ? lo + w : n, hi = lo + 2 * w < n ? lo + 2 * w : n;
      u64 i = lo, j = mid, k = lo;
      while (i < mid && j < hi) tmp[k++] = key_less(c, perm[j], perm[i]) ? perm[j++] : perm[i++];
      while (i < mid) tmp[k++] = perm[i++];
      while (j < hi) tmp[k++] = perm[j++];
    }
    memcpy(perm, tmp, n * sizeof(u64));
  }
}

/* Stable in-place sort of the COO arrays by inds[keys[0]], inds[keys[1]], ... */
int orc_sort_coo(int nd, u64 nnz, u64* const* inds, float* vals, const int* keys, int nkeys) {
  if (nnz < 2) return 0;
  u64* perm = (u64*)malloc(nnz * sizeof(u64));
  u64* tmp = (u64*)malloc(nnz * sizeof(u64));
  if (!perm || !tmp) return 1;
  for (u64 i = 0; i < nnz; ++i) perm[i] = i;
  sort_ctx c = {inds, keys, nkeys};
  merge_sort(&c, perm, tmp, nnz);
  for (int m = 0; m < nd; ++m) {
    for (u64 i = 0; i < nnz; ++i) tmp[i] = inds[m][perm[i]];
    memcpy(inds[m], tmp, nnz * sizeof(u64));
  }
  float* fv = (float*)tmp;
  for (u64 i = 0; i < nnz; ++i) fv[i] = vals[perm[i]];
  memcpy(vals, fv, nnz * sizeof(float));
  free(perm);
  free(tmp);
  return 0;
}

/* ---- CSF construction: src/util.h:1320-1436 (create_TiledHCSR) and
 * src/util.h:760-850 (create_HCSR, the same loop without the 4-D fbrS split).
 * ptr[l]/idx[l] (l = 0..nd-2) need capacity nnz+2; counts are returned in
 * nptr[l]/nidx[l]. `fbrSTh` is 128 for MM-CSF (-t 12) and "infinite"
 * otherwise. Where the reference reads one element past the last nonzero
 * (the inner scan at :1366-1374 when the last fiber has 2+ nonzeros) this
 * restatement reads 0, like the reference's oracle build whose allocations
 * are zero-padded; that value only reaches the sentinel idx[nd-2][F]. */
static u64 rd(u64* const* inds, int mode, u64 i, u64 nnz) { return i < nnz ? inds[mode][i] : 0; }

int orc_create_csf(int nd, u64 nnz, u64* const* inds, const int* order, u64 fbrTh, u64 fbrSTh,
                   u64** ptr, u64** idx, u64* nptr, u64* nidx) {
  const int L = nd - 1;
  u64 prevId[8], fbrId[8];
  for (int i = 0; i < L; ++i) nptr[i] = nidx[i] = 0;
  if (nnz == 0) return 0;
  for (int i = 0; i < L; ++i) {
    prevId[i] = inds[order[i]][0];
    ptr[i][nptr[i]++] = 0;
    idx[i][nidx[i]++] = prevId[i];
  }
  u64 x = 1, fiberSNnz = 1;
  /* the reference's fbrId vector starts zeroed; with one nonzero it is never
     read from the tensor and the sentinel is 0 */
  for (int i = 0; i < L; ++i) fbrId[i] = 0;
  while (x < nnz) {
    for (int i = 0; i < L; ++i) fbrId[i] = inds[order[i]][x];
    u64 fiberNnz = 1;
    int sameFbr = 1;
    for (int i = 0; i < L; ++i)
      if (fbrId[i] != prevId[i]) sameFbr = 0;
    while (sameFbr && x < nnz && fiberNnz < fbrTh) {
      ++x;
      ++fiberNnz;
      ++fiberSNnz;
      for (int i = 0; i < L; ++i) {
        fbrId[i] = rd(inds, order[i], x, nnz);
        if (fbrId[i] != prevId[i]) sameFbr = 0;
      }
    }
    if (x == nnz) break;
    ptr[L - 1][nptr[L - 1]++] = x;
    idx[L - 1][nidx[L - 1]++] = fbrId[L - 1];
    for (int i = nd - 3; i > -1; --i) {
      int diff = 0;
      for (int d = i; d > -1; --d) {
        if (fbrId[d] != prevId[d]) diff = 1;
        else if (nd == 4 && d == 1 && fiberSNnz > fbrSTh) diff = 1;
      }
      if (diff) {
        if (nd == 4 && i == 1) fiberSNnz = 1;
        idx[i][nidx[i]++] = fbrId[i];
        ptr[i][nptr[i]++] = nptr[i + 1] - 1;
      }
    }
    for (int i = 0; i < L; ++i) prevId[i] = fbrId[i];
    ++x;
    ++fiberSNnz;
  }
  ptr[L - 1][nptr[L - 1]++] = x;
  idx[L - 1][nidx[L - 1]++] = fbrId[L - 1];
  for (int i = nd - 3; i > -1; --i) ptr[i][nptr[i]++] = nptr[i + 1] - 1;
  return 0;
}

/* ---- fiber-to-slice map: src/util.h:1768-1783 (create_fbrLikeSlcInds).
 * Writes nFibers-1 entries (the reference leaves the last one unset). */
void orc_fbr_like_slc(const u64* ptr0, const u64* idx0, u64 nslc, u64* out) {
  for (u64 s = 0; s < nslc; ++s)
    for (u64 f = ptr0[s]; f < ptr0[s + 1]; ++f) out[f] = idx0[s];
}

/* ---- slice binning: src/util.h:1887-1952 (make_TiledBin), nBin = 10.
 * bin_of[s] receives the bin of slice s, or -1 when no bin's open interval
 * (LB, UB) contains the slice's (#children + #nonzeros) count. */
void orc_tiled_bins(int nd, const u64* const* ptr, u64 nslc, u64 totNnz, int* bin_of) {
  const u64 TB = 512;
  u64 LB[10] = {0, 2, 4, 8, 16, 1024, 4 * TB, 8 * TB, 16 * TB, 32 * TB};
  u64 UB[10] = {1025, 5, 9, 17, 1025, 4 * TB + 1, 8 * TB + 1, 16 * TB + 1, 32 * TB + 1, totNnz + 1};
  for (u64 s = 0; s < nslc; ++s) {
    long long n = (long long)(ptr[0][s + 1] - ptr[0][s]);
    for (u64 c = ptr[0][s]; c < ptr[0][s + 1]; ++c) {
      if (nd == 3) n += (long long)(ptr[1][c + 1] - ptr[1][c]);
      else
        for (u64 g = ptr[1][c]; g < ptr[1][c + 1]; ++g) n += (long long)(ptr[2][g + 1] - ptr[2][g]);
    }
    bin_of[s] = -1;
    for (int b = 0; b < 10; ++b)
      if ((u64)n > LB[b] && (u64)n < UB[b]) { bin_of[s] = b; break; }
  }
}

/* ---- HB-CSF bins: src/util.h:1786-1885 (make_HybBin): the count is the
 * slice's nonzeros only (no child count); CSL slices count their fibers. */
void orc_hyb_bins(int nd, const u64* const* ptr, u64 nslc, u64 totNnz, int* bin_of) {
  const u64 TB = 512;
  u64 LB[10] = {0, 2, 4, 8, 16, 1024, 4 * TB, 8 * TB, 16 * TB, 32 * TB};
  u64 UB[10] = {1025, 5, 9, 17, 1025, 4 * TB + 1, 8 * TB + 1, 16 * TB + 1, 32 * TB + 1, totNnz + 1};
  for (u64 s = 0; s < nslc; ++s) {
    long long n = 0;
    for (u64 c = ptr[0][s]; c < ptr[0][s + 1]; ++c) {
      if (nd == 3) n += (long long)(ptr[1][c + 1] - ptr[1][c]);
      else
        for (u64 g = ptr[1][c]; g < ptr[1][c + 1]; ++g) n += (long long)(ptr[2][g + 1] - ptr[2][g]);
    }
    bin_of[s] = -1;
    for (int b = 0; b < 10; ++b)
      if ((u64)n > LB[b] && (u64)n < UB[b]) { bin_of[s] = b; break; }
  }
}

/* ---- COO MTTKRP: src/mttkrp_cpu.cpp:60-113 (MTTKRP_COO_CPU[_4D]).
 * Cyclic mode order (m + mode) % nd; U[mode] is accumulated into. Float
 * arithmetic in the reference's association order ((v*a)*b)*c, no FMA
 * contraction (compile with -ffp-contract=off). */
/* TTM_CPU (src/ttm_cpu.cpp:60-86) on a 3-D CSF: per leaf fiber f (fptr[f] ..
 * fptr[f+1]) an FP32 running sum over its nonzeros of vals[x] * U[leaf[x]],
 * added into y[f] (zeroed here). nfib real fibers (no sentinel row). */
void orc_ttm_f32(u64 nfib, const u64* fptr, const u64* leaf, const float* vals, const float* U, int R, float* y) {
  float tmp[1024];
  for (u64 f = 0; f < nfib; ++f) {
    for (int r = 0; r < R; ++r) tmp[r] = 0.f;
    for (u64 x = fptr[f]; x < fptr[f + 1]; ++x) {
      const float* u = U + leaf[x] * (u64)R;
      for (int r = 0; r < R; ++r) tmp[r] += vals[x] * u[r];
    }
    for (int r = 0; r < R; ++r) y[f * (u64)R + r] = 0.f + tmp[r];
  }
}

void orc_mttkrp_coo_f32(int nd, u64 nnz, u64* const* inds, const float* vals, int mode, int R,
                        float* const* U) {
  int cm[8];
  for (int m = 0; m < nd; ++m) cm[m] = (m + mode) % nd;
  for (u64 x = 0; x < nnz; ++x) {
    float* out = U[cm[0]] + inds[cm[0]][x] * (u64)R;
    const float* a = U[cm[1]] + inds[cm[1]][x] * (u64)R;
    const float* b = U[cm[2]] + inds[cm[2]][x] * (u64)R;
    if (nd == 3) {
      for (int r = 0; r < R; ++r) {
        float t = vals[x] * a[r] * b[r];
        out[r] += t;
      }
    } else {
      const float* c = U[cm[3]] + inds[cm[3]][x] * (u64)R;
      for (int r = 0; r < R; ++r) {
        float t = vals[x] * a[r] * b[r] * c[r];
        out[r] += t;
      }
    }
  }
}

/* FP64 MTTKRP over float inputs: the precision oracle. out is overwritten. */
void orc_mttkrp_coo_f64(int nd, u64 nnz, u64* const* inds, const float* vals, int mode, int R,
                        const float* const* U, const u64* dims, double* out) {
  memset(out, 0, dims[mode] * (u64)R * sizeof(double));
  for (u64 x = 0; x < nnz; ++x) {
    double* o = out + inds[mode][x] * (u64)R;
    for (int r = 0; r < R; ++r) {
      double t = (double)vals[x];
      for (int m = 0; m < nd; ++m)
        if (m != mode) t *= (double)U[m][inds[m][x] * (u64)R + r];
      o[r] += t;
    }
  }
}

/* ---- HB-CSF split: src/util.h:852-998 (create_HYB, 3-D) and
 * src/util.h:1000-1142 (create_HYB_4D). Input: a CSF built by
 * orc_create_csf (no fbrS split) over COO arrays sorted for that CSF.
 * Slices with one nonzero go to the COO part; (3-D only) slices whose fibers
 * all hold one nonzero go to the CSL part; the rest stay CSF. Outputs need
 * capacity nnz+2 each. counts[] = {COOnnz, CSLnnz, HCSRnnz, nCSLslc,
 * n hptr0, n hptr1, n hptr2, n hidx0, n hidx1, n hidx2}. */
void orc_create_hyb(int nd, u64 nnz, u64* const* inds, const float* vals, const int* order,
                    u64* const* ptr, u64* const* idx, const u64* nidx,
                    u64* const* cooInds, float* cooVals, u64* cslPtr, u64* cslIdx, u64* cslI1,
                    u64* cslI2, float* cslVals, u64* const* hptr, u64* const* hidx, u64* hLeaf,
                    float* hVals, u64* counts) {
  const u64 nslc = nidx[0];
  const int leaf = order[nd - 1];
  u64 cur = 0, curCSL = 0, curCOO = 0, usedCOO = 0, usedCSL = 0, usedH = 0;
  u64 nh[3] = {0, 0, 0}, nhi[3] = {0, 0, 0}, ncslSlc = 0;
  for (u64 s = 0; s < nslc; ++s) {
    u64 slcNnz = 0;
    int lenOne = 1;
    if (nd == 3) {
      for (u64 f = ptr[0][s]; f < ptr[0][s + 1]; ++f) {
        u64 fl = ptr[1][f + 1] - ptr[1][f];
        slcNnz += fl;
        if (fl > 1) lenOne = 0;
      }
    } else {
      for (u64 fs = ptr[0][s]; fs < ptr[0][s + 1]; ++fs)
        for (u64 f = ptr[1][fs]; f < ptr[1][fs + 1]; ++f) {
          u64 fl = ptr[2][f + 1] - ptr[2][f];
          slcNnz += fl;
          if (fl > 1) lenOne = 0;
        }
    }
    if (nd == 3) {
      const u64 stF = ptr[0][s], enF = ptr[0][s + 1];
      const u64 x0 = ptr[1][stF];
      if (slcNnz == 1) {
        cooInds[0][curCOO] = idx[0][s];
        cooInds[1][curCOO] = idx[1][stF];
        cooInds[2][curCOO] = inds[leaf][x0];
        cooVals[curCOO] = vals[x0];
        ++curCOO;
        ++usedCOO;
      } else if (lenOne) {
        cslPtr[ncslSlc] = ptr[0][s] - (usedCOO + usedH);
        cslIdx[ncslSlc] = idx[0][s];
        ++ncslSlc;
        for (u64 k = 0; k < slcNnz; ++k) {
          cslI1[curCSL + k] = idx[1][stF + k];
          cslI2[curCSL + k] = inds[leaf][x0 + k];
          cslVals[curCSL + k] = vals[x0 + k];
        }
        curCSL += slcNnz;
        usedCSL += enF - stF;
      } else {
        hptr[0][nh[0]++] = ptr[0][s] - (usedCOO + usedCSL);
        hidx[0][nhi[0]++] = idx[0][s];
        for (u64 f = stF; f < enF; ++f) {
          hptr[1][nh[1]++] = ptr[1][f] - (usedCOO + usedCSL);
          hidx[1][nhi[1]++] = idx[1][f];
        }
        for (u64 k = 0; k < slcNnz; ++k) {
          hLeaf[cur + k] = inds[leaf][x0 + k];
          hVals[cur + k] = vals[x0 + k];
        }
        cur += slcNnz;
        usedH += enF - stF;
      }
    } else {
      const u64 stS = ptr[0][s], enS = ptr[0][s + 1];
      const u64 stF = ptr[1][stS];
      const u64 x0 = ptr[2][stF];
      if (slcNnz == 1) {
        cooInds[0][curCOO] = idx[0][s];
        cooInds[1][curCOO] = idx[1][stS];
        cooInds[2][curCOO] = idx[2][stF];
        cooInds[3][curCOO] = inds[leaf][x0];
        cooVals[curCOO] = vals[x0];
        ++curCOO;
        ++usedCOO;
      } else {
        hptr[0][nh[0]++] = ptr[0][s] - usedCOO;
        hidx[0][nhi[0]++] = idx[0][s];
        for (u64 fs = stS; fs < enS; ++fs) {
          hptr[1][nh[1]++] = ptr[1][fs] - usedCOO;
          hidx[1][nhi[1]++] = idx[1][fs];
          for (u64 f = ptr[1][fs]; f < ptr[1][fs + 1]; ++f) {
            hptr[2][nh[2]++] = ptr[2][f] - usedCOO;
            hidx[2][nhi[2]++] = idx[2][f];
          }
        }
        for (u64 k = 0; k < slcNnz; ++k) {
          hLeaf[cur + k] = inds[leaf][x0 + k];
          hVals[cur + k] = vals[x0 + k];
        }
        cur += slcNnz;
      }
    }
  }
  if (nd == 3) {
    hptr[1][nh[1]++] = cur;
    hptr[0][nh[0]++] = nh[1] - 1;
    cslPtr[ncslSlc] = curCSL;
  } else {
    hptr[2][nh[2]++] = cur;
    hptr[1][nh[1]++] = nh[2] - 1;
    hptr[0][nh[0]++] = nh[1] - 1;
  }
  counts[0] = curCOO;
  counts[1] = curCSL;
  counts[2] = cur;
  counts[3] = ncslSlc;
  counts[4] = nh[0];
  counts[5] = nh[1];
  counts[6] = nh[2];
  counts[7] = nhi[0];
  counts[8] = nhi[1];
  counts[9] = nhi[2];
}

/* ---- MM-CSF partition heuristic: src/util.h:2167-2516 (mm_partition_reuseBased)
 * without the unconditional `mode = 2;` of :2517, nonzeros visited in order
 * (the reference's `omp for` on one thread). inds are X's arrays at the time
 * of the call (after the chain of per-mode sorts); orders[m] is arrX[m]'s
 * mode order; redun is Opt.redunMode; fbTh is Opt.MIfbTh (-h). Writes the
 * partition of every nonzero. Returns 0, or a negative code where the
 * reference would read or write out of bounds (-2: binarySearch1 runs off
 * the front, -3: a fiber number below 0, -4: a decrement of the redundant
 * mode's unallocated counters, -5: out of memory). */
typedef struct { u64 a, b, pos; } orc_ab;
static int ab_cmp(const void* x, const void* y) {
  const orc_ab* p = (const orc_ab*)x;
  const orc_ab* q = (const orc_ab*)y;
  if (p->a != q->a) return p->a < q->a ? -1 : 1;
  if (p->b != q->b) return p->b < q->b ? -1 : 1;
  return p->pos < q->pos ? -1 : (p->pos > q->pos);
}

/* binarySearch1 (src/util.h:2128-2141): ITYPE bounds, 32-bit unsigned midpoint */
static long long orc_bsearch1(const u64* arr, u64 len_avail, u64 left, u64 right, u64 value, int* err) {
  while (left <= right) {
    int middle = (int)(((unsigned int)left + (unsigned int)right) >> 1);
    if ((u64)(unsigned int)middle >= len_avail) { *err = -2; return 0; }
    if (arr[middle] == value) return middle;
    else if (arr[middle] > value) right = (u64)(long long)(middle - 1);
    else left = (u64)(long long)(middle + 1);
  }
  return -1;
}

typedef struct {
  u64 nfib;       /* distinct (o0, o1) groups: the reference's level-1 entries */
  u64* fidx1;     /* o1 of every group, then one extra entry (the next level-1 index read past the slice) */
  u64* cnt;       /* nnzPerFiber, nfib + 1 entries (the last stays 0) */
  u64* dsp;       /* denseSlcPtr, dims[o0] + 1 entries */
} orc_mode_csf;

int orc_mm_partition(int nd, u64 nnz, u64* const* inds, const u64* dims, const int orders[][8], const int* xorder,
                     int redun, int fbTh, int* part) {
  orc_mode_csf C[4];
  memset(C, 0, sizeof C);
  int rc = 0;
  /* nnzPerFiber / nnzPerSlice / denseSlcPtr per non-redundant mode (:2175-2240) */
  for (int m = 0; m < nd && rc == 0; ++m) {
    if (m == redun) continue;
    const int o0 = orders[m][0], o1 = orders[m][1];
    orc_ab* v = (orc_ab*)malloc((nnz ? nnz : 1) * sizeof(orc_ab));
    if (!v) { rc = -5; break; }
    for (u64 i = 0; i < nnz; ++i) { v[i].a = inds[o0][i]; v[i].b = inds[o1][i]; v[i].pos = i; }
    qsort(v, nnz, sizeof(orc_ab), ab_cmp);
    u64 nf = 0;
    for (u64 i = 0; i < nnz; ++i)
      if (i == 0 || v[i].a != v[i - 1].a || v[i].b != v[i - 1].b) ++nf;
    C[m].nfib = nf;
    C[m].fidx1 = (u64*)calloc(nf + 2, sizeof(u64));
    C[m].cnt = (u64*)calloc(nf + 2, sizeof(u64));
    C[m].dsp = (u64*)calloc(dims[o0] + 2, sizeof(u64));
    u64* sfirst = (u64*)calloc(nf + 2, sizeof(u64)); /* first group of each slice */
    u64* sidx = (u64*)calloc(nf + 2, sizeof(u64));
    if (!C[m].fidx1 || !C[m].cnt || !C[m].dsp || !sfirst || !sidx) { free(v); free(sfirst); free(sidx); rc = -5; break; }
    u64 g = 0, ns = 0;
    for (u64 i = 0; i < nnz; ++i) {
      const int newg = i == 0 || v[i].a != v[i - 1].a || v[i].b != v[i - 1].b;
      if (newg) {
        if (i == 0 || v[i].a != v[i - 1].a) { sfirst[ns] = g; sidx[ns] = v[i].a; ++ns; }
        C[m].fidx1[g] = v[i].b;
        ++g;
      }
      C[m].cnt[g - 1]++;
    }
    sfirst[ns] = nf;
    /* the entry after the last group: the reference's leaf-level sentinel is
       never reached by a search that stays inside the slices it covers */
    C[m].fidx1[nf] = 0;
    for (u64 s = 0; s < ns; ++s) {
      C[m].dsp[sidx[s]] = sfirst[s];
      C[m].dsp[sidx[s] + 1] = s == ns - 1 ? sfirst[s] : sfirst[s + 1]; /* :2203-2206 */
    }
    free(v);
    free(sfirst);
    free(sidx);
  }
  /* sameFm flags, shortMode / longMode (:2263-2308) */
  int s01 = 0, s02 = 0, s12 = 0, s03 = 0, s13 = 0, s23 = 0, shortMode = 0, longMode = -1;
  for (int m = 0; m < nd; ++m) {
    if (m == 1) {
      if (same_pair(orders[1], orders[0])) { s01 = 1; shortMode = dims[0] <= dims[1] ? 0 : 1; longMode = dims[0] <= dims[1] ? 1 : 0; }
    } else if (m == 2) {
      if (same_pair(orders[2], orders[0])) { s02 = 1; shortMode = dims[0] <= dims[2] ? 0 : 2; longMode = dims[0] <= dims[2] ? 2 : 0; }
      else if (same_pair(orders[2], orders[1])) { s12 = 1; shortMode = dims[1] <= dims[2] ? 1 : 2; longMode = dims[1] <= dims[2] ? 2 : 1; }
    } else if (m == 3) {
      if (same_pair(orders[3], orders[0])) { s03 = 1; shortMode = dims[0] <= dims[3] ? 0 : 3; longMode = dims[0] <= dims[3] ? 3 : 0; }
      else if (same_pair(orders[3], orders[1])) { s13 = 1; shortMode = dims[1] <= dims[3] ? 1 : 3; longMode = dims[1] <= dims[3] ? 3 : 1; }
      else if (same_pair(orders[3], orders[2])) { s23 = 1; shortMode = dims[2] <= dims[3] ? 2 : 3; longMode = dims[2] <= dims[3] ? 3 : 2; }
    }
  }
  const int shortestMode = dims[xorder[0]] <= dims[xorder[1]] ? xorder[0] : xorder[1]; /* :2261 */
  const u64 th = (u64)(long long)fbTh;
  /* the nonzero loop (:2331-2511) */
  for (u64 idx = 0; idx < nnz && rc == 0; ++idx) {
    u64 f[4] = {0, 0, 0, 0}, no[4] = {0, 0, 0, 0};
    for (int m = 0; m < nd && rc == 0; ++m) {
      if ((m == 1 && s01) || (m == 2 && s12) || (m == 3 && s23)) { f[m] = f[m - 1]; no[m] = 99999; }
      else if ((m == 2 && s02) || (m == 3 && s13)) { f[m] = f[m - 2]; no[m] = 99999; }
      else if (m == 3 && s03) { f[m] = f[m - 3]; no[m] = 99999; }
      else {
        if (m == redun) { rc = -4; break; }
        const u64 j = inds[orders[m][1]][idx];
        const u64 slc = inds[m][idx];
        const int n = (int)(C[m].dsp[slc + 1] - C[m].dsp[slc]);
        const u64 fbr = C[m].dsp[slc];
        int err = 0;
        long long r = orc_bsearch1(C[m].fidx1 + fbr, C[m].nfib + 1 - fbr, 0, (u64)(long long)n, j, &err);
        if (err) { rc = err; break; }
        const u64 at = (u64)r + fbr;
        if (at > C[m].nfib) { rc = -3; break; }
        f[m] = C[m].cnt[at];
        no[m] = at;
      }
    }
    if (rc) break;
    int mode = shortestMode, done = 0;
    if (nd == 3) {
      u64 mx;
      mx = f[1] > f[2] ? f[1] : f[2];
      if (f[0] >= th * mx) { done = 1; mode = (s01 || s02 || s03) ? shortMode : 0; }
      if (!done) { mx = f[0] > f[2] ? f[0] : f[2]; if (f[1] >= th * mx) { done = 1; mode = (s12 || s13) ? shortMode : 1; } }
      if (!done) { mx = f[0] > f[1] ? f[0] : f[1]; if (f[2] >= th * mx) { done = 1; mode = s23 ? shortMode : 2; } }
    } else {
      /* maxOf3(int, int, int) (:2142-2146) on ITYPE arguments, times an int */
      int a[4];
      for (int m = 0; m < 4; ++m) a[m] = (int)(unsigned int)f[m];
      for (int m = 0; m < 4 && !done; ++m) {
        int x = -1, y = -1, z = -1, k = 0, o[3];
        for (int q = 0; q < 4; ++q) if (q != m) o[k++] = a[q];
        x = o[0]; y = o[1]; z = o[2];
        int mx = x < y ? y : x;
        mx = mx < z ? z : mx;
        const int prod = (int)((unsigned int)fbTh * (unsigned int)mx);
        if (f[m] >= (u64)(long long)prod) {
          done = 1;
          if (m == 0) mode = (s01 || s02 || s03) ? shortMode : 0;
          else if (m == 1) mode = (s12 || s13) ? shortMode : 1;
          else if (m == 2) mode = s23 ? shortMode : 2;
          else mode = 3;
        }
      }
    }
    if (!done) mode = shortestMode;
    for (int i = 0; i < nd; ++i) {
      int dec;
      if (mode == shortMode) dec = i != shortMode && i != longMode;
      else dec = i != redun && i != mode;
      if (!dec) continue;
      if (i == redun || !C[i].cnt) { rc = -4; break; }
      C[i].cnt[no[i]]--;
    }
    part[idx] = mode;
  }
  for (int m = 0; m < 4; ++m) { free(C[m].fidx1); free(C[m].cnt); free(C[m].dsp); }
  return rc;
}
