// Test infrastructure, not product code.
//
// Harness linked against a patched build of the reference (isratnisa/MM-CSF)
// so the reference's own host code can serve as the oracle for format
// construction and for the COO CPU MTTKRP. Only tests/, the golden-fixture
// script and bench.py's CPU-baseline leg load the library this builds.
//
// Each entry point replays, call for call, the sequence the reference's
// `main` runs for one implementation type (src/mttkrp.cu:72-389) and dumps
// every array it builds to a text file: one line per array,
// "<name> <count> v0 v1 ...".
#include "util.h"
#include "mttkrp_cpu.h"
#include "ttm_cpu.h"

#include <cstdio>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <omp.h>
#include <new>

// Zero-filled, padded allocations. The reference reads one element past the
// end of its index arrays while scanning the last fiber (src/util.h:1366-1374,
// src/util.h:800-806); padding makes that read land in owned, zeroed memory so
// the dump is deterministic.
void* operator new[](std::size_t n) {
  void* p = std::calloc(1, n + 64);
  if (!p) throw std::bad_alloc();
  return p;
}
void operator delete[](void* p) noexcept { std::free(p); }
void operator delete[](void* p, std::size_t) noexcept { std::free(p); }

namespace {

void dump_vec(FILE* f, const char* name, const std::vector<ITYPE>& v) {
  std::fprintf(f, "%s %zu", name, v.size());
  for (ITYPE x : v) std::fprintf(f, " %zu", (size_t)x);
  std::fprintf(f, "\n");
}
void dump_arr(FILE* f, const char* name, const ITYPE* a, size_t n) {
  std::fprintf(f, "%s %zu", name, n);
  for (size_t i = 0; i < n; ++i) std::fprintf(f, " %zu", (size_t)a[i]);
  std::fprintf(f, "\n");
}
void dump_vals(FILE* f, const char* name, const DTYPE* a, size_t n) {
  std::fprintf(f, "%s %zu", name, n);
  for (size_t i = 0; i < n; ++i) std::fprintf(f, " %.9g", (double)a[i]);
  std::fprintf(f, "\n");
}

void dump_tiled(FILE* f, const TiledTensor& T, const char* pfx, bool with_fbr_like) {
  char nm[128];
  std::fprintf(f, "%s.nnz 1 %zu\n", pfx, (size_t)T.totNnz);
  std::snprintf(nm, sizeof nm, "%s.modeOrder", pfx);
  dump_vec(f, nm, T.modeOrder);
  for (size_t l = 0; l < T.fbrPtr.size(); ++l) {
    std::snprintf(nm, sizeof nm, "%s.fbrPtr%zu", pfx, l);
    dump_vec(f, nm, T.fbrPtr[l]);
    std::snprintf(nm, sizeof nm, "%s.fbrIdx%zu", pfx, l);
    dump_vec(f, nm, T.fbrIdx[l]);
  }
  std::fprintf(f, "%s.nFibers 1 %zu\n", pfx, (size_t)T.nFibers);
  if (with_fbr_like && T.nFibers > 0) {
    // Only the first nFibers-1 entries are written by the reference
    // (src/util.h:1768-1783); the last one is uninitialised.
    std::snprintf(nm, sizeof nm, "%s.fbrLikeSlcInds", pfx);
    dump_arr(f, nm, T.fbrLikeSlcInds, T.nFibers - 1);
  }
  for (size_t m = 0; m < T.ndims; ++m) {
    std::snprintf(nm, sizeof nm, "%s.inds%zu", pfx, m);
    dump_arr(f, nm, T.inds[m], T.totNnz);
  }
  std::snprintf(nm, sizeof nm, "%s.vals", pfx);
  dump_vals(f, nm, T.vals, T.totNnz);
}

Options make_opts(const char* tns, int impType, int mode, long fbrTh) {
  Options Opt;
  Opt.inFileName = tns;
  Opt.impType = impType;
  Opt.mode = mode;
  if (fbrTh > 0) Opt.fbrThreashold = fbrTh;
  return Opt;
}

}  // namespace

extern "C" {

// OpenMP threads for the builders (1 makes the partition heuristic's nonzero
// loop run in order; it decrements shared counters).
void ref_set_threads(int n) { omp_set_num_threads(n); }

// mttkrp -t 12 (MM-CSF): src/mttkrp.cu:72-389, with -h (Opt.MIfbTh, the
// partition heuristic's fiber ratio; it decides only in the build without
// the partition override).
int ref_mmcsf_dump_h(const char* tns, int mode, long fbrTh, long mifbTh, const char* out) {
  Options Opt = make_opts(tns, 12, mode, fbrTh);
  Opt.MIfbTh = mifbTh;
  Tensor X;
  load_tensor(X, Opt);
  sort_COOtensor(X);
  check_opt(X, Opt);

  int redunMode = -1;
  Tensor* arrX = new Tensor[X.ndims];
  for (int m = 0; m < (int)X.ndims; ++m) {
    init_tensor(arrX, X, Opt, m);
    if (m == 1) {
      if (arrX[m].modeOrder[1] == arrX[m - 1].modeOrder[0] && arrX[m].modeOrder[0] == arrX[m - 1].modeOrder[1])
        redunMode = m;
    } else if (m == 2) {
      if ((arrX[m].modeOrder[1] == arrX[m - 2].modeOrder[0] && arrX[m].modeOrder[0] == arrX[m - 2].modeOrder[1]) ||
          (arrX[m].modeOrder[1] == arrX[m - 1].modeOrder[0] && arrX[m].modeOrder[0] == arrX[m - 1].modeOrder[1]))
        redunMode = m;
    } else if (m == 3) {
      if ((arrX[m].modeOrder[1] == arrX[m - 3].modeOrder[0] && arrX[m].modeOrder[0] == arrX[m - 3].modeOrder[1]) ||
          (arrX[m].modeOrder[1] == arrX[m - 2].modeOrder[0] && arrX[m].modeOrder[0] == arrX[m - 2].modeOrder[1]) ||
          (arrX[m].modeOrder[1] == arrX[m - 1].modeOrder[0] && arrX[m].modeOrder[0] == arrX[m - 1].modeOrder[1]))
        redunMode = m;
    }
    if (m != redunMode) sort_COOtensor(arrX[m]);
    if (m != redunMode) create_HCSR(arrX[m], Opt);
  }
  Opt.redunMode = redunMode;

  TiledTensor* MTX = new TiledTensor[X.ndims];
  mm_partition_reuseBased(arrX, X, MTX, Opt);
  populate_paritions(X, MTX);
  for (int m = 0; m < (int)X.ndims; ++m) {
    if (MTX[m].totNnz > 0) {
      sort_MI_CSF(X, MTX, m);
      create_TiledHCSR(MTX, Opt, m);
      create_fbrLikeSlcInds(MTX, m);
    }
  }

  FILE* f = std::fopen(out, "w");
  if (!f) return 1;
  std::fprintf(f, "redunMode 1 %d\n", redunMode);
  std::fprintf(f, "X.modeOrder %zu", X.modeOrder.size());
  for (auto v : X.modeOrder) std::fprintf(f, " %zu", (size_t)v);
  std::fprintf(f, "\n");
  for (int m = 0; m < (int)X.ndims; ++m) {
    char pfx[32];
    std::snprintf(pfx, sizeof pfx, "part%d", m);
    if (MTX[m].totNnz > 0) {
      dump_tiled(f, MTX[m], pfx, true);
    } else {
      std::fprintf(f, "%s.nnz 1 0\n", pfx);
      std::snprintf(pfx, sizeof pfx, "part%d.modeOrder", m);
      dump_vec(f, pfx, MTX[m].modeOrder);
    }
  }
  std::fclose(f);
  return 0;
}

int ref_mmcsf_dump(const char* tns, int mode, long fbrTh, const char* out) {
  return ref_mmcsf_dump_h(tns, mode, fbrTh, 1, out);
}

// mttkrp -t 8 (B-CSF): src/mttkrp.cu:72-100 and :167-236.
int ref_bcsf_dump(const char* tns, int mode, long fbrTh, const char* out) {
  Options Opt = make_opts(tns, 8, mode, fbrTh);
  Tensor X;
  load_tensor(X, Opt);
  sort_COOtensor(X);
  check_opt(X, Opt);
  create_HCSR(X, Opt);
  TiledTensor TiledX[1];
  make_KTiling(X, TiledX, Opt);
  if (TiledX[0].totNnz > 0) create_TiledHCSR(TiledX, Opt, 0);
  if (TiledX[0].totNnz > 0) make_TiledBin(TiledX, Opt, 0);
  create_fbrLikeSlcInds(TiledX, 0);

  FILE* f = std::fopen(out, "w");
  if (!f) return 1;
  dump_tiled(f, TiledX[0], "bcsf", true);
  for (size_t b = 0; b < TiledX[0].slcMapperBin.size(); ++b) {
    char nm[64];
    std::snprintf(nm, sizeof nm, "bcsf.bin%zu", b);
    dump_vec(f, nm, TiledX[0].slcMapperBin[b]);
  }
  std::fclose(f);
  return 0;
}

// mttkrp -t 10 (HB-CSF): src/mttkrp.cu:138-151.
int ref_hyb_dump(const char* tns, int mode, long fbrTh, const char* out) {
  Options Opt = make_opts(tns, 10, mode, fbrTh);
  Tensor X;
  load_tensor(X, Opt);
  sort_COOtensor(X);
  check_opt(X, Opt);
  create_HCSR(X, Opt);
  HYBTensor H(X);
  if (X.ndims == 3) create_HYB(H, X, Opt); else create_HYB_4D(H, X, Opt);
  make_HybBin(H, Opt);

  FILE* f = std::fopen(out, "w");
  if (!f) return 1;
  std::fprintf(f, "hyb.COOnnz 1 %zu\nhyb.CSLnnz 1 %zu\nhyb.HCSRnnz 1 %zu\n", (size_t)H.COOnnz,
               (size_t)H.CSLnnz, (size_t)H.HCSRnnz);
  dump_vec(f, "hyb.modeOrder", H.modeOrder);
  char nm[64];
  for (size_t m = 0; m < H.ndims; ++m) {
    std::snprintf(nm, sizeof nm, "hyb.COOinds%zu", m);
    dump_arr(f, nm, H.COOinds[H.modeOrder[m]], H.COOnnz);
  }
  dump_vals(f, "hyb.COOvals", H.COOvals, H.COOnnz);
  if (H.ndims == 3) {
    dump_vec(f, "hyb.CSLslicePtr", H.CSLslicePtr);
    dump_vec(f, "hyb.CSLsliceIdx", H.CSLsliceIdx);
    dump_arr(f, "hyb.CSLinds1", H.CSLinds[H.modeOrder[1]], H.CSLnnz);
    dump_arr(f, "hyb.CSLinds2", H.CSLinds[H.modeOrder[2]], H.CSLnnz);
    dump_vals(f, "hyb.CSLvals", H.CSLvals, H.CSLnnz);
  }
  for (size_t l = 0; l < H.fbrPtr.size(); ++l) {
    std::snprintf(nm, sizeof nm, "hyb.fbrPtr%zu", l);
    dump_vec(f, nm, H.fbrPtr[l]);
    std::snprintf(nm, sizeof nm, "hyb.fbrIdx%zu", l);
    dump_vec(f, nm, H.fbrIdx[l]);
  }
  dump_arr(f, "hyb.indsLeaf", H.inds[H.modeOrder[H.ndims - 1]], H.HCSRnnz);
  dump_vals(f, "hyb.vals", H.vals, H.HCSRnnz);
  for (size_t b = 0; b < H.slcMapperBin.size(); ++b) {
    std::snprintf(nm, sizeof nm, "hyb.bin%zu", b);
    dump_vec(f, nm, H.slcMapperBin[b]);
  }
  if (H.ndims == 3) {
    for (size_t b = 0; b < H.CSLslcMapperBin.size(); ++b) {
      std::snprintf(nm, sizeof nm, "hyb.cslbin%zu", b);
      dump_vec(f, nm, H.CSLslcMapperBin[b]);
    }
  }
  std::fclose(f);
  return 0;
}

// MTTKRP_COO_CPU / MTTKRP_COO_CPU_4D (src/mttkrp_cpu.cpp:60-113) on caller
// arrays. inds[m] are 0-based uint64 per mode; factors[m] are row-major
// dims[m] x R float. factors[mode] is the output and is accumulated into, as
// the reference does: callers zero it first for a plain MTTKRP.
// ttm (src/ttm.cu:55-229 with the -f split of create_HCSR): TTM_CPU on the
// CSF of `mode` after the reference's sort. Y holds up to cap x R floats;
// *nfib gets the number of real fibers (the reference's Y has one more,
// unused, sentinel row).
int ref_ttm(const char* tns, int mode, long fbrTh, int R, const float* u_leaf, float* y, uint64_t cap,
            uint64_t* nfib) {
  Options Opt = make_opts(tns, 8, mode, fbrTh);
  Opt.R = R;
  Tensor X;
  load_tensor(X, Opt);
  sort_COOtensor(X);
  check_opt(X, Opt);
  create_HCSR(X, Opt);
  const ITYPE leaf = X.modeOrder[X.ndims - 1];
  Matrix* U = new Matrix[X.ndims];
  for (int m = 0; m < (int)X.ndims; ++m) {
    U[m].nRows = X.dims[m];
    U[m].nCols = R;
    U[m].vals = static_cast<DTYPE*>(std::calloc((size_t)X.dims[m] * R, sizeof(DTYPE)));
  }
  std::memcpy(U[leaf].vals, u_leaf, (size_t)X.dims[leaf] * R * sizeof(float));
  semiSpTensor Y;
  Y.nRows = X.nFibers;
  Y.nCols = R;
  Y.vals = static_cast<DTYPE*>(std::calloc((size_t)X.nFibers * R, sizeof(DTYPE)));
  TTM_CPU(X, Y, U, Opt);
  const uint64_t F = X.nFibers ? X.nFibers - 1 : 0;
  *nfib = F;
  if (F <= cap) std::memcpy(y, Y.vals, (size_t)F * R * sizeof(float));
  for (int m = 0; m < (int)X.ndims; ++m) std::free(U[m].vals);
  delete[] U;
  std::free(Y.vals);
  return F <= cap ? 0 : 1;
}

int ref_coo_mttkrp(int nd, const uint64_t* dims, uint64_t nnz, const uint64_t* const* inds,
                   const float* vals, int mode, int R, float* const* factors) {
  if (nd != 3 && nd != 4) return 1;
  Tensor X;
  X.ndims = nd;
  X.dims = new ITYPE[nd];
  X.totNnz = nnz;
  X.inds = new ITYPE*[nd];
  for (int m = 0; m < nd; ++m) {
    X.dims[m] = dims[m];
    X.inds[m] = const_cast<ITYPE*>(reinterpret_cast<const ITYPE*>(inds[m]));
  }
  X.vals = const_cast<DTYPE*>(vals);
  Matrix U[4];
  for (int m = 0; m < nd; ++m) {
    U[m].nRows = dims[m];
    U[m].nCols = R;
    U[m].vals = factors[m];
  }
  Options Opt;
  Opt.R = R;
  Opt.mode = mode;
  if (nd == 3) MTTKRP_COO_CPU(X, U, Opt); else MTTKRP_COO_CPU_4D(X, U, Opt);
  delete[] X.inds;
  delete[] X.dims;
  return 0;
}

}  // extern "C"
