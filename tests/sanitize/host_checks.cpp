// Host-side memory and undefined-behaviour checks (test infrastructure): built
// with -fsanitize=address,undefined by tests/test_host_sanitizers.py together
// with the library's host COO MTTKRP (mm-csf_b200/csrc/coo_host.cpp) and the
// oracle's C sources. Exercises the seeded generator, the sort, the CSF
// builder and both COO MTTKRPs on 3-D and 4-D tensors, and checks the host
// MTTKRP against the oracle: bit-exact with one thread, within FP32 rounding
// with several. Exit status 0 = clean; a sanitizer report aborts the run.
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "../../mm-csf_b200/csrc/common.h"

typedef uint64_t u64;
typedef uint32_t u32;
extern "C" {
int orc_generate(int nd, const u64* dims, u64 nnz, const int* dist, const double* zipf_s, int val_dist, u64 seed,
                 int threads, u32** inds, float* vals);
int orc_sort_coo(int nd, u64 nnz, u64* const* inds, float* vals, const int* keys, int nkeys);
void orc_order_modes(int nd, const u64* dims, int mode, int natural, int* order);
int orc_create_csf(int nd, u64 nnz, u64* const* inds, const int* order, u64 fbrTh, u64 fbrSTh, u64** ptr,
                   u64** idx, u64* nptr, u64* nidx);
void orc_mttkrp_coo_f32(int nd, u64 nnz, u64* const* inds, const float* vals, int mode, int R, float* const* U);
void orc_mttkrp_coo_f64(int nd, u64 nnz, u64* const* inds, const float* vals, int mode, int R,
                        const float* const* U, const u64* dims, double* out);
}

static int fail(const char* what) {
  std::fprintf(stderr, "FAIL: %s\n", what);
  return 1;
}

static int run_case(int nd, const u64* dims, u64 nnz, int R, u64 seed) {
  const int dist[4] = {1, 0, 1, 0};
  const double zs[4] = {1.2, 1.0, 1.1, 1.0};
  std::vector<std::vector<u32>> i32(nd, std::vector<u32>(nnz));
  std::vector<float> vals(nnz);
  u32* ip[4] = {nullptr, nullptr, nullptr, nullptr};
  for (int m = 0; m < nd; ++m) ip[m] = i32[m].data();
  if (orc_generate(nd, dims, nnz, dist, zs, 1, seed, 3, ip, vals.data()) != 0) return fail("orc_generate");
  for (int m = 0; m < nd; ++m)
    for (u64 x = 0; x < nnz; ++x)
      if (i32[m][x] >= dims[m]) return fail("generated index out of range");

  // library host COO MTTKRP against the oracle's, every mode
  mmcsf_coo X;
  X.nd = nd;
  X.nnz = nnz;
  for (int m = 0; m < nd; ++m) {
    X.dims[m] = dims[m];
    X.h_inds[m] = i32[m];
  }
  X.h_vals = vals;
  X.host_valid = true;
  std::vector<std::vector<u64>> i64(nd, std::vector<u64>(nnz));
  u64* ip64[4] = {nullptr, nullptr, nullptr, nullptr};
  for (int m = 0; m < nd; ++m) {
    for (u64 x = 0; x < nnz; ++x) i64[m][x] = i32[m][x];
    ip64[m] = i64[m].data();
  }
  std::vector<std::vector<float>> U(nd);
  srand((unsigned)seed);
  for (int m = 0; m < nd; ++m) {
    U[m].resize(dims[m] * (u64)R);
    for (auto& u : U[m]) u = (float)rand() / (float)RAND_MAX;
  }
  for (int mode = 0; mode < nd; ++mode) {
    std::vector<std::vector<float>> W = U;  // the oracle accumulates into the output factor in place
    std::fill(W[mode].begin(), W[mode].end(), 0.f);
    float* wp[4] = {nullptr, nullptr, nullptr, nullptr};
    const float* up[4] = {nullptr, nullptr, nullptr, nullptr};
    for (int m = 0; m < nd; ++m) {
      wp[m] = W[m].data();
      up[m] = U[m].data();
    }
    orc_mttkrp_coo_f32(nd, nnz, ip64, vals.data(), mode, R, wp);
    std::vector<float> out1(dims[mode] * (u64)R, 0.f), outT(dims[mode] * (u64)R, 0.f);
    if (mmcsf_mttkrp_coo_host(&X, mode, R, up, out1.data(), 1) != MMCSF_OK) return fail("host MTTKRP, 1 thread");
    if (std::memcmp(out1.data(), W[mode].data(), out1.size() * 4) != 0) return fail("1 thread not bit-exact");
    if (mmcsf_mttkrp_coo_host(&X, mode, R, up, outT.data(), 4) != MMCSF_OK) return fail("host MTTKRP, 4 threads");
    std::vector<double> ref(dims[mode] * (u64)R);
    orc_mttkrp_coo_f64(nd, nnz, ip64, vals.data(), mode, R, up, dims, ref.data());
    double num = 0, den = 0;
    for (size_t e = 0; e < ref.size(); ++e) {
      num += (outT[e] - ref[e]) * (outT[e] - ref[e]);
      den += ref[e] * ref[e];
    }
    if (std::sqrt(num / (den > 0 ? den : 1)) > 1e-5) return fail("4 threads outside 1e-5 of FP64");
  }
  // invalid arguments come back as errors
  std::vector<float> o(dims[0] * (u64)R);
  const float* up[4] = {U[0].data(), U[1].data(), U[2].data(), nd == 4 ? U[3].data() : nullptr};
  if (mmcsf_mttkrp_coo_host(&X, nd, R, up, o.data(), 1) != MMCSF_ERR_INVALID) return fail("bad mode accepted");
  if (mmcsf_mttkrp_coo_host(&X, 0, 0, up, o.data(), 1) != MMCSF_ERR_INVALID) return fail("R = 0 accepted");

  // sort and CSF construction for every mode (the oracle's builders)
  for (int mode = 0; mode < nd; ++mode) {
    int order[8];
    orc_order_modes(nd, dims, mode, 0, order);
    std::vector<std::vector<u64>> s64 = i64;
    std::vector<float> sv = vals;
    u64* sp[4] = {nullptr, nullptr, nullptr, nullptr};
    for (int m = 0; m < nd; ++m) sp[m] = s64[m].data();
    if (orc_sort_coo(nd, nnz, sp, sv.data(), order, nd) != 0) return fail("orc_sort_coo");
    std::vector<std::vector<u64>> ptr(nd - 1, std::vector<u64>(nnz + 2)), idx(nd - 1, std::vector<u64>(nnz + 2));
    u64* pp[8];
    u64* xp[8];
    for (int l = 0; l < nd - 1; ++l) {
      pp[l] = ptr[l].data();
      xp[l] = idx[l].data();
    }
    u64 nptr[8], nidx[8];
    if (orc_create_csf(nd, nnz, sp, order, 4, 128, pp, xp, nptr, nidx) != 0) return fail("orc_create_csf");
    if (ptr[nd - 2][nptr[nd - 2] - 1] != nnz) return fail("leaf pointers do not end at nnz");
  }
  return 0;
}

int main() {
  const u64 d3[3] = {300, 1000, 50};
  const u64 d4[4] = {60, 40, 200, 30};
  if (run_case(3, d3, 20000, 16, 7)) return 1;
  if (run_case(3, d3, 1, 8, 8)) return 1;  // one nonzero
  if (run_case(4, d4, 15000, 12, 9)) return 1;
  std::printf("host checks passed\n");
  return 0;
}
