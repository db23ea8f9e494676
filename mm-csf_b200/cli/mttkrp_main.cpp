// mttkrp — command-line driver with the reference's flags (src/util.h:3341-3442,
// src/mttkrp.cu:72-472), on top of the C ABI in include/mmcsf.h.
//
//   mttkrp -i X.tns [-m mode] [-R rank] [-t 1|8|10|12] [-f fiber-threshold]
//          [-w warps] [-b block] [-e budget] [-v 0|1] [-c 0|1] [-o out.txt]
//
// Differences from the reference, by design:
//   * errors print a message and return a nonzero exit status (the reference
//     exit(0)s);
//   * -t 1 runs the library's host COO MTTKRP (mmcsf_mttkrp_coo_host) on one
//     thread, the reference's loop in its order; like the reference it adds
//     to U[mode] = mode + 0.5 without zeroing it (src/mttkrp.cu:89-92, 105-109);
//   * -w keeps its meaning, w warps per fiber (src/util.h:194,
//     src/mttkrp_gpu.cu:3616-3630): the reference launches w warps for each
//     of the F fibers and every warp takes a share of one fiber's nonzeros.
//     The kernels here walk nonzero-balanced chunks instead of fibers, so -w
//     sets the chunk that gives the same number of workers: with G lanes per
//     factor row (32/G teams per warp), chunk = max(1, N*G / (32*w*F))
//     nonzeros per team. Without -w the per-mode autotuner chooses, and
//     without -f as well it also picks -f among none, 128 and 32 (each
//     candidate format built and tuned, mmcsf_autotune); -e (no counterpart
//     in the reference) lets it run modes on BF16 factor copies within that
//     error budget;
//   * -o writes the output of mode -m (every mode is computed for -t 12);
//   * -i accepts a binary COO file (name ending in .bin, mmcsf_coo_write_bin).
// Factors are the reference's non-CPD constants U[m] = m + 0.5
// (src/util.h:3209-3227), so printed values are directly comparable.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "mmcsf.h"

namespace {

struct Options {  // the reference's Options fields this driver uses (src/util.h:189-236)
  int R = 32, mode = 0, impType = 1, warpPerSlice = 0, TBsize = 0, MIfbTh = 1, partitionRule = 0;
  uint64_t fbrThreashold = 0;
  double errBudget = 0;  // -e: BF16-factor error budget for the per-mode precision tuner (0: FP32 only)
  bool verbose = false, correctness = false;
  std::string inFileName, outFileName;
};

void usage() {
  std::printf(
      "options:\n"
      "        -R rank/feature : set the rank (default 32)\n"
      "        -m mode : set the mode of MTTKRP (default 0, MM-CSF evaluates all modes)\n"
      "        -t implementation type: 1: COO on CPU 8: B-CSF 10: HB-CSF 12: MM-CSF on GPU\n"
      "        -f fiber-splitting threshold: maximum nonzeros per fiber (default none)\n"
      "        -h MM-CSF partition ratio: a mode takes a nonzero when its fiber is h times the others' (default 1)\n"
      "        -P MM-CSF partition rule: 0 all nonzeros to partition 2 as the reference ships (default),\n"
      "           1 the reference's partition heuristic decides\n"
      "        -w warps per fiber: as many workers as w warps for every fiber (default: autotuned)\n"
      "        -e error budget: without -w, run modes on BF16 factor copies where faster and within this\n"
      "           relative change of their output (default 0: FP32 only). Without -w and -f the tuner also\n"
      "           picks -f among none, 128 and 32 (-v 1 prints the choice)\n"
      "        -b threads per CTA (default 256)\n"
      "        -v verbose: 1 to enable\n"
      "        -c correctness: 1 to check the last mode against a host COO MTTKRP\n"
      "        -i input file name (.tns)\n"
      "        -o output file name\n");
}

bool parse(int argc, char** argv, Options& o) {
  for (int i = 1; i < argc; i++) {
    if (argv[i][0] != '-' || i + 1 >= argc) return false;
    const char c = argv[i][1];
    const char* v = argv[++i];
    switch (c) {
      case 'R': o.R = std::atoi(v); break;
      case 'm': o.mode = std::atoi(v); break;
      case 't': o.impType = std::atoi(v); break;
      case 'w': o.warpPerSlice = std::atoi(v); break;
      case 'f': o.fbrThreashold = std::strtoull(v, nullptr, 10); break;
      case 'b': o.TBsize = std::atoi(v); break;
      case 'v': o.verbose = std::atoi(v) == 1; break;
      case 'c': o.correctness = std::atoi(v) == 1; break;
      case 'i': o.inFileName = v; break;
      case 'o': o.outFileName = v; break;
      case 'h': o.MIfbTh = std::atoi(v); break;
      case 'P': o.partitionRule = std::atoi(v); break;
      case 'e': o.errBudget = std::atof(v); break;
      case 's': case 'g': case 'l': case 'p': case 'q': case 'r': break;  // accepted, unused
      default: std::fprintf(stderr, "unknown option: -%c\n", c); return false;
    }
  }
  return !o.inFileName.empty();
}

int fail(const char* what, int st) {
  std::fprintf(stderr, "%s failed: %s (%s)\n", what, mmcsf_status_string(st), mmcsf_last_error());
  return 1;
}

// -t 1: the COO CPU path (src/mttkrp.cu:105-109) on the reference's
// constant factors; U[mode] keeps its initial mode + 0.5 (never zeroed).
int coo_cpu(const Options& o, mmcsf_coo* X, int nd, const uint64_t* dims) {
  const int R = o.R;
  std::vector<std::vector<float>> U(nd);
  std::vector<const float*> fac(nd);
  for (int m = 0; m < nd; ++m) {
    U[m].assign(dims[m] * (uint64_t)R, (float)m + 0.5f);
    fac[m] = U[m].data();
  }
  int st = mmcsf_coo_to_host(X);
  if (st) return fail("host copy", st);
  auto t0 = std::chrono::steady_clock::now();
  st = mmcsf_mttkrp_coo_host(X, o.mode, R, fac.data(), U[o.mode].data(), 1);
  const double sec = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  if (st) return fail("COO CPU MTTKRP", st);
  std::printf("COO CPU - time: %.3f sec \n", sec);
  if (!o.outFileName.empty()) {
    FILE* fo = std::fopen(o.outFileName.c_str(), "w");
    if (!fo) { std::fprintf(stderr, "cannot write %s\n", o.outFileName.c_str()); return 1; }
    std::fprintf(fo, "%llu x %d matrix\n", (unsigned long long)dims[o.mode], R);
    for (uint64_t i = 0; i < dims[o.mode]; ++i) {
      for (int j = 0; j < R; ++j) std::fprintf(fo, "%.2f\t", U[o.mode][i * R + j]);
      std::fprintf(fo, "\n");
    }
    std::fclose(fo);
  }
  mmcsf_coo_destroy(X);
  return 0;
}

}  // namespace

int main(int argc, char** argv) {
  Options o;
  if (!parse(argc, argv, o)) {
    usage();
    return 1;
  }
  if (o.impType != MMCSF_IMPL_COO_CPU && o.impType != MMCSF_IMPL_MMCSF && o.impType != MMCSF_IMPL_BCSF &&
      o.impType != MMCSF_IMPL_HBCSF) {
    std::fprintf(stderr, "-t %d is not provided by this library (1: COO CPU; GPU formats: 8, 10, 12)\n",
                 o.impType);
    return 1;
  }
  mmcsf_coo* X = nullptr;
  const std::string& in = o.inFileName;
  const bool bin = in.size() > 4 && in.compare(in.size() - 4, 4, ".bin") == 0;
  int st = bin ? mmcsf_coo_load_bin(in.c_str(), &X) : mmcsf_coo_load_tns(in.c_str(), &X);
  if (st) return fail("load_tensor", st);
  int nd = 0;
  uint64_t dims[4] = {0, 0, 0, 0}, nnz = 0;
  mmcsf_coo_info(X, &nd, dims, &nnz);
  if (o.mode < 0 || o.mode >= nd) {
    std::fprintf(stderr, "Mode cannot be larger than tensor dimension.\n");
    return 1;
  }
  if (o.impType == MMCSF_IMPL_COO_CPU) return coo_cpu(o, X, nd, dims);
  mmcsf_build_opts bo{};
  bo.impl = o.impType;
  bo.mode = o.impType == MMCSF_IMPL_MMCSF ? 0 : o.mode;  // check_opt forces mode 0 for -t 12
  bo.fiber_threshold = o.fbrThreashold;
  bo.views = o.impType == MMCSF_IMPL_MMCSF ? 1 : 0;
  bo.partition_rule = o.impType == MMCSF_IMPL_MMCSF ? o.partitionRule : 0;
  bo.partition_ratio = o.MIfbTh;
  cudaStream_t s = nullptr;
  mmcsf_format* F = nullptr;
  const int R = o.R;
  std::vector<float*> dU(nd), dOut(nd);
  std::vector<std::vector<float>> hU(nd);
  for (int m = 0; m < nd; ++m) {
    hU[m].assign(dims[m] * (uint64_t)R, (float)m + 0.5f);
    cudaMalloc(&dU[m], dims[m] * (uint64_t)R * 4);
    cudaMalloc(&dOut[m], dims[m] * (uint64_t)R * 4);
    cudaMemcpy(dU[m], hU[m].data(), dims[m] * (uint64_t)R * 4, cudaMemcpyHostToDevice);
  }
  const void* fac[4] = {dU[0], dU[1], dU[2], nd == 4 ? dU[3] : nullptr};
  const float* facf[4] = {dU[0], dU[1], dU[2], nd == 4 ? dU[3] : nullptr};
  // without -w and -f the tuner also picks -f (each candidate format built and tuned)
  const bool autotune = o.warpPerSlice <= 0 && o.fbrThreashold == 0;
  mmcsf_plan plan{};
  auto t0 = std::chrono::steady_clock::now();
  if (autotune) {
    if ((st = mmcsf_autotune(X, &bo, nullptr, 0, R, facf, dOut.data(), o.errBudget, s, &F, &plan)))
      return fail("autotune", st);
  } else {
    if ((st = mmcsf_build(X, &bo, s, &F))) return fail("format construction", st);
  }
  double build_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
  if (o.verbose) std::printf("format construction (device)%s: %.3f ms\n", autotune ? " and autotuning" : "", build_ms);
  if (o.verbose && autotune)
    std::printf("autotuned -f %d%s\n", plan.fiber_threshold, plan.fiber_threshold ? "" : " (no split)");

  mmcsf_kernel_cfg cfg{};
  if (o.warpPerSlice > 0) {
    // workers of the reference's launch: w warps per fiber, summed over the partitions
    uint64_t fibers = 0;
    for (int p = 0; p < (o.impType == MMCSF_IMPL_MMCSF ? nd : 1); ++p) {
      mmcsf_part_info pi{};
      if (mmcsf_format_info(F, p, &pi) == MMCSF_OK && pi.present) fibers += pi.n_fibers;
    }
    const int R4 = (R + 3) / 4;
    const uint64_t G = R4 >= 32 ? 32 : (R4 >= 16 ? 16 : (R4 >= 8 ? 8 : (R4 >= 4 ? 4 : (R4 >= 2 ? 2 : 1))));
    const uint64_t workers = 32ull * (uint64_t)o.warpPerSlice * (fibers ? fibers : 1);
    cfg.chunk = (int)std::max<uint64_t>(1, std::min<uint64_t>(1u << 20, nnz * G / workers));
    if (o.verbose) std::printf("-w %d: %llu nonzeros per worker team\n", o.warpPerSlice, (unsigned long long)cfg.chunk);
  }
  if (o.TBsize > 0) cfg.block_threads = o.TBsize;
  const int nmodes = o.impType == MMCSF_IMPL_MMCSF ? nd : 1;
  if (!autotune && o.warpPerSlice <= 0) {
    st = (o.impType == MMCSF_IMPL_MMCSF && o.errBudget > 0)
             ? mmcsf_tune_precision(F, R, facf, dOut.data(), o.errBudget, s, &plan)
             : mmcsf_tune(F, R, MMCSF_DTYPE_F32, fac, dOut.data(), s, &plan);
    if (st) return fail("autotune", st);
  }
  if (o.verbose && o.warpPerSlice <= 0 && plan.mixed)
    for (int m = 0; m < nd; ++m)
      std::printf("mode %d: %s factors (relative change %.2e)\n", m,
                  plan.mode_dtype[m] == MMCSF_DTYPE_BF16 ? "BF16" : "FP32", plan.bf16_error[m]);
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  float total = 0;
  const bool all_call = o.impType == MMCSF_IMPL_MMCSF && o.warpPerSlice <= 0;
  if (all_call) {  // the tuned all-mode call (two-output walk, per-mode precision)
    cudaEventRecord(e0, s);
    if ((st = mmcsf_mttkrp_all(F, R, MMCSF_DTYPE_F32, fac, dOut.data(), nullptr, s))) return fail("MTTKRP", st);
    cudaEventRecord(e1, s);
    cudaEventSynchronize(e1);
    cudaEventElapsedTime(&total, e0, e1);
  }
  for (int q = 0; q < nmodes && !all_call; ++q) {
    const int m = o.impType == MMCSF_IMPL_MMCSF ? q : o.mode;
    cudaEventRecord(e0, s);
    if ((st = mmcsf_mttkrp(F, m, R, MMCSF_DTYPE_F32, fac, dOut[m], o.warpPerSlice > 0 ? &cfg : nullptr, s)))
      return fail("MTTKRP", st);
    cudaEventRecord(e1, s);
    cudaEventSynchronize(e1);
    float ms = 0;
    cudaEventElapsedTime(&ms, e0, e1);
    total += ms;
    if (o.verbose) std::printf("mode %d: %.3f ms\n", m, ms);
  }
  // totals over the partitions, as src/mttkrp_gpu.cu:3740-3766 prints them
  unsigned long long tslc = 0, tsfib = 0, tfib = 0, tnnz = 0;
  for (int p = 0; p < (o.impType == MMCSF_IMPL_MMCSF ? nd : 1); ++p) {
    mmcsf_part_info pi{};
    mmcsf_format_info(F, p, &pi);
    if (!pi.present) continue;
    tslc += pi.n_slices;
    tsfib += pi.n_fbrs + 1;
    tfib += pi.n_fibers + 1;
    tnnz += pi.nnz;
    if (o.verbose) std::printf("partition %d: %llu nonzeros\n", p, (unsigned long long)pi.nnz);
  }
  std::printf("Total GPU time: %f", total);
  if (nd == 3)
    std::printf(" nSlc:%llu, nFibers:%llu, nnz:%llu\n", tslc, tfib, tnnz);
  else
    std::printf(" nSlc:%llu, nSFibers:%llu, nFibers:%llu, nnz:%llu\n", tslc, tsfib, tfib, tnnz);

  const int check_mode = o.impType == MMCSF_IMPL_MMCSF ? nd - 1 : o.mode;
  std::vector<float> res(dims[check_mode] * (uint64_t)R);
  cudaMemcpy(res.data(), dOut[check_mode], res.size() * 4, cudaMemcpyDeviceToHost);
  if (o.correctness) {
    // host COO MTTKRP in double (src/util.h:3285-3311 compares with |diff| > 0.1)
    const uint32_t* inds[4];
    const float* vals;
    mmcsf_coo_to_host(X);
    mmcsf_coo_host_arrays(X, inds, &vals);
    std::vector<double> ref(res.size(), 0.0);
    for (uint64_t x = 0; x < nnz; ++x) {
      double p = vals[x];
      for (int m = 0; m < nd; ++m)
        if (m != check_mode) p *= (double)m + 0.5;
      for (int r = 0; r < R; ++r) ref[(uint64_t)inds[check_mode][x] * R + r] += p;
    }
    uint64_t mism = 0;
    double maxd = 0;
    for (size_t i = 0; i < res.size(); ++i) {
      double d = std::fabs(res[i] - ref[i]);
      if (d > 1e-5 * std::fabs(ref[i]) + 1e-6) ++mism;
      if (d > maxd) maxd = d;
    }
    if (mism == 0) std::printf("Correctness pass!\n");
    else std::printf("%llu mismatches; maximum diff %g\n", (unsigned long long)mism, maxd);
  }
  if (!o.outFileName.empty()) {
    std::vector<float> om(dims[o.mode] * (uint64_t)R);
    cudaMemcpy(om.data(), dOut[o.mode], om.size() * 4, cudaMemcpyDeviceToHost);
    FILE* fo = std::fopen(o.outFileName.c_str(), "w");
    if (!fo) { std::fprintf(stderr, "cannot write %s\n", o.outFileName.c_str()); return 1; }
    std::fprintf(fo, "%llu x %d matrix\n", (unsigned long long)dims[o.mode], R);
    for (uint64_t i = 0; i < dims[o.mode]; ++i) {
      for (int j = 0; j < R; ++j) std::fprintf(fo, "%.2f\t", om[i * R + j]);
      std::fprintf(fo, "\n");
    }
    std::fclose(fo);
  }
  for (int m = 0; m < nd; ++m) { cudaFree(dU[m]); cudaFree(dOut[m]); }
  mmcsf_format_destroy(F);
  mmcsf_coo_destroy(X);
  return 0;
}
