// ttm — command-line driver with the reference's ttm flags (src/ttm.cu:55-229,
// src/util.h:3341-3442) on top of the C ABI in include/mmcsf.h.
//
//   ttm -i X.tns [-m mode] [-R rank] [-t 2|3] [-f fiber-threshold] [-c 0|1] [-o Y.txt]
//
// Computes, on the device, the semi-sparse Y (one R-vector per fiber of the
// mode's CSF) with the leaf mode's factor set to the reference's constants
// U[m] = m + 0.5 (src/util.h:3209-3227), prints the reference's
// "TTM GPU - time" line and writes Y like write_output_ttmY
// (src/util.h:3239-3252), without the reference's unused sentinel row.
// Differences, by design: the input need not be pre-sorted for the mode (the
// reference's ttm refuses files whose name lacks the mode digit); errors end
// with a message and a nonzero status; -t 1 (serial CPU) is not provided.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <string>
#include <vector>

#include "mmcsf.h"

int main(int argc, char** argv) {
  int R = 32, mode = 0, impType = 2;
  uint64_t fth = 0;
  bool check = false;
  std::string in, out;
  for (int i = 1; i + 1 < argc; i += 2) {
    const char c = argv[i][0] == '-' ? argv[i][1] : 0;
    const char* v = argv[i + 1];
    switch (c) {
      case 'R': R = std::atoi(v); break;
      case 'm': mode = std::atoi(v); break;
      case 't': impType = std::atoi(v); break;
      case 'f': fth = std::strtoull(v, nullptr, 10); break;
      case 'c': check = std::atoi(v) == 1; break;
      case 'i': in = v; break;
      case 'o': out = v; break;
      case 'w': case 'v': case 'b': break;  // accepted, unused
      default: std::fprintf(stderr, "unknown option: %s\n", argv[i]); return 1;
    }
  }
  if (in.empty() || (argc % 2) == 0) {
    std::printf("usage: ttm -i X.tns [-m mode] [-R rank] [-t 2|3] [-f fiber-threshold] [-c 0|1] [-o Y.txt]\n");
    return 1;
  }
  if (impType != 2 && impType != 3) {
    std::fprintf(stderr, "-t %d is not provided by this library (GPU TTM: 2, 3)\n", impType);
    return 1;
  }
  mmcsf_coo* X = nullptr;
  const bool bin = in.size() > 4 && in.compare(in.size() - 4, 4, ".bin") == 0;
  int st = bin ? mmcsf_coo_load_bin(in.c_str(), &X) : mmcsf_coo_load_tns(in.c_str(), &X);
  if (st) { std::fprintf(stderr, "load_tensor failed: %s\n", mmcsf_last_error()); return 1; }
  int nd = 0;
  uint64_t dims[4] = {0, 0, 0, 0}, nnz = 0;
  mmcsf_coo_info(X, &nd, dims, &nnz);
  if (nd != 3 || mode < 0 || mode >= nd) { std::fprintf(stderr, "TTM needs a 3-D tensor and a mode in [0, 3)\n"); return 1; }
  mmcsf_build_opts bo{};
  bo.impl = MMCSF_IMPL_BCSF;
  bo.mode = mode;
  bo.fiber_threshold = fth;
  bo.keep_coo = check ? 1 : 0;
  mmcsf_format* F = nullptr;
  if ((st = mmcsf_build(X, &bo, nullptr, &F))) { std::fprintf(stderr, "format construction failed: %s\n", mmcsf_last_error()); return 1; }
  mmcsf_part_info pi{};
  mmcsf_format_info(F, 0, &pi);
  const int leaf = pi.mode_order[2];
  std::vector<float> hU(dims[leaf] * (uint64_t)R, (float)leaf + 0.5f);
  float* dU = nullptr;
  float* dY = nullptr;
  uint64_t nf = 0;
  mmcsf_ttm(F, R, MMCSF_DTYPE_F32, nullptr, nullptr, &nf, nullptr);
  if (cudaMalloc(&dU, hU.size() * 4) != cudaSuccess || cudaMalloc(&dY, (nf ? nf : 1) * (uint64_t)R * 4) != cudaSuccess) {
    std::fprintf(stderr, "device allocation failed\n");
    return 1;
  }
  cudaMemcpy(dU, hU.data(), hU.size() * 4, cudaMemcpyHostToDevice);
  if ((st = mmcsf_ttm(F, R, MMCSF_DTYPE_F32, dU, dY, &nf, nullptr))) { std::fprintf(stderr, "TTM failed: %s\n", mmcsf_last_error()); return 1; }
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  cudaEventRecord(e0);
  mmcsf_ttm(F, R, MMCSF_DTYPE_F32, dU, dY, &nf, nullptr);
  cudaEventRecord(e1);
  cudaEventSynchronize(e1);
  float ms = 0;
  cudaEventElapsedTime(&ms, e0, e1);
  std::printf("TTM GPU - time %fms\n", ms);
  std::vector<float> Y(nf * (uint64_t)R);
  cudaMemcpy(Y.data(), dY, Y.size() * 4, cudaMemcpyDeviceToHost);
  if (check) {  // host TTM in double over the format's own fiber pointers and leaf indices
    std::vector<uint64_t> fptr(nf + 1), leafi(nnz);
    std::vector<float> vals(nnz);
    uint64_t cnt = 0;
    mmcsf_format_export(F, 0, "fbrPtr1", fptr.data(), fptr.size(), &cnt);
    mmcsf_format_export(F, 0, "indsLeaf", leafi.data(), leafi.size(), &cnt);
    mmcsf_format_export_f32(F, 0, "vals", vals.data(), vals.size(), &cnt);
    uint64_t mism = 0;
    for (uint64_t f = 0; f < nf; ++f) {
      double s = 0;
      for (uint64_t x = fptr[f]; x < fptr[f + 1]; ++x) s += vals[x] * ((double)leaf + 0.5);
      for (int r = 0; r < R; ++r)
        if (std::fabs(Y[f * R + r] - s) > 1e-5 * std::fabs(s) + 1e-6) ++mism;
    }
    if (mism == 0) std::printf("Correctness pass!\n");
    else std::printf("%llu mismatches\n", (unsigned long long)mism);
  }
  if (!out.empty()) {
    FILE* fo = std::fopen(out.c_str(), "w");
    if (!fo) { std::fprintf(stderr, "cannot write %s\n", out.c_str()); return 1; }
    std::fprintf(fo, "%llu x %d semiSpTensor\n", (unsigned long long)nf, R);
    for (uint64_t f = 0; f < nf; ++f) {
      for (int r = 0; r < R; ++r) std::fprintf(fo, "%.2f\t", Y[f * R + r]);
      std::fprintf(fo, "\n");
    }
    std::fclose(fo);
  }
  cudaFree(dU);
  cudaFree(dY);
  mmcsf_format_destroy(F);
  mmcsf_coo_destroy(X);
  return 0;
}
