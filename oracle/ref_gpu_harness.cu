// Test infrastructure, not product code.
//
// Harness that runs the reference's own GPU MTTKRP, MTTKRP_MIHCSR_GPU
// (src/mttkrp_gpu.cu:3380-3784), compiled for sm_100a from the reference's
// sources by oracle/build_ref.py, on an MM-CSF partition given as arrays
// under the reference's names (the arrays mmcsf_format_export writes, which
// the tests prove bit-exact to the reference's builders). It fills one
// TiledTensor (src/util.h:107-136) with them, sets the factors to the
// reference's non-CPD constants U[m] = m + 0.5 (src/util.h:3223; its driver
// resets each finished mode to that constant, src/mttkrp_gpu.cu:3552-3557),
// calls MTTKRP_MIHCSR_GPU, and returns the "Total GPU time" it prints
// (src/mttkrp_gpu.cu:3757: the sum of its per-launch CUDA-event times) and
// the last mode's output it copies back. Only bench.py's reference-GPU
// section loads the library this builds, as a baseline.
#include "util.h"
#include "mttkrp_gpu.h"

#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <iostream>
#include <sstream>
#include <string>

extern "C" int ref_mihcsr_gpu(int nd, const uint64_t* dims, int R, int warpPerSlice, int TBsize, int fiberPerWarp,
                              int part,
                              const int* modeOrder, const uint64_t* const* fbrPtr, const uint64_t* fbrPtrLen,
                              const uint64_t* const* fbrIdx, const uint64_t* fbrIdxLen, const uint64_t* fbrLike,
                              uint64_t nFibers, uint64_t* const* inds, float* vals, uint64_t nnz,
                              float* last_mode_out, double* total_ms) {
  if (nd < 3 || nd > 4 || part < 0 || part >= nd || !total_ms) return 1;
  TiledTensor* TX = new TiledTensor[nd];
  for (int m = 0; m < nd; ++m) {
    TX[m].ndims = nd;
    TX[m].totNnz = 0;
    TX[m].nFibers = 0;
    TX[m].dims = new ITYPE[nd];
    for (int q = 0; q < nd; ++q) {
      TX[m].dims[q] = dims[q];
      TX[m].modeOrder.push_back((ITYPE)((q + m) % nd));  // empty partitions: any valid order
    }
  }
  TiledTensor& T = TX[part];
  for (int q = 0; q < nd; ++q) T.modeOrder[q] = (ITYPE)modeOrder[q];
  T.totNnz = nnz;
  T.nFibers = nFibers;
  T.fbrPtr.resize(nd - 1);
  T.fbrIdx.resize(nd - 1);
  for (int l = 0; l < nd - 1; ++l) {
    T.fbrPtr[l].assign(fbrPtr[l], fbrPtr[l] + fbrPtrLen[l]);
    T.fbrIdx[l].assign(fbrIdx[l], fbrIdx[l] + fbrIdxLen[l]);
  }
  T.fbrLikeSlcInds = const_cast<ITYPE*>(reinterpret_cast<const ITYPE*>(fbrLike));
  T.inds = new ITYPE*[nd];
  for (int q = 0; q < nd; ++q) T.inds[q] = reinterpret_cast<ITYPE*>(inds[q]);
  T.vals = vals;

  Matrix* U = new Matrix[nd];
  for (int m = 0; m < nd; ++m) {
    U[m].nRows = dims[m];
    U[m].nCols = R;
    U[m].vals = new DTYPE[dims[m] * (uint64_t)R];
    for (uint64_t i = 0; i < dims[m] * (uint64_t)R; ++i) U[m].vals[i] = (DTYPE)m + 0.5f;
  }
  Options Opt;
  Opt.R = R;
  Opt.impType = 12;
  Opt.mode = 0;
  if (warpPerSlice > 0) Opt.warpPerSlice = warpPerSlice;
  if (TBsize > 0) Opt.TBsize = TBsize;
  if (fiberPerWarp > 0) Opt.fiberPerWarp = fiberPerWarp;

  // the driver prints its timings on std::cout
  std::ostringstream cap;
  std::streambuf* old = std::cout.rdbuf(cap.rdbuf());
  MTTKRP_MIHCSR_GPU(TX, U, Opt);
  std::cout.rdbuf(old);
  const std::string text = cap.str();
  const size_t at = text.find("Total GPU time: ");
  int rc = 0;
  if (at == std::string::npos) rc = 2;
  else *total_ms = std::strtod(text.c_str() + at + 16, nullptr);
  if (last_mode_out)
    std::memcpy(last_mode_out, U[nd - 1].vals, dims[nd - 1] * (uint64_t)R * sizeof(float));
  for (int m = 0; m < nd; ++m) delete[] U[m].vals;
  delete[] U;
  delete[] T.inds;
  for (int m = 0; m < nd; ++m) delete[] TX[m].dims;
  delete[] TX;
  return rc;
}
