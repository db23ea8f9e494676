// Array export (device -> host, widened to uint64) under the reference's
// array names, for bit-exact comparison with the reference's builders.
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "format.h"

using mmcsf::set_error;
using mmcsf::CsfPart;
using mmcsf::DevBuf;

namespace {

int copy_u32(const DevBuf& b, uint64_t n, uint64_t* dst, uint64_t cap, uint64_t* count, uint32_t mask = ~0u) {
  if (count) *count = n;
  if (!dst) return MMCSF_OK;
  if (cap < n) return set_error(MMCSF_ERR_INVALID, "export buffer too small (%llu < %llu)",
                                (unsigned long long)cap, (unsigned long long)n);
  if (n == 0) return MMCSF_OK;
  std::vector<uint32_t> h(n);
  MMCSF_CUDA(cudaDeviceSynchronize());
  MMCSF_CUDA(cudaMemcpy(h.data(), b.p, n * 4, cudaMemcpyDeviceToHost));
  for (uint64_t i = 0; i < n; ++i) dst[i] = h[i] & mask;
  return MMCSF_OK;
}

int copy_bins(const DevBuf& bin_of, uint64_t nslc, int b, uint64_t* dst, uint64_t cap, uint64_t* count) {
  std::vector<int32_t> h(nslc);
  if (nslc) {
    MMCSF_CUDA(cudaDeviceSynchronize());
    MMCSF_CUDA(cudaMemcpy(h.data(), bin_of.p, nslc * 4, cudaMemcpyDeviceToHost));
  }
  uint64_t n = 0;
  for (uint64_t s = 0; s < nslc; ++s)
    if (h[s] == b) {
      if (dst) {
        if (n >= cap) return set_error(MMCSF_ERR_INVALID, "export buffer too small");
        dst[n] = s;
      }
      ++n;
    }
  if (count) *count = n;
  return MMCSF_OK;
}

bool starts(const char* s, const char* p, int* num) {
  size_t n = strlen(p);
  if (strncmp(s, p, n) != 0) return false;
  if (s[n] < '0' || s[n] > '9') return false;
  *num = atoi(s + n);
  return true;
}

}  // namespace

extern "C" int mmcsf_format_export(const mmcsf_format* F, int part, const char* name, uint64_t* dst, uint64_t cap,
                                   uint64_t* count) {
  MMCSF_RANGE("mmcsf_format_export");
  if (!F || !name) return set_error(MMCSF_ERR_INVALID, "null argument");
  if (part < 0 || part > 3) return set_error(MMCSF_ERR_INVALID, "bad part %d", part);
  const int nd = F->nd;
  if (F->impl == MMCSF_IMPL_HBCSF && part > 0) {
    const auto& H = F->hyb;
    int l;
    if (part == 1) {  // COO part
      if (starts(name, "COOinds", &l) && l < nd) return copy_u32(H.coo_inds[l], H.coo_nnz, dst, cap, count);
    } else if (part == 2 && nd == 3) {  // CSL part
      if (!strcmp(name, "CSLslicePtr")) return copy_u32(H.csl_ptr, H.n_csl_slices + 1, dst, cap, count);
      if (!strcmp(name, "CSLsliceIdx")) return copy_u32(H.csl_idx, H.n_csl_slices, dst, cap, count);
      if (!strcmp(name, "CSLinds1")) return copy_u32(H.csl_i1, H.csl_nnz, dst, cap, count);
      if (!strcmp(name, "CSLinds2")) return copy_u32(H.csl_i2, H.csl_nnz, dst, cap, count);
      if (starts(name, "cslbin", &l) && l < 10) return copy_bins(H.csl_bin_of, H.n_csl_slices, l, dst, cap, count);
    }
    return set_error(MMCSF_ERR_INVALID, "unknown array %s for part %d", name, part);
  }
  const CsfPart& P = F->parts[part];
  if (!P.present) {
    if (count) *count = 0;
    return MMCSF_OK;
  }
  int l;
  // level array lengths, as the reference stores them
  auto ptr_len = [&](int lv) -> uint64_t { return P.n[lv] + 1; };
  auto idx_len = [&](int lv) -> uint64_t {
    const bool leaf_level = lv == nd - 2;
    if (F->impl == MMCSF_IMPL_HBCSF) return P.n[lv];  // create_HYB pushes no sentinel
    return leaf_level ? P.n[lv] + 1 : P.n[lv];
  };
  if (starts(name, "fbrPtr", &l) && l < nd - 1) return copy_u32(P.ptr[l], ptr_len(l), dst, cap, count);
  if (starts(name, "fbrIdx", &l) && l < nd - 1) return copy_u32(P.idx[l], idx_len(l), dst, cap, count);
  if (!strcmp(name, "fbrLikeSlcInds")) return copy_u32(P.fbr_like, P.n[1], dst, cap, count);
  // the leaf array carries fiber-start flags in bit 31 (see build.cu)
  if (!strcmp(name, "indsLeaf")) return copy_u32(P.leaf, P.nnz, dst, cap, count, 0x7fffffffu);
  if (starts(name, "inds", &l) && l < nd) {
    if (!P.coo[l].p) return set_error(MMCSF_ERR_INVALID, "build with keep_coo=1 to export inds%d", l);
    return copy_u32(P.coo[l], P.nnz, dst, cap, count);
  }
  if (starts(name, "bin", &l) && l < 10) {
    if (!P.bin_of.p) return set_error(MMCSF_ERR_INVALID, "this format has no slice bins");
    return copy_bins(P.bin_of, P.n[0], l, dst, cap, count);
  }
  return set_error(MMCSF_ERR_INVALID, "unknown array %s", name);
}

extern "C" int mmcsf_format_export_f32(const mmcsf_format* F, int part, const char* name, float* dst, uint64_t cap,
                                       uint64_t* count) {
  if (!F || !name) return set_error(MMCSF_ERR_INVALID, "null argument");
  if (part < 0 || part > 3) return set_error(MMCSF_ERR_INVALID, "bad part %d", part);
  const DevBuf* b = nullptr;
  uint64_t n = 0;
  if (F->impl == MMCSF_IMPL_HBCSF && part == 1 && !strcmp(name, "COOvals")) {
    b = &F->hyb.coo_vals;
    n = F->hyb.coo_nnz;
  } else if (F->impl == MMCSF_IMPL_HBCSF && part == 2 && !strcmp(name, "CSLvals")) {
    b = &F->hyb.csl_vals;
    n = F->hyb.csl_nnz;
  } else if (!strcmp(name, "vals")) {
    b = &F->parts[part].vals;
    n = F->parts[part].present ? F->parts[part].nnz : 0;
  } else {
    return set_error(MMCSF_ERR_INVALID, "unknown array %s", name);
  }
  if (count) *count = n;
  if (!dst || n == 0) return MMCSF_OK;
  if (cap < n) return set_error(MMCSF_ERR_INVALID, "export buffer too small");
  MMCSF_CUDA(cudaDeviceSynchronize());
  MMCSF_CUDA(cudaMemcpy(dst, b->p, n * 4, cudaMemcpyDeviceToHost));
  return MMCSF_OK;
}
