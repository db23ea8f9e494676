// HB-CSF (-t 10): the reference's hybrid of COO, CSL and CSF slices
// (create_HYB / create_HYB_4D, src/util.h:852-1142; make_HybBin,
// src/util.h:1786-1885), built on the device from the CSF of the computed
// mode, and its MTTKRP (MTTKRP_HYB_GPU, src/mttkrp_gpu.cu:2530-2851).
//
// Slices with one nonzero go to the COO part; in 3-D, slices whose fibers
// all hold one nonzero go to the CSL part (slice -> nonzeros); the rest stay
// CSF. Every output array is produced by a per-slice classification, exclusive
// scans of per-class counts, and scatters into the compacted positions.
#include <cuda_bf16.h>

#include "format.h"
#include "prims.cuh"

namespace mmcsf {
namespace {

constexpr uint32_t FLAG = 0x80000000u;

// cls: 0 COO, 1 CSL, 2 CSF. cnt_nnz / cnt_fib / cnt_fs: per-slice counts.
__global__ void k_classify(int nd, const uint32_t* __restrict__ p0, const uint32_t* __restrict__ p1,
                           const uint32_t* __restrict__ p2, uint64_t nslc, uint32_t* __restrict__ cls,
                           uint32_t* __restrict__ cnt_nnz, uint32_t* __restrict__ cnt_fib,
                           uint32_t* __restrict__ cnt_fs) {
  for (uint64_t s = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; s < nslc; s += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t c0 = p0[s], c1 = p0[s + 1];
    uint32_t nnz, nfib;
    if (nd == 3) {
      nnz = p1[c1] - p1[c0];
      nfib = c1 - c0;
    } else {
      const uint32_t f0 = p1[c0], f1 = p1[c1];
      nnz = p2[f1] - p2[f0];
      nfib = f1 - f0;
    }
    uint32_t c = 2;
    if (nnz == 1) c = 0;
    else if (nd == 3 && nnz == nfib) c = 1;  // every fiber holds one nonzero
    cls[s] = c;
    cnt_nnz[s] = nnz;
    cnt_fib[s] = nfib;
    cnt_fs[s] = c1 - c0;
  }
}

// masked[s] = cls[s] == want ? val[s] : 0
__global__ void k_mask(const uint32_t* __restrict__ cls, const uint32_t* __restrict__ val, uint32_t want,
                       uint64_t n, uint32_t* __restrict__ out) {
  for (uint64_t s = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; s < n; s += (uint64_t)gridDim.x * blockDim.x)
    out[s] = cls[s] == want ? (val ? val[s] : 1u) : 0u;
}

// parent[c] = the slice owning level-1 entry c
__global__ void k_mark_starts(const uint32_t* __restrict__ p0, uint64_t nslc, uint32_t* __restrict__ flag) {
  for (uint64_t s = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; s < nslc; s += (uint64_t)gridDim.x * blockDim.x)
    flag[p0[s]] = 1;
}
__global__ void k_parent_of(const uint32_t* __restrict__ excl, uint64_t n, uint32_t* __restrict__ out) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
    out[i] = excl[i + 1] - 1;
}

struct HybScan {
  const uint32_t *cls, *slot, *nnz_before, *fib_before, *fs_before;  // exclusive scans per class
};

// COO part and CSF/CSL slice-level arrays
__global__ void k_hyb_slices(int nd, HybScan h, const uint32_t* __restrict__ p0, const uint32_t* __restrict__ p1,
                             const uint32_t* __restrict__ p2, const uint32_t* __restrict__ i0,
                             const uint32_t* __restrict__ i1, const uint32_t* __restrict__ i2,
                             const uint32_t* __restrict__ leaf, const float* __restrict__ vals, uint64_t nslc,
                             uint32_t* c0, uint32_t* c1, uint32_t* c2, uint32_t* c3, float* cv,
                             uint32_t* csl_ptr, uint32_t* csl_idx, uint32_t* h_p0, uint32_t* h_i0) {
  for (uint64_t s = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; s < nslc; s += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t c = h.cls[s], k = h.slot[s];
    const uint32_t fs0 = p0[s];
    if (c == 0) {
      const uint32_t f0 = (nd == 3) ? fs0 : p1[fs0];
      const uint32_t x0 = (nd == 3) ? p1[f0] : p2[f0];
      c0[k] = i0[s];
      c1[k] = i1[fs0];
      if (nd == 3) {
        c2[k] = leaf[x0] & ~FLAG;
      } else {
        c2[k] = i2[f0];
        c3[k] = leaf[x0] & ~FLAG;
      }
      cv[k] = vals[x0];
    } else if (c == 1) {
      csl_ptr[k] = h.fib_before[s];
      csl_idx[k] = i0[s];
    } else {
      h_p0[k] = (nd == 3) ? h.fib_before[s] : h.fs_before[s];
      h_i0[k] = i0[s];
    }
  }
}

// 3-D level-1 (fiber) arrays of the CSL and CSF parts, plus their nonzeros
__global__ void k_hyb_fibers3(HybScan h, const uint32_t* __restrict__ parent, const uint32_t* __restrict__ p0,
                              const uint32_t* __restrict__ p1, const uint32_t* __restrict__ i1,
                              const uint32_t* __restrict__ leaf, const float* __restrict__ vals, uint64_t nfib,
                              uint32_t* csl_i1, uint32_t* csl_i2, float* csl_v, uint32_t* h_p1, uint32_t* h_i1,
                              uint32_t* h_leaf, float* h_vals) {
  for (uint64_t f = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; f < nfib; f += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t s = parent[f], c = h.cls[s];
    const uint32_t rel = (uint32_t)f - p0[s];  // fiber within its slice
    if (c == 1) {
      const uint32_t pos = h.fib_before[s] + rel, x = p1[f];
      csl_i1[pos] = i1[f];
      csl_i2[pos] = leaf[x] & ~FLAG;
      csl_v[pos] = vals[x];
    } else if (c == 2) {
      const uint32_t g = h.fib_before[s] + rel;
      const uint32_t xs = p1[p0[s]];
      const uint32_t nb = h.nnz_before[s];
      h_p1[g] = nb + (p1[f] - xs);
      h_i1[g] = i1[f];
      for (uint32_t x = p1[f]; x < p1[f + 1]; ++x) {
        h_leaf[nb + (x - xs)] = leaf[x] & ~FLAG;
        h_vals[nb + (x - xs)] = vals[x];
      }
    }
  }
}

// 4-D fbrS- and fiber-level arrays of the CSF part, plus its nonzeros
__global__ void k_hyb_fbrs4(HybScan h, const uint32_t* __restrict__ parent, const uint32_t* __restrict__ p0,
                            const uint32_t* __restrict__ p1, const uint32_t* __restrict__ p2,
                            const uint32_t* __restrict__ i1, const uint32_t* __restrict__ i2,
                            const uint32_t* __restrict__ leaf, const float* __restrict__ vals, uint64_t nfs,
                            uint32_t* h_p1, uint32_t* h_i1, uint32_t* h_p2, uint32_t* h_i2, uint32_t* h_leaf,
                            float* h_vals) {
  for (uint64_t q = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; q < nfs; q += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t s = parent[q];
    if (h.cls[s] != 2) continue;
    const uint32_t fs_new = h.fs_before[s] + ((uint32_t)q - p0[s]);
    const uint32_t fslc0 = p1[p0[s]];                 // first fiber of the slice
    const uint32_t xs = p2[fslc0];                    // first nonzero of the slice
    const uint32_t fb = h.fib_before[s], nb = h.nnz_before[s];
    h_p1[fs_new] = fb + (p1[q] - fslc0);
    h_i1[fs_new] = i1[q];
    for (uint32_t f = p1[q]; f < p1[q + 1]; ++f) {
      const uint32_t g = fb + (f - fslc0);
      h_p2[g] = nb + (p2[f] - xs);
      h_i2[g] = i2[f];
      for (uint32_t x = p2[f]; x < p2[f + 1]; ++x) {
        h_leaf[nb + (x - xs)] = leaf[x] & ~FLAG;
        h_vals[nb + (x - xs)] = vals[x];
      }
    }
  }
}

__global__ void k_set(uint32_t* p, uint64_t i, uint32_t v) { p[i] = v; }

// CSF-part derived arrays: fbr_like (o0 per level-1 entry), fpar (4-D),
// fiber-start flags in the leaf index
__global__ void k_like_from_slices(const uint32_t* __restrict__ hp0, const uint32_t* __restrict__ hi0,
                                   uint64_t nslc, uint32_t* __restrict__ like) {
  for (uint64_t s = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; s < nslc; s += (uint64_t)gridDim.x * blockDim.x)
    for (uint32_t c = hp0[s]; c < hp0[s + 1]; ++c) like[c] = hi0[s];
}
__global__ void k_fpar(const uint32_t* __restrict__ hp1, uint64_t nfs, uint32_t* __restrict__ fpar) {
  for (uint64_t q = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; q < nfs; q += (uint64_t)gridDim.x * blockDim.x)
    for (uint32_t f = hp1[q]; f < hp1[q + 1]; ++f) fpar[f] = (uint32_t)q;
}
__global__ void k_flags(uint32_t* __restrict__ leaf, const uint32_t* __restrict__ fptr, uint64_t nfib) {
  for (uint64_t f = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; f < nfib; f += (uint64_t)gridDim.x * blockDim.x)
    leaf[fptr[f]] |= FLAG;
}

// make_HybBin counts: CSF slices count their nonzeros; CSL slices their fibers
__global__ void k_hyb_bins(const uint32_t* __restrict__ sptr, const uint32_t* __restrict__ nzstart, uint64_t nslc,
                           uint64_t tot, int32_t* __restrict__ bin_of) {
  const uint64_t TB = 512;
  for (uint64_t s = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; s < nslc; s += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t c0 = sptr[s], c1 = sptr[s + 1];
    const uint64_t n = nzstart ? (uint64_t)(nzstart[c1] - nzstart[c0]) : c1 - c0;
    const uint64_t LB[10] = {0, 2, 4, 8, 16, 1024, 4 * TB, 8 * TB, 16 * TB, 32 * TB};
    const uint64_t UB[10] = {1025, 5, 9, 17, 1025, 4 * TB + 1, 8 * TB + 1, 16 * TB + 1, 32 * TB + 1, tot + 1};
    int b = -1;
    for (int i = 0; i < 10; ++i)
      if (n > LB[i] && n < UB[i]) { b = i; break; }
    bin_of[s] = b;
  }
}

int scan_to(const uint32_t* in, uint64_t n, DevBuf& out, uint32_t* total, cudaStream_t s) {
  MMCSF_CUDA(out.alloc((n + 1) * 4));
  MMCSF_CUDA(exclusive_scan_u32(in, out.as<uint32_t>(), n, s));
  MMCSF_CUDA(cudaMemcpyAsync(total, out.as<uint32_t>() + n, 4, cudaMemcpyDeviceToHost, s));
  MMCSF_CUDA(cudaStreamSynchronize(s));
  return MMCSF_OK;
}

}  // namespace

int build_hyb(mmcsf_format* F, CsfPart& X, cudaStream_t s, int* launches) {
  const int nd = F->nd;
  HybExtra& H = F->hyb;
  if (!X.present) return MMCSF_OK;
  const uint64_t S_ = X.n[0];
  const uint32_t* p0 = X.ptr[0].as<uint32_t>();
  const uint32_t* p1 = X.ptr[1].as<uint32_t>();
  const uint32_t* p2 = nd == 4 ? X.ptr[2].as<uint32_t>() : nullptr;
  const int G = grid_for(S_, 256);
  int L = 0;
  DevBuf cls, cn, cf, cs;
  MMCSF_CUDA(cls.alloc(S_ * 4));
  MMCSF_CUDA(cn.alloc(S_ * 4));
  MMCSF_CUDA(cf.alloc(S_ * 4));
  MMCSF_CUDA(cs.alloc(S_ * 4));
  k_classify<<<G, 256, 0, s>>>(nd, p0, p1, p2, S_, cls.as<uint32_t>(), cn.as<uint32_t>(), cf.as<uint32_t>(),
                               cs.as<uint32_t>());
  ++L;
  MMCSF_LAUNCH_CHECK();
  // per-class slot numbers and counts before each slice (a slice belongs to
  // one class, so one scan of the class-masked counts serves its class)
  DevBuf m0, m1, m2, slot, nb, fb, fsb, tmpm;
  MMCSF_CUDA(tmpm.alloc(S_ * 4));
  uint32_t ncls[3] = {0, 0, 0};
  DevBuf sl[3], nbv[3], fbv[3], fsv[3];
  uint32_t tot_n[3], tot_f[3], tot_s[3];
  for (uint32_t c = 0; c < 3; ++c) {
    k_mask<<<G, 256, 0, s>>>(cls.as<uint32_t>(), nullptr, c, S_, tmpm.as<uint32_t>());
    MMCSF_LAUNCH_CHECK();
    MMCSF_TRY(scan_to(tmpm.as<uint32_t>(), S_, sl[c], &ncls[c], s));
    k_mask<<<G, 256, 0, s>>>(cls.as<uint32_t>(), cn.as<uint32_t>(), c, S_, tmpm.as<uint32_t>());
    MMCSF_LAUNCH_CHECK();
    MMCSF_TRY(scan_to(tmpm.as<uint32_t>(), S_, nbv[c], &tot_n[c], s));
    k_mask<<<G, 256, 0, s>>>(cls.as<uint32_t>(), cf.as<uint32_t>(), c, S_, tmpm.as<uint32_t>());
    MMCSF_LAUNCH_CHECK();
    MMCSF_TRY(scan_to(tmpm.as<uint32_t>(), S_, fbv[c], &tot_f[c], s));
    k_mask<<<G, 256, 0, s>>>(cls.as<uint32_t>(), cs.as<uint32_t>(), c, S_, tmpm.as<uint32_t>());
    MMCSF_LAUNCH_CHECK();
    MMCSF_TRY(scan_to(tmpm.as<uint32_t>(), S_, fsv[c], &tot_s[c], s));
    L += 4 * 4;
  }
  // combine: each slice reads the scans of its own class
  DevBuf cslot, cnb, cfb, cfsb;
  MMCSF_CUDA(cslot.alloc(S_ * 4));
  MMCSF_CUDA(cnb.alloc(S_ * 4));
  MMCSF_CUDA(cfb.alloc(S_ * 4));
  MMCSF_CUDA(cfsb.alloc(S_ * 4));
  {
    std::vector<uint32_t> hc(S_), a[3], b[3], c_[3], d[3];
    MMCSF_CUDA(cudaMemcpyAsync(hc.data(), cls.p, S_ * 4, cudaMemcpyDeviceToHost, s));
    for (int c = 0; c < 3; ++c) {
      a[c].resize(S_); b[c].resize(S_); c_[c].resize(S_); d[c].resize(S_);
      MMCSF_CUDA(cudaMemcpyAsync(a[c].data(), sl[c].p, S_ * 4, cudaMemcpyDeviceToHost, s));
      MMCSF_CUDA(cudaMemcpyAsync(b[c].data(), nbv[c].p, S_ * 4, cudaMemcpyDeviceToHost, s));
      MMCSF_CUDA(cudaMemcpyAsync(c_[c].data(), fbv[c].p, S_ * 4, cudaMemcpyDeviceToHost, s));
      MMCSF_CUDA(cudaMemcpyAsync(d[c].data(), fsv[c].p, S_ * 4, cudaMemcpyDeviceToHost, s));
    }
    MMCSF_CUDA(cudaStreamSynchronize(s));
    std::vector<uint32_t> o1(S_), o2(S_), o3(S_), o4(S_);
    for (uint64_t i = 0; i < S_; ++i) {
      const uint32_t c = hc[i];
      o1[i] = a[c][i];
      o2[i] = b[c][i];
      o3[i] = c_[c][i];
      o4[i] = d[c][i];
    }
    MMCSF_CUDA(cudaMemcpyAsync(cslot.p, o1.data(), S_ * 4, cudaMemcpyHostToDevice, s));
    MMCSF_CUDA(cudaMemcpyAsync(cnb.p, o2.data(), S_ * 4, cudaMemcpyHostToDevice, s));
    MMCSF_CUDA(cudaMemcpyAsync(cfb.p, o3.data(), S_ * 4, cudaMemcpyHostToDevice, s));
    MMCSF_CUDA(cudaMemcpyAsync(cfsb.p, o4.data(), S_ * 4, cudaMemcpyHostToDevice, s));
    MMCSF_CUDA(cudaStreamSynchronize(s));
  }
  HybScan hs{cls.as<uint32_t>(), cslot.as<uint32_t>(), cnb.as<uint32_t>(), cfb.as<uint32_t>(), cfsb.as<uint32_t>()};

  // output sizes
  H.coo_nnz = ncls[0];
  H.csl_nnz = tot_n[1];
  H.n_csl_slices = ncls[1];
  const uint64_t hs_ = ncls[2], hfs = tot_s[2], hf = (nd == 3) ? tot_f[2] : tot_f[2], hn = tot_n[2];
  for (int l = 0; l < nd; ++l) MMCSF_CUDA(H.coo_inds[l].alloc((uint64_t)H.coo_nnz * 4));
  MMCSF_CUDA(H.coo_vals.alloc((uint64_t)H.coo_nnz * 4));
  MMCSF_CUDA(H.csl_ptr.alloc(((uint64_t)H.n_csl_slices + 1) * 4));
  MMCSF_CUDA(H.csl_idx.alloc((uint64_t)H.n_csl_slices * 4));
  MMCSF_CUDA(H.csl_i1.alloc((uint64_t)H.csl_nnz * 4));
  MMCSF_CUDA(H.csl_i2.alloc((uint64_t)H.csl_nnz * 4));
  MMCSF_CUDA(H.csl_vals.alloc((uint64_t)H.csl_nnz * 4));
  CsfPart P;  // the CSF part
  P.present = true;  // the reference always emits the CSF part's terminal pointers
  P.nd = nd;
  for (int i = 0; i < nd; ++i) P.order[i] = X.order[i];
  P.nnz = hn;
  P.n[0] = hs_;
  P.n[1] = nd == 3 ? hf : hfs;
  if (nd == 4) P.n[2] = hf;
  MMCSF_CUDA(P.ptr[0].alloc((hs_ + 1) * 4));
  MMCSF_CUDA(P.idx[0].alloc((hs_ + 1) * 4));
  MMCSF_CUDA(P.ptr[1].alloc((P.n[1] + 1) * 4));
  MMCSF_CUDA(P.idx[1].alloc((P.n[1] + 1) * 4));
  if (nd == 4) {
    MMCSF_CUDA(P.ptr[2].alloc((hf + 1) * 4));
    MMCSF_CUDA(P.idx[2].alloc((hf + 1) * 4));
  }
  MMCSF_CUDA(P.leaf.alloc(hn * 4));
  MMCSF_CUDA(P.vals.alloc(hn * 4));

  k_hyb_slices<<<G, 256, 0, s>>>(nd, hs, p0, p1, p2, X.idx[0].as<uint32_t>(), X.idx[1].as<uint32_t>(),
                                 nd == 4 ? X.idx[2].as<uint32_t>() : nullptr, X.leaf.as<uint32_t>(),
                                 X.vals.as<float>(), S_, H.coo_inds[0].as<uint32_t>(), H.coo_inds[1].as<uint32_t>(),
                                 H.coo_inds[2].as<uint32_t>(), nd == 4 ? H.coo_inds[3].as<uint32_t>() : nullptr,
                                 H.coo_vals.as<float>(), H.csl_ptr.as<uint32_t>(), H.csl_idx.as<uint32_t>(),
                                 P.ptr[0].as<uint32_t>(), P.idx[0].as<uint32_t>());
  ++L;
  MMCSF_LAUNCH_CHECK();
  // parent slice of every level-1 entry of the base CSF
  const uint64_t n1 = X.n[1];
  DevBuf flag, ex, parent;
  MMCSF_CUDA(flag.alloc(n1 * 4));
  MMCSF_CUDA(cudaMemsetAsync(flag.p, 0, n1 * 4, s));
  k_mark_starts<<<G, 256, 0, s>>>(p0, S_, flag.as<uint32_t>());
  MMCSF_LAUNCH_CHECK();
  // inclusive count of starts: exclusive scan then +flag handled via excl[i+1]
  MMCSF_CUDA(ex.alloc((n1 + 1) * 4));
  MMCSF_CUDA(exclusive_scan_u32(flag.as<uint32_t>(), ex.as<uint32_t>(), n1, s));
  MMCSF_CUDA(parent.alloc(n1 * 4));
  k_parent_of<<<grid_for(n1, 256), 256, 0, s>>>(ex.as<uint32_t>(), n1, parent.as<uint32_t>());
  MMCSF_LAUNCH_CHECK();
  L += 5;
  if (nd == 3) {
    k_hyb_fibers3<<<grid_for(n1, 256), 256, 0, s>>>(hs, parent.as<uint32_t>(), p0, p1, X.idx[1].as<uint32_t>(),
                                                    X.leaf.as<uint32_t>(), X.vals.as<float>(), n1,
                                                    H.csl_i1.as<uint32_t>(), H.csl_i2.as<uint32_t>(),
                                                    H.csl_vals.as<float>(), P.ptr[1].as<uint32_t>(),
                                                    P.idx[1].as<uint32_t>(), P.leaf.as<uint32_t>(),
                                                    P.vals.as<float>());
  } else {
    k_hyb_fbrs4<<<grid_for(n1, 256), 256, 0, s>>>(hs, parent.as<uint32_t>(), p0, p1, p2, X.idx[1].as<uint32_t>(),
                                                  X.idx[2].as<uint32_t>(), X.leaf.as<uint32_t>(), X.vals.as<float>(),
                                                  n1, P.ptr[1].as<uint32_t>(), P.idx[1].as<uint32_t>(),
                                                  P.ptr[2].as<uint32_t>(), P.idx[2].as<uint32_t>(),
                                                  P.leaf.as<uint32_t>(), P.vals.as<float>());
  }
  ++L;
  MMCSF_LAUNCH_CHECK();
  // terminal pointers (create_HYB pushes them after the slice loop)
  if (nd == 3) {
    k_set<<<1, 1, 0, s>>>(P.ptr[1].as<uint32_t>(), hf, (uint32_t)hn);
    k_set<<<1, 1, 0, s>>>(P.ptr[0].as<uint32_t>(), hs_, (uint32_t)hf);
    k_set<<<1, 1, 0, s>>>(H.csl_ptr.as<uint32_t>(), H.n_csl_slices, (uint32_t)H.csl_nnz);
  } else {
    k_set<<<1, 1, 0, s>>>(P.ptr[2].as<uint32_t>(), hf, (uint32_t)hn);
    k_set<<<1, 1, 0, s>>>(P.ptr[1].as<uint32_t>(), hfs, (uint32_t)hf);
    k_set<<<1, 1, 0, s>>>(P.ptr[0].as<uint32_t>(), hs_, (uint32_t)hfs);
  }
  L += 3;
  MMCSF_LAUNCH_CHECK();
  // derived arrays used by the MTTKRP kernels
  const int lf = nd - 2;
  const uint64_t nfib = P.n[lf];
  MMCSF_CUDA(P.fbr_like.alloc((P.n[1] + 1) * 4));
  MMCSF_CUDA(cudaMemsetAsync(P.fbr_like.p, 0, (P.n[1] + 1) * 4, s));
  if (hs_) {
    k_like_from_slices<<<grid_for(hs_, 256), 256, 0, s>>>(P.ptr[0].as<uint32_t>(), P.idx[0].as<uint32_t>(), hs_,
                                                          P.fbr_like.as<uint32_t>());
    MMCSF_LAUNCH_CHECK();
  }
  if (nd == 4 && hfs) {
    MMCSF_CUDA(P.fpar.alloc(hf * 4));
    k_fpar<<<grid_for(hfs, 256), 256, 0, s>>>(P.ptr[1].as<uint32_t>(), hfs, P.fpar.as<uint32_t>());
    MMCSF_LAUNCH_CHECK();
  }
  if (nfib) {
    k_flags<<<grid_for(nfib, 256), 256, 0, s>>>(P.leaf.as<uint32_t>(), P.ptr[lf].as<uint32_t>(), nfib);
    MMCSF_LAUNCH_CHECK();
  }
  // bins: CSF slices by nonzeros, CSL slices by fibers (UB[9] = all nonzeros + 1)
  MMCSF_CUDA(P.bin_of.alloc(hs_ * 4 + 4));
  if (hs_) {
    DevBuf nzs;
    if (nd == 3) {
      k_hyb_bins<<<grid_for(hs_, 256), 256, 0, s>>>(P.ptr[0].as<uint32_t>(), P.ptr[1].as<uint32_t>(), hs_, F->nnz,
                                                    P.bin_of.as<int32_t>());
    } else {
      // nonzero start of every fbrS: ptr2[ptr1[q]]
      std::vector<uint32_t> h1(hfs + 1), h2(hf + 1), z(hfs + 1);
      MMCSF_CUDA(cudaMemcpyAsync(h1.data(), P.ptr[1].p, (hfs + 1) * 4, cudaMemcpyDeviceToHost, s));
      MMCSF_CUDA(cudaMemcpyAsync(h2.data(), P.ptr[2].p, (hf + 1) * 4, cudaMemcpyDeviceToHost, s));
      MMCSF_CUDA(cudaStreamSynchronize(s));
      for (uint64_t q = 0; q <= hfs; ++q) z[q] = h2[h1[q]];
      MMCSF_CUDA(nzs.alloc((hfs + 1) * 4));
      MMCSF_CUDA(cudaMemcpyAsync(nzs.p, z.data(), (hfs + 1) * 4, cudaMemcpyHostToDevice, s));
      k_hyb_bins<<<grid_for(hs_, 256), 256, 0, s>>>(P.ptr[0].as<uint32_t>(), nzs.as<uint32_t>(), hs_, F->nnz,
                                                    P.bin_of.as<int32_t>());
    }
    MMCSF_LAUNCH_CHECK();
    MMCSF_CUDA(cudaStreamSynchronize(s));
  }
  if (nd == 3) {
    MMCSF_CUDA(H.csl_bin_of.alloc(H.n_csl_slices * 4 + 4));
    if (H.n_csl_slices) {
      k_hyb_bins<<<grid_for(H.n_csl_slices, 256), 256, 0, s>>>(H.csl_ptr.as<uint32_t>(), nullptr, H.n_csl_slices,
                                                               F->nnz, H.csl_bin_of.as<int32_t>());
      MMCSF_LAUNCH_CHECK();
    }
  }
  MMCSF_CUDA(cudaStreamSynchronize(s));
  L += 6;
  X = std::move(P);
  *launches += L;
  return MMCSF_OK;
}

// ---- HB-CSF MTTKRP: the COO and CSL parts (the CSF part runs k_mttkrp) ----

template <class T> __device__ __forceinline__ float ldf(const T* p);
template <> __device__ __forceinline__ float ldf<float>(const float* p) { return __ldg(p); }
template <> __device__ __forceinline__ float ldf<__nv_bfloat16>(const __nv_bfloat16* p) {
  return __bfloat162float(*p);
}

// COO part: one output row per nonzero (its slice holds only that nonzero),
// written without atomics as the reference does (src/mttkrp_gpu.cu:196-275).
template <class T>
__global__ void k_hyb_coo(int nd, uint64_t n, const uint32_t* i0, const uint32_t* i1, const uint32_t* i2,
                          const uint32_t* i3, const float* v, const T* U1, const T* U2, const T* U3, int R,
                          float* out) {
  const uint64_t total = n * (uint64_t)R;
  for (uint64_t t = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; t < total; t += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t x = t / R;
    const int r = (int)(t % R);
    float p = v[x] * ldf(U1 + (uint64_t)i1[x] * R + r) * ldf(U2 + (uint64_t)i2[x] * R + r);
    if (nd == 4) p *= ldf(U3 + (uint64_t)i3[x] * R + r);
    out[(uint64_t)i0[x] * R + r] += p;
  }
}

// CSL part (3-D): slice s owns nonzeros [ptr[s], ptr[s+1]); one thread per
// (slice, column) sums them and adds to the slice's output row.
template <class T>
__global__ void k_hyb_csl(uint64_t nslc, const uint32_t* ptr, const uint32_t* sidx, const uint32_t* i1,
                          const uint32_t* i2, const float* v, const T* U1, const T* U2, int R, float* out) {
  const uint64_t total = nslc * (uint64_t)R;
  for (uint64_t t = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; t < total; t += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t s = t / R;
    const int r = (int)(t % R);
    float acc = 0.f;
    for (uint32_t x = ptr[s]; x < ptr[s + 1]; ++x)
      acc += v[x] * ldf(U1 + (uint64_t)i1[x] * R + r) * ldf(U2 + (uint64_t)i2[x] * R + r);
    out[(uint64_t)sidx[s] * R + r] += acc;
  }
}

int hyb_extra_mttkrp(const mmcsf_format* F, int R, int dtype, const void* const* U, float* out, cudaStream_t s,
                     int* launches) {
  const HybExtra& H = F->hyb;
  const int nd = F->nd;
  const int* o = F->parts[0].order;  // level -> tensor mode
  auto run = [&](auto tag) -> int {
    using T = decltype(tag);
    const T* u[4];
    for (int l = 0; l < nd; ++l) u[l] = static_cast<const T*>(U[o[l]]);
    if (H.coo_nnz) {
      const uint64_t tot = H.coo_nnz * (uint64_t)R;
      k_hyb_coo<T><<<grid_for(tot, 256), 256, 0, s>>>(
          nd, H.coo_nnz, H.coo_inds[0].as<uint32_t>(), H.coo_inds[1].as<uint32_t>(), H.coo_inds[2].as<uint32_t>(),
          nd == 4 ? H.coo_inds[3].as<uint32_t>() : nullptr, H.coo_vals.as<float>(), u[1], u[2],
          nd == 4 ? u[3] : nullptr, R, out);
      MMCSF_LAUNCH_CHECK();
      ++*launches;
    }
    if (nd == 3 && H.n_csl_slices) {
      const uint64_t tot = H.n_csl_slices * (uint64_t)R;
      k_hyb_csl<T><<<grid_for(tot, 256), 256, 0, s>>>(H.n_csl_slices, H.csl_ptr.as<uint32_t>(),
                                                      H.csl_idx.as<uint32_t>(), H.csl_i1.as<uint32_t>(),
                                                      H.csl_i2.as<uint32_t>(), H.csl_vals.as<float>(), u[1], u[2], R,
                                                      out);
      MMCSF_LAUNCH_CHECK();
      ++*launches;
    }
    return MMCSF_OK;
  };
  if (dtype == MMCSF_DTYPE_F32) return run(float{});
  return run(__nv_bfloat16{});
}

}  // namespace mmcsf
