// MTTKRP kernels for MM-CSF / B-CSF / HB-CSF parts on sm_100a.
//
// The reference launches one warp (or -w warps) per fiber, strides lanes over
// the rank with scalar 4-byte loads, and issues atomicAdd per fiber (slice and
// fiber modes) or per nonzero (leaf mode) (src/mttkrp_gpu.cu:716-1509).
// Here every mode uses the same nonzero-balanced traversal:
//   * a TEAM of G lanes owns one factor row (R = 4*G*V floats, each lane V
//     float4 = 16 B vectors), so one warp works on 32/G nonzeros at once;
//   * a team walks a fixed, contiguous range of `chunk` nonzeros — skewed
//     fibers and slices cost the same as uniform ones — locating its first
//     fiber by binary search over the fiber pointers;
//   * the team loads G leaf indices and values with one coalesced access,
//     broadcasts them by shuffle, and issues all G row gathers before using
//     any, so G independent 16-byte loads per lane are in flight;
//   * products are accumulated in registers along the fiber / fbrS / slice
//     hierarchy and flushed with ONE vector atomic (red.global.add.v4.f32) per
//     output row segment: per slice run for the slice mode, per fiber or fbrS
//     for the middle modes, per nonzero for the leaf mode (which scatters).
// Correct for every R (the reference's kernels keep one scalar accumulator per
// lane across the rank loop and are wrong for R > 32).
#include <algorithm>
#include <cuda_bf16.h>

#include <cmath>
#include <cstring>
#include <type_traits>

#include "mttkrp_args.h"
#include "prims.cuh"

using mmcsf::set_error;

namespace mmcsf {
namespace {

bool native_R(int R) { return R == 4 || R == 8 || R == 16 || R == 32 || R == 64 || R == 128 || R == 256; }
int padded_R(int R) {
  const int opts[] = {4, 8, 16, 32, 64, 128, 256};
  for (int r : opts)
    if (r >= R) return r;
  return -1;
}

__global__ void k_pad_rows(const void* in, int esz, uint64_t rows, int R, int Rp, void* out) {
  const uint64_t n = rows * (uint64_t)Rp;
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
    uint64_t r = i / Rp, c = i % Rp;
    if (esz == 4) static_cast<float*>(out)[i] = c < (uint64_t)R ? static_cast<const float*>(in)[r * R + c] : 0.f;
    else static_cast<uint16_t*>(out)[i] = c < (uint64_t)R ? static_cast<const uint16_t*>(in)[r * R + c] : 0;
  }
}
__global__ void k_unpad_rows(const float* in, uint64_t rows, int R, int Rp, float* out) {
  const uint64_t n = rows * (uint64_t)R;
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
    out[i] = in[(i / R) * Rp + i % R];
}

int default_chunk(int R) {
  (void)R;
  return 512;
}

// Kernel arguments for part P (factors U by tensor mode, reordered by level).
template <class T>
void fill_args(Args<T>& a, const CsfPart& P, const float* vals_override, int slot, int chunk, int R,
               const void* const* U, float* out) {
  a.vals = vals_override ? vals_override : P.vals.as<float>();
  a.leaf = P.leaf.as<uint32_t>();
  const int lf = P.nd - 2;
  a.fptr = P.ptr[lf].as<uint32_t>();
  a.fidx = P.idx[lf].as<uint32_t>();
  a.fpar = P.fpar.as<uint32_t>();
  a.sidx1 = P.nd == 4 ? P.idx[1].as<uint32_t>() : nullptr;
  a.like = P.fbr_like.as<uint32_t>();
  a.cfib = slot >= 0 && P.cfib[slot].p ? P.cfib[slot].as<uint32_t>() : nullptr;
  a.mid = P.mid.as<uint32_t>();
  a.mid2 = P.mid2.as<uint32_t>();
  a.snz = P.snz.as<uint32_t>();
  a.sidx = P.idx[0].as<uint32_t>();
  a.cslc = slot >= 0 && P.cslc[slot].p ? P.cslc[slot].as<uint32_t>() : nullptr;
  a.nslc = (uint32_t)P.n[0];
  a.nnz = P.nnz;
  a.nfib = (uint32_t)P.n_fibers();
  a.chunk = (uint32_t)chunk;
  a.R = (uint32_t)R;
  for (int l = 0; l < P.nd; ++l) a.U[l] = static_cast<const T*>(U[P.order[l]]);
  a.out = out;
}

__global__ void k_add_f64(const double* __restrict__ in, uint64_t n, float* __restrict__ out) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
    out[i] = (float)((double)out[i] + in[i]);
}

// The format's scratch buffers grow on first use. cudaMalloc and cudaFree are
// not allowed while a stream is being captured (the failed call would also
// invalidate the capture), so a growth needed under capture is refused with a
// clear error instead: run the same call once uncaptured first (mmcsf_cpd
// allocates what its loop needs before it captures).
int no_alloc_in_capture(cudaStream_t s) {
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  if (cudaStreamIsCapturing(s, &cs) == cudaSuccess && cs != cudaStreamCaptureStatusNone)
    return set_error(MMCSF_ERR_UNSUPPORTED,
                     "a scratch buffer of the format must grow, which cannot happen during stream capture: "
                     "run the call once before capturing it");
  return MMCSF_OK;
}

// MTTKRP on one part for tensor mode `mode`; out must be zeroed by the caller.
int part_mttkrp(const mmcsf_format* F, const CsfPart& P, int mode, int R, int dtype, const void* const* U,
                float* out, const mmcsf_kernel_cfg* cfg, cudaStream_t s, int* launches,
                const float* vals_override = nullptr) {
  if (!P.present || P.nnz == 0) return MMCSF_OK;
  int lvl = -1;
  for (int l = 0; l < P.nd; ++l)
    if (P.order[l] == mode) lvl = l;
  if (lvl < 0) return set_error(MMCSF_ERR_INVALID, "mode %d not in part", mode);
  int chunk = cfg && cfg->chunk > 0 ? cfg->chunk : default_chunk(R);
  int threads = cfg && cfg->block_threads > 0 ? cfg->block_threads : 256;
  const int mb = cfg && cfg->min_blocks > 0 ? cfg->min_blocks : 2;
  int kern = cfg && cfg->kernel > 0 ? cfg->kernel : (P.nd == 3 ? 2 : 1);
  if (kern < 1 || kern > 7) return set_error(MMCSF_ERR_INVALID, "kernel must be 0 .. 7");
  if (kern == 7 && (P.nd != 3 || lvl != 0 || R < 16 || R > 128)) kern = 6;  // staged rows: 3-D slice level, R 16..128
  if (kern == 4 && (P.nd != 3 || lvl != 0)) kern = 3;  // per-fiber middle rows: the 3-D slice level only
  if (kern == 6 && (P.nd != 3 || lvl != 0)) kern = 5;  // warp-interleaved walk: the 3-D slice level only
  if (kern == 5 && P.nd != 3) kern = 3;                 // vector index loads: 3-D
  if ((kern == 4 || kern == 5 || kern == 6 || kern == 7) && !P.mid.p) kern = 2;
  if (kern == 3 && (!P.mid.p || (P.nd == 4 && lvl != 0 && lvl != 3))) kern = 2;  // per-nonzero walk not applicable
  if (kern == 2 && P.nd == 4) kern = 1;                                         // no 4-D branch-free fiber walk
  const int slot = CsfPart::cfib_slot((uint64_t)chunk);
  if (threads % 32 || threads > 256) return set_error(MMCSF_ERR_INVALID, "block_threads must be a multiple of 32, <= 256");
  // the leaf level scatters one reduction per nonzero: accumulate in FP64
  // (kept by the format), then add into the output once
  const bool leaf = lvl == P.nd - 1;
  const uint64_t nout = F->dims[mode] * (uint64_t)R;
  double* o64 = nullptr;
  if (leaf) {
    mmcsf_format* Fm = const_cast<mmcsf_format*>(F);
    if (Fm->leaf64.bytes < nout * 8) {
      MMCSF_TRY(no_alloc_in_capture(s));
      MMCSF_CUDA(Fm->leaf64.alloc(nout * 8));
    }
    o64 = Fm->leaf64.as<double>();
    MMCSF_CUDA(cudaMemsetAsync(o64, 0, nout * 8, s));
  }
  cudaError_t e;
  if (dtype == MMCSF_DTYPE_F32) {
    Args<float> a{};
    fill_args(a, P, vals_override, slot, chunk, R, U, out);
    a.out64 = o64;
    e = launch_R<float>(a, P.nd, lvl, kern, threads, mb, s);
  } else {
    Args<__nv_bfloat16> a{};
    fill_args(a, P, vals_override, slot, chunk, R, U, out);
    a.out64 = o64;
    e = launch_R<__nv_bfloat16>(a, P.nd, lvl, kern, threads, mb, s);
  }
  if (e != cudaSuccess) return set_error(MMCSF_ERR_CUDA, "MTTKRP launch failed: %s", cudaGetErrorString(e));
  if (launches) ++*launches;
  if (leaf) {
    k_add_f64<<<grid_for(nout, 256), 256, 0, s>>>(o64, nout, out);
    MMCSF_LAUNCH_CHECK();
    if (launches) ++*launches;
  }
  return MMCSF_OK;
}

}  // namespace

int hyb_extra_mttkrp(const mmcsf_format* F, int R, int dtype, const void* const* U, float* out, cudaStream_t s,
                     int* launches);  // hyb.cu

__global__ void k_reorder_vals(const float* __restrict__ in, const uint32_t* __restrict__ from, uint64_t n,
                               float* __restrict__ out) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
    out[i] = in[from[i]];
}

// One mode over every part that holds nonzeros (the reference's per-mode loop
// over partitions, src/mttkrp_gpu.cu:3578-3724). vals: optional values in the
// format's nonzero order replacing the tensor's (the sampled model's adjoint).
int mttkrp_mode_vals(const mmcsf_format* F, int mode, int R, int dtype, const void* const* U, const float* vals,
                     float* out, const mmcsf_kernel_cfg* cfg, cudaStream_t s, int* launches) {
  MMCSF_CUDA(cudaMemsetAsync(out, 0, F->dims[mode] * (uint64_t)R * sizeof(float), s));
  int trav = cfg ? cfg->traversal : 0;
  const int d = dtype == MMCSF_DTYPE_BF16 ? 1 : 0;  // the plan tuned for this factor type
  if (trav == 0) trav = F->plan_traversal[d][mode] ? F->plan_traversal[d][mode] : (F->views[mode].present ? 2 : 1);
  mmcsf_kernel_cfg c{};
  if (cfg) c = *cfg;
  if (c.chunk == 0) c.chunk = F->plan_chunk[d][mode];
  if (c.min_blocks == 0) c.min_blocks = F->plan_mb[d][mode];
  if (c.kernel == 0) c.kernel = F->plan_kernel[d][mode];
  if (trav == 2) {
    const CsfPart& V = F->views[mode];
    if (!V.present) return set_error(MMCSF_ERR_INVALID, "no view for mode %d (build with views)", mode);
    const float* vv = nullptr;
    if (vals) {
      mmcsf_format* Fm = const_cast<mmcsf_format*>(F);
      if (Fm->vals_scratch.bytes < V.nnz * 4) {
        MMCSF_TRY(no_alloc_in_capture(s));
        MMCSF_CUDA(Fm->vals_scratch.alloc(V.nnz * 4));
      }
      k_reorder_vals<<<grid_for(V.nnz, 256), 256, 0, s>>>(vals, V.from_part.as<uint32_t>(), V.nnz,
                                                          Fm->vals_scratch.as<float>());
      MMCSF_LAUNCH_CHECK();
      if (launches) ++*launches;
      vv = Fm->vals_scratch.as<float>();
    }
    return part_mttkrp(F, V, mode, R, dtype, U, out, &c, s, launches, vv);
  }
  uint64_t off = 0;  // caller values are in the format's order: partitions 0..nd-1
  for (int p = 0; p < F->nd; ++p) {
    MMCSF_TRY(part_mttkrp(F, F->parts[p], mode, R, dtype, U, out, &c, s, launches, vals ? vals + off : nullptr));
    if (F->parts[p].present) off += F->parts[p].nnz;
  }
  if (F->impl == MMCSF_IMPL_HBCSF) {
    if (vals) return set_error(MMCSF_ERR_UNSUPPORTED, "MTTKRP on other values is not available for HB-CSF");
    MMCSF_TRY(hyb_extra_mttkrp(F, R, dtype, U, out, s, launches));
  }
  return MMCSF_OK;
}

int mttkrp_mode(const mmcsf_format* F, int mode, int R, int dtype, const void* const* U, float* out,
                const mmcsf_kernel_cfg* cfg, cudaStream_t s, int* launches) {
  return mttkrp_mode_vals(F, mode, R, dtype, U, nullptr, out, cfg, s, launches);
}

// Allocate, now, the FP64 scratch that mttkrp_mode (default cfg) needs for
// every mode it walks at a partition's leaf level, so that later calls,
// captured ones included, allocate nothing.
int reserve_leaf_scratch(mmcsf_format* F, int R, int dtype) {
  const int d = dtype == MMCSF_DTYPE_BF16 ? 1 : 0;
  uint64_t need = 0;
  for (int m = 0; m < F->nd; ++m) {
    const int trav = F->plan_traversal[d][m] ? F->plan_traversal[d][m] : (F->views[m].present ? 2 : 1);
    if (trav == 2) continue;  // a view walks the mode at level 0
    for (int p = 0; p < F->nd; ++p) {
      const CsfPart& P = F->parts[p];
      if (P.present && P.nnz && P.order[P.nd - 1] == m) need = std::max(need, F->dims[m] * (uint64_t)R * 8);
    }
  }
  if (need > F->leaf64.bytes) MMCSF_CUDA(F->leaf64.alloc(need));
  return MMCSF_OK;
}

}  // namespace mmcsf

using namespace mmcsf;

namespace {
int check_call(const mmcsf_format* F, int R, int dtype) {
  if (!F) return set_error(MMCSF_ERR_INVALID, "null format");
  if (R < 1) return set_error(MMCSF_ERR_INVALID, "rank must be >= 1");
  if (dtype != MMCSF_DTYPE_F32 && dtype != MMCSF_DTYPE_BF16) return set_error(MMCSF_ERR_INVALID, "bad dtype");
  if (R > 256) return set_error(MMCSF_ERR_UNSUPPORTED, "rank %d > 256", R);
  return MMCSF_OK;
}

// Run `fn(U, out_for_mode)` with rank padded to a native kernel width when R is
// not one (factors copied into zero-padded buffers, outputs copied back).
template <class Fn>
int with_padding(const mmcsf_format* F, int R, int dtype, const void* const* U, Fn fn, cudaStream_t s) {
  if (native_R(R)) return fn(R, U);
  const int Rp = padded_R(R);
  const int esz = dtype == MMCSF_DTYPE_F32 ? 4 : 2;
  DevBuf pu[4];
  const void* pp[4] = {nullptr, nullptr, nullptr, nullptr};
  for (int m = 0; m < F->nd; ++m) {
    MMCSF_CUDA(pu[m].alloc(F->dims[m] * (uint64_t)Rp * esz));
    k_pad_rows<<<grid_for(F->dims[m] * (uint64_t)Rp, 256), 256, 0, s>>>(U[m], esz, F->dims[m], R, Rp, pu[m].p);
    MMCSF_LAUNCH_CHECK();
    pp[m] = pu[m].p;
  }
  int st = fn(Rp, pp);
  MMCSF_CUDA(cudaStreamSynchronize(s));
  return st;
}
}  // namespace

extern "C" int mmcsf_mttkrp(const mmcsf_format* F, int mode, int R, int factor_dtype, const void* const* d_factors,
                            float* d_out, const mmcsf_kernel_cfg* cfg, void* stream) {
  MMCSF_RANGE("mmcsf_mttkrp");
  MMCSF_TRY(check_call(F, R, factor_dtype));
  if (mode < 0 || mode >= F->nd) return set_error(MMCSF_ERR_INVALID, "Mode cannot be larger than tensor dimension.");
  MMCSF_TRY(bounds_gate(F, stream));
  if (!d_factors || !d_out) return set_error(MMCSF_ERR_INVALID, "null pointer");
  if (F->impl != MMCSF_IMPL_MMCSF && mode != F->mode)
    return set_error(MMCSF_ERR_INVALID, "this format was built for mode %d only", F->mode);
  cudaStream_t s = S(stream);
  mmcsf_format* Fm = const_cast<mmcsf_format*>(F);
  int launches = 0;
  int st = with_padding(F, R, factor_dtype, d_factors, [&](int Rk, const void* const* U) -> int {
    if (Rk == R) return mttkrp_mode(F, mode, R, factor_dtype, U, d_out, cfg, s, &launches);
    DevBuf tmp;
    MMCSF_CUDA(tmp.alloc(F->dims[mode] * (uint64_t)Rk * 4));
    MMCSF_TRY(mttkrp_mode(F, mode, Rk, factor_dtype, U, tmp.as<float>(), cfg, s, &launches));
    k_unpad_rows<<<grid_for(F->dims[mode] * (uint64_t)R, 256), 256, 0, s>>>(tmp.as<float>(), F->dims[mode], R, Rk,
                                                                           d_out);
    MMCSF_LAUNCH_CHECK();
    MMCSF_CUDA(cudaStreamSynchronize(s));
    return MMCSF_OK;
  }, s);
  Fm->last_launches = launches;
  return st;
}

__global__ void k_to_bf16(const float* __restrict__ in, __nv_bfloat16* __restrict__ out, uint64_t n) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
    out[i] = __float2bfloat16_rn(in[i]);
}

// sums[0] += sum (a - b)^2, sums[1] += sum b^2 (FP64)
__global__ void k_diff_norms(const float* __restrict__ a, const float* __restrict__ b, uint64_t n,
                             double* __restrict__ sums) {
  __shared__ double p0[256], p1[256];
  double s0 = 0, s1 = 0;
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
    const double d = (double)a[i] - (double)b[i];
    s0 += d * d;
    s1 += (double)b[i] * (double)b[i];
  }
  p0[threadIdx.x] = s0;
  p1[threadIdx.x] = s1;
  __syncthreads();
  for (int w = 128; w > 0; w >>= 1) {
    if (threadIdx.x < w) { p0[threadIdx.x] += p0[threadIdx.x + w]; p1[threadIdx.x] += p1[threadIdx.x + w]; }
    __syncthreads();
  }
  if (threadIdx.x == 0) { atomicAdd(sums, p0[0]); atomicAdd(sums + 1, p1[0]); }
}

__global__ void k_scale_cols(float* __restrict__ M, uint64_t rows, int R, const float* __restrict__ lam) {
  const uint64_t n = rows * (uint64_t)R;
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
    M[i] *= __ldg(lam + i % R);
}

extern "C" int mmcsf_cp_adjoint(const mmcsf_format* F, int mode, int R, int factor_dtype,
                                const void* const* d_factors, const float* d_lambda, const float* d_grad,
                                float* d_out, const mmcsf_kernel_cfg* cfg, void* stream) {
  MMCSF_RANGE("mmcsf_cp_adjoint");
  MMCSF_TRY(check_call(F, R, factor_dtype));
  if (mode < 0 || mode >= F->nd) return set_error(MMCSF_ERR_INVALID, "Mode cannot be larger than tensor dimension.");
  MMCSF_TRY(bounds_gate(F, stream));
  if (!d_factors || !d_out || !d_grad) return set_error(MMCSF_ERR_INVALID, "null pointer");
  if (F->impl == MMCSF_IMPL_HBCSF) return set_error(MMCSF_ERR_UNSUPPORTED, "not available for HB-CSF formats");
  if (F->impl != MMCSF_IMPL_MMCSF && mode != F->mode)
    return set_error(MMCSF_ERR_INVALID, "this format was built for mode %d only", F->mode);
  cudaStream_t s = S(stream);
  mmcsf_format* Fm = const_cast<mmcsf_format*>(F);
  int launches = 0;
  int st = with_padding(F, R, factor_dtype, d_factors, [&](int Rk, const void* const* U) -> int {
    if (Rk == R) return mttkrp_mode_vals(F, mode, R, factor_dtype, U, d_grad, d_out, cfg, s, &launches);
    DevBuf tmp;
    MMCSF_CUDA(tmp.alloc(F->dims[mode] * (uint64_t)Rk * 4));
    MMCSF_TRY(mttkrp_mode_vals(F, mode, Rk, factor_dtype, U, d_grad, tmp.as<float>(), cfg, s, &launches));
    k_unpad_rows<<<grid_for(F->dims[mode] * (uint64_t)R, 256), 256, 0, s>>>(tmp.as<float>(), F->dims[mode], R, Rk,
                                                                           d_out);
    MMCSF_LAUNCH_CHECK();
    MMCSF_CUDA(cudaStreamSynchronize(s));
    return MMCSF_OK;
  }, s);
  if (st == MMCSF_OK && d_lambda) {
    k_scale_cols<<<grid_for(F->dims[mode] * (uint64_t)R, 256), 256, 0, s>>>(d_out, F->dims[mode], R, d_lambda);
    MMCSF_LAUNCH_CHECK();
    ++launches;
  }
  Fm->last_launches = launches;
  return st;
}

extern "C" int mmcsf_mttkrp_pair(const mmcsf_format* F, int R, int factor_dtype, const void* const* d_factors,
                                 float* d_out_slice, float* d_out_mid, int* modes, const mmcsf_kernel_cfg* cfg,
                                 void* stream) {
  MMCSF_RANGE("mmcsf_mttkrp_pair");
  MMCSF_TRY(check_call(F, R, factor_dtype));
  if (F->impl != MMCSF_IMPL_MMCSF) return set_error(MMCSF_ERR_INVALID, "the two-output walk needs an MM-CSF format");
  const CsfPart* P = nullptr;
  int np = 0;
  for (int p = 0; p < F->nd; ++p)
    if (F->parts[p].present) { P = &F->parts[p]; ++np; }
  if (np > 1) return set_error(MMCSF_ERR_UNSUPPORTED, "the two-output walk needs a single-partition format");
  if (!P || !P->mid.p || (P->nd == 4 && !P->mid2.p))
    return set_error(MMCSF_ERR_UNSUPPORTED, "the two-output walk needs the per-nonzero middle indices");
  if (modes) { modes[0] = P->order[0]; modes[1] = P->order[1]; }
  if (!d_factors || !d_out_slice || !d_out_mid) return modes ? MMCSF_OK : set_error(MMCSF_ERR_INVALID, "null pointer");
  MMCSF_TRY(bounds_gate(F, stream));
  if (!native_R(R) || R > 128) return set_error(MMCSF_ERR_UNSUPPORTED, "the two-output walk runs R in 4..128");
  cudaStream_t s = S(stream);
  MMCSF_CUDA(cudaMemsetAsync(d_out_slice, 0, F->dims[P->order[0]] * (uint64_t)R * sizeof(float), s));
  MMCSF_CUDA(cudaMemsetAsync(d_out_mid, 0, F->dims[P->order[1]] * (uint64_t)R * sizeof(float), s));
  const int d = factor_dtype == MMCSF_DTYPE_BF16 ? 1 : 0;
  const int chunk = cfg && cfg->chunk > 0 ? cfg->chunk : (F->pair_chunk[d] ? F->pair_chunk[d] : 256);
  const int threads = cfg && cfg->block_threads > 0 ? cfg->block_threads : 256;
  const int mb = cfg && cfg->min_blocks > 0 ? cfg->min_blocks : (F->pair_mb[d] ? F->pair_mb[d] : 3);
  const int kern = cfg && cfg->kernel > 0 ? cfg->kernel : F->pair_kernel[d];
  if (kern < 0 || kern > 7) return set_error(MMCSF_ERR_INVALID, "kernel must be 0 .. 7");
  if (threads % 32 || threads > 256) return set_error(MMCSF_ERR_INVALID, "block_threads must be a multiple of 32, <= 256");
  const int slot = CsfPart::cfib_slot((uint64_t)chunk);
  cudaError_t e;
  if (factor_dtype == MMCSF_DTYPE_F32) {
    Args<float> a{};
    fill_args(a, *P, nullptr, slot, chunk, R, d_factors, d_out_slice);
    a.out2 = d_out_mid;
    e = launch_pair_R<float>(a, P->nd, threads, mb, kern, s);
  } else {
    Args<__nv_bfloat16> a{};
    fill_args(a, *P, nullptr, slot, chunk, R, d_factors, d_out_slice);
    a.out2 = d_out_mid;
    e = launch_pair_R<__nv_bfloat16>(a, P->nd, threads, mb, kern, s);
  }
  if (e != cudaSuccess) return set_error(MMCSF_ERR_CUDA, "two-output walk launch: %s", cudaGetErrorString(e));
  const_cast<mmcsf_format*>(F)->last_launches = 1;
  return MMCSF_OK;
}

namespace {
// The tuned plan runs the partition's two upper modes in one walk (only
// without a caller override of the traversal or kernel). modes[0..1] get
// them.
bool pair_active(const mmcsf_format* F, int R, bool want, const mmcsf_kernel_cfg* cfg, int* modes) {
  if (!want || F->impl != MMCSF_IMPL_MMCSF || !native_R(R) || R > 128) return false;
  if (cfg && (cfg->traversal != 0 || cfg->kernel != 0)) return false;
  const CsfPart* P = nullptr;
  for (int p = 0; p < F->nd; ++p)
    if (F->parts[p].present) {
      if (P) return false;  // several partitions
      P = &F->parts[p];
    }
  if (!P || !P->mid.p) return false;
  modes[0] = P->order[0];
  modes[1] = P->order[1];
  return true;
}
}  // namespace

extern "C" int mmcsf_mttkrp_all(const mmcsf_format* F, int R, int factor_dtype, const void* const* d_factors,
                                float* const* d_outs, const mmcsf_kernel_cfg* cfg, void* stream) {
  MMCSF_RANGE("mmcsf_mttkrp_all");
  MMCSF_TRY(check_call(F, R, factor_dtype));
  if (!d_factors || !d_outs) return set_error(MMCSF_ERR_INVALID, "null pointer");
  MMCSF_TRY(bounds_gate(F, stream));
  if (F->impl != MMCSF_IMPL_MMCSF)
    return set_error(MMCSF_ERR_INVALID, "all-mode MTTKRP needs an MM-CSF format (-t 12)");
  int total = 0;
  int pm[2] = {-1, -1};
  // a per-mode precision plan (mmcsf_tune_precision) with FP32 factors: the
  // launches it assigns to BF16 read BF16 copies of the factors, converted here
  const bool mixed = F->mixed && factor_dtype == MMCSF_DTYPE_F32 && !(cfg && (cfg->traversal || cfg->kernel));
  const void* bf[4] = {nullptr, nullptr, nullptr, nullptr};
  auto dt_of = [&](int m) { return mixed ? F->mode_dtype[m] : factor_dtype; };
  const int pdt = mixed ? F->pair_dtype : factor_dtype;
  bool need_bf16 = false;
  if (mixed) {
    for (int m = 0; m < F->nd; ++m) need_bf16 = need_bf16 || F->mode_dtype[m] == MMCSF_DTYPE_BF16;
    need_bf16 = need_bf16 || (F->mixed_pair && F->pair_dtype == MMCSF_DTYPE_BF16);
  }
  if (need_bf16) {
    cudaStream_t s = S(stream);
    for (int m = 0; m < F->nd; ++m) {
      const uint64_t n = F->dims[m] * (uint64_t)R;
      if (F->bf16_fac[m].bytes < n * 2)  // kept by the format between calls (allocated on first use)
        MMCSF_CUDA(const_cast<mmcsf_format*>(F)->bf16_fac[m].alloc(n * 2));
      k_to_bf16<<<grid_for(n, 256), 256, 0, s>>>(static_cast<const float*>(d_factors[m]),
                                                 F->bf16_fac[m].as<__nv_bfloat16>(), n);
      MMCSF_LAUNCH_CHECK();
      bf[m] = F->bf16_fac[m].p;
      ++total;
    }
  }
  auto fac = [&](int dt) { return dt == MMCSF_DTYPE_BF16 && need_bf16 ? bf : d_factors; };
  const bool pair = pair_active(F, R, mixed ? F->mixed_pair : F->pair_use[factor_dtype == MMCSF_DTYPE_BF16 ? 1 : 0],
                                cfg, pm);
  if (pair) {
    MMCSF_TRY(mmcsf_mttkrp_pair(F, R, pdt, fac(pdt), d_outs[pm[0]], d_outs[pm[1]], nullptr, nullptr, stream));
    total += F->last_launches;
  }
  for (int m = 0; m < F->nd; ++m) {
    if (pair && (m == pm[0] || m == pm[1])) continue;
    MMCSF_TRY(mmcsf_mttkrp(F, m, R, dt_of(m), fac(dt_of(m)), d_outs[m], cfg, stream));
    total += F->last_launches;
  }
  const_cast<mmcsf_format*>(F)->last_launches = total;
  return MMCSF_OK;
}

// Host-buffer all-mode MTTKRP with the copies overlapped with the kernels:
// the mode whose inputs exclude the largest factor runs first, as soon as the
// other factors are on the device, while the largest factor is uploaded on a
// second stream; every output is downloaded on a third stream right after its
// mode finishes. With pinned host buffers the copies and kernels overlap.
extern "C" int mmcsf_mttkrp_all_host(mmcsf_format* F, int R, const float* const* h_factors, float* const* h_outs,
                                     const mmcsf_kernel_cfg* cfg, void* stream) {
  MMCSF_RANGE("mmcsf_mttkrp_all_host");
  MMCSF_TRY(check_call(F, R, MMCSF_DTYPE_F32));
  if (!h_factors || !h_outs) return set_error(MMCSF_ERR_INVALID, "null pointer");
  MMCSF_TRY(bounds_gate(F, stream));
  if (F->impl != MMCSF_IMPL_MMCSF)
    return set_error(MMCSF_ERR_INVALID, "all-mode MTTKRP needs an MM-CSF format (-t 12)");
  cudaStream_t s = S(stream);
  const int nd = F->nd;
  if (F->stage_R != R) {
    for (int m = 0; m < nd; ++m) {
      MMCSF_CUDA(F->stage_in[m].alloc(F->dims[m] * (uint64_t)R * 4));
      MMCSF_CUDA(F->stage_out[m].alloc(F->dims[m] * (uint64_t)R * 4));
    }
    F->stage_R = R;
  }
  if (!F->copy_in) {
    MMCSF_CUDA(cudaStreamCreateWithFlags(&F->copy_in, cudaStreamNonBlocking));
    MMCSF_CUDA(cudaStreamCreateWithFlags(&F->copy_out, cudaStreamNonBlocking));
    for (int m = 0; m < 4; ++m) {
      MMCSF_CUDA(cudaEventCreateWithFlags(&F->ev_in[m], cudaEventDisableTiming));
      MMCSF_CUDA(cudaEventCreateWithFlags(&F->ev_done[m], cudaEventDisableTiming));
    }
    MMCSF_CUDA(cudaEventCreateWithFlags(&F->ev_start, cudaEventDisableTiming));
  }
  // order: the largest factor is uploaded last; its own mode (which does not
  // read it) runs first, and its output's download overlaps that upload. The
  // two-output walk is not used here: once the last factor has arrived, one
  // launch per mode lets the first output's download overlap the next launch
  // (measured 9.23 against 9.45 ms per call on the 100M-nonzero skewed 3-D
  // tensor, where the copies take ~6 ms each way).
  int big = 0;
  for (int m = 1; m < nd; ++m)
    if (F->dims[m] > F->dims[big]) big = m;
  int order[4], n = 0;
  order[n++] = big;
  for (int m = 0; m < nd; ++m)
    if (m != big) order[n++] = m;
  // then the larger outputs first, so that their downloads start earlier
  std::stable_sort(order + 1, order + nd, [&](int x, int y) { return F->dims[x] > F->dims[y]; });
  const void* din[4];
  MMCSF_CUDA(cudaEventRecord(F->ev_start, s));  // staging buffers are free once earlier work on s is done
  MMCSF_CUDA(cudaStreamWaitEvent(F->copy_in, F->ev_start, 0));
  for (int m = 0; m < nd; ++m) din[m] = F->stage_in[m].p;
  for (int q = 0; q < nd; ++q) {  // upload: all but the largest, then the largest
    const int m = q < nd - 1 ? order[q + 1] : big;
    MMCSF_CUDA(cudaMemcpyAsync(F->stage_in[m].p, h_factors[m], F->dims[m] * (uint64_t)R * 4,
                               cudaMemcpyHostToDevice, F->copy_in));
    MMCSF_CUDA(cudaEventRecord(F->ev_in[m], F->copy_in));
  }
  int total = 0;
  auto download = [&](int m) -> int {
    MMCSF_CUDA(cudaEventRecord(F->ev_done[m], s));
    MMCSF_CUDA(cudaStreamWaitEvent(F->copy_out, F->ev_done[m], 0));
    MMCSF_CUDA(cudaMemcpyAsync(h_outs[m], F->stage_out[m].p, F->dims[m] * (uint64_t)R * 4, cudaMemcpyDeviceToHost,
                               F->copy_out));
    return MMCSF_OK;
  };
  for (int q = 0; q < nd; ++q) {
    const int m = order[q];
    for (int p = 0; p < nd; ++p)
      if (p != m) MMCSF_CUDA(cudaStreamWaitEvent(s, F->ev_in[p], 0));
    MMCSF_TRY(mmcsf_mttkrp(F, m, R, MMCSF_DTYPE_F32, din, F->stage_out[m].as<float>(), cfg, stream));
    total += F->last_launches;
    MMCSF_TRY(download(m));
  }
  MMCSF_CUDA(cudaStreamSynchronize(F->copy_out));
  MMCSF_CUDA(cudaStreamSynchronize(s));
  F->last_launches = total;
  return MMCSF_OK;
}

extern "C" int mmcsf_tune(mmcsf_format* F, int R, int factor_dtype, const void* const* d_factors,
                          float* const* d_outs, void* stream, mmcsf_plan* plan) {
  MMCSF_RANGE("mmcsf_tune");
  MMCSF_TRY(check_call(F, R, factor_dtype));
  if (!d_factors || !d_outs) return set_error(MMCSF_ERR_INVALID, "null pointer");
  const int d = factor_dtype == MMCSF_DTYPE_BF16 ? 1 : 0;
  cudaStream_t s = S(stream);
  cudaEvent_t e0, e1;
  MMCSF_CUDA(cudaEventCreate(&e0));
  MMCSF_CUDA(cudaEventCreate(&e1));
  const int chunks[] = {128, 256, 512, 1024, 2048, 4096};
  const int nmodes = F->impl == MMCSF_IMPL_MMCSF ? F->nd : 1;
  float best_ms[4] = {0, 0, 0, 0};
  int st = MMCSF_OK;
  F->mixed = false;  // a plain tune runs every launch at the caller's factor type
  for (int i = 0; i < nmodes && st == MMCSF_OK; ++i) {
    const int m = F->impl == MMCSF_IMPL_MMCSF ? i : F->mode;
    float best = 1e30f;
    int bt = 1, bc = 512, bm = 2, bk = 1;
    const int nkern = 7;
    for (int trav = 1; trav <= 2 && st == MMCSF_OK; ++trav) {
      if (trav == 2 && !F->views[m].present) continue;
      for (int kern = 1; kern <= nkern && st == MMCSF_OK; ++kern) {
      if (kern == 2 && F->nd == 4) continue;  // 4-D has no branch-free fiber walk
      if (kern == 5 && (F->nd != 3 || R < 16)) continue;  // vector index loads: 3-D, teams of >= 4 lanes
      if (kern == 6 && (F->nd != 3 || R < 8)) continue;   // warp-interleaved walk: 3-D
      if (kern == 7 && (F->nd != 3 || R < 16 || R > 128)) continue;  // staged rows: 3-D, R 16..128
      if (kern == 4 || kern == 7) {  // per-fiber middle rows: only where the mode is the slice level of a 3-D part with `mid`
        const CsfPart* tp = nullptr;
        if (trav == 2) tp = &F->views[m];
        else
          for (int p = 0; p < F->nd; ++p)
            if (F->parts[p].present) { tp = &F->parts[p]; break; }
        if (!tp || tp->nd != 3 || tp->order[0] != m || !tp->mid.p) continue;
        if (trav == 1 && F->impl == MMCSF_IMPL_MMCSF) {  // every partition must have m at level 0
          bool all0 = true;
          for (int p = 0; p < F->nd; ++p)
            if (F->parts[p].present && F->parts[p].order[0] != m) all0 = false;
          if (!all0) continue;
        }
      }
      // one launch to warm up, the next one timed
      auto time_cfg = [&](int c, int mbv, float* ms) {
        mmcsf_kernel_cfg cfg{};
        cfg.chunk = c;
        cfg.traversal = trav;
        cfg.min_blocks = mbv;
        cfg.kernel = kern;
        if ((st = mmcsf_mttkrp(F, m, R, factor_dtype, d_factors, d_outs[m], &cfg, stream)) != MMCSF_OK) return;
        if (cudaEventRecord(e0, s) != cudaSuccess) { st = MMCSF_ERR_CUDA; return; }
        if ((st = mmcsf_mttkrp(F, m, R, factor_dtype, d_factors, d_outs[m], &cfg, stream)) != MMCSF_OK) return;
        if (cudaEventRecord(e1, s) != cudaSuccess || cudaEventSynchronize(e1) != cudaSuccess) {
          st = MMCSF_ERR_CUDA;
          return;
        }
        cudaEventElapsedTime(ms, e0, e1);
        if (*ms < best) { best = *ms; bt = trav; bc = c; bm = mbv; bk = kern; }
      };
      // a traversal and kernel more than twice as slow as the best so far at
      // a middle launch shape is not swept over every shape
      if (best < 1e30f) {
        float probe = 0;
        time_cfg(512, 2, &probe);
        if (st != MMCSF_OK) break;
        if (probe > 2.f * best) continue;
      }
      for (int mbv = 1; mbv <= 4 && st == MMCSF_OK; ++mbv) {
        for (int c : chunks) {
          if (kern == 7 && c != chunks[0]) break;  // kernel 7 sizes its own ranges: one timing per level
          float ms = 0;
          time_cfg(c, mbv, &ms);
          if (st != MMCSF_OK) break;
        }
      }
      }
    }
    F->plan_traversal[d][m] = bt;
    F->plan_chunk[d][m] = bc;
    F->plan_mb[d][m] = bm;
    F->plan_kernel[d][m] = bk;
    F->plan_ms[d][m] = best;
    best_ms[m] = best;
    if (plan) {
      plan->traversal[m] = bt;
      plan->chunk[m] = bc;
      plan->min_blocks[m] = bm;
      plan->kernel[m] = bk;
      plan->ms[m] = best;
    }
  }
  // the two upper modes of the partition in one walk, kept when it beats the
  // two modes' best single-mode plans
  F->pair_use[d] = false;
  F->pair_ms[d] = 0.f;
  int pm[2] = {-1, -1};
  if (st == MMCSF_OK && F->impl == MMCSF_IMPL_MMCSF &&
      mmcsf_mttkrp_pair(F, R, factor_dtype, nullptr, nullptr, nullptr, pm, nullptr, stream) == MMCSF_OK &&
      native_R(R) && R <= 128) {
    float bestp = 1e30f;
    int bpc = 0, bpm = 0, bpk = 0;
    for (int kern : {2, 3, 4, 5, 6, 7})
    for (int mbv = 1; mbv <= (kern == 7 ? 4 : 3) && st == MMCSF_OK && (kern == 3 || F->nd == 3) &&
                      (kern != 5 || R >= 16) && (kern != 6 || R >= 8) && (kern != 7 || R >= 16);
         ++mbv)
      for (int c : {256, 512, 1024}) {
        if (kern == 7 && c != 256) break;  // kernel 7 sizes its own ranges
        mmcsf_kernel_cfg cfg{};
        cfg.chunk = c;
        cfg.min_blocks = mbv;
        cfg.kernel = kern;
        float ms = 0;
        for (int rep = 0; rep < 2; ++rep) {
          if ((st = mmcsf_mttkrp_pair(F, R, factor_dtype, d_factors, d_outs[pm[0]], d_outs[pm[1]], nullptr, &cfg,
                                      stream)) != MMCSF_OK)
            break;
          if (cudaEventRecord(e0, s) != cudaSuccess) { st = MMCSF_ERR_CUDA; break; }
          if ((st = mmcsf_mttkrp_pair(F, R, factor_dtype, d_factors, d_outs[pm[0]], d_outs[pm[1]], nullptr, &cfg,
                                      stream)) != MMCSF_OK)
            break;
          if (cudaEventRecord(e1, s) != cudaSuccess || cudaEventSynchronize(e1) != cudaSuccess) {
            st = MMCSF_ERR_CUDA;
            break;
          }
          cudaEventElapsedTime(&ms, e0, e1);
        }
        if (st != MMCSF_OK) break;
        if (ms < bestp) { bestp = ms; bpc = c; bpm = mbv; bpk = kern; }
      }
    if (st == MMCSF_OK) {
      F->pair_use[d] = bestp < best_ms[pm[0]] + best_ms[pm[1]];
      F->pair_chunk[d] = bpc;
      F->pair_mb[d] = bpm;
      F->pair_kernel[d] = bpk;
      F->pair_ms[d] = bestp;
    }
    if (plan && st == MMCSF_OK) {
      plan->pair = F->pair_use[d] ? 1 : 0;
      plan->pair_chunk = bpc;
      plan->pair_min_blocks = bpm;
      plan->pair_kernel = bpk;
      plan->pair_ms = bestp;
    }
  } else if (plan) {
    plan->pair = 0;
    plan->pair_chunk = plan->pair_min_blocks = plan->pair_kernel = 0;
    plan->pair_ms = 0.f;
  }
  if (plan) {
    plan->factor_dtype = factor_dtype;
    plan->mixed = 0;
    for (int m = 0; m < 4; ++m) {
      plan->mode_dtype[m] = factor_dtype;
      plan->bf16_error[m] = 0.f;
    }
    plan->pair_dtype = factor_dtype;
    // -f of the format: 0 for no split (the reference's default 99999999, src/util.h:212)
    plan->fiber_threshold = F->fiber_threshold_tuned >= 0 ? F->fiber_threshold_tuned
                            : (F->fbr_th >= 99999999ull ? 0 : (int)std::min<uint64_t>(F->fbr_th, 0x7fffffff));
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  return st;
}

namespace {
// Relative Frobenius norm ||a - b|| / ||b|| of two device arrays.
int rel_frob(const float* a, const float* b, uint64_t n, cudaStream_t s, double* out) {
  DevBuf sums;
  MMCSF_CUDA(sums.alloc(16));
  MMCSF_CUDA(cudaMemsetAsync(sums.p, 0, 16, s));
  k_diff_norms<<<std::min<uint64_t>(grid_for(n, 256), (uint64_t)sm_count() * 8), 256, 0, s>>>(a, b, n,
                                                                                                sums.as<double>());
  MMCSF_LAUNCH_CHECK();
  double h[2] = {0, 0};
  MMCSF_CUDA(cudaMemcpyAsync(h, sums.p, 16, cudaMemcpyDeviceToHost, s));
  MMCSF_CUDA(cudaStreamSynchronize(s));
  *out = h[1] > 0 ? std::sqrt(h[0] / h[1]) : (h[0] > 0 ? 1.0 : 0.0);
  return MMCSF_OK;
}
}  // namespace

extern "C" int mmcsf_tune_precision(mmcsf_format* F, int R, const float* const* d_factors, float* const* d_outs,
                                    double error_budget, void* stream, mmcsf_plan* plan) {
  MMCSF_RANGE("mmcsf_tune_precision");
  MMCSF_TRY(check_call(F, R, MMCSF_DTYPE_F32));
  if (!d_factors || !d_outs) return set_error(MMCSF_ERR_INVALID, "null pointer");
  if (F->impl != MMCSF_IMPL_MMCSF)
    return set_error(MMCSF_ERR_INVALID, "per-mode precision plans are for MM-CSF formats (-t 12)");
  if (!(error_budget >= 0)) return set_error(MMCSF_ERR_INVALID, "error budget must be >= 0");
  cudaStream_t s = S(stream);
  const int nd = F->nd;
  const void* f32[4] = {d_factors[0], d_factors[1], d_factors[2], nd == 4 ? d_factors[3] : nullptr};
  const void* b16[4] = {nullptr, nullptr, nullptr, nullptr};
  uint64_t maxrows = 0;
  for (int m = 0; m < nd; ++m) {
    const uint64_t n = F->dims[m] * (uint64_t)R;
    if (F->bf16_fac[m].bytes < n * 2) MMCSF_CUDA(F->bf16_fac[m].alloc(n * 2));
    b16[m] = F->bf16_fac[m].p;
    maxrows = std::max(maxrows, F->dims[m]);
  }
  // the conversion every mixed all-mode call makes, timed
  cudaEvent_t e0, e1;
  MMCSF_CUDA(cudaEventCreate(&e0));
  MMCSF_CUDA(cudaEventCreate(&e1));
  float conv_ms = 0;
  for (int rep = 0; rep < 2; ++rep) {
    MMCSF_CUDA(cudaEventRecord(e0, s));
    for (int m = 0; m < nd; ++m) {
      const uint64_t n = F->dims[m] * (uint64_t)R;
      k_to_bf16<<<grid_for(n, 256), 256, 0, s>>>(d_factors[m], F->bf16_fac[m].as<__nv_bfloat16>(), n);
      MMCSF_LAUNCH_CHECK();
    }
    MMCSF_CUDA(cudaEventRecord(e1, s));
    MMCSF_CUDA(cudaEventSynchronize(e1));
    cudaEventElapsedTime(&conv_ms, e0, e1);
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  mmcsf_plan p32{}, p16{};
  MMCSF_TRY(mmcsf_tune(F, R, MMCSF_DTYPE_F32, f32, d_outs, stream, &p32));
  MMCSF_TRY(mmcsf_tune(F, R, MMCSF_DTYPE_BF16, b16, d_outs, stream, &p16));
  // the error BF16 factors cost, per mode: the BF16-factor output against the FP32-factor output
  DevBuf tmp;
  MMCSF_CUDA(tmp.alloc(maxrows * R * 4));
  double err[4] = {0, 0, 0, 0};
  for (int m = 0; m < nd; ++m) {
    MMCSF_TRY(mmcsf_mttkrp(F, m, R, MMCSF_DTYPE_F32, f32, d_outs[m], nullptr, stream));
    MMCSF_TRY(mmcsf_mttkrp(F, m, R, MMCSF_DTYPE_BF16, b16, tmp.as<float>(), nullptr, stream));
    MMCSF_TRY(rel_frob(tmp.as<float>(), d_outs[m], F->dims[m] * (uint64_t)R, s, &err[m]));
  }
  // choose: per mode the faster type within the budget; the two-output walk
  // at the faster admissible type when it beats its two modes
  int dt[4] = {0, 0, 0, 0};
  float unit_ms[4] = {0, 0, 0, 0};
  for (int m = 0; m < nd; ++m) {
    const bool ok16 = err[m] <= error_budget;
    dt[m] = (ok16 && p16.ms[m] < p32.ms[m]) ? MMCSF_DTYPE_BF16 : MMCSF_DTYPE_F32;
    unit_ms[m] = dt[m] == MMCSF_DTYPE_BF16 ? p16.ms[m] : p32.ms[m];
  }
  bool use_pair = false;
  int pdt = MMCSF_DTYPE_F32;
  int pm[2] = {-1, -1};
  if (mmcsf_mttkrp_pair(F, R, MMCSF_DTYPE_F32, nullptr, nullptr, nullptr, pm, nullptr, stream) == MMCSF_OK &&
      p32.pair_ms > 0) {
    const bool ok16 = err[pm[0]] <= error_budget && err[pm[1]] <= error_budget && p16.pair_ms > 0;
    pdt = (ok16 && p16.pair_ms < p32.pair_ms) ? MMCSF_DTYPE_BF16 : MMCSF_DTYPE_F32;
    const float pms = pdt == MMCSF_DTYPE_BF16 ? p16.pair_ms : p32.pair_ms;
    use_pair = pms < unit_ms[pm[0]] + unit_ms[pm[1]];
  }
  bool any16 = use_pair && pdt == MMCSF_DTYPE_BF16;
  for (int m = 0; m < nd; ++m)
    if (!(use_pair && (m == pm[0] || m == pm[1])) && dt[m] == MMCSF_DTYPE_BF16) any16 = true;
  // the conversion is paid once per call: drop BF16 where it does not pay for it
  if (any16) {
    float saved = 0;
    if (use_pair && pdt == MMCSF_DTYPE_BF16) saved += p32.pair_ms - p16.pair_ms;
    for (int m = 0; m < nd; ++m)
      if (!(use_pair && (m == pm[0] || m == pm[1])) && dt[m] == MMCSF_DTYPE_BF16) saved += p32.ms[m] - p16.ms[m];
    if (saved <= conv_ms) {
      any16 = false;
      for (int m = 0; m < nd; ++m) dt[m] = MMCSF_DTYPE_F32;
      pdt = MMCSF_DTYPE_F32;
      use_pair = F->pair_use[0];
    }
  }
  F->mixed = any16;
  for (int m = 0; m < nd; ++m) F->mode_dtype[m] = dt[m];
  F->pair_dtype = pdt;
  F->mixed_pair = use_pair;
  if (plan) {
    *plan = mmcsf_plan{};
    for (int m = 0; m < nd; ++m) {
      const mmcsf_plan& q = dt[m] == MMCSF_DTYPE_BF16 ? p16 : p32;
      plan->traversal[m] = q.traversal[m];
      plan->chunk[m] = q.chunk[m];
      plan->min_blocks[m] = q.min_blocks[m];
      plan->kernel[m] = q.kernel[m];
      plan->ms[m] = q.ms[m];
      plan->mode_dtype[m] = dt[m];
      plan->bf16_error[m] = (float)err[m];
      plan->ms_f32[m] = p32.ms[m];
      plan->ms_bf16[m] = p16.ms[m];
    }
    const mmcsf_plan& q = pdt == MMCSF_DTYPE_BF16 ? p16 : p32;
    plan->pair = use_pair ? 1 : 0;
    plan->pair_chunk = q.pair_chunk;
    plan->pair_min_blocks = q.pair_min_blocks;
    plan->pair_kernel = q.pair_kernel;
    plan->pair_ms = q.pair_ms;
    plan->pair_dtype = pdt;
    plan->pair_ms_f32 = p32.pair_ms;
    plan->pair_ms_bf16 = p16.pair_ms;
    plan->factor_dtype = MMCSF_DTYPE_F32;
    plan->mixed = any16 ? 1 : 0;
    plan->convert_ms = conv_ms;
    plan->fiber_threshold = p32.fiber_threshold;
  }
  return MMCSF_OK;
}

namespace {
// Device time of one call under a tuned plan: the launches it runs (the
// two-output walk or its two modes, the other modes) plus the conversion of a
// mixed plan. B-CSF / HB-CSF formats: their one mode.
float plan_step_ms(const mmcsf_format* F, const mmcsf_plan& p) {
  if (F->impl != MMCSF_IMPL_MMCSF) return p.ms[F->mode];
  int pm[2] = {-1, -1};
  const bool pair = p.pair && mmcsf_mttkrp_pair(F, 32, MMCSF_DTYPE_F32, nullptr, nullptr, nullptr, pm, nullptr,
                                                nullptr) == MMCSF_OK;
  float t = pair ? p.pair_ms : 0.f;
  for (int m = 0; m < F->nd; ++m)
    if (!(pair && (m == pm[0] || m == pm[1]))) t += p.ms[m];
  return t + (p.mixed ? p.convert_ms : 0.f);
}
}  // namespace

extern "C" int mmcsf_autotune(mmcsf_coo* X, const mmcsf_build_opts* base, const uint64_t* f_candidates,
                              int n_candidates, int R, const float* const* d_factors, float* const* d_outs,
                              double error_budget, void* stream, mmcsf_format** out, mmcsf_plan* plan) {
  MMCSF_RANGE("mmcsf_autotune");
  if (!X || !base || !d_factors || !d_outs || !out) return set_error(MMCSF_ERR_INVALID, "null argument");
  static const uint64_t defaults[] = {0, 128, 32};
  if (!f_candidates || n_candidates <= 0) {
    f_candidates = defaults;
    n_candidates = 3;
  }
  mmcsf_format* best = nullptr;
  mmcsf_plan best_plan{};
  float best_ms = 0.f;
  for (int i = 0; i < n_candidates; ++i) {
    mmcsf_build_opts o = *base;
    o.fiber_threshold = f_candidates[i];
    mmcsf_format* F = nullptr;
    int st = mmcsf_build(X, &o, stream, &F);
    mmcsf_plan p{};
    if (st == MMCSF_OK)
      st = F->impl == MMCSF_IMPL_MMCSF
               ? mmcsf_tune_precision(F, R, d_factors, d_outs, error_budget, stream, &p)
               : mmcsf_tune(F, R, MMCSF_DTYPE_F32, reinterpret_cast<const void* const*>(d_factors), d_outs, stream,
                            &p);
    if (st != MMCSF_OK) {
      if (F) mmcsf_format_destroy(F);
      if (best) mmcsf_format_destroy(best);
      return st;
    }
    F->fiber_threshold_tuned = (int)std::min<uint64_t>(f_candidates[i], 0x7fffffff);
    p.fiber_threshold = F->fiber_threshold_tuned;
    const float t = plan_step_ms(F, p);
    if (!best || t < best_ms) {
      if (best) mmcsf_format_destroy(best);
      best = F;
      best_ms = t;
      best_plan = p;
    } else {
      mmcsf_format_destroy(F);
    }
  }
  *out = best;
  if (plan) *plan = best_plan;
  return MMCSF_OK;
}

extern "C" int mmcsf_set_plan(mmcsf_format* F, const mmcsf_plan* plan) {
  if (!F || !plan) return set_error(MMCSF_ERR_INVALID, "null argument");
  if (plan->factor_dtype != MMCSF_DTYPE_F32 && plan->factor_dtype != MMCSF_DTYPE_BF16)
    return set_error(MMCSF_ERR_INVALID, "plan factor_dtype must be MMCSF_DTYPE_F32 or MMCSF_DTYPE_BF16");
  for (int m = 0; m < F->nd; ++m) {
    if (plan->traversal[m] == 2 && !F->views[m].present)
      return set_error(MMCSF_ERR_INVALID, "plan uses a view for mode %d that was not built", m);
    if (plan->traversal[m] < 0 || plan->traversal[m] > 2 || plan->chunk[m] < 0 || plan->kernel[m] < 0 ||
        plan->kernel[m] > 7)
      return set_error(MMCSF_ERR_INVALID, "bad plan entry for mode %d", m);
    if (plan->mixed && plan->mode_dtype[m] != MMCSF_DTYPE_F32 && plan->mode_dtype[m] != MMCSF_DTYPE_BF16)
      return set_error(MMCSF_ERR_INVALID, "bad mode_dtype for mode %d", m);
  }
  if (plan->pair_chunk < 0 || plan->pair_min_blocks < 0 || plan->pair_kernel < 0 || plan->pair_kernel > 7)
    return set_error(MMCSF_ERR_INVALID, "bad pair entry");
  if (plan->mixed && plan->pair_dtype != MMCSF_DTYPE_F32 && plan->pair_dtype != MMCSF_DTYPE_BF16)
    return set_error(MMCSF_ERR_INVALID, "bad pair_dtype");
  for (int m = 0; m < F->nd; ++m) {
    // a mixed plan's per-mode entries belong to the type chosen for the mode
    const int d = plan->mixed ? (plan->mode_dtype[m] == MMCSF_DTYPE_BF16) : (plan->factor_dtype == MMCSF_DTYPE_BF16);
    F->plan_traversal[d][m] = plan->traversal[m];
    F->plan_chunk[d][m] = plan->chunk[m];
    F->plan_mb[d][m] = plan->min_blocks[m];
    F->plan_kernel[d][m] = plan->kernel[m];
  }
  const int pd = plan->mixed ? (plan->pair_dtype == MMCSF_DTYPE_BF16) : (plan->factor_dtype == MMCSF_DTYPE_BF16);
  F->pair_chunk[pd] = plan->pair_chunk;
  F->pair_mb[pd] = plan->pair_min_blocks;
  F->pair_kernel[pd] = plan->pair_kernel;
  if (plan->mixed) {
    F->mixed = true;
    F->mixed_pair = plan->pair != 0;
    F->pair_dtype = plan->pair_dtype;
    for (int m = 0; m < F->nd; ++m) F->mode_dtype[m] = plan->mode_dtype[m];
    if (F->impl != MMCSF_IMPL_MMCSF) return set_error(MMCSF_ERR_INVALID, "mixed plans are for MM-CSF formats");
  } else {
    F->mixed = false;
    F->pair_use[pd] = plan->pair != 0;
  }
  return MMCSF_OK;
}
