// Row-gather probe (measurement only; no counterpart in the reference): the
// rate at which this GPU gathers random factor rows for a given index stream,
// with the MTTKRP kernels' team layout (G lanes per row, R = 4*G floats, rows
// summed in registers) and nothing else. It is the ceiling the MTTKRP kernels'
// per-nonzero gathers run against: bench.py reports it beside the HBM roofline.
#include "prims.cuh"
#include "common.h"

using mmcsf::set_error;

namespace {

constexpr unsigned FULL = 0xffffffffu;

template <int G, int PF>
__global__ void __launch_bounds__(256, 4) k_probe_gather(const uint32_t* __restrict__ idx, uint64_t n,
                                                        const float* __restrict__ rows, uint32_t chunk,
                                                        float* __restrict__ sink) {
  constexpr uint32_t R = 4 * G;
  const int lane = threadIdx.x & 31, tl = lane & (G - 1), tb = lane - tl;
  const uint64_t team = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) / G;
  const uint64_t x0 = team * chunk;
  const uint64_t x1 = x0 < n ? min(x0 + chunk, n) : x0;
  float4 acc = make_float4(0.f, 0.f, 0.f, 0.f);
  for (uint32_t it = 0; it < chunk; it += G) {  // same trip count for every team (uniform shuffles)
    const uint64_t xb = x0 + it;
    const uint32_t k = xb + tl < x1 ? __ldg(idx + xb + tl) : 0u;
#pragma unroll
    for (int jb = 0; jb < G; jb += PF) {
      float4 r[PF];
#pragma unroll
      for (int j = 0; j < PF; ++j) {
        const uint32_t kj = __shfl_sync(FULL, k, tb + jb + j);
        r[j] = __ldg(reinterpret_cast<const float4*>(rows + (uint64_t)kj * R) + tl);
      }
#pragma unroll
      for (int j = 0; j < PF; ++j) { acc.x += r[j].x; acc.y += r[j].y; acc.z += r[j].z; acc.w += r[j].w; }
    }
  }
  // keep the loads: one store per lane of a value that is never the sentinel in practice
  if (acc.x + acc.y + acc.z + acc.w == -1.2345e-30f) sink[0] = acc.x;
}

// The same gather with the rows landed in shared memory by the copy engine:
// every lane of a warp issues one bulk copy (cp.async.bulk, no multicast) of
// its nonzero's row into a per-warp ring of S stages of 32 rows, completion
// tracked by one mbarrier per stage (transaction bytes); the warp then reads
// the stage's rows from shared memory with the MTTKRP team layout (G lanes per
// row) and sums them. Rows in flight are bounded by shared memory instead of
// registers. Every wait is bounded: after `limit` polls the warp records an
// error in *err, waits (bounded again) for its copies in flight and leaves.
__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
__device__ __forceinline__ void bulk_row(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                   smem_u32(dst)),
               "l"(src), "r"(bytes), "r"(smem_u32(bar))
               : "memory");
}
// bounded wait: true when the phase completed
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity, uint32_t limit) {
  for (uint32_t i = 0; i < limit; ++i)
    if (mbar_try_wait(bar, parity)) return true;
  return false;
}

template <int G, int S>
__global__ void __launch_bounds__(256, 1) k_probe_gather_tma(const uint32_t* __restrict__ idx, uint64_t n,
                                                             const float* __restrict__ rows, uint32_t chunk,
                                                             float* __restrict__ sink, int* __restrict__ err,
                                                             uint32_t limit) {
  constexpr uint32_t R = 4 * G;
  constexpr uint32_t RB = R * 4;  // row bytes
  extern __shared__ __align__(128) unsigned char smem[];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
  uint64_t* bars = reinterpret_cast<uint64_t*>(smem) + warp * S;
  float* ring = reinterpret_cast<float*>(smem + ((nwarps * S * 8 + 127) / 128) * 128) + (size_t)warp * S * 32 * R;
  if (lane == 0)
    for (int s = 0; s < S; ++s) mbar_init(bars + s, 1);
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  __syncwarp();
  const uint64_t gw = blockIdx.x * (uint64_t)nwarps + warp;  // this warp's range
  const uint64_t x0 = gw * chunk;
  const uint64_t x1 = x0 < n ? min(x0 + chunk, n) : x0;
  const uint32_t nblk = (uint32_t)((x1 - x0 + 31) / 32);
  auto issue = [&](uint32_t b) {  // block b of 32 rows into stage b % S
    const int s = (int)(b % S);
    const uint64_t x = x0 + (uint64_t)b * 32 + lane;
    const uint32_t cnt = (uint32_t)(uint32_t)min((uint64_t)32, x1 - (x0 + (uint64_t)b * 32));
    if (lane == 0) mbar_expect_tx(bars + s, cnt * RB);
    __syncwarp();
    if (x < x1) bulk_row(ring + ((size_t)s * 32 + lane) * R, rows + (uint64_t)__ldg(idx + x) * R, RB, bars + s);
  };
  for (uint32_t b = 0; b < (uint32_t)S && b < nblk; ++b) issue(b);
  const int tl = lane & (G - 1), tb = lane / G;
  float4 acc = make_float4(0.f, 0.f, 0.f, 0.f);
  bool ok = true;
  uint32_t b = 0;
  for (; b < nblk; ++b) {
    const int s = (int)(b % S);
    if (!mbar_wait_bounded(bars + s, (b / S) & 1u, limit)) { ok = false; break; }
    const uint32_t cnt = (uint32_t)(uint32_t)min((uint64_t)32, x1 - (x0 + (uint64_t)b * 32));
    const float* st = ring + (size_t)s * 32 * R;
#pragma unroll 4
    for (uint32_t r = tb; r < cnt; r += 32 / G) {
      const float4 v = reinterpret_cast<const float4*>(st + (size_t)r * R)[tl];
      acc.x += v.x; acc.y += v.y; acc.z += v.z; acc.w += v.w;
    }
    __syncwarp();
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");  // reads done before the copy engine refills
    if (b + S < nblk) issue(b + S);
  }
  if (!ok) {
    if (lane == 0) atomicExch(err, 1);
    // the copies already issued still land in this warp's ring: wait for them (bounded) before leaving
    for (uint32_t q = b; q < nblk && q < b + S; ++q) mbar_wait_bounded(bars + (q % S), (q / S) & 1u, limit);
  }
  if (acc.x + acc.y + acc.z + acc.w == -1.2345e-30f) sink[0] = acc.x;
}

}  // namespace

extern "C" int mmcsf_probe_gather_tma(const uint32_t* d_idx, uint64_t n, const float* d_rows, uint64_t nrows, int R,
                                      int stages, int warps, int reps, float* ms_out, void* stream) {
  if (!d_idx || !d_rows || !ms_out || n == 0) return set_error(MMCSF_ERR_INVALID, "null or empty argument");
  if (R != 16 && R != 32 && R != 64) return set_error(MMCSF_ERR_UNSUPPORTED, "TMA probe runs R 16, 32, 64");
  if (stages != 2 && stages != 4 && stages != 8) return set_error(MMCSF_ERR_UNSUPPORTED, "stages 2, 4 or 8");
  if (warps < 1 || warps > 8) return set_error(MMCSF_ERR_INVALID, "warps per block in 1..8");
  (void)nrows;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  mmcsf::DevBuf sink, err;
  MMCSF_CUDA(sink.alloc(16));
  MMCSF_CUDA(err.alloc(16));
  MMCSF_CUDA(cudaMemsetAsync(err.p, 0, 16, s));
  const size_t smem = ((size_t)(warps * stages * 8 + 127) / 128) * 128 + (size_t)warps * stages * 32 * R * 4;
  if (smem > 227 * 1024) return set_error(MMCSF_ERR_INVALID, "ring of %zu bytes exceeds shared memory", smem);
  const int nsm = mmcsf::sm_count();
  const uint64_t total_warps = (uint64_t)nsm * warps;  // one block per SM
  const uint32_t chunk = (uint32_t)(((n + total_warps - 1) / total_warps + 31) / 32 * 32);
  const uint32_t limit = 1u << 22;  // polls per wait before the warp gives up (seconds at most)
  cudaError_t e = cudaSuccess;
  auto launch = [&]() {
#define MMCSF_PT(GG, SS)                                                                                     \
  {                                                                                                           \
    auto k = k_probe_gather_tma<GG, SS>;                                                                      \
    e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);                      \
    if (e == cudaSuccess)                                                                                     \
      k<<<nsm, warps * 32, smem, s>>>(d_idx, n, d_rows, chunk, sink.as<float>(), err.as<int>(), limit);      \
  }
    const int G = R / 4;
    if (G == 4 && stages == 2) MMCSF_PT(4, 2) else if (G == 4 && stages == 4) MMCSF_PT(4, 4) else if (G == 4) MMCSF_PT(4, 8)
    else if (G == 8 && stages == 2) MMCSF_PT(8, 2) else if (G == 8 && stages == 4) MMCSF_PT(8, 4) else if (G == 8) MMCSF_PT(8, 8)
    else if (stages == 2) MMCSF_PT(16, 2) else if (stages == 4) MMCSF_PT(16, 4) else MMCSF_PT(16, 8)
#undef MMCSF_PT
  };
  cudaEvent_t e0, e1;
  MMCSF_CUDA(cudaEventCreate(&e0));
  MMCSF_CUDA(cudaEventCreate(&e1));
  launch();
  MMCSF_CUDA(e);
  launch();
  MMCSF_CUDA(cudaEventRecord(e0, s));
  for (int i = 0; i < (reps > 0 ? reps : 5); ++i) launch();
  MMCSF_CUDA(cudaEventRecord(e1, s));
  MMCSF_CUDA(cudaEventSynchronize(e1));
  float ms = 0;
  cudaEventElapsedTime(&ms, e0, e1);
  *ms_out = ms / (reps > 0 ? reps : 5);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  MMCSF_CUDA(cudaGetLastError());
  int herr = 0;
  MMCSF_CUDA(cudaMemcpy(&herr, err.p, sizeof(int), cudaMemcpyDeviceToHost));
  if (herr) return set_error(MMCSF_ERR_TIMEOUT, "TMA probe: a wait gave up");
  return MMCSF_OK;
}

extern "C" int mmcsf_probe_gather(const uint32_t* d_idx, uint64_t n, const float* d_rows, uint64_t nrows, int R,
                                  int reps, float* ms_out, void* stream) {
  if (!d_idx || !d_rows || !ms_out || n == 0) return set_error(MMCSF_ERR_INVALID, "null or empty argument");
  if (R != 16 && R != 32 && R != 64 && R != 128) return set_error(MMCSF_ERR_UNSUPPORTED, "probe runs R 16..128");
  (void)nrows;  // indices must be < nrows (the caller's contract, as for the format's indices)
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  mmcsf::DevBuf sink;
  MMCSF_CUDA(sink.alloc(16));
  const uint32_t chunk = 512;
  const int G = R / 4;
  const uint64_t teams = (n + chunk - 1) / chunk, blocks = (teams * G + 255) / 256;
  auto launch = [&]() {
    switch (R) {
      case 16: k_probe_gather<4, 4><<<(unsigned)blocks, 256, 0, s>>>(d_idx, n, d_rows, chunk, sink.as<float>()); break;
      case 32: k_probe_gather<8, 4><<<(unsigned)blocks, 256, 0, s>>>(d_idx, n, d_rows, chunk, sink.as<float>()); break;
      case 64: k_probe_gather<16, 4><<<(unsigned)blocks, 256, 0, s>>>(d_idx, n, d_rows, chunk, sink.as<float>()); break;
      default: k_probe_gather<32, 4><<<(unsigned)blocks, 256, 0, s>>>(d_idx, n, d_rows, chunk, sink.as<float>()); break;
    }
  };
  cudaEvent_t e0, e1;
  MMCSF_CUDA(cudaEventCreate(&e0));
  MMCSF_CUDA(cudaEventCreate(&e1));
  launch();
  launch();
  MMCSF_CUDA(cudaEventRecord(e0, s));
  for (int i = 0; i < (reps > 0 ? reps : 5); ++i) launch();
  MMCSF_CUDA(cudaEventRecord(e1, s));
  MMCSF_CUDA(cudaEventSynchronize(e1));
  float ms = 0;
  cudaEventElapsedTime(&ms, e0, e1);
  *ms_out = ms / (reps > 0 ? reps : 5);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  MMCSF_CUDA(cudaGetLastError());
  return MMCSF_OK;
}
