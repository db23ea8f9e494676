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

}  // namespace

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
