// Exclusive scan and stable LSD radix sort for sm_100a.
//
// The scan is the classic reduce / scan-partials / downsweep scheme with
// 2048-element tiles. The radix sort moves 8 bits per pass: a per-tile
// digit histogram, a digit-major exclusive scan of all histograms, and a
// scatter that ranks keys stably inside the tile (warp match + per-warp
// digit counters, warps owning contiguous 512-key runs). Stability is what
// makes the reference's chain of sorts reproducible as one composite sort.
#include <cuda_runtime.h>

#include "prims.cuh"

namespace mmcsf {

namespace {
constexpr unsigned FULL = 0xffffffffu;
constexpr int SCAN_T = 256, SCAN_I = 8, SCAN_TILE = SCAN_T * SCAN_I;
constexpr int RS_T = 256, RS_I = 16, RS_TILE = RS_T * RS_I, RS_WARPS = RS_T / 32, RS_RADIX = 256;

__device__ __forceinline__ uint32_t warp_incl_scan(uint32_t v) {
  const int lane = threadIdx.x & 31;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    uint32_t t = __shfl_up_sync(FULL, v, o);
    if (lane >= o) v += t;
  }
  return v;
}

// Exclusive scan of one value per thread across the block.
__device__ __forceinline__ uint32_t block_excl_scan(uint32_t v, uint32_t* total) {
  __shared__ uint32_t ws[32];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
  uint32_t inc = warp_incl_scan(v);
  if (lane == 31) ws[wid] = inc;
  __syncthreads();
  if (wid == 0) {
    uint32_t w = lane < nw ? ws[lane] : 0;
    w = warp_incl_scan(w);
    ws[lane] = w;
  }
  __syncthreads();
  uint32_t pre = wid ? ws[wid - 1] : 0;
  *total = ws[nw - 1];
  __syncthreads();
  return pre + inc - v;
}

__global__ void __launch_bounds__(SCAN_T) k_scan_reduce(const uint32_t* __restrict__ in, uint64_t n,
                                                        uint32_t* __restrict__ partials) {
  uint64_t base = (uint64_t)blockIdx.x * SCAN_TILE;
  uint32_t s = 0;
#pragma unroll
  for (int i = 0; i < SCAN_I; ++i) {
    uint64_t idx = base + (uint64_t)i * SCAN_T + threadIdx.x;
    if (idx < n) s += in[idx];
  }
  uint32_t tot;
  block_excl_scan(s, &tot);
  if (threadIdx.x == 0) partials[blockIdx.x] = tot;
}

// Each thread owns SCAN_I consecutive elements of the tile.
__global__ void __launch_bounds__(SCAN_T) k_scan_down(const uint32_t* in, uint32_t* out, uint64_t n,
                                                      const uint32_t* __restrict__ partials, uint64_t nblocks) {
  uint64_t base = (uint64_t)blockIdx.x * SCAN_TILE + (uint64_t)threadIdx.x * SCAN_I;
  uint32_t v[SCAN_I];
  uint32_t s = 0;
#pragma unroll
  for (int i = 0; i < SCAN_I; ++i) {
    v[i] = (base + i < n) ? in[base + i] : 0u;
    s += v[i];
  }
  uint32_t tot;
  uint32_t pre = block_excl_scan(s, &tot) + (partials ? partials[blockIdx.x] : 0u);
#pragma unroll
  for (int i = 0; i < SCAN_I; ++i) {
    if (base + i < n) out[base + i] = pre;
    pre += v[i];
  }
  if (blockIdx.x == nblocks - 1 && threadIdx.x == 0)
    out[n] = (partials ? partials[blockIdx.x] : 0u) + tot;
}

__global__ void __launch_bounds__(RS_T) k_rs_hist(const uint64_t* __restrict__ keys, uint64_t n, int shift,
                                                  uint32_t* __restrict__ hist, uint32_t ntiles) {
  __shared__ uint32_t cnt[RS_RADIX];
  cnt[threadIdx.x] = 0;
  __syncthreads();
  const int lane = threadIdx.x & 31;
  uint64_t base = (uint64_t)blockIdx.x * RS_TILE;
#pragma unroll 4
  for (int i = 0; i < RS_I; ++i) {
    uint64_t idx = base + (uint64_t)i * RS_T + threadIdx.x;
    uint32_t d = idx < n ? (uint32_t)((keys[idx] >> shift) & (RS_RADIX - 1)) : RS_RADIX;
    unsigned peers = __match_any_sync(FULL, d);
    if (d < RS_RADIX && lane == __ffs(peers) - 1) atomicAdd(&cnt[d], (uint32_t)__popc(peers));
  }
  __syncthreads();
  hist[(uint64_t)threadIdx.x * ntiles + blockIdx.x] = cnt[threadIdx.x];
}

__global__ void __launch_bounds__(RS_T) k_rs_scatter(const uint64_t* __restrict__ kin,
                                                     const uint32_t* __restrict__ vin,
                                                     uint64_t* __restrict__ kout, uint32_t* __restrict__ vout,
                                                     uint64_t n, int shift,
                                                     const uint32_t* __restrict__ offs, uint32_t ntiles) {
  __shared__ uint32_t wcnt[RS_WARPS][RS_RADIX];
  __shared__ uint32_t base[RS_RADIX];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  for (int i = threadIdx.x; i < RS_WARPS * RS_RADIX; i += RS_T) (&wcnt[0][0])[i] = 0;
  base[threadIdx.x] = offs[(uint64_t)threadIdx.x * ntiles + blockIdx.x];
  __syncthreads();
  const unsigned lt = (1u << lane) - 1u;
  const uint64_t wbase = (uint64_t)blockIdx.x * RS_TILE + (uint64_t)w * (RS_I * 32);
  uint64_t k[RS_I];
  uint32_t v[RS_I], rank[RS_I];
  uint32_t dg[RS_I];
#pragma unroll
  for (int i = 0; i < RS_I; ++i) {
    uint64_t idx = wbase + (uint64_t)i * 32 + lane;
    bool ok = idx < n;
    k[i] = ok ? kin[idx] : 0ull;
    v[i] = ok ? vin[idx] : 0u;
    dg[i] = ok ? (uint32_t)((k[i] >> shift) & (RS_RADIX - 1)) : RS_RADIX;
  }
#pragma unroll
  for (int i = 0; i < RS_I; ++i) {
    unsigned peers = __match_any_sync(FULL, dg[i]);
    uint32_t before = dg[i] < RS_RADIX ? wcnt[w][dg[i]] : 0u;
    rank[i] = before + (uint32_t)__popc(peers & lt);
    __syncwarp();
    if (dg[i] < RS_RADIX && lane == __ffs(peers) - 1) wcnt[w][dg[i]] = before + (uint32_t)__popc(peers);
    __syncwarp();
  }
  __syncthreads();
  {  // exclusive prefix of the per-warp counts, digit by digit
    const int d = threadIdx.x;
    uint32_t run = 0;
#pragma unroll
    for (int ww = 0; ww < RS_WARPS; ++ww) {
      uint32_t c = wcnt[ww][d];
      wcnt[ww][d] = run;
      run += c;
    }
  }
  __syncthreads();
#pragma unroll
  for (int i = 0; i < RS_I; ++i) {
    if (dg[i] < RS_RADIX) {
      uint32_t pos = base[dg[i]] + wcnt[w][dg[i]] + rank[i];
      kout[pos] = k[i];
      vout[pos] = v[i];
    }
  }
}

__global__ void k_iota(uint32_t* v, uint64_t n) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
    v[i] = (uint32_t)i;
}

__global__ void k_gather(const uint32_t* __restrict__ in, const uint32_t* __restrict__ perm,
                         uint32_t* __restrict__ out, uint64_t n) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
    out[i] = in[perm[i]];
}

int g_sms = 0;
}  // namespace

int sm_count() {
  if (g_sms == 0) {
    int dev = 0;
    cudaGetDevice(&dev);
    if (cudaDeviceGetAttribute(&g_sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || g_sms <= 0)
      g_sms = 148;
  }
  return g_sms;
}

int grid_for(uint64_t n, int threads) {
  uint64_t b = (n + threads - 1) / threads;
  uint64_t cap = (uint64_t)sm_count() * (2048 / threads);
  if (b > cap) b = cap;
  return b ? (int)b : 1;
}

cudaError_t exclusive_scan_u32(const uint32_t* in, uint32_t* out, uint64_t n, cudaStream_t s) {
  if (n == 0) return cudaMemsetAsync(out, 0, sizeof(uint32_t), s);
  uint64_t nb = (n + SCAN_TILE - 1) / SCAN_TILE;
  if (nb == 1) {
    k_scan_down<<<1, SCAN_T, 0, s>>>(in, out, n, nullptr, 1);
    return cudaGetLastError();
  }
  Tmp part;
  cudaError_t e = part.alloc((nb + 1) * sizeof(uint32_t), s);
  if (e != cudaSuccess) return e;
  k_scan_reduce<<<(unsigned)nb, SCAN_T, 0, s>>>(in, n, part.as<uint32_t>());
  if ((e = cudaGetLastError()) != cudaSuccess) return e;
  if ((e = exclusive_scan_u32(part.as<uint32_t>(), part.as<uint32_t>(), nb, s)) != cudaSuccess) return e;
  k_scan_down<<<(unsigned)nb, SCAN_T, 0, s>>>(in, out, n, part.as<uint32_t>(), nb);
  return cudaGetLastError();
}

cudaError_t radix_sort_pairs(uint64_t* keys, uint32_t* vals, uint64_t* keys_alt, uint32_t* vals_alt,
                             uint64_t n, int key_bits, cudaStream_t s) {
  if (n <= 1 || key_bits <= 0) return cudaSuccess;
  const uint32_t ntiles = (uint32_t)((n + RS_TILE - 1) / RS_TILE);
  const uint64_t nh = (uint64_t)ntiles * RS_RADIX;
  Tmp hist;
  cudaError_t e = hist.alloc((nh + 1) * sizeof(uint32_t), s);
  if (e != cudaSuccess) return e;
  uint64_t *ka = keys, *kb = keys_alt;
  uint32_t *va = vals, *vb = vals_alt;
  int passes = 0;
  for (int shift = 0; shift < key_bits; shift += 8, ++passes) {
    k_rs_hist<<<ntiles, RS_T, 0, s>>>(ka, n, shift, hist.as<uint32_t>(), ntiles);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    if ((e = exclusive_scan_u32(hist.as<uint32_t>(), hist.as<uint32_t>(), nh, s)) != cudaSuccess) return e;
    k_rs_scatter<<<ntiles, RS_T, 0, s>>>(ka, va, kb, vb, n, shift, hist.as<uint32_t>(), ntiles);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    uint64_t* tk = ka; ka = kb; kb = tk;
    uint32_t* tv = va; va = vb; vb = tv;
  }
  if (passes & 1) {
    if ((e = cudaMemcpyAsync(keys, ka, n * sizeof(uint64_t), cudaMemcpyDeviceToDevice, s)) != cudaSuccess) return e;
    if ((e = cudaMemcpyAsync(vals, va, n * sizeof(uint32_t), cudaMemcpyDeviceToDevice, s)) != cudaSuccess) return e;
  }
  return cudaSuccess;
}

cudaError_t iota_u32(uint32_t* v, uint64_t n, cudaStream_t s) {
  if (!n) return cudaSuccess;
  k_iota<<<grid_for(n, 256), 256, 0, s>>>(v, n);
  return cudaGetLastError();
}

cudaError_t gather_u32(const uint32_t* in, const uint32_t* perm, uint32_t* out, uint64_t n, cudaStream_t s) {
  if (!n) return cudaSuccess;
  k_gather<<<grid_for(n, 256), 256, 0, s>>>(in, perm, out, n);
  return cudaGetLastError();
}

}  // namespace mmcsf
