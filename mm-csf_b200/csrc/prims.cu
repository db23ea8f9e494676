// Exclusive scan and stable LSD radix sort for sm_100a.
//
// The scan is the classic reduce / scan-partials / downsweep scheme with
// 2048-element tiles. The radix sort moves 8 bits per pass: a per-tile
// digit histogram, a digit-major exclusive scan of all histograms, and a
// scatter that ranks keys stably inside the tile (warp match + per-warp
// digit counters, warps owning contiguous 512-key runs). Stability is what
// makes the reference's chain of sorts reproducible as one composite sort.
#include <cuda_runtime.h>

#include <utility>

#include "common.h"
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

// ---------------------------------------------------------------------------
// Construction sort without device allocation.
//
// Some callers cannot allocate device memory once they are running: a
// process whose device memory was reserved up front by another allocator
// (a serving runtime or framework memory pool) finds cudaMalloc failing or
// fragmenting that pool, and a latency-critical loop cannot afford the
// implicit synchronisation of cudaMalloc/cudaFree. For them,
// mmcsf_sort_coo_noalloc runs the format builder's stable radix sort with
// all of its scratch (keys, permutation, digit histograms, scan partials) in
// one file-scope device array of NOALLOC_BYTES (about 12.2 MiB), which every
// GPU that loads this library holds until the process exits.
// ---------------------------------------------------------------------------
namespace mmcsf {
namespace {

constexpr uint64_t NOALLOC_MAX_NNZ = 1ull << 19;  // 524,288 nonzeros
constexpr uint64_t NA_TILES = (NOALLOC_MAX_NNZ + RS_TILE - 1) / RS_TILE;
constexpr uint64_t NA_HIST = NA_TILES * RS_RADIX + 1;          // digit histograms + total
constexpr uint64_t NA_PART = (NA_HIST + SCAN_TILE - 1) / SCAN_TILE + 1;
constexpr uint64_t NA_KEYS_OFF = 0;                                          // 2 x u64[MAX]
constexpr uint64_t NA_PERM_OFF = NA_KEYS_OFF + 2 * NOALLOC_MAX_NNZ * 8;      // 2 x u32[MAX]
constexpr uint64_t NA_HIST_OFF = NA_PERM_OFF + 2 * NOALLOC_MAX_NNZ * 4;      // u32[NA_HIST]
constexpr uint64_t NA_PART_OFF = NA_HIST_OFF + ((NA_HIST * 4 + 255) / 256) * 256;
constexpr uint64_t NOALLOC_BYTES = NA_PART_OFF + ((NA_PART * 4 + 255) / 256) * 256;

// The scratch. Host code must not use this symbol as an address (on the host
// it names a stand-in, not device memory); it asks for the device address with
// cudaGetSymbolAddress, once per device.
static __device__ __align__(256) unsigned char g_noalloc_scratch[NOALLOC_BYTES];

constexpr int NA_MAX_DEVICES = 64;
// Per device: the scratch's device address and the id of the context it was
// taken in. A caller that resets the device (cudaDeviceReset) gets a new
// primary context whose module, and so whose array, may sit elsewhere; the
// address is looked up again whenever the current context's id differs.
unsigned char* g_noalloc_ptr[NA_MAX_DEVICES] = {};
unsigned long long g_noalloc_ctx[NA_MAX_DEVICES] = {};

// Id of the current context (cuCtxGetCurrent + cuCtxGetId, reached through
// the runtime's driver entry points so that the library needs no link to the
// driver library). 0 when the driver does not provide them.
unsigned long long current_ctx_id() {
  typedef int (*get_current_t)(void**);
  typedef int (*get_id_t)(void*, unsigned long long*);
  static get_current_t get_current = nullptr;
  static get_id_t get_id = nullptr;
  static bool looked_up = false;
  if (!looked_up) {
    void* f = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      get_current = reinterpret_cast<get_current_t>(f);
    f = nullptr;
    if (cudaGetDriverEntryPoint("cuCtxGetId", &f, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      get_id = reinterpret_cast<get_id_t>(f);
    looked_up = true;
  }
  void* ctx = nullptr;
  unsigned long long id = 0;
  if (!get_current || !get_id || get_current(&ctx) != 0 || !ctx || get_id(ctx, &id) != 0) return 0;
  return id;
}

__global__ void k_na_pack(const uint32_t* __restrict__ i0, const uint32_t* __restrict__ i1,
                          const uint32_t* __restrict__ i2, const uint32_t* __restrict__ i3,
                          const uint32_t* __restrict__ perm, int nk, int4 modes, int4 shifts, uint64_t n,
                          uint64_t* __restrict__ keys) {
  const uint32_t* in[4] = {i0, i1, i2, i3};
  const int md[4] = {modes.x, modes.y, modes.z, modes.w};
  const int sh[4] = {shifts.x, shifts.y, shifts.z, shifts.w};
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t src = perm[i];
    uint64_t k = 0;
    for (int j = 0; j < nk; ++j) k |= (uint64_t)in[md[j]][src] << sh[j];
    keys[i] = k;
  }
}

__global__ void k_na_gather_f32(const float* __restrict__ in, const uint32_t* __restrict__ perm, uint64_t n,
                                float* __restrict__ out) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
    out[i] = in[perm[i]];
}

// Exclusive scan of n <= SCAN_TILE * SCAN_TILE elements with caller scratch
// for the partials (no allocation).
cudaError_t na_scan(uint32_t* data, uint64_t n, uint32_t* part, cudaStream_t s) {
  const uint64_t nb = (n + SCAN_TILE - 1) / SCAN_TILE;
  if (nb == 1) {
    k_scan_down<<<1, SCAN_T, 0, s>>>(data, data, n, nullptr, 1);
    return cudaGetLastError();
  }
  k_scan_reduce<<<(unsigned)nb, SCAN_T, 0, s>>>(data, n, part);
  k_scan_down<<<1, SCAN_T, 0, s>>>(part, part, nb, nullptr, 1);
  k_scan_down<<<(unsigned)nb, SCAN_T, 0, s>>>(data, data, n, part, nb);
  return cudaGetLastError();
}

int bits_of(uint64_t dim) {
  int b = 0;
  while (b < 64 && ((dim - 1) >> b)) ++b;
  return b;
}

}  // namespace
}  // namespace mmcsf

extern "C" int mmcsf_sort_coo_noalloc(int impl, int mode, int nd, const uint64_t* dims, uint64_t nnz,
                                      const uint32_t* const* d_inds, const float* d_vals,
                                      uint32_t* const* d_out_inds, float* d_out_vals, void* stream) {
  using namespace mmcsf;
  if (!dims || (nnz && (!d_inds || !d_vals || !d_out_inds || !d_out_vals)))
    return set_error(MMCSF_ERR_INVALID, "null argument");
  if (nd < 3 || nd > 4) return set_error(MMCSF_ERR_INVALID, "Supported tensor dimension is 3 or 4 (got %d)", nd);
  if (impl != MMCSF_IMPL_MMCSF && impl != MMCSF_IMPL_BCSF && impl != MMCSF_IMPL_HBCSF)
    return set_error(MMCSF_ERR_INVALID, "unknown implementation type -t %d", impl);
  if (mode < 0 || mode >= nd) return set_error(MMCSF_ERR_INVALID, "Mode cannot be larger than tensor dimension.");
  if (nnz > NOALLOC_MAX_NNZ)
    return set_error(MMCSF_ERR_INVALID,
                     "mmcsf_sort_coo_noalloc handles at most %llu nonzeros (got %llu); use mmcsf_build",
                     (unsigned long long)NOALLOC_MAX_NNZ, (unsigned long long)nnz);
  for (int m = 0; m < nd; ++m)
    if (dims[m] == 0 || dims[m] >= (1ull << 31))
      return set_error(MMCSF_ERR_INVALID, "mode %d length %llu out of range [1, 2^31)", m,
                       (unsigned long long)dims[m]);
  if (nnz == 0) return MMCSF_OK;
  cudaStream_t s = S(stream);

  // Set-up, once per device (and again after the device's context was
  // replaced), with that device current: the device address of the scratch
  // array. The first call on a device does this.
  int dev = 0;
  MMCSF_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= NA_MAX_DEVICES) return set_error(MMCSF_ERR_UNSUPPORTED, "device ordinal %d", dev);
  const unsigned long long ctx = current_ctx_id();  // 0: no context current yet, or no driver entry points
  if (!g_noalloc_ptr[dev] || ctx == 0 || ctx != g_noalloc_ctx[dev]) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);  // makes the primary context current
    if (e != cudaSuccess || !p)
      return set_error(MMCSF_ERR_CUDA, "cudaGetSymbolAddress(scratch) failed: %s", cudaGetErrorString(e));
    g_noalloc_ptr[dev] = static_cast<unsigned char*>(p);
    g_noalloc_ctx[dev] = current_ctx_id();
  }
  unsigned char* base = g_noalloc_ptr[dev];
  uint64_t* keysA = reinterpret_cast<uint64_t*>(base + NA_KEYS_OFF);
  uint64_t* keysB = keysA + NOALLOC_MAX_NNZ;
  uint32_t* permA = reinterpret_cast<uint32_t*>(base + NA_PERM_OFF);
  uint32_t* permB = permA + NOALLOC_MAX_NNZ;
  uint32_t* hist = reinterpret_cast<uint32_t*>(base + NA_HIST_OFF);
  uint32_t* part = reinterpret_cast<uint32_t*>(base + NA_PART_OFF);

  int keys[4];
  const int nk = sort_key_plan(impl, nd, dims, mode, keys);
  // Every scratch region is fully written before it is read (the
  // permutation by iota, keys by packing, histograms by k_rs_hist, partials
  // by the scan), so nothing left by the previous call is used.
  MMCSF_CUDA(iota_u32(permA, nnz, s));
  // LSD over <= 64-bit key groups, least significant group first
  int g_end = nk;
  while (g_end > 0) {
    int g_beg = g_end, bits = 0;
    while (g_beg > 0 && bits + bits_of(dims[keys[g_beg - 1]]) <= 64 && g_end - g_beg < 4) {
      bits += bits_of(dims[keys[g_beg - 1]]);
      --g_beg;
    }
    int md[4] = {0, 0, 0, 0}, sh[4] = {0, 0, 0, 0}, tot = 0;
    for (int j = g_end - 1; j >= g_beg; --j) {
      md[j - g_beg] = keys[j];
      sh[j - g_beg] = tot;
      tot += bits_of(dims[keys[j]]);
    }
    if (tot > 0) {
      const uint32_t* ip[4] = {d_inds[0], d_inds[1], d_inds[2], nd == 4 ? d_inds[3] : d_inds[0]};
      k_na_pack<<<grid_for(nnz, 256), 256, 0, s>>>(ip[0], ip[1], ip[2], ip[3], permA, g_end - g_beg,
                                                   make_int4(md[0], md[1], md[2], md[3]),
                                                   make_int4(sh[0], sh[1], sh[2], sh[3]), nnz, keysA);
      MMCSF_LAUNCH_CHECK();
      const uint32_t ntiles = (uint32_t)((nnz + RS_TILE - 1) / RS_TILE);
      const uint64_t nh = (uint64_t)ntiles * RS_RADIX;
      uint64_t *ka = keysA, *kb = keysB;
      uint32_t *va = permA, *vb = permB;
      int passes = 0;
      for (int shift = 0; shift < tot; shift += 8, ++passes) {
        k_rs_hist<<<ntiles, RS_T, 0, s>>>(ka, nnz, shift, hist, ntiles);
        MMCSF_LAUNCH_CHECK();
        MMCSF_CUDA(na_scan(hist, nh, part, s));
        k_rs_scatter<<<ntiles, RS_T, 0, s>>>(ka, va, kb, vb, nnz, shift, hist, ntiles);
        MMCSF_LAUNCH_CHECK();
        std::swap(ka, kb);
        std::swap(va, vb);
      }
      if (passes & 1) MMCSF_CUDA(cudaMemcpyAsync(permA, permB, nnz * 4, cudaMemcpyDeviceToDevice, s));
    }
    g_end = g_beg;
  }
  for (int m = 0; m < nd; ++m) MMCSF_CUDA(gather_u32(d_inds[m], permA, d_out_inds[m], nnz, s));
  k_na_gather_f32<<<grid_for(nnz, 256), 256, 0, s>>>(d_vals, permA, nnz, d_out_vals);
  MMCSF_LAUNCH_CHECK();
  return MMCSF_OK;
}
