// Seeded synthetic sparse tensors, generated on the device.
//
// Candidate j (a global counter) gets, for every mode m, a coordinate drawn
// from a counter-based hash of (seed, m, j): uniform over the mode, or a Zipf
// rank (P(k) ~ k^-s, k = 1..dim) mapped through a seeded permutation of the
// mode. The tensor is the first `nnz` candidates, in candidate order, whose
// coordinates were not taken by an earlier candidate. Because every
// candidate's coordinates depend only on j, the result does not depend on how
// candidates are batched. Values depend only on the kept candidate's j.
#include <cmath>
#include <cstring>
#include <vector>

#include "common.h"
#include "prims.cuh"

using mmcsf::set_error;

namespace {

__host__ __device__ __forceinline__ uint64_t splitmix(uint64_t x) {
  x += 0x9e3779b97f4a7c15ull;
  x = (x ^ (x >> 30)) * 0xbf58476d1ce4e5b9ull;
  x = (x ^ (x >> 27)) * 0x94d049bb133111ebull;
  return x ^ (x >> 31);
}
__host__ __device__ __forceinline__ uint64_t hash3(uint64_t seed, uint64_t stream, uint64_t j) {
  return splitmix(splitmix(seed ^ (stream * 0xd1b54a32d192ed03ull)) ^ j);
}
// Uniform in the open interval (0, 1).
__host__ __device__ __forceinline__ double u01(uint64_t h) {
  return ((double)(h >> 11) + 0.5) * (1.0 / 9007199254740992.0);
}

struct ModeGen {
  uint64_t dim;
  int dist;
  const double* cdf;     // Zipf CDF (dim entries), device
  const uint32_t* perm;  // rank -> index permutation, device
};
struct GenArgs {
  int nd;
  uint64_t seed;
  ModeGen m[4];
  uint64_t radix[4];  // mixed-radix multipliers of the linear key
};

__device__ __forceinline__ uint32_t draw_coord(const GenArgs& a, int m, uint64_t j) {
  const ModeGen& g = a.m[m];
  double u = u01(hash3(a.seed, (uint64_t)m + 1, j));
  if (g.dist == MMCSF_DIST_UNIFORM) {
    uint64_t k = (uint64_t)(u * (double)g.dim);
    return (uint32_t)(k < g.dim ? k : g.dim - 1);
  }
  // first rank whose CDF reaches u
  uint64_t lo = 0, hi = g.dim - 1;
  while (lo < hi) {
    uint64_t mid = (lo + hi) >> 1;
    if (g.cdf[mid] < u) lo = mid + 1; else hi = mid;
  }
  return g.perm[lo];
}

__global__ void k_candidates(GenArgs a, uint64_t j0, uint64_t cnt, uint64_t* keys, uint32_t* cand) {
  for (uint64_t t = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; t < cnt; t += (uint64_t)gridDim.x * blockDim.x) {
    uint64_t j = j0 + t, key = 0;
    for (int m = 0; m < a.nd; ++m) key += (uint64_t)draw_coord(a, m, j) * a.radix[m];
    keys[t] = key;
    cand[t] = (uint32_t)j;
  }
}

// flag[i] = 1 if sorted entry i starts a new key group (first occurrence).
__global__ void k_first_of_group(const uint64_t* keys, uint64_t n, uint32_t* flag) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
    flag[i] = (i == 0 || keys[i] != keys[i - 1]) ? 1u : 0u;
}

__global__ void k_compact(const uint64_t* keys, const uint32_t* cand, const uint32_t* flag, const uint32_t* pos,
                          uint64_t n, uint64_t* okeys, uint32_t* ocand) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
    if (flag[i]) {
      okeys[pos[i]] = keys[i];
      ocand[pos[i]] = cand[i];
    }
}

__global__ void k_emit(GenArgs a, const uint32_t* cand, uint64_t n, int val_dist, uint32_t* i0, uint32_t* i1,
                       uint32_t* i2, uint32_t* i3, float* vals) {
  for (uint64_t t = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; t < n; t += (uint64_t)gridDim.x * blockDim.x) {
    uint64_t j = cand[t];
    uint32_t* outs[4] = {i0, i1, i2, i3};
    for (int m = 0; m < a.nd; ++m) outs[m][t] = draw_coord(a, m, j);
    double u1 = u01(hash3(a.seed, 101, j)), u2 = u01(hash3(a.seed, 102, j));
    float v;
    if (val_dist == MMCSF_VAL_LOGNORMAL) {
      double z = sqrt(-2.0 * log(u1)) * cos(6.283185307179586 * u2);
      v = (float)exp(z);
    } else if (val_dist == MMCSF_VAL_INT1_50) {
      v = (float)(1 + (int)(u1 * 50.0 < 50.0 ? u1 * 50.0 : 49.0));
    } else {
      v = (float)(1.0 - u1 * (1.0 - 1e-7));  // (0, 1]
    }
    vals[t] = v;
  }
}

__global__ void k_widen(const uint32_t* in, uint64_t* out, uint64_t n) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
    out[i] = in[i];
}

// okeys[i] = ck[slot[i]], ocand[i] = cidx[i] (ascending candidate index)
__global__ void k_regather(const uint64_t* ck, const uint32_t* slot, const uint64_t* cidx, uint64_t* okeys,
                           uint32_t* ocand, uint64_t n) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
    okeys[i] = ck[slot[i]];
    ocand[i] = (uint32_t)cidx[i];
  }
}

// Planted CP model value of nonzero t: sum_r prod_m A_m[i_m, r], A_m[i, r]
// uniform in [0,1) from a hash of (seed, m, r, i).
__device__ __forceinline__ double planted_value(uint64_t seed, int nd, const uint32_t* const* inds, uint64_t t, int K) {
  double v = 0;
  for (int r = 0; r < K; ++r) {
    double p = 1;
    for (int m = 0; m < nd; ++m) p *= u01(hash3(seed ^ 0x5bd1e995ull, (uint64_t)(m * 4096 + r + 7), inds[m][t]));
    v += p;
  }
  return v;
}

__global__ void k_planted(uint64_t seed, int nd, const uint32_t* i0, const uint32_t* i1, const uint32_t* i2,
                          const uint32_t* i3, uint64_t n, int K, float* vals, double* sumsq) {
  const uint32_t* in[4] = {i0, i1, i2, i3};
  double acc = 0;
  for (uint64_t t = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; t < n; t += (uint64_t)gridDim.x * blockDim.x) {
    const double v = planted_value(seed, nd, in, t, K);
    vals[t] = (float)v;
    acc += v * v;
  }
  atomicAdd(sumsq, acc);
}

// noise N(0, sigma^2) by Box-Muller; or a Poisson draw with mean vals[t]
// (inversion for small means, a rounded normal for large ones), at least 1.
__global__ void k_perturb(uint64_t seed, uint64_t n, const uint32_t* cand, double sigma, int poisson, float* vals) {
  for (uint64_t t = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; t < n; t += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t j = cand[t];
    const double u1 = u01(hash3(seed, 201, j)), u2 = u01(hash3(seed, 202, j));
    if (poisson) {
      const double mu = vals[t];
      double k;
      if (mu < 30) {
        double pk = exp(-mu), cdf = pk;
        k = 0;
        while (cdf < u1 && k < 1000) { k += 1; pk *= mu / k; cdf += pk; }
      } else {
        const double z = sqrt(-2.0 * log(u1)) * cos(6.283185307179586 * u2);
        k = floor(mu + sqrt(mu) * z + 0.5);
      }
      vals[t] = (float)(k < 1 ? 1 : k);
    } else {
      const double z = sqrt(-2.0 * log(u1)) * cos(6.283185307179586 * u2);
      vals[t] = (float)(vals[t] + sigma * z);
    }
  }
}

int bits_for(uint64_t v) {  // bits to hold values 0..v-1
  int b = 0;
  while (b < 64 && (v - 1) >> b) ++b;
  return b;
}

}  // namespace

extern "C" int mmcsf_generate(const mmcsf_gen_spec* spec, void* stream, mmcsf_coo** out) {
  MMCSF_RANGE("mmcsf_generate");
  using namespace mmcsf;
  if (!spec || !out) return set_error(MMCSF_ERR_INVALID, "null argument");
  const int nd = spec->nd;
  if (nd < 3 || nd > 4) return set_error(MMCSF_ERR_INVALID, "Supported tensor dimension is 3 or 4 (got %d)", nd);
  cudaStream_t s = S(stream);
  long double space = 1;
  for (int m = 0; m < nd; ++m) {
    if (spec->dims[m] == 0 || spec->dims[m] >= (1ull << 32)) return set_error(MMCSF_ERR_INVALID, "bad mode length");
    space *= (long double)spec->dims[m];
  }
  if (space >= 18446744073709551615.0L)
    return set_error(MMCSF_ERR_UNSUPPORTED, "coordinate space exceeds 2^64");
  if ((long double)spec->nnz > space) return set_error(MMCSF_ERR_INVALID, "more nonzeros than coordinates");
  if (spec->nnz >= (1ull << 31)) return set_error(MMCSF_ERR_INVALID, "nonzero count too large");
  const uint64_t N = spec->nnz;

  GenArgs a{};
  a.nd = nd;
  a.seed = spec->seed;
  DevBuf cdf[4], perm[4];
  uint64_t mult = 1;
  for (int m = nd - 1; m >= 0; --m) {
    a.radix[m] = mult;
    mult *= spec->dims[m];
  }
  for (int m = 0; m < nd; ++m) {
    const uint64_t d = spec->dims[m];
    a.m[m].dim = d;
    a.m[m].dist = spec->dist[m];
    if (spec->dist[m] == MMCSF_DIST_ZIPF) {
      const double sx = spec->zipf_s[m];
      std::vector<double> c(d);
      double acc = 0;
      for (uint64_t k = 0; k < d; ++k) {
        acc += pow((double)(k + 1), -sx);
        c[k] = acc;
      }
      for (uint64_t k = 0; k < d; ++k) c[k] /= acc;
      c[d - 1] = 1.0;
      std::vector<uint32_t> p(d);
      for (uint64_t k = 0; k < d; ++k) p[k] = (uint32_t)k;
      uint64_t st = splitmix(spec->seed ^ (0xabcdef12345ull + (uint64_t)m));
      for (uint64_t k = d - 1; k > 0; --k) {  // Fisher-Yates with a seeded stream
        st = splitmix(st);
        uint64_t r = st % (k + 1);
        uint32_t t = p[k]; p[k] = p[r]; p[r] = t;
      }
      MMCSF_CUDA(cdf[m].alloc(d * sizeof(double)));
      MMCSF_CUDA(perm[m].alloc(d * sizeof(uint32_t)));
      MMCSF_CUDA(cudaMemcpyAsync(cdf[m].p, c.data(), d * sizeof(double), cudaMemcpyHostToDevice, s));
      MMCSF_CUDA(cudaMemcpyAsync(perm[m].p, p.data(), d * sizeof(uint32_t), cudaMemcpyHostToDevice, s));
      MMCSF_CUDA(cudaStreamSynchronize(s));
      a.m[m].cdf = cdf[m].as<double>();
      a.m[m].perm = perm[m].as<uint32_t>();
    } else if (spec->dist[m] != MMCSF_DIST_UNIFORM) {
      return set_error(MMCSF_ERR_INVALID, "unknown distribution %d", spec->dist[m]);
    }
  }
  const int key_bits = bits_for((uint64_t)space);

  // pool of kept candidates (sorted by candidate index) plus new candidates
  uint64_t cap = N + N / 4 + 4096;
  DevBuf keys, cand, keys2, cand2, flag;
  MMCSF_CUDA(keys.alloc(cap * 8));
  MMCSF_CUDA(cand.alloc(cap * 4));
  MMCSF_CUDA(keys2.alloc(cap * 8));
  MMCSF_CUDA(cand2.alloc(cap * 4));
  MMCSF_CUDA(flag.alloc((cap + 1) * 4));
  uint64_t kept = 0, next = 0;
  for (int round = 0; kept < N; ++round) {
    if (round > 200) return set_error(MMCSF_ERR_INVALID, "could not draw %llu distinct coordinates",
                                      (unsigned long long)N);
    uint64_t need = N - kept;
    uint64_t draw = need + need / 4 + 1024;
    if (kept + draw > cap) {
      // grow the pool
      uint64_t ncap = kept + draw;
      DevBuf k2, c2;
      MMCSF_CUDA(k2.alloc(ncap * 8));
      MMCSF_CUDA(c2.alloc(ncap * 4));
      if (kept) {
        MMCSF_CUDA(cudaMemcpyAsync(k2.p, keys.p, kept * 8, cudaMemcpyDeviceToDevice, s));
        MMCSF_CUDA(cudaMemcpyAsync(c2.p, cand.p, kept * 4, cudaMemcpyDeviceToDevice, s));
      }
      keys = std::move(k2);
      cand = std::move(c2);
      MMCSF_CUDA(keys2.alloc(ncap * 8));
      MMCSF_CUDA(cand2.alloc(ncap * 4));
      MMCSF_CUDA(flag.alloc((ncap + 1) * 4));
      cap = ncap;
    }
    k_candidates<<<grid_for(draw, 256), 256, 0, s>>>(a, next, draw, keys.as<uint64_t>() + kept,
                                                     cand.as<uint32_t>() + kept);
    MMCSF_LAUNCH_CHECK();
    next += draw;
    const uint64_t n = kept + draw;
    // stable sort by key: equal keys stay in candidate order
    MMCSF_CUDA(radix_sort_pairs(keys.as<uint64_t>(), cand.as<uint32_t>(), keys2.as<uint64_t>(),
                                cand2.as<uint32_t>(), n, key_bits, s));
    k_first_of_group<<<grid_for(n, 256), 256, 0, s>>>(keys.as<uint64_t>(), n, flag.as<uint32_t>());
    MMCSF_LAUNCH_CHECK();
    MMCSF_CUDA(exclusive_scan_u32(flag.as<uint32_t>(), keys2.as<uint32_t>(), n, s));  // positions in keys2 scratch
    uint32_t total = 0;
    MMCSF_CUDA(cudaMemcpyAsync(&total, keys2.as<uint32_t>() + n, 4, cudaMemcpyDeviceToHost, s));
    MMCSF_CUDA(cudaStreamSynchronize(s));
    // compact the first occurrences (still in key order)
    DevBuf ck, cc;
    MMCSF_CUDA(ck.alloc((uint64_t)total * 8));
    MMCSF_CUDA(cc.alloc((uint64_t)total * 4));
    k_compact<<<grid_for(n, 256), 256, 0, s>>>(keys.as<uint64_t>(), cand.as<uint32_t>(), flag.as<uint32_t>(),
                                               keys2.as<uint32_t>(), n, ck.as<uint64_t>(), cc.as<uint32_t>());
    MMCSF_LAUNCH_CHECK();
    kept = total;
    // restore candidate order: sort (candidate index, slot) pairs, then gather
    uint64_t* cidx = keys.as<uint64_t>();
    uint32_t* slot = cand.as<uint32_t>();
    k_widen<<<grid_for(kept, 256), 256, 0, s>>>(cc.as<uint32_t>(), cidx, kept);
    MMCSF_LAUNCH_CHECK();
    MMCSF_CUDA(iota_u32(slot, kept, s));
    MMCSF_CUDA(radix_sort_pairs(cidx, slot, keys2.as<uint64_t>(), cand2.as<uint32_t>(), kept, 32, s));
    k_regather<<<grid_for(kept, 256), 256, 0, s>>>(ck.as<uint64_t>(), slot, cidx, keys2.as<uint64_t>(),
                                                   cand2.as<uint32_t>(), kept);
    MMCSF_LAUNCH_CHECK();
    MMCSF_CUDA(cudaMemcpyAsync(keys.p, keys2.p, kept * 8, cudaMemcpyDeviceToDevice, s));
    MMCSF_CUDA(cudaMemcpyAsync(cand.p, cand2.p, kept * 4, cudaMemcpyDeviceToDevice, s));
    if (next >= (1ull << 32) - cap) return set_error(MMCSF_ERR_INVALID, "candidate counter overflow");
  }
  // first N kept candidates in candidate order
  mmcsf_coo* X = new (std::nothrow) mmcsf_coo;
  if (!X) return set_error(MMCSF_ERR_NOMEM, "host allocation failed");
  X->nd = nd;
  X->nnz = N;
  for (int m = 0; m < nd; ++m) X->dims[m] = spec->dims[m];
  uint32_t* outs[4] = {nullptr, nullptr, nullptr, nullptr};
  for (int m = 0; m < nd; ++m) {
    if (X->d_inds[m].alloc(N * 4) != cudaSuccess) { delete X; return set_error(MMCSF_ERR_NOMEM, "cudaMalloc"); }
    outs[m] = X->d_inds[m].as<uint32_t>();
  }
  if (X->d_vals.alloc(N * 4) != cudaSuccess) { delete X; return set_error(MMCSF_ERR_NOMEM, "cudaMalloc"); }
  if (N) {
    k_emit<<<grid_for(N, 256), 256, 0, s>>>(a, cand.as<uint32_t>(), N, spec->val_dist, outs[0], outs[1], outs[2],
                                            outs[3] ? outs[3] : outs[0], X->d_vals.as<float>());
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess && spec->planted_rank > 0) {
      DevBuf ss;
      e = ss.alloc(8);
      if (e == cudaSuccess) e = cudaMemsetAsync(ss.p, 0, 8, s);
      if (e == cudaSuccess) {
        k_planted<<<grid_for(N, 256), 256, 0, s>>>(spec->seed, nd, outs[0], outs[1], outs[2], outs[3] ? outs[3] : outs[0],
                                                   N, spec->planted_rank, X->d_vals.as<float>(), ss.as<double>());
        e = cudaGetLastError();
      }
      double sumsq = 0;
      if (e == cudaSuccess) e = cudaMemcpyAsync(&sumsq, ss.p, 8, cudaMemcpyDeviceToHost, s);
      if (e == cudaSuccess) e = cudaStreamSynchronize(s);
      if (e == cudaSuccess && (spec->noise > 0 || spec->poisson)) {
        const double sigma = spec->noise * sqrt(sumsq / (double)N);
        k_perturb<<<grid_for(N, 256), 256, 0, s>>>(spec->seed, N, cand.as<uint32_t>(), sigma, spec->poisson,
                                                   X->d_vals.as<float>());
        e = cudaGetLastError();
      }
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) { delete X; return set_error(MMCSF_ERR_CUDA, "generator: %s", cudaGetErrorString(e)); }
  }
  X->dev_valid = true;
  *out = X;
  return MMCSF_OK;
}

