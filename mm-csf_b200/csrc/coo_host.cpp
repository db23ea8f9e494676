// Host COO MTTKRP: the reference's `-t 1` path (MTTKRP_COO_CPU[_4D],
// src/mttkrp_cpu.cpp:60-113) as a library entry point, so the `mttkrp`
// command serves -t 1 itself.
//
// Per nonzero x and column r, with the cyclic mode order
// (mode, mode+1, ...) mod nd of src/mttkrp_cpu.cpp:65-66:
//   out[i0, r] += ((v * U1[i1, r]) * U2[i2, r]) [* U3[i3, r]]
// in FP32 with the reference's association. With one thread the nonzeros
// are visited in order, so the result is the reference's bit for bit. With T
// threads, thread t runs the same loop over the t-th contiguous range of
// nonzeros into a private zeroed buffer and the buffers are added to `out`
// in thread order, rows split across the threads (the reference's loop has
// its OpenMP pragma commented out, src/mttkrp_cpu.cpp:79, so it has no
// parallel form to follow; this one stays deterministic for a given T).
#include <stdint.h>

#include <algorithm>
#include <cstring>
#include <new>
#include <thread>
#include <vector>

#include "common.h"

using mmcsf::set_error;

namespace {

template <int ND>
void coo_range(const uint32_t* const* ind, const float* vals, uint64_t x0, uint64_t x1, const int* md, int R,
               const float* const* U, float* out) {
  const uint32_t* i0 = ind[md[0]];
  const uint32_t* i1 = ind[md[1]];
  const uint32_t* i2 = ind[md[2]];
  const uint32_t* i3 = ND == 4 ? ind[md[3]] : nullptr;
  const float* U1 = U[md[1]];
  const float* U2 = U[md[2]];
  const float* U3 = ND == 4 ? U[md[3]] : nullptr;
  for (uint64_t x = x0; x < x1; ++x) {
    float* o = out + (uint64_t)i0[x] * R;
    const float* a = U1 + (uint64_t)i1[x] * R;
    const float* b = U2 + (uint64_t)i2[x] * R;
    const float v = vals[x];
    if constexpr (ND == 3) {
      for (int r = 0; r < R; ++r) {
        const float t = v * a[r] * b[r];
        o[r] += t;
      }
    } else {
      const float* c = U3 + (uint64_t)i3[x] * R;
      for (int r = 0; r < R; ++r) {
        const float t = v * a[r] * b[r] * c[r];
        o[r] += t;
      }
    }
  }
}

}  // namespace

extern "C" int mmcsf_mttkrp_coo_host(const mmcsf_coo* X, int mode, int R, const float* const* h_factors,
                                     float* h_out, int threads) {
  MMCSF_RANGE("mmcsf_mttkrp_coo_host");
  if (!X || !h_factors || !h_out) return set_error(MMCSF_ERR_INVALID, "null argument");
  const int nd = X->nd;
  if (mode < 0 || mode >= nd) return set_error(MMCSF_ERR_INVALID, "Mode cannot be larger than tensor dimension.");
  if (R <= 0) return set_error(MMCSF_ERR_INVALID, "rank must be positive (got %d)", R);
  if (!X->host_valid)
    return set_error(MMCSF_ERR_INVALID, "the tensor has no host copy (mmcsf_coo_to_host first)");
  for (int m = 0; m < nd; ++m)
    if (m != mode && !h_factors[m]) return set_error(MMCSF_ERR_INVALID, "factor %d is null", m);
  const uint64_t n = X->nnz;
  if (n == 0) return MMCSF_OK;
  int md[4];
  for (int m = 0; m < nd; ++m) md[m] = (m + mode) % nd;
  const uint32_t* ind[4] = {nullptr, nullptr, nullptr, nullptr};
  for (int m = 0; m < nd; ++m) ind[m] = X->h_inds[m].data();
  const float* vals = X->h_vals.data();
  auto run = [&](uint64_t x0, uint64_t x1, float* out) {
    if (nd == 3) coo_range<3>(ind, vals, x0, x1, md, R, h_factors, out);
    else coo_range<4>(ind, vals, x0, x1, md, R, h_factors, out);
  };

  int T = threads > 0 ? threads : (int)std::max(1u, std::thread::hardware_concurrency());
  const uint64_t out_elems = X->dims[mode] * (uint64_t)R;
  // bound the private buffers at about 8 GiB
  const uint64_t cap_t = std::max<uint64_t>(1, (8ull << 30) / std::max<uint64_t>(1, out_elems * 4));
  T = (int)std::min<uint64_t>({(uint64_t)T, cap_t, n, 256});
  if (T <= 1) {
    run(0, n, h_out);
    return MMCSF_OK;
  }
  std::vector<float*> priv(T, nullptr);
  for (int t = 0; t < T; ++t) {
    priv[t] = new (std::nothrow) float[out_elems];
    if (!priv[t]) {
      for (int u = 0; u < t; ++u) delete[] priv[u];
      return set_error(MMCSF_ERR_NOMEM, "host allocation of %d private outputs failed", T);
    }
  }
  std::vector<std::thread> pool;
  pool.reserve(T);
  for (int t = 0; t < T; ++t)
    pool.emplace_back([&, t]() {
      std::memset(priv[t], 0, out_elems * 4);
      run(n * t / T, n * (t + 1) / T, priv[t]);
    });
  for (auto& th : pool) th.join();
  pool.clear();
  // out += priv[0] + ... + priv[T-1], rows split across the threads
  for (int t = 0; t < T; ++t)
    pool.emplace_back([&, t]() {
      const uint64_t e0 = out_elems * t / T, e1 = out_elems * (t + 1) / T;
      for (int u = 0; u < T; ++u) {
        const float* p = priv[u];
        for (uint64_t e = e0; e < e1; ++e) h_out[e] += p[e];
      }
    });
  for (auto& th : pool) th.join();
  for (int t = 0; t < T; ++t) delete[] priv[t];
  return MMCSF_OK;
}
