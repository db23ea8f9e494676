// CP-ALS on the device (the reference's cpd(), src/cpd_cpu.cu:484-691, with
// its GPU hooks init_GPU / MTTKRP_MIHCSR_GPU_oneMode_forCPD,
// src/mttkrp_gpu.cu:3786-4052).
//
// Per iteration and mode m: MTTKRP into M; V = Hadamard of the other modes'
// Gram matrices; U_m = M V^-1 (Cholesky, Gauss-Jordan with pivoting if V is not
// positive definite, as the reference falls back to gesv); column norms ->
// lambda (2-norm in the first iteration, max-norm after); the Gram of the new
// factor. After the last mode, the fit. Everything stays on the device.
//
// Two forms:
//   * precision MMCSF_CPD_FP32: FP32 factors and FP32 small-matrix math;
//   * precision MMCSF_CPD_BF16: BF16 factors (the MTTKRP inputs) with FP32
//     accumulation, and the Gram Hadamard / Cholesky solve / lambda / fit in
//     FP64.
// Either form runs the whole loop as ONE CUDA graph launch (a WHILE
// conditional node whose body is one iteration, the fit kernel setting the
// condition) unless opts.no_graph is set; on the default stream, which cannot
// be captured, the FP32 forms run host-driven instead (one iteration at a time,
// the fit read back to test convergence, like the reference's structure) and
// the BF16 form is refused.
//
// Deviations from the reference, on purpose: the fit uses the full symmetric
// Gram product (the reference reads the unwritten triangle,
// src/cpd_cpu.cu:383-385 vs the 'L' ssyrk at :543-546), the max-norm is a true
// column maximum clamped below at 1 (the reference's loop compares against the
// zeroed lambda and sums per-thread values, :298-303), and there is no write
// past the R x R Gram (:119).
#include <cuda_bf16.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <type_traits>
#include <vector>

#include "format.h"
#include "prims.cuh"

using mmcsf::set_error;

namespace mmcsf {
int mttkrp_mode(const mmcsf_format* F, int mode, int R, int dtype, const void* const* U, float* out,
                const mmcsf_kernel_cfg* cfg, cudaStream_t s, int* launches);
int reserve_leaf_scratch(mmcsf_format* F, int R, int dtype);

namespace {

constexpr int MAXR = 64;

template <class T> __device__ __forceinline__ double tod(T x);
template <> __device__ __forceinline__ double tod<float>(float x) { return (double)x; }
template <> __device__ __forceinline__ double tod<double>(double x) { return x; }
template <> __device__ __forceinline__ double tod<__nv_bfloat16>(__nv_bfloat16 x) { return (double)__bfloat162float(x); }
template <class T> __device__ __forceinline__ T fromd(double x);
template <> __device__ __forceinline__ float fromd<float>(double x) { return (float)x; }
template <> __device__ __forceinline__ double fromd<double>(double x) { return x; }
template <> __device__ __forceinline__ __nv_bfloat16 fromd<__nv_bfloat16>(double x) { return __float2bfloat16((float)x); }

// order-preserving map of floats to unsigned (for atomicMax on signed values)
__device__ __forceinline__ unsigned f2ord(float f) {
  const unsigned u = __float_as_uint(f);
  return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
__device__ __forceinline__ float ord2f(unsigned u) {
  return __uint_as_float((u & 0x80000000u) ? (u & 0x7fffffffu) : ~u);
}

// Uniform [0,1) initial factors from a counter-based hash (seeded).
__device__ __forceinline__ uint64_t mix64(uint64_t x) {
  x += 0x9e3779b97f4a7c15ull;
  x = (x ^ (x >> 30)) * 0xbf58476d1ce4e5b9ull;
  x = (x ^ (x >> 27)) * 0x94d049bb133111ebull;
  return x ^ (x >> 31);
}
template <class T>
__global__ void k_init(T* U, uint64_t n, uint64_t seed, int m) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
    U[i] = fromd<T>((double)(mix64(mix64(seed + 0x51ed27u * (uint64_t)(m + 1)) ^ i) >> 11) * (1.0 / 9007199254740992.0));
}
template <class T>
__global__ void k_convert(const float* in, T* out, uint64_t n) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
    out[i] = fromd<T>((double)in[i]);
}

// Gram G += U^T U over this block's row tiles (G pre-zeroed, full R x R).
template <class T, class A>
__global__ void __launch_bounds__(256) k_gram(const T* __restrict__ U, uint64_t rows, int R, A* __restrict__ G) {
  constexpr int TR = 32;
  __shared__ A tile[TR * MAXR];
  constexpr int EPT = MAXR * MAXR / 256;
  A acc[EPT];
#pragma unroll
  for (int e = 0; e < EPT; ++e) acc[e] = 0;
  const int RR = R * R;
  for (uint64_t r0 = (uint64_t)blockIdx.x * TR; r0 < rows; r0 += (uint64_t)gridDim.x * TR) {
    const int nr = (int)min((uint64_t)TR, rows - r0);
    __syncthreads();
    for (int t = threadIdx.x; t < nr * R; t += blockDim.x) tile[t] = (A)tod(U[r0 * R + t]);
    __syncthreads();
#pragma unroll
    for (int e = 0; e < EPT; ++e) {
      const int q = threadIdx.x + e * 256;
      if (q < RR) {
        const int a = q / R, b = q % R;
        A s = 0;
        for (int i = 0; i < nr; ++i) s += tile[i * R + a] * tile[i * R + b];
        acc[e] += s;
      }
    }
  }
#pragma unroll
  for (int e = 0; e < EPT; ++e) {
    const int q = threadIdx.x + e * 256;
    if (q < RR) atomicAdd(&G[q], acc[e]);
  }
}

// V = Hadamard of the Grams of every mode but `mode`; Vinv = V^-1 by Cholesky
// (Gauss-Jordan with partial pivoting when V is not positive definite).
// One block; dynamic shared memory: V[R*R], W[R*R], fac[R] of A.
// status[0] = 1 when the fallback ran.
template <class A>
__global__ void __launch_bounds__(256) k_solve(const A* __restrict__ grams, int nd, int mode, int R,
                                               A* __restrict__ Vinv, int* status) {
  extern __shared__ __align__(16) unsigned char sm_raw[];
  A* V = reinterpret_cast<A*>(sm_raw);
  A* W = V + R * R;
  A* fac = W + R * R;
  __shared__ int ok, piv;
  const int RR = R * R;
  auto build_v = [&]() {
    for (int q = threadIdx.x; q < RR; q += blockDim.x) {
      A v = 1;
      for (int p = 0; p < nd; ++p)
        if (p != mode) v *= grams[(size_t)p * RR + q];
      V[q] = v;
    }
  };
  build_v();
  if (threadIdx.x == 0) ok = 1;
  __syncthreads();
  // Cholesky V = L L^T in place (lower), right-looking
  for (int j = 0; j < R; ++j) {
    if (threadIdx.x == 0) {
      const A d = V[j * R + j];
      if (!(d > 0)) ok = 0;
      else V[j * R + j] = sqrt(d);
    }
    __syncthreads();
    if (!ok) break;
    const A dj = V[j * R + j];
    for (int i = j + 1 + threadIdx.x; i < R; i += blockDim.x) V[i * R + j] /= dj;
    __syncthreads();
    for (int q = threadIdx.x; q < (R - j - 1) * (R - j - 1); q += blockDim.x) {
      const int i = j + 1 + q / (R - j - 1), k = j + 1 + q % (R - j - 1);
      if (k <= i) V[i * R + k] -= V[i * R + j] * V[k * R + j];
    }
    __syncthreads();
  }
  if (ok) {
    // Linv (lower) into W: column c by forward substitution, one thread per column
    for (int c = threadIdx.x; c < R; c += blockDim.x) {
      for (int i = 0; i < R; ++i) {
        A sacc = (i == c) ? (A)1 : (A)0;
        for (int k = c; k < i; ++k) sacc -= V[i * R + k] * W[k * R + c];
        W[i * R + c] = (i < c) ? (A)0 : sacc / V[i * R + i];
      }
    }
    __syncthreads();
    // Vinv = Linv^T Linv
    for (int q = threadIdx.x; q < RR; q += blockDim.x) {
      const int a = q / R, b = q % R;
      A sacc = 0;
      for (int k = max(a, b); k < R; ++k) sacc += W[k * R + a] * W[k * R + b];
      Vinv[q] = sacc;
    }
    if (threadIdx.x == 0 && status) status[0] = 0;
    return;
  }
  // fallback: Gauss-Jordan on [V | W = I] with partial pivoting (V rebuilt)
  __syncthreads();
  build_v();
  for (int q = threadIdx.x; q < RR; q += blockDim.x) W[q] = (q / R == q % R) ? (A)1 : (A)0;
  __syncthreads();
  for (int j = 0; j < R; ++j) {
    if (threadIdx.x == 0) {
      int p = j;
      A best = fabs(V[j * R + j]);
      for (int i = j + 1; i < R; ++i)
        if (fabs(V[i * R + j]) > best) { best = fabs(V[i * R + j]); p = i; }
      piv = p;
    }
    __syncthreads();
    if (piv != j)
      for (int c = threadIdx.x; c < R; c += blockDim.x) {
        A t = V[j * R + c]; V[j * R + c] = V[piv * R + c]; V[piv * R + c] = t;
        t = W[j * R + c]; W[j * R + c] = W[piv * R + c]; W[piv * R + c] = t;
      }
    __syncthreads();
    const A d = V[j * R + j];
    __syncthreads();
    for (int c = threadIdx.x; c < R; c += blockDim.x) {
      V[j * R + c] /= (d != 0 ? d : (A)1);
      W[j * R + c] /= (d != 0 ? d : (A)1);
    }
    for (int i = threadIdx.x; i < R; i += blockDim.x) fac[i] = V[i * R + j];
    __syncthreads();
    for (int q = threadIdx.x; q < RR; q += blockDim.x) {
      const int i = q / R, c = q % R;
      if (i != j) {
        V[i * R + c] -= fac[i] * V[j * R + c];
        W[i * R + c] -= fac[i] * W[j * R + c];
      }
    }
    __syncthreads();
  }
  for (int q = threadIdx.x; q < RR; q += blockDim.x) Vinv[q] = W[q];
  if (threadIdx.x == 0 && status) status[0] = 1;
}

// Ut[i,:] = M[i,:] Vinv, plus per-column sum of squares (FP64) and maximum.
template <class A>
__global__ void __launch_bounds__(256) k_apply(const float* __restrict__ M, uint64_t rows, int R,
                                               const A* __restrict__ Vinv, float* __restrict__ Ut,
                                               double* __restrict__ colsq, unsigned* __restrict__ colmax) {
  __shared__ A vi[MAXR * MAXR];
  __shared__ double sq[MAXR];
  __shared__ unsigned mx[MAXR];
  for (int q = threadIdx.x; q < R * R; q += blockDim.x) vi[q] = Vinv[q];
  for (int q = threadIdx.x; q < R; q += blockDim.x) { sq[q] = 0; mx[q] = 0u; }
  __syncthreads();
  const uint64_t n = rows * (uint64_t)R;
  for (uint64_t t = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; t < n; t += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t i = t / R;
    const int c = (int)(t % R);
    const float* mr = M + i * R;
    A s = 0;
    for (int k = 0; k < R; ++k) s += (A)mr[k] * vi[k * R + c];
    const float o = (float)s;
    Ut[t] = o;
    atomicAdd(&sq[c], (double)s * (double)s);
    atomicMax(&mx[c], f2ord(o));
  }
  __syncthreads();
  for (int q = threadIdx.x; q < R; q += blockDim.x) {
    atomicAdd(&colsq[q], sq[q]);
    atomicMax(&colmax[q], mx[q]);
  }
}

struct State {  // device-resident loop state
  int iter;
  int converged;
  int keep_going;
  int solve_fallbacks;
  double fit, oldfit;
};

// lambda: column 2-norms in the first iteration, else max(column max, 1)
__global__ void k_lambda(const double* colsq, const unsigned* colmax, int R, const State* st, double* lambda) {
  for (int r = threadIdx.x; r < R; r += blockDim.x) {
    double l;
    if (st->iter == 0) {
      l = sqrt(colsq[r]);
      if (!(l > 0)) l = 1;
    } else {
      l = (double)ord2f(colmax[r]);
      if (l < 1) l = 1;
    }
    lambda[r] = l;
  }
}

// U = Ut / lambda stored as T; G += U^T U (of the stored values); for the last
// mode also inner[r] += sum_i U[i,r] M[i,r].
template <class T, class A>
__global__ void __launch_bounds__(256) k_finish(const float* __restrict__ Ut, uint64_t rows, int R,
                                                const double* __restrict__ lambda, T* __restrict__ U,
                                                A* __restrict__ G, const float* __restrict__ M,
                                                double* __restrict__ inner) {
  constexpr int TR = 32;
  __shared__ A tile[TR * MAXR];
  __shared__ double inn[MAXR];
  constexpr int EPT = MAXR * MAXR / 256;
  A acc[EPT];
#pragma unroll
  for (int e = 0; e < EPT; ++e) acc[e] = 0;
  for (int q = threadIdx.x; q < R; q += blockDim.x) inn[q] = 0;
  const int RR = R * R;
  for (uint64_t r0 = (uint64_t)blockIdx.x * TR; r0 < rows; r0 += (uint64_t)gridDim.x * TR) {
    const int nr = (int)min((uint64_t)TR, rows - r0);
    __syncthreads();
    for (int t = threadIdx.x; t < nr * R; t += blockDim.x) {
      const uint64_t g = r0 * R + t;
      const T u = fromd<T>((double)Ut[g] / lambda[t % R]);
      U[g] = u;
      const double ud = tod(u);
      tile[t] = (A)ud;
      if (M) atomicAdd(&inn[t % R], ud * (double)M[g]);
    }
    __syncthreads();
#pragma unroll
    for (int e = 0; e < EPT; ++e) {
      const int q = threadIdx.x + e * 256;
      if (q < RR) {
        const int a = q / R, b = q % R;
        A s = 0;
        for (int i = 0; i < nr; ++i) s += tile[i * R + a] * tile[i * R + b];
        acc[e] += s;
      }
    }
  }
#pragma unroll
  for (int e = 0; e < EPT; ++e) {
    const int q = threadIdx.x + e * 256;
    if (q < RR) atomicAdd(&G[q], acc[e]);
  }
  __syncthreads();
  if (M)
    for (int q = threadIdx.x; q < R; q += blockDim.x) atomicAdd(&inner[q], inn[q]);
}

// fit = 1 - sqrt(|X|^2 + lambda^T (Hadamard of all Grams) lambda - 2 <X, model>) / |X|
template <class A>
__global__ void k_fit(const A* __restrict__ grams, int nd, int R, const double* __restrict__ lambda,
                      const double* __restrict__ inner, double xnormsq, double tol, int maxit, State* st,
                      double* history, cudaGraphConditionalHandle handle, int use_handle) {
  __shared__ double part[256];
  double s = 0;
  for (int q = threadIdx.x; q < R * R; q += blockDim.x) {
    double v = lambda[q / R] * lambda[q % R];
    for (int p = 0; p < nd; ++p) v *= (double)grams[(size_t)p * R * R + q];
    s += v;
  }
  part[threadIdx.x] = s;
  __syncthreads();
  for (int w = 128; w > 0; w >>= 1) {
    if (threadIdx.x < w) part[threadIdx.x] += part[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    const double norm_mats = fabs(part[0]);
    double in = 0;
    for (int r = 0; r < R; ++r) in += lambda[r] * inner[r];
    double residual = xnormsq + norm_mats - 2 * in;
    if (residual > 0.0) residual = sqrt(residual);
    const double fit = 1 - residual / sqrt(xnormsq);
    const int it = st->iter;
    history[it] = fit;
    const int conv = (it > 0 && fabs(fit - st->oldfit) < tol) ? 1 : 0;
    st->oldfit = fit;
    st->fit = fit;
    st->converged = conv;
    st->iter = it + 1;
    st->keep_going = (!conv && it + 1 < maxit) ? 1 : 0;
    if (use_handle) cudaGraphSetConditional(handle, st->keep_going ? 1u : 0u);
  }
}

__global__ void k_sumsq_vals(const float* __restrict__ v, uint64_t n, double* out) {
  __shared__ double part[256];
  double s = 0;
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
    s += (double)v[i] * (double)v[i];
  part[threadIdx.x] = s;
  __syncthreads();
  for (int w = 128; w > 0; w >>= 1) {
    if (threadIdx.x < w) part[threadIdx.x] += part[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) atomicAdd(out, part[0]);
}

// GetFinalLambda (src/cpd_cpu.cu:406-424): lambda *= column 2-norms of every
// factor, factors divided by them; written out as FP32.
template <class T>
__global__ void k_colsq(const T* __restrict__ U, uint64_t rows, int R, double* __restrict__ colsq) {
  __shared__ double sq[MAXR];
  for (int q = threadIdx.x; q < R; q += blockDim.x) sq[q] = 0;
  __syncthreads();
  for (uint64_t t = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; t < rows * (uint64_t)R;
       t += (uint64_t)gridDim.x * blockDim.x) {
    const double u = tod(U[t]);
    atomicAdd(&sq[t % R], u * u);
  }
  __syncthreads();
  for (int q = threadIdx.x; q < R; q += blockDim.x) atomicAdd(&colsq[q], sq[q]);
}
template <class T>
__global__ void k_final(const T* __restrict__ U, uint64_t rows, int R, const double* __restrict__ colsq,
                        float* __restrict__ out) {
  for (uint64_t t = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; t < rows * (uint64_t)R;
       t += (uint64_t)gridDim.x * blockDim.x) {
    const double n = sqrt(colsq[t % R]);
    out[t] = (float)(tod(U[t]) / (n > 0 ? n : 1.0));
  }
}
__global__ void k_final_lambda(const double* colsq, int nd, int R, double* lambda) {
  for (int r = threadIdx.x; r < R; r += blockDim.x) {
    double l = lambda[r];
    for (int m = 0; m < nd; ++m) {
      const double n = sqrt(colsq[m * MAXR + r]);
      l *= (n > 0 ? n : 1.0);
    }
    lambda[r] = l;
  }
}

template <class T, class A>
struct Als {
  mmcsf_format* F;
  int nd, R, dtype;
  cudaStream_t s;
  DevBuf fac[4], M, Ut, grams, Vinv, colsq, colmax, lambda, inner, xn, st, hist, status;
  double tol;
  int maxit;
  int launches = 0;

  size_t solve_smem() const { return (size_t)(2 * R * R + R) * sizeof(A); }

  int setup(const mmcsf_cpd_opts* o, const float* const* d_init) {
    if (solve_smem() > 48 * 1024)
      MMCSF_CUDA(cudaFuncSetAttribute(k_solve<A>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)solve_smem()));
    uint64_t maxd = 0;
    for (int m = 0; m < nd; ++m) maxd = std::max(maxd, F->dims[m]);
    for (int m = 0; m < nd; ++m) MMCSF_CUDA(fac[m].alloc(F->dims[m] * (uint64_t)R * sizeof(T)));
    MMCSF_CUDA(M.alloc(maxd * R * 4));
    MMCSF_CUDA(Ut.alloc(maxd * R * 4));
    MMCSF_CUDA(grams.alloc((uint64_t)nd * R * R * sizeof(A)));
    MMCSF_CUDA(Vinv.alloc((uint64_t)R * R * sizeof(A)));
    MMCSF_CUDA(colsq.alloc(4 * MAXR * sizeof(double)));
    MMCSF_CUDA(colmax.alloc(MAXR * sizeof(unsigned)));
    MMCSF_CUDA(lambda.alloc(MAXR * sizeof(double)));
    MMCSF_CUDA(inner.alloc(MAXR * sizeof(double)));
    MMCSF_CUDA(xn.alloc(sizeof(double)));
    MMCSF_CUDA(st.alloc(sizeof(State)));
    MMCSF_CUDA(hist.alloc((uint64_t)maxit * sizeof(double)));
    MMCSF_CUDA(status.alloc(sizeof(int)));
    MMCSF_TRY(reserve_leaf_scratch(F, R, dtype));  // nothing allocates inside the iteration (it may be captured)
    MMCSF_CUDA(cudaMemsetAsync(st.p, 0, sizeof(State), s));
    MMCSF_CUDA(cudaMemsetAsync(hist.p, 0, (uint64_t)maxit * sizeof(double), s));
    MMCSF_CUDA(cudaMemsetAsync(grams.p, 0, (uint64_t)nd * R * R * sizeof(A), s));
    for (int m = 0; m < nd; ++m) {
      const uint64_t n = F->dims[m] * (uint64_t)R;
      if (d_init && d_init[m]) k_convert<T><<<grid_for(n, 256), 256, 0, s>>>(d_init[m], fac[m].as<T>(), n);
      else k_init<T><<<grid_for(n, 256), 256, 0, s>>>(fac[m].as<T>(), n, o->seed, m);
      MMCSF_LAUNCH_CHECK();
      k_gram<T, A><<<std::min<uint64_t>(grid_for(F->dims[m], 32) , (uint64_t)sm_count() * 4), 256, 0, s>>>(
          fac[m].as<T>(), F->dims[m], R, grams.as<A>() + (size_t)m * R * R);
      MMCSF_LAUNCH_CHECK();
    }
    MMCSF_CUDA(cudaMemsetAsync(xn.p, 0, sizeof(double), s));
    for (int p = 0; p < 4; ++p) {
      const CsfPart& P = F->parts[p];
      if (!P.present || !P.nnz) continue;
      k_sumsq_vals<<<grid_for(P.nnz, 256), 256, 0, s>>>(P.vals.as<float>(), P.nnz, xn.as<double>());
      MMCSF_LAUNCH_CHECK();
    }
    return MMCSF_OK;
  }

  // Per-phase timing (opts.profile): an event at every phase boundary of one
  // iteration, read back after the iteration.
  struct Prof {
    static constexpr int NEV = 4 * 6 + 2;  // up to 4 modes x 6 boundaries + fit
    cudaEvent_t ev[NEV] = {};
    int phase[NEV] = {};  // phase that ends at event i
    int n = 0;
    double ms[MMCSF_CPD_PHASES] = {};
    bool ok = false;
    int init() {
      for (auto& e : ev) MMCSF_CUDA(cudaEventCreate(&e));
      ok = true;
      return MMCSF_OK;
    }
    ~Prof() {
      if (ok)
        for (auto& e : ev) cudaEventDestroy(e);
    }
    void mark(cudaStream_t s, int ph) {  // phase `ph` ends here (-1: start)
      if (n < NEV) { cudaEventRecord(ev[n], s); phase[n] = ph; ++n; }
    }
    int collect() {  // after the stream has synchronised
      for (int i = 1; i < n; ++i) {
        float t = 0;
        MMCSF_CUDA(cudaEventElapsedTime(&t, ev[i - 1], ev[i]));
        if (phase[i] >= 0) ms[phase[i]] += t;
      }
      n = 0;
      return MMCSF_OK;
    }
  };

  // one ALS iteration, stream-ordered (capturable when prof is null)
  int iteration(double xnormsq, cudaGraphConditionalHandle h, int use_handle, Prof* prof = nullptr) {
    MMCSF_RANGE("mmcsf_cpd.iteration");
    const void* U[4];
    for (int m = 0; m < nd; ++m) U[m] = fac[m].p;
    auto mark = [&](int ph) { if (prof) prof->mark(s, ph); };
    mark(-1);
    MMCSF_CUDA(cudaMemsetAsync(inner.p, 0, MAXR * sizeof(double), s));
    for (int m = 0; m < nd; ++m) {
      const uint64_t rows = F->dims[m];
      MMCSF_TRY(mttkrp_mode(F, m, R, dtype, U, M.as<float>(), nullptr, s, &launches));
      mark(0);
      k_solve<A><<<1, 256, solve_smem(), s>>>(grams.as<A>(), nd, m, R, Vinv.as<A>(), status.as<int>());
      MMCSF_LAUNCH_CHECK();
      mark(1);
      MMCSF_CUDA(cudaMemsetAsync(colsq.p, 0, MAXR * sizeof(double), s));
      MMCSF_CUDA(cudaMemsetAsync(colmax.p, 0, MAXR * sizeof(unsigned), s));
      k_apply<A><<<grid_for(rows * (uint64_t)R, 256), 256, 0, s>>>(M.as<float>(), rows, R, Vinv.as<A>(),
                                                                   Ut.as<float>(), colsq.as<double>(),
                                                                   colmax.as<unsigned>());
      MMCSF_LAUNCH_CHECK();
      mark(2);
      k_lambda<<<1, 64, 0, s>>>(colsq.as<double>(), colmax.as<unsigned>(), R, st.as<State>(), lambda.as<double>());
      MMCSF_LAUNCH_CHECK();
      mark(3);
      MMCSF_CUDA(cudaMemsetAsync(grams.as<A>() + (size_t)m * R * R, 0, (uint64_t)R * R * sizeof(A), s));
      k_finish<T, A><<<std::min<uint64_t>(grid_for(rows, 32), (uint64_t)sm_count() * 4), 256, 0, s>>>(
          Ut.as<float>(), rows, R, lambda.as<double>(), fac[m].as<T>(), grams.as<A>() + (size_t)m * R * R,
          m == nd - 1 ? M.as<float>() : nullptr, inner.as<double>());
      MMCSF_LAUNCH_CHECK();
      mark(4);
      launches += 4;
    }
    k_fit<A><<<1, 256, 0, s>>>(grams.as<A>(), nd, R, lambda.as<double>(), inner.as<double>(), xnormsq, tol, maxit,
                               st.as<State>(), hist.as<double>(), h, use_handle);
    MMCSF_LAUNCH_CHECK();
    mark(5);
    ++launches;
    return MMCSF_OK;
  }

  int finish(float* const* d_out, double* h_lambda) {
    MMCSF_CUDA(cudaMemsetAsync(colsq.p, 0, 4 * MAXR * sizeof(double), s));
    for (int m = 0; m < nd; ++m) {
      const uint64_t n = F->dims[m] * (uint64_t)R;
      k_colsq<T><<<grid_for(n, 256), 256, 0, s>>>(fac[m].as<T>(), F->dims[m], R, colsq.as<double>() + m * MAXR);
      MMCSF_LAUNCH_CHECK();
    }
    k_final_lambda<<<1, 64, 0, s>>>(colsq.as<double>(), nd, R, lambda.as<double>());
    MMCSF_LAUNCH_CHECK();
    for (int m = 0; m < nd; ++m) {
      const uint64_t n = F->dims[m] * (uint64_t)R;
      if (d_out && d_out[m]) {
        k_final<T><<<grid_for(n, 256), 256, 0, s>>>(fac[m].as<T>(), F->dims[m], R, colsq.as<double>() + m * MAXR,
                                                    d_out[m]);
        MMCSF_LAUNCH_CHECK();
      }
    }
    if (h_lambda) MMCSF_CUDA(cudaMemcpyAsync(h_lambda, lambda.p, R * sizeof(double), cudaMemcpyDeviceToHost, s));
    return MMCSF_OK;
  }
};

template <class T, class A>
int run_cpd(mmcsf_format* F, const mmcsf_cpd_opts* o, const float* const* d_init, float* const* d_out,
            double* h_lambda, mmcsf_cpd_result* res, cudaStream_t s) {
  Als<T, A> als;
  als.F = F;
  als.nd = F->nd;
  als.R = o->rank;
  als.dtype = std::is_same<T, float>::value ? MMCSF_DTYPE_F32 : MMCSF_DTYPE_BF16;
  als.s = s;
  als.tol = o->tol > 0 ? o->tol : 1e-5;
  als.maxit = o->max_iters > 0 ? o->max_iters : 10;
  cudaEvent_t e0, e1;
  MMCSF_CUDA(cudaEventCreate(&e0));
  MMCSF_CUDA(cudaEventCreate(&e1));
  MMCSF_TRY(als.setup(o, d_init));
  double xnormsq = 0;
  MMCSF_CUDA(cudaMemcpyAsync(&xnormsq, als.xn.p, sizeof(double), cudaMemcpyDeviceToHost, s));
  MMCSF_CUDA(cudaStreamSynchronize(s));
  State hst{};
  int graph_used = 0;
  MMCSF_CUDA(cudaEventRecord(e0, s));
  typename Als<T, A>::Prof prof;
  if (o->profile) MMCSF_TRY(prof.init());
  if (!o->no_graph && !o->profile && (o->precision == MMCSF_CPD_BF16 || s != nullptr)) {
    // the whole loop as one graph: WHILE node, body = one iteration
    cudaGraph_t g = nullptr;
    cudaGraphExec_t ge = nullptr;
    MMCSF_CUDA(cudaGraphCreate(&g, 0));
    cudaGraphConditionalHandle h;
    int st = MMCSF_OK;
    cudaError_t e = cudaGraphConditionalHandleCreate(&h, g, 1, cudaGraphCondAssignDefault);
    cudaGraphNodeParams cp = {};
    cudaGraphNode_t node;
    if (e == cudaSuccess) {
      cp.type = cudaGraphNodeTypeConditional;
      cp.conditional.handle = h;
      cp.conditional.type = cudaGraphCondTypeWhile;
      cp.conditional.size = 1;
      e = cudaGraphAddNode(&node, g, nullptr, 0, &cp);
    }
    if (e == cudaSuccess) {
      cudaGraph_t body = cp.conditional.phGraph_out[0];
      e = cudaStreamBeginCaptureToGraph(s, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal);
      if (e == cudaSuccess) {
        st = als.iteration(xnormsq, h, 1);
        cudaError_t e2 = cudaStreamEndCapture(s, &body);
        if (st == MMCSF_OK && e2 != cudaSuccess) e = e2;
      }
    }
    if (e == cudaSuccess && st == MMCSF_OK) e = cudaGraphInstantiate(&ge, g, 0);
    if (e == cudaSuccess && st == MMCSF_OK) e = cudaGraphLaunch(ge, s);
    if (e == cudaSuccess && st == MMCSF_OK) e = cudaStreamSynchronize(s);
    if (ge) cudaGraphExecDestroy(ge);
    cudaGraphDestroy(g);
    if (st != MMCSF_OK) return st;
    if (e != cudaSuccess) return set_error(MMCSF_ERR_CUDA, "CP-ALS graph: %s", cudaGetErrorString(e));
    graph_used = 1;
  } else {
    for (int it = 0; it < als.maxit; ++it) {
      MMCSF_TRY(als.iteration(xnormsq, cudaGraphConditionalHandle{}, 0, o->profile ? &prof : nullptr));
      MMCSF_CUDA(cudaMemcpyAsync(&hst, als.st.p, sizeof(State), cudaMemcpyDeviceToHost, s));
      MMCSF_CUDA(cudaStreamSynchronize(s));
      if (o->profile) MMCSF_TRY(prof.collect());
      if (!hst.keep_going) break;
    }
  }
  MMCSF_CUDA(cudaEventRecord(e1, s));
  MMCSF_CUDA(cudaEventSynchronize(e1));
  float ms = 0;
  cudaEventElapsedTime(&ms, e0, e1);
  MMCSF_CUDA(cudaMemcpy(&hst, als.st.p, sizeof(State), cudaMemcpyDeviceToHost));
  MMCSF_TRY(als.finish(d_out, h_lambda));
  MMCSF_CUDA(cudaStreamSynchronize(s));
  if (res) {
    memset(res, 0, sizeof *res);
    res->iters = hst.iter;
    res->fit = hst.fit;
    res->converged = hst.converged;
    res->seconds = ms / 1e3;
    res->graph = graph_used;
    res->launches = als.launches;
    for (int p = 0; p < MMCSF_CPD_PHASES; ++p) res->phase_ms[p] = o->profile ? prof.ms[p] : 0.0;
    const int nh = std::min(hst.iter, MMCSF_CPD_MAX_HISTORY);
    if (nh > 0) MMCSF_CUDA(cudaMemcpy(res->fit_history, als.hist.p, nh * sizeof(double), cudaMemcpyDeviceToHost));
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  return MMCSF_OK;
}

}  // namespace
}  // namespace mmcsf

extern "C" int mmcsf_cpd(mmcsf_format* F, const mmcsf_cpd_opts* opts, const float* const* d_init,
                         float* const* d_factors_out, double* lambda_out, mmcsf_cpd_result* result, void* stream) {
  MMCSF_RANGE("mmcsf_cpd");
  using namespace mmcsf;
  if (!F || !opts) return set_error(MMCSF_ERR_INVALID, "null argument");
  MMCSF_TRY(bounds_gate(F, stream));
  if (F->impl != MMCSF_IMPL_MMCSF) return set_error(MMCSF_ERR_INVALID, "CP-ALS needs an MM-CSF format (-t 12)");
  const int R = opts->rank;
  if (R < 1 || R > MAXR) return set_error(MMCSF_ERR_INVALID, "CP-ALS rank must be in [1, %d]", MAXR);
  if (R != 4 && R != 8 && R != 16 && R != 32 && R != 64)
    return set_error(MMCSF_ERR_UNSUPPORTED, "CP-ALS runs ranks 4, 8, 16, 32 or 64");
  if (opts->max_iters > MMCSF_CPD_MAX_HISTORY)
    return set_error(MMCSF_ERR_INVALID, "max_iters must be <= %d", MMCSF_CPD_MAX_HISTORY);
  cudaStream_t s = S(stream);
  if (s == nullptr && opts->precision == MMCSF_CPD_BF16 && !opts->no_graph)
    return set_error(MMCSF_ERR_INVALID, "the graph form needs a non-default stream (capture)");
  if (opts->precision == MMCSF_CPD_FP32) return run_cpd<float, float>(F, opts, d_init, d_factors_out, lambda_out, result, s);
  if (opts->precision == MMCSF_CPD_BF16)
    return run_cpd<__nv_bfloat16, double>(F, opts, d_init, d_factors_out, lambda_out, result, s);
  if (opts->precision == MMCSF_CPD_FP64_SOLVE)
    return run_cpd<float, double>(F, opts, d_init, d_factors_out, lambda_out, result, s);
  return set_error(MMCSF_ERR_INVALID, "unknown CP-ALS precision %d", opts->precision);
}
