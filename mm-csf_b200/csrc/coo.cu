// COO tensor handles and .tns text I/O.
//
// The .tns reader replaces load_tensor (src/util.h:313-370): same format
// (order, mode lengths, then 1-based coordinates and a value per line), read
// once with a hand-rolled parser over the whole file instead of two passes of
// iostream extraction. The nonzero count is the number of complete entries
// parsed; the reference takes (#lines - 2), which differs only for files with
// trailing blank lines.
#include <cerrno>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>

#include "common.h"

using mmcsf::set_error;

namespace {

int check_shape(int nd, const uint64_t* dims, uint64_t nnz) {
  if (nd < 3 || nd > 4)
    return set_error(MMCSF_ERR_INVALID, "Supported tensor dimension is 3 or 4 (got %d)", nd);
  for (int m = 0; m < nd; ++m)
    if (dims[m] == 0 || dims[m] >= (1ull << 32))
      return set_error(MMCSF_ERR_INVALID, "mode %d length %llu out of range [1, 2^32)", m,
                       (unsigned long long)dims[m]);
  if (nnz >= (1ull << 32) - 1)
    return set_error(MMCSF_ERR_INVALID, "nonzero count %llu out of range", (unsigned long long)nnz);
  return MMCSF_OK;
}

inline const char* skip_ws(const char* p, const char* e) {
  while (p < e && (*p == ' ' || *p == '\t' || *p == '\n' || *p == '\r')) ++p;
  return p;
}

// Parse an unsigned integer; returns nullptr if none.
inline const char* parse_u64(const char* p, const char* e, uint64_t* out) {
  p = skip_ws(p, e);
  if (p >= e || *p < '0' || *p > '9') return nullptr;
  uint64_t v = 0;
  while (p < e && *p >= '0' && *p <= '9') v = v * 10 + (uint64_t)(*p++ - '0');
  *out = v;
  return p;
}

// Parse a float token with strtof semantics (the reference uses
// `ifstream >> float`, i.e. the same decimal-to-float rounding).
inline const char* parse_f32(const char* p, const char* e, float* out) {
  p = skip_ws(p, e);
  if (p >= e) return nullptr;
  char buf[64];
  int n = 0;
  while (p < e && n < 63 && !(*p == ' ' || *p == '\t' || *p == '\n' || *p == '\r')) buf[n++] = *p++;
  buf[n] = 0;
  char* end = nullptr;
  *out = strtof(buf, &end);
  if (end == buf) return nullptr;
  return p;
}

}  // namespace

extern "C" int mmcsf_coo_create(int nd, const uint64_t* dims, uint64_t nnz, const uint32_t* const* inds,
                                const float* vals, mmcsf_coo** out) {
  if (!out || !dims || (nnz && (!inds || !vals))) return set_error(MMCSF_ERR_INVALID, "null argument");
  MMCSF_TRY(check_shape(nd, dims, nnz));
  mmcsf_coo* X = new (std::nothrow) mmcsf_coo;
  if (!X) return set_error(MMCSF_ERR_NOMEM, "host allocation failed");
  X->nd = nd;
  X->nnz = nnz;
  for (int m = 0; m < nd; ++m) {
    X->dims[m] = dims[m];
    X->h_inds[m].assign(inds ? inds[m] : nullptr, inds ? inds[m] + nnz : nullptr);
    for (uint64_t x = 0; x < nnz; ++x)
      if (X->h_inds[m][x] >= dims[m]) {
        delete X;
        return set_error(MMCSF_ERR_INVALID, "index %u of mode %d at nonzero %llu exceeds length %llu",
                         inds[m][x], m, (unsigned long long)x, (unsigned long long)dims[m]);
      }
  }
  X->h_vals.assign(vals ? vals : nullptr, vals ? vals + nnz : nullptr);
  X->host_valid = true;
  *out = X;
  return MMCSF_OK;
}

extern "C" int mmcsf_coo_create_device(int nd, const uint64_t* dims, uint64_t nnz, const uint32_t* const* d_inds,
                                       const float* d_vals, void* stream, mmcsf_coo** out) {
  if (!out || !dims || (nnz && (!d_inds || !d_vals))) return set_error(MMCSF_ERR_INVALID, "null argument");
  MMCSF_TRY(check_shape(nd, dims, nnz));
  mmcsf_coo* X = new (std::nothrow) mmcsf_coo;
  if (!X) return set_error(MMCSF_ERR_NOMEM, "host allocation failed");
  X->nd = nd;
  X->nnz = nnz;
  for (int m = 0; m < nd; ++m) X->dims[m] = dims[m];
  for (int m = 0; m < nd; ++m) {
    if (X->d_inds[m].alloc(nnz * 4) != cudaSuccess) { delete X; return set_error(MMCSF_ERR_NOMEM, "cudaMalloc"); }
    if (nnz && cudaMemcpyAsync(X->d_inds[m].p, d_inds[m], nnz * 4, cudaMemcpyDeviceToDevice, mmcsf::S(stream)) != cudaSuccess) {
      delete X;
      return set_error(MMCSF_ERR_CUDA, "device copy failed");
    }
  }
  if (X->d_vals.alloc(nnz * 4) != cudaSuccess) { delete X; return set_error(MMCSF_ERR_NOMEM, "cudaMalloc"); }
  if (nnz && cudaMemcpyAsync(X->d_vals.p, d_vals, nnz * 4, cudaMemcpyDeviceToDevice, mmcsf::S(stream)) != cudaSuccess) {
    delete X;
    return set_error(MMCSF_ERR_CUDA, "device copy failed");
  }
  X->dev_valid = true;
  *out = X;
  return MMCSF_OK;
}

extern "C" int mmcsf_coo_load_tns(const char* path, mmcsf_coo** out) {
  if (!path || !out) return set_error(MMCSF_ERR_INVALID, "null argument");
  FILE* f = fopen(path, "rb");
  if (!f) return set_error(MMCSF_ERR_IO, "%s does not exist!", path);
  fseek(f, 0, SEEK_END);
  long sz = ftell(f);
  fseek(f, 0, SEEK_SET);
  std::vector<char> buf((size_t)(sz > 0 ? sz : 0) + 1);
  size_t got = sz > 0 ? fread(buf.data(), 1, (size_t)sz, f) : 0;
  fclose(f);
  const char* p = buf.data();
  const char* e = p + got;
  uint64_t nd64 = 0;
  if (!(p = parse_u64(p, e, &nd64))) return set_error(MMCSF_ERR_IO, "%s: missing tensor order", path);
  int nd = (int)nd64;
  if (nd < 3 || nd > 4) return set_error(MMCSF_ERR_INVALID, "Supported tensor dimension is 3 or 4 (got %d)", nd);
  uint64_t dims[4] = {0, 0, 0, 0};
  for (int m = 0; m < nd; ++m)
    if (!(p = parse_u64(p, e, &dims[m]))) return set_error(MMCSF_ERR_IO, "%s: missing mode lengths", path);
  mmcsf_coo* X = new (std::nothrow) mmcsf_coo;
  if (!X) return set_error(MMCSF_ERR_NOMEM, "host allocation failed");
  X->nd = nd;
  for (int m = 0; m < nd; ++m) X->dims[m] = dims[m];
  // rough capacity guess: ~4 bytes per token
  size_t guess = got / (size_t)(4 * (nd + 1)) + 16;
  for (int m = 0; m < nd; ++m) X->h_inds[m].reserve(guess);
  X->h_vals.reserve(guess);
  for (;;) {
    uint64_t c[4];
    const char* q = p;
    int m = 0;
    for (; m < nd; ++m)
      if (!(q = parse_u64(q, e, &c[m]))) break;
    if (m < nd) break;
    float v;
    if (!(q = parse_f32(q, e, &v))) break;
    for (int k = 0; k < nd; ++k) {
      if (c[k] == 0 || c[k] > dims[k]) {
        delete X;
        return set_error(MMCSF_ERR_IO, "%s: coordinate %llu of mode %d outside [1, %llu]", path,
                         (unsigned long long)c[k], k, (unsigned long long)dims[k]);
      }
      X->h_inds[k].push_back((uint32_t)(c[k] - 1));
    }
    X->h_vals.push_back(v);
    p = q;
  }
  X->nnz = X->h_vals.size();
  int st = check_shape(nd, dims, X->nnz);
  if (st != MMCSF_OK) { delete X; return st; }
  X->host_valid = true;
  *out = X;
  return MMCSF_OK;
}

extern "C" int mmcsf_coo_info(const mmcsf_coo* X, int* nd, uint64_t* dims, uint64_t* nnz) {
  if (!X) return set_error(MMCSF_ERR_INVALID, "null tensor");
  if (nd) *nd = X->nd;
  if (dims)
    for (int m = 0; m < X->nd; ++m) dims[m] = X->dims[m];
  if (nnz) *nnz = X->nnz;
  return MMCSF_OK;
}

extern "C" int mmcsf_coo_to_host(mmcsf_coo* X) {
  if (!X) return set_error(MMCSF_ERR_INVALID, "null tensor");
  if (X->host_valid) return MMCSF_OK;
  if (!X->dev_valid) return set_error(MMCSF_ERR_INVALID, "tensor has no data");
  MMCSF_CUDA(cudaDeviceSynchronize());
  for (int m = 0; m < X->nd; ++m) {
    X->h_inds[m].resize(X->nnz);
    if (X->nnz) MMCSF_CUDA(cudaMemcpy(X->h_inds[m].data(), X->d_inds[m].p, X->nnz * 4, cudaMemcpyDeviceToHost));
  }
  X->h_vals.resize(X->nnz);
  if (X->nnz) MMCSF_CUDA(cudaMemcpy(X->h_vals.data(), X->d_vals.p, X->nnz * 4, cudaMemcpyDeviceToHost));
  X->host_valid = true;
  return MMCSF_OK;
}

extern "C" int mmcsf_coo_to_device(mmcsf_coo* X, void* stream) {
  if (!X) return set_error(MMCSF_ERR_INVALID, "null tensor");
  if (X->dev_valid) return MMCSF_OK;
  for (int m = 0; m < X->nd; ++m) {
    MMCSF_CUDA(X->d_inds[m].alloc(X->nnz * 4));
    if (X->nnz)
      MMCSF_CUDA(cudaMemcpyAsync(X->d_inds[m].p, X->h_inds[m].data(), X->nnz * 4, cudaMemcpyHostToDevice,
                                 mmcsf::S(stream)));
  }
  MMCSF_CUDA(X->d_vals.alloc(X->nnz * 4));
  if (X->nnz)
    MMCSF_CUDA(cudaMemcpyAsync(X->d_vals.p, X->h_vals.data(), X->nnz * 4, cudaMemcpyHostToDevice, mmcsf::S(stream)));
  MMCSF_CUDA(cudaStreamSynchronize(mmcsf::S(stream)));
  X->dev_valid = true;
  return MMCSF_OK;
}

extern "C" int mmcsf_coo_host_arrays(const mmcsf_coo* X, const uint32_t** inds, const float** vals) {
  if (!X || !inds || !vals) return set_error(MMCSF_ERR_INVALID, "null argument");
  for (int m = 0; m < X->nd; ++m) inds[m] = X->host_valid ? X->h_inds[m].data() : nullptr;
  *vals = X->host_valid ? X->h_vals.data() : nullptr;
  return MMCSF_OK;
}

extern "C" int mmcsf_coo_device_arrays(const mmcsf_coo* X, const uint32_t** d_inds, const float** d_vals) {
  if (!X || !d_inds || !d_vals) return set_error(MMCSF_ERR_INVALID, "null argument");
  for (int m = 0; m < X->nd; ++m) d_inds[m] = X->dev_valid ? X->d_inds[m].as<uint32_t>() : nullptr;
  *d_vals = X->dev_valid ? X->d_vals.as<float>() : nullptr;
  return MMCSF_OK;
}

extern "C" int mmcsf_coo_write_tns(mmcsf_coo* X, const char* path) {
  if (!X || !path) return set_error(MMCSF_ERR_INVALID, "null argument");
  MMCSF_TRY(mmcsf_coo_to_host(X));
  FILE* f = fopen(path, "w");
  if (!f) return set_error(MMCSF_ERR_IO, "cannot open %s", path);
  fprintf(f, "%d\n", X->nd);
  for (int m = 0; m < X->nd; ++m) fprintf(f, m ? " %llu" : "%llu", (unsigned long long)X->dims[m]);
  fprintf(f, "\n");
  for (uint64_t x = 0; x < X->nnz; ++x) {
    for (int m = 0; m < X->nd; ++m) fprintf(f, "%u ", X->h_inds[m][x] + 1);
    fprintf(f, "%.9g\n", (double)X->h_vals[x]);
  }
  fclose(f);
  return MMCSF_OK;
}

extern "C" void mmcsf_coo_destroy(mmcsf_coo* X) { delete X; }
