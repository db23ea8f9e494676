// COO tensor handles and .tns text I/O.
//
// The .tns reader replaces load_tensor (src/util.h:313-370): same format
// (order, mode lengths, then 1-based coordinates and a value per line), read
// once with a hand-rolled parser over the whole file instead of two passes of
// iostream extraction, split across host threads at line ends (one nonzero
// per line) and concatenated in file order, so the result is the sequential
// parse. The nonzero count is the number of complete entries parsed; the
// reference takes (#lines - 2), which differs only for files with trailing
// blank lines. A binary COO file (mmcsf_coo_write_bin / mmcsf_coo_load_bin)
// skips the text parse on later runs.
#include <algorithm>
#include <cerrno>
#include <thread>
#include <vector>
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
  MMCSF_RANGE("mmcsf_coo_create");
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
  MMCSF_RANGE("mmcsf_coo_create_device");
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
  MMCSF_RANGE("mmcsf_coo_load_tns");
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
  // entries, split into per-thread chunks that start after a newline
  struct Chunk {
    std::vector<uint32_t> inds[4];
    std::vector<float> vals;
    bool stopped = false;  // an unparsable token before the chunk's end: the file's entries end here
    uint64_t bad = 0;      // a coordinate outside its mode (1-based value), with its mode in bad_mode
    int bad_mode = -1;
  };
  const size_t body = (size_t)(e - p);
  unsigned T = std::max(1u, std::min(32u, std::thread::hardware_concurrency()));
  T = (unsigned)std::min<size_t>(T, body / (256 * 1024) + 1);
  std::vector<const char*> cut(T + 1);
  cut[0] = p;
  cut[T] = e;
  for (unsigned t = 1; t < T; ++t) {
    const char* c = std::max(cut[t - 1], p + body * t / T);
    while (c < e && *c != '\n') ++c;
    cut[t] = c < e ? c + 1 : e;
  }
  std::vector<Chunk> ch(T);
  auto work = [&](unsigned t) {
    Chunk& C = ch[t];
    const size_t guess = (size_t)(cut[t + 1] - cut[t]) / (size_t)(4 * (nd + 1)) + 16;
    for (int m = 0; m < nd; ++m) C.inds[m].reserve(guess);
    C.vals.reserve(guess);
    const char* q0 = cut[t];
    const char* ce = cut[t + 1];
    for (;;) {
      uint64_t c[4];
      const char* q = q0;
      int m = 0;
      for (; m < nd; ++m)
        if (!(q = parse_u64(q, ce, &c[m]))) break;
      float v;
      if (m < nd || !(q = parse_f32(q, ce, &v))) {
        C.stopped = skip_ws(q0, ce) < ce;
        break;
      }
      for (int k = 0; k < nd; ++k) {
        if (c[k] == 0 || c[k] > dims[k]) {
          C.bad = c[k];
          C.bad_mode = k;
          return;
        }
        C.inds[k].push_back((uint32_t)(c[k] - 1));
      }
      C.vals.push_back(v);
      q0 = q;
    }
  };
  {
    std::vector<std::thread> th;
    for (unsigned t = 1; t < T; ++t) th.emplace_back(work, t);
    work(0);
    for (auto& x : th) x.join();
  }
  uint64_t total = 0;
  unsigned used = 0;
  for (; used < T; ++used) {
    const Chunk& C = ch[used];
    if (C.bad_mode >= 0) {
      delete X;
      return set_error(MMCSF_ERR_IO, "%s: coordinate %llu of mode %d outside [1, %llu]", path,
                       (unsigned long long)C.bad, C.bad_mode, (unsigned long long)dims[C.bad_mode]);
    }
    total += C.vals.size();
    if (C.stopped) { ++used; break; }
  }
  for (int m = 0; m < nd; ++m) X->h_inds[m].reserve(total);
  X->h_vals.reserve(total);
  for (unsigned t = 0; t < used; ++t) {
    for (int m = 0; m < nd; ++m) X->h_inds[m].insert(X->h_inds[m].end(), ch[t].inds[m].begin(), ch[t].inds[m].end());
    X->h_vals.insert(X->h_vals.end(), ch[t].vals.begin(), ch[t].vals.end());
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

// Binary COO file: "MMCSFCOO", u32 version (1), u32 order, u64 nonzeros,
// u64 mode lengths[4], then the order's uint32 index arrays (0-based) and the
// float32 values, little-endian as written by this host.
namespace {
constexpr char BIN_MAGIC[8] = {'M', 'M', 'C', 'S', 'F', 'C', 'O', 'O'};
struct BinHeader {
  char magic[8];
  uint32_t version, nd;
  uint64_t nnz, dims[4];
};
}  // namespace

extern "C" int mmcsf_coo_write_bin(mmcsf_coo* X, const char* path) {
  if (!X || !path) return set_error(MMCSF_ERR_INVALID, "null argument");
  MMCSF_TRY(mmcsf_coo_to_host(X));
  FILE* f = fopen(path, "wb");
  if (!f) return set_error(MMCSF_ERR_IO, "cannot open %s", path);
  BinHeader h{};
  memcpy(h.magic, BIN_MAGIC, 8);
  h.version = 1;
  h.nd = (uint32_t)X->nd;
  h.nnz = X->nnz;
  for (int m = 0; m < X->nd; ++m) h.dims[m] = X->dims[m];
  bool ok = fwrite(&h, sizeof h, 1, f) == 1;
  for (int m = 0; m < X->nd && ok; ++m)
    ok = X->nnz == 0 || fwrite(X->h_inds[m].data(), 4, X->nnz, f) == X->nnz;
  ok = ok && (X->nnz == 0 || fwrite(X->h_vals.data(), 4, X->nnz, f) == X->nnz);
  ok = (fclose(f) == 0) && ok;
  return ok ? MMCSF_OK : set_error(MMCSF_ERR_IO, "write to %s failed", path);
}

extern "C" int mmcsf_coo_load_bin(const char* path, mmcsf_coo** out) {
  MMCSF_RANGE("mmcsf_coo_load_bin");
  if (!path || !out) return set_error(MMCSF_ERR_INVALID, "null argument");
  FILE* f = fopen(path, "rb");
  if (!f) return set_error(MMCSF_ERR_IO, "%s does not exist!", path);
  BinHeader h{};
  if (fread(&h, sizeof h, 1, f) != 1 || memcmp(h.magic, BIN_MAGIC, 8) != 0 || h.version != 1) {
    fclose(f);
    return set_error(MMCSF_ERR_IO, "%s is not a binary COO file of this library", path);
  }
  const int st0 = check_shape((int)h.nd, h.dims, h.nnz);
  if (st0 != MMCSF_OK) { fclose(f); return st0; }
  mmcsf_coo* X = new (std::nothrow) mmcsf_coo;
  if (!X) { fclose(f); return set_error(MMCSF_ERR_NOMEM, "host allocation failed"); }
  X->nd = (int)h.nd;
  X->nnz = h.nnz;
  bool ok = true;
  for (int m = 0; m < X->nd; ++m) {
    X->dims[m] = h.dims[m];
    X->h_inds[m].resize(h.nnz);
    ok = ok && (h.nnz == 0 || fread(X->h_inds[m].data(), 4, h.nnz, f) == h.nnz);
  }
  X->h_vals.resize(h.nnz);
  ok = ok && (h.nnz == 0 || fread(X->h_vals.data(), 4, h.nnz, f) == h.nnz);
  fclose(f);
  for (int m = 0; m < X->nd && ok; ++m)
    for (uint64_t x = 0; x < h.nnz; ++x)
      if (X->h_inds[m][x] >= h.dims[m]) { ok = false; break; }
  if (!ok) { delete X; return set_error(MMCSF_ERR_IO, "%s: truncated or out-of-range entries", path); }
  X->host_valid = true;
  *out = X;
  return MMCSF_OK;
}

extern "C" void mmcsf_coo_destroy(mmcsf_coo* X) { delete X; }
