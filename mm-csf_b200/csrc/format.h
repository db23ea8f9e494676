// Device-resident sparse formats (internal layout).
//
// One CSF "part" holds, for a mode order (o0, ..., o_{nd-1}):
//   3-D: ptr[0] slices->fibers [S+1], idx[0] slice index (o0) [S],
//        ptr[1] fibers->nonzeros [F+1], idx[1] fiber index (o1) [F+1, last = sentinel]
//   4-D: ptr[0] slices->fbrS [S+1], idx[0] [S],
//        ptr[1] fbrS->fibers [FS+1], idx[1] fbrS index (o1) [FS],
//        ptr[2] fibers->nonzeros [F+1], idx[2] fiber index (o2) [F+1, last = sentinel]
//   leaf[N] (index of the last mode per nonzero), vals[N],
//   fbr_like[n1]: o0 index per level-1 entry (the reference's fbrLikeSlcInds),
//   fpar[F] (4-D): fbrS id of every fiber.
// These are the reference's TiledTensor arrays (src/util.h:107-136) with
// uint32 instead of size_t entries.
#pragma once
#include <stdint.h>

#include <vector>

#include "common.h"

namespace mmcsf {

struct CsfPart {
  bool present = false;
  int nd = 0;
  int order[4] = {0, 1, 2, 3};
  uint64_t nnz = 0;
  uint64_t n[3] = {0, 0, 0};  // entries per index level: S, (3-D) F | (4-D) FS, F
  DevBuf ptr[3], idx[3];
  DevBuf leaf, vals, fbr_like, fpar;
  DevBuf coo[4];    // optional: sorted index array of every tensor mode (keep_coo)
  DevBuf bin_of;    // optional: int32 bin per slice (B-CSF / HB-CSF export)
  DevBuf from_part; // views: partition position of every view position (value reordering)
  // first leaf fiber of every chunk of (128 << i) nonzeros, i < 6: the worker
  // teams' starting points for the chunk sizes the tuner tries
  static constexpr int N_CHUNK_SIZES = 6;
  DevBuf cfib[N_CHUNK_SIZES];
  DevBuf cslc[N_CHUNK_SIZES];  // ... and its slice (3-D parts with `mid`)
  DevBuf mid;                  // o_{nd-2} of every nonzero (per-nonzero traversal), or empty
  DevBuf mid2;                 // 4-D: o1 of every nonzero
  DevBuf snz;                  // with mid: first nonzero of every slice [S+1]
  static int cfib_slot(uint64_t chunk) {
    for (int i = 0; i < N_CHUNK_SIZES; ++i)
      if (chunk == (128ull << i)) return i;
    return -1;
  }
  uint64_t bytes() const {
    uint64_t b = 0;
    for (int l = 0; l < 3; ++l) b += ptr[l].bytes + idx[l].bytes;
    for (int i = 0; i < N_CHUNK_SIZES; ++i) b += cfib[i].bytes + cslc[i].bytes;
    b += mid.bytes + mid2.bytes + snz.bytes;
    b += leaf.bytes + vals.bytes + fbr_like.bytes + fpar.bytes + bin_of.bytes + from_part.bytes;
    for (int m = 0; m < 4; ++m) b += coo[m].bytes;
    return b;
  }
  uint64_t n_slices() const { return n[0]; }
  uint64_t n_level1() const { return n[1]; }
  uint64_t n_fibers() const { return nd == 3 ? n[1] : n[2]; }
};

// HB-CSF extra parts (src/util.h:852-1142).
struct HybExtra {
  uint64_t coo_nnz = 0, csl_nnz = 0, n_csl_slices = 0;
  DevBuf coo_inds[4], coo_vals;                       // by level
  DevBuf csl_ptr, csl_idx, csl_i1, csl_i2, csl_vals;  // 3-D only
  DevBuf csl_bin_of;
};

// The MM-CSF partition heuristic (partition.cu).
int mm_partition_heuristic(int nd, const uint64_t* dims, const int (*orders)[4], const int* xorder, int redun,
                           int fbth, const uint32_t* const* sx, uint64_t n, uint8_t* part, int* rounds,
                           int* launches, cudaStream_t s);
int partition_members(const uint8_t* part, int p, const uint32_t* perm, uint64_t n, DevBuf& out, uint64_t* count,
                      int* launches, cudaStream_t s);

}  // namespace mmcsf

struct mmcsf_format {
  int impl = 0;
  int nd = 0;
  uint64_t dims[4] = {0, 0, 0, 0};
  uint64_t nnz = 0;
  int mode = 0;      // -m
  int redun = -1;    // redunMode (MM-CSF)
  int partition_rule = 0;
  int heur_rounds = 0;  // rounds the partition heuristic took (partition_rule 1)
  mmcsf::DevBuf all_vals;  // several partitions: their values concatenated (the format's nonzero order)
  int xorder[4] = {0, 1, 2, 3};
  uint64_t fbr_th = 0;
  mmcsf::CsfPart parts[4];
  mmcsf::CsfPart views[4];  // views[m]: a CSF with mode m at level 0 (order_modes(m))
  // tuned plans, one per factor type (index: MMCSF_DTYPE_F32 / _BF16)
  int plan_traversal[2][4] = {};  // 1 partitions, 2 view (0 = untuned)
  int plan_chunk[2][4] = {};
  int plan_mb[2][4] = {};
  int plan_kernel[2][4] = {};
  float plan_ms[2][4] = {};
  int pair_chunk[2] = {}, pair_mb[2] = {}, pair_kernel[2] = {};  // the two-output walk's launch shape (0: defaults)
  bool pair_use[2] = {};      // mmcsf_mttkrp_all runs the partition's two upper modes in one walk
  float pair_ms[2] = {};
  // per-mode precision (mmcsf_tune_precision): with FP32 factors, mmcsf_mttkrp_all runs mode m's kernel on
  // BF16 copies of the factors where mode_dtype[m] (or pair_dtype, for the two-output walk) says so
  bool mixed = false;
  int mode_dtype[4] = {};
  bool mixed_pair = false;  // the mixed plan runs the two-output walk
  int pair_dtype = 0;
  mmcsf::DevBuf bf16_fac[4];  // BF16 copies of the caller's factors (mixed plans)
  int fiber_threshold_tuned = -1;  // mmcsf_autotune: the -f the format was chosen with
  mmcsf::HybExtra hyb;
  int last_launches = 0;
  bool checked = false;  // bounds-checked build: mmcsf_format_check passed once
  // staging for the host-buffer MTTKRP entry point
  mmcsf::DevBuf stage_in[4], stage_out[4];
  int stage_R = 0;
  mmcsf::DevBuf vals_scratch;  // caller values reordered for a view traversal
  mmcsf::DevBuf leaf64;        // FP64 accumulation of leaf-level (per-nonzero scatter) MTTKRP outputs
  mmcsf::DevBuf ttm_side;      // TTM: per-chunk partial rows of fibers that cross chunk starts
  cudaStream_t copy_in = nullptr, copy_out = nullptr;
  cudaEvent_t ev_in[4] = {}, ev_done[4] = {}, ev_start = nullptr;
  ~mmcsf_format() {
    if (copy_in) cudaStreamDestroy(copy_in);
    if (copy_out) cudaStreamDestroy(copy_out);
    for (int m = 0; m < 4; ++m) {
      if (ev_in[m]) cudaEventDestroy(ev_in[m]);
      if (ev_done[m]) cudaEventDestroy(ev_done[m]);
    }
    if (ev_start) cudaEventDestroy(ev_start);
  }
};

namespace mmcsf {
// Bounds-checked build (-DMMCSF_BOUNDS): every compute entry point validates
// the format once (mmcsf_format_check) before its first launch on it, so no
// kernel follows an index the check has not seen. Otherwise a no-op.
inline int bounds_gate(const mmcsf_format* F, void* stream) {
#ifdef MMCSF_BOUNDS
  if (F && !F->checked) {
    const int st = mmcsf_format_check(F, nullptr, stream);
    if (st != MMCSF_OK) return st;
    const_cast<mmcsf_format*>(F)->checked = true;
  }
#else
  (void)F;
  (void)stream;
#endif
  return MMCSF_OK;
}
}  // namespace mmcsf
