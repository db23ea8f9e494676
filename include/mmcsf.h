/*
 * mmcsf.h — C ABI of the B200-native MM-CSF sparse MTTKRP library.
 *
 * Plain C types only (pointers, sizes, integers); CUDA streams are passed as
 * `void*` (a cudaStream_t, NULL = the legacy default stream). Every call
 * returns an mmcsf_status and never exits or asserts; mmcsf_last_error()
 * gives a message for the last failure on the calling thread.
 *
 * Each declaration names the reference (isratnisa/MM-CSF) interface it
 * replaces. The reference has no plugin layer; its boundary is the C++
 * function API in src/mttkrp_gpu.h:59-81 plus the builders in src/util.h.
 *
 * Threads and streams: different tensors and formats are independent. A
 * format keeps small per-format state between calls (its tuned plan, staging
 * buffers of the host-buffer MTTKRP, reordered values for the adjoint, TTM's
 * side rows, the launch count), so calls on ONE format must not overlap from
 * several host threads, nor run on several streams at once; serialise them.
 *
 * Index limits: the nonzero count must be below 2^32 and, to build a format,
 * every mode length below 2^31 (indices are stored as uint32 on the device,
 * the leaf index carrying a fiber-start flag in bit 31; the reference uses
 * size_t).
 */
#ifndef MMCSF_H
#define MMCSF_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status ------------------------------------------------------------ */
typedef enum {
  MMCSF_OK = 0,
  MMCSF_ERR_INVALID = 1,     /* bad argument; the reference prints and exit(0)s (src/util.h:238-248) */
  MMCSF_ERR_CUDA = 2,        /* a CUDA call failed; the reference asserts (src/mttkrp_gpu.cu:60-67) */
  MMCSF_ERR_NOMEM = 3,       /* host or device allocation failed */
  MMCSF_ERR_IO = 4,          /* file missing or malformed; the reference exit(0)s (src/util.h:327-330) */
  MMCSF_ERR_UNSUPPORTED = 5, /* valid request this build does not implement */
  MMCSF_ERR_TIMEOUT = 6      /* a bounded device-side wait gave up */
} mmcsf_status;

/* Text for a status code. */
const char* mmcsf_status_string(int status);
/* Message for the last failure on this thread ("" if none). */
const char* mmcsf_last_error(void);
/* Library version as 10000*major + 100*minor + patch. */
int mmcsf_version(void);

/* ---- implementation types: the reference's -t values (src/mttkrp.cu) --- */
#define MMCSF_IMPL_COO_CPU 1 /* -t 1: COO MTTKRP on the host (mmcsf_mttkrp_coo_host) */
#define MMCSF_IMPL_BCSF 8    /* -t 8: B-CSF, single mode */
#define MMCSF_IMPL_HBCSF 10  /* -t 10: HB-CSF, single mode */
#define MMCSF_IMPL_MMCSF 12  /* -t 12: MM-CSF, all modes from one partitioned format */

/* Factor element types for MTTKRP inputs (outputs are always float32). */
#define MMCSF_DTYPE_F32 0
#define MMCSF_DTYPE_BF16 1

/* ---- COO tensors --------------------------------------------------------
 * Replaces Tensor + load_tensor (src/util.h:80-104, 313-370). A COO handle
 * holds 0-based uint32 indices per mode and float32 values, on the host, on
 * the device, or both. */
typedef struct mmcsf_coo mmcsf_coo;

/* Parse a .tns file (line 1: order; line 2: mode lengths; then 1-based
 * coordinates and a value per line). Replaces load_tensor
 * (src/util.h:313-370); the nonzero count is the number of parsed entries. */
int mmcsf_coo_load_tns(const char* path, mmcsf_coo** out);
/* Copy caller host arrays into a new handle (inds[m][x] 0-based). */
int mmcsf_coo_create(int nd, const uint64_t* dims, uint64_t nnz, const uint32_t* const* inds,
                     const float* vals, mmcsf_coo** out);
/* Wrap-copy caller DEVICE arrays into a new handle (stream-ordered copy). */
int mmcsf_coo_create_device(int nd, const uint64_t* dims, uint64_t nnz, const uint32_t* const* d_inds,
                            const float* d_vals, void* stream, mmcsf_coo** out);
int mmcsf_coo_info(const mmcsf_coo* X, int* nd, uint64_t* dims, uint64_t* nnz);
/* Make sure the host (resp. device) copy exists; synchronous. */
int mmcsf_coo_to_host(mmcsf_coo* X);
int mmcsf_coo_to_device(mmcsf_coo* X, void* stream);
/* Borrow array pointers (host or device copy; NULL if absent). inds must
 * have room for nd pointers. */
int mmcsf_coo_host_arrays(const mmcsf_coo* X, const uint32_t** inds, const float** vals);
int mmcsf_coo_device_arrays(const mmcsf_coo* X, const uint32_t** d_inds, const float** d_vals);
/* Write as .tns (1-based). */
int mmcsf_coo_write_tns(mmcsf_coo* X, const char* path);
/* Binary COO file (no counterpart in the reference): the same tensor without
 * the text parse, for loading large tensors repeatedly. Written and read on
 * hosts of the same byte order. */
int mmcsf_coo_write_bin(mmcsf_coo* X, const char* path);
int mmcsf_coo_load_bin(const char* path, mmcsf_coo** out);
void mmcsf_coo_destroy(mmcsf_coo* X);

/* ---- synthetic tensors --------------------------------------------------
 * Seeded generator for the benchmark shapes (no counterpart in the
 * reference, whose tools/generate_tensor.py writes .tns text). Coordinates
 * per mode are uniform or Zipf(s) mapped through a seeded permutation;
 * duplicates are dropped keeping the first occurrence, and new candidates are
 * drawn until `nnz` distinct coordinates exist. Runs on the device. */
#define MMCSF_DIST_UNIFORM 0
#define MMCSF_DIST_ZIPF 1
#define MMCSF_VAL_UNIFORM01 0 /* uniform in (0, 1] */
#define MMCSF_VAL_LOGNORMAL 1 /* lognormal(0, 1) */
#define MMCSF_VAL_INT1_50 2   /* integer counts 1..50 stored as float */
typedef struct {
  int nd;
  uint64_t dims[4];
  uint64_t nnz;
  int dist[4];        /* MMCSF_DIST_* per mode */
  double zipf_s[4];   /* exponent for Zipf modes */
  int val_dist;       /* MMCSF_VAL_* */
  uint64_t seed;
  int planted_rank;   /* > 0: values from a planted CP model sum_r prod_m A_m[i_m, r] with A_m uniform
                         in [0,1) (seeded), replacing val_dist */
  double noise;       /* planted: add N(0, (noise * RMS of the model values)^2) */
  int poisson;        /* planted: replace each value by a Poisson draw with that mean (counts, >= 1) */
} mmcsf_gen_spec;
int mmcsf_generate(const mmcsf_gen_spec* spec, void* stream, mmcsf_coo** out);

/* ---- formats ------------------------------------------------------------
 * Replaces the host-side builders the reference's main runs before a GPU
 * call: sort_COOtensor, create_HCSR, mm_partition_reuseBased,
 * populate_paritions, sort_MI_CSF, create_TiledHCSR, create_fbrLikeSlcInds,
 * make_TiledBin, create_HYB, make_HybBin (src/util.h:389-2526,
 * src/mttkrp.cu:72-389). Built on the device with radix-sort and scan
 * kernels; every index array is bit-exact to the reference's (with its sort
 * made stable). */
typedef struct {
  int impl;                 /* MMCSF_IMPL_MMCSF, _BCSF or _HBCSF (-t) */
  int mode;                 /* -m: drives the first sort; the computed mode for B-CSF/HB-CSF */
  uint64_t fiber_threshold; /* -f: max nonzeros per fiber; 0 = the reference default (99999999) */
  int partition_rule;       /* 0: the reference as shipped (all nonzeros to partition 2, src/util.h:2517);
                               1: the partition heuristic above that line decides (mm_partition_reuseBased,
                               src/util.h:2167-2516, nonzeros visited in order), each partition sorted and
                               built as sort_MI_CSF / create_TiledHCSR do */
  int keep_coo;             /* 1: keep every mode's sorted index array on the device for export */
  int views;                /* slice-major views for MTTKRP (no counterpart in the reference):
                               0 none, 1 = modes at the leaf level of the MM-CSF partition, 2 = every mode */
  int partition_ratio;      /* -h (Opt.MIfbTh): a mode wins a nonzero when its fiber is at least this many
                               times the others' (0 = the reference default 1); partition_rule 1 only */
  int view_order;           /* mode order of the views (no counterpart in the reference): 0 the reference's
                               order for a mode-m CSF (the rest by ascending length), 1 the rest by descending
                               length, so the shortest mode (the smallest factor) sits at the leaf level */
} mmcsf_build_opts;

typedef struct mmcsf_format mmcsf_format;
int mmcsf_build(mmcsf_coo* X, const mmcsf_build_opts* opts, void* stream, mmcsf_format** out);
void mmcsf_format_destroy(mmcsf_format* F);

/* Per-partition summary (the numbers the reference prints at
 * src/mttkrp_gpu.cu:3757-3767). part: 0..nd-1 for MM-CSF (a partition per
 * mode), 0 for B-CSF, 0 = CSF part / 1 = COO part / 2 = CSL part for HB-CSF;
 * 4 + m = the slice-major view of mode m (MM-CSF built with views). */
typedef struct {
  int present;
  int nd;
  int mode_order[4];
  uint64_t nnz;
  uint64_t n_slices;  /* level-0 entries */
  uint64_t n_fbrs;    /* level-1 entries (4-D: fbrS) */
  uint64_t n_fibers;  /* leaf-fiber entries (3-D: = n_fbrs) */
  uint64_t device_bytes;
} mmcsf_part_info;
int mmcsf_format_info(const mmcsf_format* F, int part, mmcsf_part_info* info);
/* Reference-side scalars: redunMode (-1 if none) and X's mode order. */
int mmcsf_format_meta(const mmcsf_format* F, int* redun_mode, int* x_mode_order);
/* partition_rule of the build, and the rounds the partition heuristic took
 * to settle (0 for partition_rule 0; no counterpart in the reference). */
int mmcsf_format_partitioning(const mmcsf_format* F, int* partition_rule, int* rounds);

/* Copy one array to host, named as the reference names it (widened to
 * uint64): "fbrPtr<l>", "fbrIdx<l>", "fbrLikeSlcInds", "inds<m>" (needs
 * keep_coo; m = tensor mode), "indsLeaf", "bin<b>" (B-CSF/HB-CSF), and for
 * HB-CSF parts 1/2 "COOinds<l>", "CSLslicePtr", "CSLsliceIdx", "CSLinds<l>",
 * "cslbin<b>". Pass dst=NULL to query the count. Values: "vals", "COOvals",
 * "CSLvals" through mmcsf_format_export_f32. */
int mmcsf_format_export(const mmcsf_format* F, int part, const char* name, uint64_t* dst, uint64_t cap,
                        uint64_t* count);
int mmcsf_format_export_f32(const mmcsf_format* F, int part, const char* name, float* dst, uint64_t cap,
                            uint64_t* count);

/* Format check (no counterpart in the reference, which trusts its builders):
 * validates on the device every index the MTTKRP kernels dereference, for
 * every part (partitions, views, HB-CSF COO/CSL/CSF parts): index arrays
 * below rows[m] (the row count of mode m's factor; NULL = the tensor's dims),
 * pointer arrays starting at 0, strictly increasing and ending at the next
 * level's count, the leaf fiber flags at exactly the fiber starts, the
 * per-nonzero middle indices, the slice starts and the chunk-start tables.
 * Reads are bounded by the allocations, so a corrupt array is reported, not
 * followed. MMCSF_ERR_INVALID names the array and the first bad position.
 * Synchronises `stream`. A library built with -DMMCSF_BOUNDS (make
 * lib/libmmcsf_bounds.so) runs it once per format before the first launch of
 * every compute entry point. */
int mmcsf_format_check(const mmcsf_format* F, const uint64_t* rows, void* stream);

/* ---- MTTKRP -------------------------------------------------------------
 * Replaces MTTKRP_MIHCSR_GPU (src/mttkrp_gpu.cu:3380-3784), MTTKRP_B_HCSR_GPU
 * (:1850-2129) and MTTKRP_HYB_GPU (:2530-2851). Factor matrices are
 * row-major dims[m] x R on the device; out (dims[mode] x R float32) is
 * overwritten with X_(mode) (Khatri-Rao of the other factors). Correct for
 * any R >= 1 (the reference's kernels are only correct for R <= 32).
 * Stream-ordered; nothing is synchronised. */
typedef struct {
  int chunk;         /* nonzeros per worker team; 0 = auto (the tuned plan, else 512) */
  int block_threads; /* threads per CTA; 0 = auto (256) */
  int traversal;     /* 0 auto (tuned plan, else a view when one exists), 1 MM-CSF partitions, 2 view */
  int min_blocks;    /* occupancy level: 0 auto; 1..4 = more resident warps per SM at the higher
                        levels, fewer rows in flight per warp */
  int kernel;        /* 0 auto (tuned plan, else 2 for 3-D and 1 for 4-D); 1 per-team fiber walk;
                        2 branch-free fiber walk (3-D; 4-D runs 1); 3 per-nonzero walk (every 3-D
                        level; 4-D slice and leaf levels; the 4-D middle levels run 1); 4 per-nonzero
                        walk gathering the middle row once per fiber (3-D slice level; elsewhere 3);
                        5 per-nonzero walk with 16-byte index/value loads (3-D, R >= 16, chunk % 4 == 0;
                        elsewhere 3); 6 per-nonzero walk with the teams of a warp interleaved over one
                        range, each team loading its own 16-byte index/value vectors (3-D slice level,
                        chunk % 4 == 0; elsewhere 5); 7 per-nonzero walk with the factor rows staged in
                        shared memory several steps ahead of their use and the middle row once per fiber
                        (3-D slice level, R 16..128; elsewhere 6; its grid is one block per SM and its teams
                        split the nonzeros evenly, so chunk is not used; min_blocks 1..4 picks steps of 4, 4, 8,
                        8 nonzeros per team with 2, 3, 2, 3 stages in flight) */
  int reserved[3];
} mmcsf_kernel_cfg;

/* One mode. factor_dtype: MMCSF_DTYPE_F32 (d_factors are float*) or
 * MMCSF_DTYPE_BF16 (d_factors are __nv_bfloat16*, FP32 accumulation). For
 * B-CSF/HB-CSF formats only the built mode is available. */
int mmcsf_mttkrp(const mmcsf_format* F, int mode, int R, int factor_dtype, const void* const* d_factors,
                 float* d_out, const mmcsf_kernel_cfg* cfg, void* stream);
/* -t 1: COO MTTKRP on the HOST, on the tensor's host copy. Replaces
 * MTTKRP_COO_CPU / MTTKRP_COO_CPU_4D (src/mttkrp_cpu.cpp:60-113): with the
 * cyclic mode order (mode, mode+1, ...) mod nd, h_out[i0, r] +=
 * ((v * U1[i1, r]) * U2[i2, r]) [* U3[i3, r]] in FP32. Like the reference it
 * ADDS to h_out (dims[mode] x R, row-major) without zeroing it. h_factors[m]
 * (m != mode) are host dims[m] x R float32. threads: 1 runs the reference's
 * loop in nonzero order (bit-exact to it); T > 1 splits the nonzeros into T
 * contiguous ranges with private outputs added in range order; 0 = every
 * hardware thread. Synchronous; touches no device. */
int mmcsf_mttkrp_coo_host(const mmcsf_coo* X, int mode, int R, const float* const* h_factors, float* h_out,
                          int threads);
/* Two modes in one walk (no counterpart in the reference; MM-CSF's reuse of a
 * partition across modes): on a 3-D or 4-D MM-CSF format, the MTTKRP of the
 * partition's slice mode (modes[0], into d_out_slice) and of its middle mode
 * (modes[1], into d_out_mid) from one traversal that gathers each nonzero's
 * factor rows once. cfg->kernel 2 runs the branch-free fiber walk (the middle
 * row gathered once per fiber), 3 the per-nonzero form, 4 the per-nonzero form
 * with the middle row gathered once per fiber (3-D), 5 the per-nonzero form
 * with 16-byte index loads (3-D, R >= 16), 6 the warp-interleaved per-nonzero
 * form (3-D), 7 the form with the rows staged in shared memory (3-D, R 16..128;
 * 0: the tuned choice);
 * chunk and min_blocks as for mmcsf_mttkrp. With null outputs only `modes` is
 * filled. R in 4..128 (powers of two). */
int mmcsf_mttkrp_pair(const mmcsf_format* F, int R, int factor_dtype, const void* const* d_factors,
                      float* d_out_slice, float* d_out_mid, int* modes, const mmcsf_kernel_cfg* cfg, void* stream);
/* All modes, each from the same input factors: d_outs[m] gets mode m. When
 * the tuned plan says so (and cfg overrides neither traversal nor kernel), the
 * partition's two upper modes run in one walk (mmcsf_mttkrp_pair).
 * (The reference's all-mode loop, src/mttkrp_gpu.cu:3548-3724.) */
int mmcsf_mttkrp_all(const mmcsf_format* F, int R, int factor_dtype, const void* const* d_factors,
                     float* const* d_outs, const mmcsf_kernel_cfg* cfg, void* stream);
/* All modes through HOST buffers: copies the factors host->device, runs
 * every mode, copies every output device->host and synchronises the stream.
 * The end-to-end form of MTTKRP_MIHCSR_GPU, which takes host Matrix objects.
 * Device staging buffers are kept by the format between calls. */
int mmcsf_mttkrp_all_host(mmcsf_format* F, int R, const float* const* h_factors, float* const* h_outs,
                          const mmcsf_kernel_cfg* cfg, void* stream);

/* Autotuner (no counterpart in the reference, whose -w/-f are set by hand):
 * times every traversal (MM-CSF partitions, the mode's view when built) and
 * worker-team size for each mode with the caller's factors, keeps the fastest
 * as the format's plan (used when mmcsf_kernel_cfg leaves chunk/traversal 0)
 * and reports it. d_outs are used as scratch outputs. */
typedef struct {
  int traversal[4]; /* 1 MM-CSF partitions, 2 view */
  int chunk[4];
  int min_blocks[4];
  int kernel[4];    /* mmcsf_kernel_cfg.kernel */
  float ms[4];      /* best time per mode */
  int pair;         /* 1: mmcsf_mttkrp_all runs the partition's two upper modes in one walk (mmcsf_mttkrp_pair) */
  int pair_chunk, pair_min_blocks;
  int pair_kernel;  /* 2: branch-free fiber walk with both outputs; 3 (or 0): per-nonzero form; 4: per-nonzero
                       form with the middle row once per fiber; 5: per-nonzero form with 16-byte index loads;
                       6: warp-interleaved per-nonzero form; 7: per-nonzero form with the rows staged in
                       shared memory */
  float pair_ms;    /* best time of that walk (both modes) */
  int factor_dtype; /* MMCSF_DTYPE_* of the factors the plan is for (mmcsf_set_plan files the entries under it) */
  /* per-mode precision (mmcsf_tune_precision): with FP32 factors, mmcsf_mttkrp_all runs each launch at the
   * type chosen here, converting the factors to BF16 once per call when any launch reads BF16 */
  int mixed;         /* 1: mode_dtype / pair_dtype apply (the per-mode entries above are those of the chosen type) */
  int mode_dtype[4];
  int pair_dtype;
  float bf16_error[4]; /* relative Frobenius difference of the mode's output with BF16-rounded factors against
                          its output with the FP32 factors */
  float ms_f32[4], ms_bf16[4]; /* best single-mode time per type */
  float pair_ms_f32, pair_ms_bf16;
  float convert_ms;    /* the once-per-call FP32 -> BF16 conversion of all factors */
  int fiber_threshold; /* -f of the format (mmcsf_autotune: the threshold it chose; 0: no split) */
} mmcsf_plan;
int mmcsf_tune(mmcsf_format* F, int R, int factor_dtype, const void* const* d_factors, float* const* d_outs,
               void* stream, mmcsf_plan* plan);
int mmcsf_set_plan(mmcsf_format* F, const mmcsf_plan* plan);
/* Per-mode precision (no counterpart in the reference): tunes the format for
 * FP32 factors and for BF16 copies of them (the plain tuner, twice), measures
 * for every mode the relative Frobenius difference its BF16-factor output
 * makes against its FP32-factor output, and picks for every launch of the
 * all-mode step (each mode, and the two-output walk) the faster type whose
 * error is within error_budget; BF16 is dropped where it does not pay for
 * the conversion. mmcsf_mttkrp_all with FP32 factors then follows the plan.
 * error_budget 0 keeps every launch FP32. */
int mmcsf_tune_precision(mmcsf_format* F, int R, const float* const* d_factors, float* const* d_outs,
                         double error_budget, void* stream, mmcsf_plan* plan);
/* Autotuner over the fiber-split threshold (the reference's -f, set by hand
 * there): builds the format of `base` for every threshold in f_candidates
 * (0 = no split), tunes each (mmcsf_tune_precision with error_budget), and
 * returns the one whose tuned all-mode step is fastest, its plan (with
 * fiber_threshold) in *plan. The formats not chosen are freed. */
int mmcsf_autotune(mmcsf_coo* X, const mmcsf_build_opts* base, const uint64_t* f_candidates, int n_candidates,
                   int R, const float* const* d_factors, float* const* d_outs, double error_budget, void* stream,
                   mmcsf_format** out, mmcsf_plan* plan);

/* Row-gather probe (measurement; no counterpart in the reference): average
 * milliseconds over `reps` launches of a kernel that only gathers and sums
 * the rows d_rows[d_idx[x]] (R floats each, R in 16..128) for x < n, with the
 * MTTKRP kernels' team layout. The ceiling for their per-nonzero gathers on
 * the same index stream. Every index must be below nrows. */
int mmcsf_probe_gather(const uint32_t* d_idx, uint64_t n, const float* d_rows, uint64_t nrows, int R, int reps,
                       float* ms_out, void* stream);
/* The same gather with the rows landed in shared memory by the copy engine
 * (measurement; no counterpart in the reference): one bulk copy
 * (cp.async.bulk) per row into a per-warp ring of `stages` x 32 rows, one
 * mbarrier per stage, one block of `warps` warps per SM. R 16, 32 or 64;
 * stages 2, 4 or 8. Returns MMCSF_ERR_TIMEOUT if a bounded wait gave up. */
int mmcsf_probe_gather_tma(const uint32_t* d_idx, uint64_t n, const float* d_rows, uint64_t nrows, int R,
                           int stages, int warps, int reps, float* ms_out, void* stream);

/* ---- TTM ------------------------------------------------------------------
 * Replaces TTM_GPU / TTM_CPU (src/ttm_gpu.cu:83-143, src/ttm_cpu.cpp:60-86):
 * on a 3-D B-CSF format built for mode m (-t 8, -m m, -f as given), for every
 * leaf fiber f of its CSF, in the format's fiber order,
 *   d_Y[f, :] = sum over the fiber's nonzeros of val * d_factor[leaf index, :]
 * (d_factor: the leaf mode's factor, dims[leaf] x R; d_Y: n_fibers x R FP32,
 * overwritten; the reference's semi-sparse Y without its unused sentinel row).
 * The fibers' coordinates are mmcsf_format_export(F, 0, "fbrIdx0/1",
 * "fbrPtr0"). With d_factor and d_Y NULL only *n_fibers is returned.
 * R in {4, 8, ..., 128}. */
int mmcsf_ttm(const mmcsf_format* F, int R, int factor_dtype, const void* d_factor, float* d_Y, uint64_t* n_fibers,
              void* stream);

/* ---- sampled model and its adjoint (gradient-based CP) -------------------
 * No counterpart in the reference. The sampled CP model at every nonzero,
 * xhat[x] = sum_r lambda_r prod_m A_m[i_m(x), r] (d_lambda may be NULL for
 * all ones), written in the format's nonzero order. */
int mmcsf_sampled_model(const mmcsf_format* F, int R, int factor_dtype, const void* const* d_factors,
                        const float* d_lambda, float* d_out, void* stream);
/* Adjoint of mmcsf_sampled_model with respect to factor `mode`:
 * d_out[i, r] = lambda_r * sum over nonzeros x with i_mode(x) = i of
 * d_grad[x] * prod_{m != mode} A_m[i_m(x), r], i.e. an MTTKRP of the tensor
 * with F's sparsity and the values d_grad (one per nonzero, in the format's
 * nonzero order) in place of its own, columns scaled by lambda (d_lambda NULL:
 * unscaled, a plain MTTKRP on other values). d_out: dims[mode] x R FP32,
 * overwritten. Not available for HB-CSF formats. No counterpart in the
 * reference. */
int mmcsf_cp_adjoint(const mmcsf_format* F, int mode, int R, int factor_dtype, const void* const* d_factors,
                     const float* d_lambda, const float* d_grad, float* d_out, const mmcsf_kernel_cfg* cfg,
                     void* stream);
/* Fused Poisson step for gradient CP on a 3-D format (no counterpart in the
 * reference): one pass that computes, for every nonzero x (format order),
 * w[x] = y[x] / (xhat[x] + eps) with xhat the CP model (no lambda) and y the
 * tensor's values, loss = sum_x y[x] log(xhat[x] + eps) (one device double),
 * and the gradient of that loss with respect to the factor of the format's
 * slice mode (*root_mode = that mode), d_grad_root: dims[root] x R FP32. The
 * gradients of the other factors are mmcsf_cp_adjoint with d_grad = d_w.
 * Overwrites d_grad_root and d_loss. R in {4, 8, 16, 32, 64}. */
int mmcsf_poisson_step(const mmcsf_format* F, int R, int factor_dtype, const void* const* d_factors, float eps,
                       float* d_w, float* d_grad_root, double* d_loss, int* root_mode, void* stream);
/* Device pointer to F's values in its nonzero order, and their count. */
int mmcsf_format_values(const mmcsf_format* F, const float** d_vals, uint64_t* nnz);

/* ---- CP-ALS ---------------------------------------------------------------
 * Replaces cpd() (src/cpd_cpu.cu:484-691) with its GPU hooks init_GPU and
 * MTTKRP_MIHCSR_GPU_oneMode_forCPD (src/mttkrp_gpu.cu:3786-4052): the whole
 * loop runs on the device over an MM-CSF format. Per iteration and mode:
 * MTTKRP, solve against the Hadamard of the other Gram matrices (Cholesky,
 * Gauss-Jordan when not positive definite), normalise (column 2-norms in the
 * first iteration, max(column max, 1) after), update the Gram; then the fit
 * 1 - ||X - model|| / ||X||. Stops when |fit - previous fit| < tol (after the
 * first iteration) or after max_iters. Differences from the reference: the fit
 * uses the full symmetric Gram product and the max-norm is a true maximum
 * (both are wrong in the reference, src/cpd_cpu.cu:383-385 and :298-303). */
#define MMCSF_CPD_FP32 0       /* FP32 factors and small-matrix math */
#define MMCSF_CPD_BF16 1       /* BF16 factors, FP32 MTTKRP accumulation, FP64 Gram/solve/lambda/fit */
#define MMCSF_CPD_FP64_SOLVE 2 /* FP32 factors with the FP64 small-matrix math */
/* Every form runs the whole loop as one CUDA graph launch (a WHILE node over one
 * captured iteration) unless no_graph is set. The graph needs a non-default
 * stream: on the default stream the FP32 forms run host-driven (the host reads
 * the fit back every iteration) and the BF16 form returns MMCSF_ERR_INVALID. */
#define MMCSF_CPD_MAX_HISTORY 1000
typedef struct {
  int rank;       /* 4, 8, 16, 32 or 64 */
  int max_iters;  /* 0 = the reference's 10 (src/util.h:210) */
  double tol;     /* 0 = the reference's 1e-5 (src/cpd_cpu.cu:494) */
  int precision;  /* MMCSF_CPD_* */
  int no_graph;   /* 1: run the loop host-driven (one iteration at a time), at any precision */
  uint64_t seed;  /* initial factors uniform in [0,1) when d_init is NULL */
  int profile;    /* 1: time every phase of every iteration with CUDA events (host-driven loop, also for
                     BF16) into mmcsf_cpd_result.phase_ms; the events add a few microseconds per phase */
} mmcsf_cpd_opts;
#define MMCSF_CPD_PHASES 6 /* MTTKRP, solve (Hadamard + Cholesky/inverse), apply (M V^-1, column norms),
                              lambda, finish (normalise, store, Gram, fit inner product), fit */
typedef struct {
  int iters, converged, graph, launches; /* launches: kernels per iteration (graph) or in total */
  double fit;
  double seconds; /* device time of the iteration loop */
  double phase_ms[MMCSF_CPD_PHASES]; /* with opts.profile: device time of each phase summed over the loop */
  double fit_history[MMCSF_CPD_MAX_HISTORY];
} mmcsf_cpd_result;
/* d_init (optional): FP32 initial factors (dims[m] x rank); d_factors_out
 * (optional): normalised FP32 factors; lambda_out (optional, host): rank
 * weights. Synchronises the stream before returning. */
int mmcsf_cpd(mmcsf_format* F, const mmcsf_cpd_opts* opts, const float* const* d_init, float* const* d_factors_out,
              double* lambda_out, mmcsf_cpd_result* result, void* stream);

/* ---- construction sort without device allocation ------------------------
 * No counterpart in the reference. Sorts a device COO tensor (stably) into
 * the nonzero order that mmcsf_build gives the format `impl` built with
 * `mode` -- the order of the arrays mmcsf_format_export("inds<m>"/"vals")
 * returns -- writing every mode's sorted indices and the values into caller
 * buffers. It allocates no device memory: for callers whose device memory is
 * owned by another allocator (a runtime or framework that reserved the GPU's
 * memory up front) or that cannot take cudaMalloc's implicit synchronisation
 * in their steady state. Its scratch is one static device array of about
 * 12.2 MiB that every GPU loading this library holds until process exit.
 * Limit: nnz <= 524288 (2^19) and every mode length below 2^31; larger
 * inputs are rejected with MMCSF_ERR_INVALID. The first call on each device
 * looks up the scratch array's device address (make that first call before
 * any stream capture). All calls share the scratch: calls that overlap on the
 * GPU (different streams, threads or processes sharing a context) race and
 * must be serialised by the caller. Stream-ordered; nothing is synchronised. */
int mmcsf_sort_coo_noalloc(int impl, int mode, int nd, const uint64_t* dims, uint64_t nnz,
                           const uint32_t* const* d_inds, const float* d_vals, uint32_t* const* d_out_inds,
                           float* d_out_vals, void* stream);

/* Number of kernel launches the last MTTKRP/build call on this format made
 * (instrumentation for launch accounting). */
int mmcsf_format_last_launches(const mmcsf_format* F, int* launches);

#ifdef __cplusplus
}
#endif
#endif /* MMCSF_H */
