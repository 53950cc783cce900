/*
 * swift_b200.h -- C ABI of the B200-native Swift SpMM library (libswiftb200.so).
 *
 * Swift computes C = A * B for a CSR sparse A (M x K) and a dense B (K x N).  The library
 * builds the Swift column-sorted tiled format ON THE GPU (column sort by nonzero count,
 * 32-nonzero regular tiles, irregular "reside" remainder, load-balance blocks), keeps it
 * resident in HBM as a plan, and runs hand-written sm_100a kernels over it.
 *
 * All entry points are plain C: pointers, sizes and enums only.  Every call returns a
 * swift_status; nothing prints and nothing exits.  Device work is stream-ordered on the
 * caller's stream (NULL = the legacy default stream).  A plan's pattern is fixed at
 * creation; its products share per-plan scratch (split-row partials and counters), so the
 * products of one plan must be ordered on one stream (or separated by events); different
 * plans run concurrently without restriction.
 *
 * Reference interface each entry point replaces (paths inside the reference project):
 *   swift_plan_create           -- csr_to_csc + col_sort/ColSort + formattransation/
 *                                  formatTransform + block_catgory + balance, as sequenced
 *                                  by src/main.cu:207-385 (src/gpu_csr2csc.h:51,
 *                                  src/coo2csc.h:82,137, src/ColSort_cuda.h:48,
 *                                  src/formatTransform_cuda.h:198, src/block_catgory.h:1,
 *                                  src/balance.h:1)
 *   swift_plan_export_*         -- the slide_matrix those functions fill (src/format.h:6-39)
 *   swift_spmm                  -- Swift_GPU / Swift_GPU_3 / Swift_GPU_4 / Swift_gpu1 /
 *                                  Swift_gpu2 kernels (src/Swift.h:15-181,
 *                                  src/Swift_3.h:6-213, src/Swift_4.h:6-302,
 *                                  src/Swift_gpu_col_major.h:6-168,
 *                                  src/Swift_gpu_row_major.h:29-133)
 *   swift_ref_*                 -- the same functions with the reference's host-buffer
 *                                  calling convention (see swift_compat.h for the C++ shims
 *                                  that carry the reference's exact signatures)
 *   swift_spmm_transposed, swift_sddmm, swift_fused_forward_backward, swift_batch_*,
 *   swift_plan_set_values       -- no counterpart in the reference (backward pass, batched
 *                                  execution and value updates added by this library)
 */
#ifndef SWIFT_B200_H
#define SWIFT_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Every declaration below is exported from the shared library (built with hidden default
 * visibility). */
#if defined(__GNUC__)
#pragma GCC visibility push(default)
#endif

#define SWIFT_B200_VERSION "0.1.0"

/* Same object as cudaStream_t; NULL selects the legacy default stream. */
typedef struct CUstream_st *swift_stream_t;

typedef enum swift_status {
  SWIFT_OK = 0,
  SWIFT_ERR_INVALID_ARG = 1, /* null pointer, negative size, unknown enum value           */
  SWIFT_ERR_BAD_CSR = 2,     /* rowptr not monotone / not 0..nnz, column index out of range */
  SWIFT_ERR_BAD_PERM = 3,    /* injected column order is not a count-sorting permutation  */
  SWIFT_ERR_UNSUPPORTED = 4, /* dtype / layout / engine combination not provided          */
  SWIFT_ERR_CUDA = 5,        /* a CUDA runtime call or kernel launch failed               */
  SWIFT_ERR_ALLOC = 6,       /* device or host allocation failed                          */
  SWIFT_ERR_OVERFLOW = 7,    /* a size exceeds the int32 index range of the format        */
  SWIFT_ERR_TIMEOUT = 8,     /* a bounded device-side wait ran out                        */
  SWIFT_ERR_NO_DEVICE = 9,   /* no CUDA device, or not an sm_100 device                   */
  SWIFT_ERR_VERIFY = 10,     /* compat entry points: result differs from the golden C     */
  SWIFT_ERR_IO = 11,         /* a file cannot be opened or read                           */
  SWIFT_ERR_FORMAT = 12      /* a MatrixMarket file is malformed                          */
} swift_status;

typedef enum swift_dtype { SWIFT_F32 = 0, SWIFT_F64 = 1, SWIFT_BF16 = 2, SWIFT_F16 = 3 } swift_dtype;
typedef enum swift_layout { SWIFT_ROW_MAJOR = 0, SWIFT_COL_MAJOR = 1 } swift_layout;
typedef enum swift_memspace { SWIFT_HOST = 0, SWIFT_DEVICE = 1 } swift_memspace;

/* Execution engines over the same plan.
 *   TILED   -- the Swift kernels proper: one warp per run of regular tiles that share their
 *              32 sorted columns, runs of equal rows reduced in registers before a vector
 *              atomic into C, plus the load-balanced reside blocks.  Any layout of B and C.
 *   ROWWISE -- row-ordered execution for C much larger than L2: each C row is accumulated
 *              in registers and written once; rows longer than the split threshold are cut
 *              into pieces combined deterministically.  Column-major B or C are transposed
 *              into row-major copies held by the plan (not with b_presorted).
 *   TILED_GROUPED -- the tiled engine in the order of Swift_GPU_4 (src/Swift_4.h:6-76): the
 *              slots of every group of 8 tiles visited in row-sorted order (the per-group row
 *              sort of src/back_process.h:23-229, run on the GPU when first needed), so equal
 *              rows of a group form one run and take one vector atomic.  Row-major B and C,
 *              FP32 or FP64.
 *   BAND    -- dense diagonal tiles for matrices whose nonzeros crowd the diagonal: every
 *              group of 8 rows keeps the columns [8g - W, 8g - W + 8 + 2W) as a dense 8-row
 *              tile (values only, no indices), multiplied from a TMA-staged B panel with the 8
 *              rows held in registers; the nonzeros outside the tiles go through the ROWWISE
 *              walk first.  The half-width W in {3, 7, 15, 31, 47, 63} comes from the plan's
 *              |col - row| profile (swift_plan_band_profile; 3 when no width pays).  FP32
 *              plans, F32 / BF16 / F16 row-major B and C with N >= 128, N % 4 == 0, 16-byte
 *              aligned B, C, ldb and ldc (else SWIFT_ERR_UNSUPPORTED).  The split is built on
 *              first use.  No counterpart in the reference.
 *   AUTO    -- the autotuned choice for (N, dtype), ROWWISE when no tuning was run and the
 *              layouts allow it. */
typedef enum swift_engine {
  SWIFT_ENGINE_AUTO = 0,
  SWIFT_ENGINE_TILED = 1,
  SWIFT_ENGINE_ROWWISE = 2,
  SWIFT_ENGINE_TILED_GROUPED = 3,
  SWIFT_ENGINE_BAND = 4
} swift_engine;

typedef struct swift_csr {
  int rows;              /* M */
  int cols;              /* K */
  int nnz;
  const int *rowptr;     /* M+1, rowptr[0] = 0, non-decreasing, rowptr[M] = nnz */
  const int *colidx;     /* nnz, each in [0, K) */
  const void *val;       /* nnz values of type val_type */
  swift_dtype val_type;  /* SWIFT_F32 or SWIFT_F64 */
  swift_memspace mem;    /* where rowptr/colidx/val live */
} swift_csr;

typedef struct swift_plan_opts {
  /* Column order to use instead of the stable count order (ascending count, ties by
   * ascending column index -- the order of the reference's thrust::sort_by_key,
   * src/ColSort_cuda.h:108).  Must sort the column counts ascending.  NULL = stable. */
  const int *col_perm;
  swift_memspace col_perm_mem;
  /* Rowwise engine: rows with more nonzeros than this are cut into pieces of this size
   * (0 = default 128). */
  int long_row_split;
  /* Also build the transposed (A^T) row layout used by swift_spmm_transposed and the
   * backward kernels (0 = build lazily on first use). */
  int build_transpose;
} swift_plan_opts;

typedef struct swift_plan swift_plan;

typedef struct swift_plan_stats {
  int rows, cols, nnz;
  int nsteps;            /* distinct nonzero counts among the sorted columns */
  int tilenum, regular_nnz;
  int reside_col, reside_nnz, numblk;
  int fmt_count[3];      /* regular tiles of format 0 / 1 / 2 (src/block_catgory.h) */
  int empty_cols, max_col_nnz, max_row_nnz;
  int long_rows, long_pieces, long_row_split;
  double build_ms;       /* device time of the format build (CUDA events) */
  size_t device_bytes;   /* HBM held by the plan */
} swift_plan_stats;

/* Host copy of the reference's slide_matrix, field for field (src/format.h:6-39).  The
 * FP32 flavour matches test/k-32/FP32/format.h; a reference slide_matrix* may be passed
 * where these are expected.  Arrays are malloc'd; free with swift_slide_free_* or the
 * reference's Tile_destroy. */
#define SWIFT_SLIDE_FIELDS(VAL_T)                                                             \
  VAL_T *sortval;                                                                             \
  int *sortrowidx;                                                                            \
  int *tile_ptr;                                                                              \
  int *tile_len;                                                                              \
  int *tile_colidx;                                                                           \
  int *tile_tall;                                                                             \
  int *tile_format;                                                                           \
  int *countrow;                                                                              \
  int *segmentoffset;                                                                         \
  int *segptr;                                                                                \
  int *seginfo;                                                                               \
  int *seglength;                                                                             \
  int *sortrowindex;                                                                          \
  int *val_position;                                                                          \
  int *val_offset;                                                                            \
  int tilenum;                                                                                \
  int segsum;                                                                                 \
  int regular_nnz;                                                                            \
  int reside_col;                                                                             \
  int reside_nnz;                                                                             \
  int *reside_cscptr;                                                                         \
  int *reside_cscrowidx;                                                                      \
  VAL_T *reside_val;                                                                          \
  int numblk;                                                                                 \
  unsigned int *colorblk;                                                                     \
  int *blkstart;                                                                              \
  int *blkstop;                                                                               \
  int *blkptr;

typedef struct swift_slide_matrix_f32 { SWIFT_SLIDE_FIELDS(float) } swift_slide_matrix_f32;
typedef struct swift_slide_matrix_f64 { SWIFT_SLIDE_FIELDS(double) } swift_slide_matrix_f64;

/* ------------------------------------------------------------------ basics */
const char *swift_status_string(swift_status s);
const char *swift_version(void);
/* Text of the last CUDA or validation failure seen by this thread ("" if none). */
const char *swift_last_error(void);
/* Checks that a CUDA device of compute capability 10.x is current. */
swift_status swift_device_check(int *sm_count, int *cc_major, int *cc_minor);

/* ------------------------------------------------------------------ plans */
/* Builds the Swift format of A on the current device.  A may live on the host or the
 * device.  Synchronises `stream` once (sizes of the format are read back). */
swift_status swift_plan_create(const swift_csr *A, const swift_plan_opts *opts,
                               swift_stream_t stream, swift_plan **out);
/* Releases the plan's device memory once the work it enqueued on each stream it ran on is done
 * (stream-ordered: the host does not wait and other streams are not stalled; when the plan was
 * used inside a stream capture, after a device synchronisation). */
swift_status swift_plan_destroy(swift_plan *plan);
swift_status swift_plan_get_stats(const swift_plan *plan, swift_plan_stats *out);
/* New values for the plan's fixed pattern (nnz values of the plan's value type, CSR order,
 * host or device memory); every value copy of the format is refilled on `stream`, the
 * pattern, column order and task layouts are kept.  No counterpart in the reference (added
 * for training loops that update A's values).  Products already queued on other streams
 * must have finished. */
swift_status swift_plan_set_values(swift_plan *plan, const void *val, swift_memspace mem,
                                   swift_stream_t stream);

/* Host copies of every reference array.  with_row_sort != 0 also runs the per-8-tile row
 * sort (src/back_process.h:23-229) and fills val_position / val_offset; the reference
 * overwrites sortrowidx with the sorted keys at that point, and so does this export.
 * blockratio (may be NULL) receives the FP32 flavour's statistic of that step. */
swift_status swift_plan_export_f32(const swift_plan *plan, swift_slide_matrix_f32 *out,
                                   int with_row_sort, float *blockratio);
swift_status swift_plan_export_f64(const swift_plan *plan, swift_slide_matrix_f64 *out,
                                   int with_row_sort, float *blockratio);
void swift_slide_free_f32(swift_slide_matrix_f32 *m);
void swift_slide_free_f64(swift_slide_matrix_f64 *m);

/* Host copies of the column sort (src/coo2csc.h:82-134 outputs): perm[K] (sorted position ->
 * column), sortnnz[K], and the sorted CSC (nnz row indices / values of the plan's type).
 * Any pointer may be NULL. */
swift_status swift_plan_export_sorted(const swift_plan *plan, int *perm, int *sortnnz,
                                      int *sortrowidx_tmp, void *sortval_tmp);

/* ------------------------------------------------------------------ products */
/* C = A * B.  B is K x N, C is M x N, both of `dtype` (F32 or F64 matching the plan's
 * values, or BF16 / F16 with an F32 plan: B and C in 16 bits, products accumulated in F32).
 * ld* are leading dimensions in elements (row-major: row stride; col-major: column
 * stride).  b_presorted != 0 means B's rows are already in the plan's sorted column order
 * (the reference's sort_dense_mtx); otherwise rows are in A's original column order.
 * C is overwritten.  Stream-ordered; no synchronisation. */
swift_status swift_spmm(const swift_plan *plan, swift_engine engine, int N, swift_dtype dtype,
                        const void *B, int64_t ldb, swift_layout b_layout, int b_presorted,
                        void *C, int64_t ldc, swift_layout c_layout, swift_stream_t stream);

/* C = A * B with 16-bit operands scaled per row, for values outside FP16's range (or that
 * would lose BF16's few mantissa bits near its extremes).  dtype BF16 or F16, F32 plan;
 * row-major B (K x N, rows in A's column order) and C (M x N).  Row k of B holds
 * B_true[k] / b_scale[k] (b_scale: K floats on the device, or NULL for all 1); each product
 * term is A[r][k] * b_scale[k] * B[k][n], accumulated in F32.  C row r is written as
 * C_true[r] / c_scale[r] with c_scale[r] (M floats on the device) the power of two that
 * puts the row's largest magnitude in [2^14, 2^15) (1 for an all-zero row), so the 16-bit
 * rows neither overflow nor flush to zero.  Row walk only: B / C / ldb / ldc 16-byte aligned
 * and N <= 256, or 32-byte aligned and N <= 512; other shapes return SWIFT_ERR_UNSUPPORTED.  No counterpart in the
 * reference (FP32 / FP64 only). */
swift_status swift_spmm_scaled(const swift_plan *plan, int N, swift_dtype dtype, const void *B, int64_t ldb,
                               const float *b_scale, void *C, int64_t ldc, float *c_scale,
                               swift_stream_t stream);

/* X = A^T * Y (row-major, K x N and M x N): the backward product dX = A^T dY. */
swift_status swift_spmm_transposed(const swift_plan *plan, int N, swift_dtype dtype,
                                   const void *Y, int64_t ldy, void *X, int64_t ldx,
                                   swift_stream_t stream);

/* out[e] = sum_n U[row_e, n] * V[col_e, n] for every nonzero e of A in CSR order
 * (U is M x N, V is K x N, row-major): the backward dA_vals = SDDMM(dY, X).  out has the
 * plan's value type (F32 plans accumulate F32, also for BF16/F16 inputs). */
swift_status swift_sddmm(const swift_plan *plan, int N, swift_dtype dtype, const void *U,
                         int64_t ldu, const void *V, int64_t ldv, void *out,
                         swift_stream_t stream);

/* Whether A equals its transpose, values included (square plans; computed once on the GPU
 * and cached; synchronises `stream` the first time).  No counterpart in the reference. */
swift_status swift_plan_is_symmetric(swift_plan *plan, int *symmetric, swift_stream_t stream);
/* use = 0 keeps swift_fused_forward_backward on the general path (one pass for Y and dA, one
 * over A^T for dX) even for a symmetric A; 1 (default) lets it use the symmetry. */
swift_status swift_plan_set_symmetry(swift_plan *plan, int use);

/* One pass over A in row order for Y = A X and dA_vals = SDDMM(dY, X) (X read once per
 * nonzero for both), then dX = A^T dY over the transposed layout.  When A == A^T with equal
 * values (checked once per plan, see swift_plan_is_symmetric), dX = A dY joins the same pass
 * and the transposed layout is not used.  Any output pointer may be NULL to skip that
 * product.  Row-major, F32 or F64. */
swift_status swift_fused_forward_backward(const swift_plan *plan, int N, swift_dtype dtype,
                                          const void *X, int64_t ldx, const void *dY,
                                          int64_t lddy, void *Y, int64_t ldy, void *dX,
                                          int64_t lddx, void *dA, swift_stream_t stream);

/* Deterministic FP64 product C = A * B (one warp per row, nonzeros summed in CSR order),
 * the GPU error reference; A's values are widened if the plan is F32.  Row-major. */
swift_status swift_spmm_f64_reference(const swift_plan *plan, int N, const double *B,
                                      int64_t ldb, double *C, int64_t ldc,
                                      swift_stream_t stream);

/* C = A * B for callers that cannot allocate device memory once running -- real-time or
 * certified deployments that forbid device allocation after start-up, and hosts whose device
 * memory belongs to another allocator (a framework's caching allocator, a fixed arena), where
 * a stray cudaMalloc can fail or fragment that memory and synchronises the device.  No
 * counterpart in the reference.
 *
 * Same result as swift_spmm with the ROWWISE engine on row-major B (K x N) and C (M x N), but
 * it calls no cudaMalloc, cudaFree or allocating routine: the scratch of the long-row pieces
 * lives in a fixed device array of SWIFT_NOALLOC_SCRATCH_BYTES that every GPU loading the
 * library holds until the process exits.  The plan must already exist (creating it
 * allocates).
 * Limits: at most SWIFT_NOALLOC_MAX_LONG_ROWS long rows and pieces * N * 4 bytes (8 for FP64)
 * of partial rows within the array minus 64 KiB; larger products return SWIFT_ERR_OVERFLOW
 * (details in swift_last_error) -- a plan made with a larger long_row_split has fewer pieces.
 * The first call on each device looks up the array's device address with that device
 * current, so make it before any stream capture.  The address is kept per device together
 * with the id of the CUDA context it belongs to; if that context is destroyed and a new one
 * made (cudaDeviceReset), the next call looks the address up again in the new context -- make
 * that call, too, outside stream capture, after creating new plans (a reset also destroys every
 * plan's device memory).  All calls share the array and it keeps the
 * last call's contents (each call clears the counters it uses): calls that overlap on the GPU
 * race, so serialise them. */
#define SWIFT_NOALLOC_SCRATCH_BYTES ((size_t)16 << 20)
#define SWIFT_NOALLOC_MAX_LONG_ROWS 16384
swift_status swift_spmm_noalloc(const swift_plan *plan, int N, swift_dtype dtype, const void *B,
                                int64_t ldb, void *C, int64_t ldc, swift_stream_t stream);

/* ------------------------------------------------------------------ tuning */
/* Diagonal profile of A, measured on the GPU once per plan (synchronises `stream` the first
 * time): hist[d] = nonzeros with |col - row| == d for d = 0..SWIFT_BAND_PROFILE_MAX (hist may
 * be NULL), and the BAND engine's half-width: the W in {3, 7, 15, 31, 47, 63} with the largest
 * (nonzeros within distance W) - M * (8 + 2W) / 8 -- the gathers the tiles save against the
 * dense work they add, a gathered nonzero costing the row walk about eight dense tile
 * elements -- if that saves at least a twentieth of the nonzeros, else -1.  AUTO's tuner
 * tries the BAND engine only when the half-width is >= 0.  No counterpart in the reference. */
#define SWIFT_BAND_PROFILE_MAX 128
swift_status swift_plan_band_profile(swift_plan *plan, long long *hist, int *half_width,
                                     swift_stream_t stream);

/* Block-density histogram of A, measured on the GPU: blocks of bh consecutive rows x bw
 * consecutive columns, columns in A's own order (order 0) or the plan's sorted column order
 * (order 1).  For each block holding a nonzero, its fill f = nonzeros / (bh * bw) lands in bin
 * k when 2^-(k+1) < f <= 2^-k (k = 0 .. nbins - 2) and in bin nbins - 1 when sparser;
 * blocks[k] counts those blocks and nnz[k] their nonzeros (both arrays nbins long, host
 * memory, 1 <= nbins <= 64).  Synchronises `stream`; temporary device memory of about 20 bytes
 * per nonzero.  The measurement behind a dense-tile path (the BAND engine, tensor cores): it
 * pays only where blocks are dense.  No counterpart in the reference. */
swift_status swift_plan_block_histogram(swift_plan *plan, int bh, int bw, int order, int nbins,
                                        long long *blocks, long long *nnz, swift_stream_t stream);

/* Measurement: the gather ceiling of the row-ordered engines on this plan's A.  Times (CUDA
 * events on `stream`, `reps` launches after two warm-up launches) a kernel that only gathers B
 * rows along A's column stream -- the row walk's 16-byte vectors and sub-warp widths, four
 * loads in flight per lane, no values, no row bookkeeping, no C -- and the same kernel with
 * every column index folded into rows 0..255 (rows resident in L1).  ms_stream and ms_l1 are
 * per launch; checksum (may be NULL) is the sum of every gathered element of the first launch
 * kind, for checking.  Row-major FP32 B (K x N), N in {32, 64, 128}, B 16-byte aligned,
 * ldb % 4 == 0, K >= 256.  Synchronises `stream`.  No counterpart in the reference. */
swift_status swift_gather_bound(const swift_plan *plan, int N, const float *B, int64_t ldb, int reps,
                                swift_stream_t stream, double *ms_stream, double *ms_l1, double *checksum);

/* Whether a BAND product's block gave up waiting for its TMA copies (a bounded wait of about
 * two seconds; the block then leaves its C rows without the tiles' part): *flag = 1 if any did
 * since the last reset.  Synchronous; reset != 0 clears the flag.  No counterpart in the
 * reference. */
swift_status swift_band_timeout_flag(int *flag, int reset);

/* Times the engines and their parameters on this plan for (N, dtype) with CUDA events and
 * stores the fastest as the plan's AUTO choice.  B and C are caller buffers of the right
 * shape (row-major); their contents are overwritten.  best_ms may be NULL. */
swift_status swift_plan_autotune(swift_plan *plan, int N, swift_dtype dtype, const void *B,
                                 void *C, swift_stream_t stream, double *best_ms,
                                 swift_engine *best_engine);

/* Row-ordered engine parameters: task_size = merged nonzero/row-end positions per sub-warp
 * task (0 clears the override and returns to the tuned / default choice); loads_in_flight =
 * B-row vector loads each lane issues before consuming them (4 = default, with registers
 * capped for 64 resident warps per SM; 8; or 16); vector_bytes = bytes per lane access (0 =
 * widest the operands allow, 32, 16 or 4); kernel = 0 (choose), 1 (lean walk), 2 (walk over
 * row-start-flagged indices staged in shared memory), 3 (general walk, any width), 4 (staged
 * walk: FP32 operands with N = 32, 64 or 128 and 16-byte vectors; each lane keeps its slices
 * of the next 7 or 15 gathered B rows -- loads_in_flight 8 or 16 -- in flight through cp.async
 * into shared memory; other shapes take the walk the other parameters select).  The override applies to
 * every later swift_spmm with the ROWWISE (or AUTO) engine on this plan. */
swift_status swift_plan_set_rowwise_params(swift_plan *plan, int task_size, int loads_in_flight,
                                           int vector_bytes, int kernel);
/* The parameters AUTO / ROWWISE would use for (N, dtype) on this plan. */
swift_status swift_plan_get_rowwise_params(swift_plan *plan, int N, swift_dtype dtype,
                                           int *task_size, int *loads_in_flight,
                                           int *vector_bytes, int *kernel);

/* ------------------------------------------------------------------ batches */
/* Many independent products C_i = A_i * B_i (FP32 plans, FP32 row-major B_i and C_i) in one
 * persistent launch: every SM runs resident blocks whose warps stride over the merge-path
 * tasks of all members.  Each member keeps its own task layout, split-row counters and
 * scratch, so a batch shares no mutable state with its plans' own products.  The plans must
 * outlive the batch.  One batch must not run on two streams at once. */
typedef struct swift_batch swift_batch;
swift_status swift_batch_create(swift_plan *const *plans, int count, swift_stream_t stream,
                                swift_batch **out);
/* Releases the batch's device memory once its own launches are done (stream-ordered, as
 * swift_plan_destroy; after a device synchronisation when a launch was captured into a
 * caller's graph). */
swift_status swift_batch_destroy(swift_batch *batch);
/* Ns[i], B[i], ldb[i], C[i], ldc[i] per member (device pointers, row-major).  N_i <= 128 with
 * 16-byte aligned operands (N_i % 4 == 0), or N_i <= 32 otherwise.  Builds the members' task
 * layouts (first call, or after autotuning) and uploads the launch table; synchronises
 * `stream`.  A graph captured by swift_batch_run_graph reads the table when it replays, so it
 * stays valid when operands are set again. */
swift_status swift_batch_set_operands(swift_batch *batch, const int *Ns, const void *const *B,
                                      const int64_t *ldb, void *const *C, const int64_t *ldc,
                                      swift_stream_t stream);
/* One launch; writes every row of every C_i. */
swift_status swift_batch_run(swift_batch *batch, swift_stream_t stream);
/* Captures swift_batch_run into a CUDA graph on the first call (on a private stream) and
 * replays it on `stream`. */
swift_status swift_batch_run_graph(swift_batch *batch, swift_stream_t stream);
/* Chooses the merge-path task size (merged positions per sub-warp task) per member class --
 * N <= 32, N <= 64, wider -- by timing whole batch launches: the best of 128, 256, 512 and 1024
 * for every class, then each class on its own against the others' current sizes; then the
 * N-split of each class (see swift_batch_set_n_split), kept where it is faster (operands must
 * be set; each C_i is overwritten with its product).  best_ms = the chosen launch's time,
 * best_task_size = the widest class's size. */
swift_status swift_batch_autotune(swift_batch *batch, swift_stream_t stream, double *best_ms,
                                  int *best_task_size);
/* The task sizes in use for the three member classes (N <= 32, N <= 64, wider). */
swift_status swift_batch_get_task_sizes(const swift_batch *batch, int *sizes);
/* N-split per member class (splits[3], each 1 or 2): with 2, every member of the class whose N
 * is a multiple of 8 is walked as two column halves, each a separate entry of the launch
 * (own tasks and split-row scratch) -- half-width B rows per gather, the walk over A twice.
 * Rebuilds the launch table when operands are set (a graph captured by swift_batch_run_graph
 * is re-captured on its next call).  SWIFT_ERR_INVALID_ARG for other values. */
swift_status swift_batch_set_n_split(swift_batch *batch, const int *splits, swift_stream_t stream);
/* The N-split in use for the three member classes. */
swift_status swift_batch_get_n_split(const swift_batch *batch, int *splits);

/* ------------------------------------------------------------------ MatrixMarket input */
/* Reads a MatrixMarket coordinate file into host CSR as the reference's reader does
 * (mmio_allinone, src/auxiliary.h:167-332): 0-based indices, entries in file order inside
 * each row (duplicates kept), off-diagonal entries of symmetric and hermitian files mirrored
 * with the same value, skew-symmetric files read as stored, pattern entries 1.0, complex
 * entries their real part.  val_type is SWIFT_F32 or SWIFT_F64.  *rowptr (m + 1), *colidx and
 * *val (nnz) are malloc'd; release each with swift_host_free.  Errors: SWIFT_ERR_IO (cannot
 * open or read), SWIFT_ERR_FORMAT (banner, size line or an entry malformed, an index outside
 * the matrix), SWIFT_ERR_UNSUPPORTED ("array" files), SWIFT_ERR_OVERFLOW.  reference_code
 * (may be NULL) receives what the reference's reader returns for the file: 0, -1 (cannot
 * open), -2 (banner), -4 (size line), or -5 where the reference would go on with undefined
 * values. */
swift_status swift_mtx_read(const char *path, swift_dtype val_type, int *m, int *n, int *nnz,
                            int *is_symmetric, int **rowptr, int **colidx, void **val,
                            int *reference_code);
void swift_host_free(void *p);

/* ------------------------------------------------------------------ reference calling convention */
/* The reference's preprocessing and kernels with its host-buffer convention: inputs and
 * outputs are host arrays, device buffers are allocated and freed inside, and *ms receives
 * the device time of the work (CUDA events) where the reference reports a time.  Column
 * sorts use the stable count order.  swift_compat.h wraps these in the reference's C++
 * signatures. */
swift_status swift_ref_csr_to_csc_f32(float *ms, int m, int n, int nnz, const float *csr_val,
                                      const int *csr_row_ptr, const int *csr_col_ind,
                                      float *csc_val, int *csc_row_ind, int *csc_col_ptr,
                                      int *nnzpercol);
swift_status swift_ref_csr_to_csc_f64(float *ms, int m, int n, int nnz, const double *csr_val,
                                      const int *csr_row_ptr, const int *csr_col_ind,
                                      double *csc_val, int *csc_row_ind, int *csc_col_ptr,
                                      int *nnzpercol);
/* src/coo2csc.h:82-134 / src/ColSort_cuda.h:48-143 */
swift_status swift_ref_col_sort_f32(float *ms, int colA, int nnz, int width, const int *nnzpercol,
                                    const int *csccolptr, const int *cscrowidx,
                                    const float *cscval, int *sortrowidx_tmp,
                                    float *sortval_tmp, int *sortnnz_tmp, const float *dense,
                                    float *sort_dense);
swift_status swift_ref_col_sort_f64(float *ms, int colA, int nnz, int width, const int *nnzpercol,
                                    const int *csccolptr, const int *cscrowidx,
                                    const double *cscval, int *sortrowidx_tmp,
                                    double *sortval_tmp, int *sortnnz_tmp, const double *dense,
                                    double *sort_dense);
/* src/coo2csc.h:137-435 (regular + reside).  reside_ratio may be NULL. */
swift_status swift_ref_formattransation_f32(float *ms, swift_slide_matrix_f32 *m,
                                            const int *sortrowidx_tmp, const float *sortval_tmp,
                                            const int *sortnnz_tmp, int nnz, int rowA, int colA,
                                            double *reside_ratio);
swift_status swift_ref_formattransation_f64(float *ms, swift_slide_matrix_f64 *m,
                                            const int *sortrowidx_tmp, const double *sortval_tmp,
                                            const int *sortnnz_tmp, int nnz, int rowA, int colA,
                                            double *reside_ratio);
/* src/formatTransform_cuda.h:198-435 (regular part only; h_count = number of steps). */
swift_status swift_ref_formatTransform_f32(float *ms, swift_slide_matrix_f32 *m,
                                           const int *sortrowidx_tmp, const float *sortval_tmp,
                                           const int *sortnnz_tmp, int nnz, int rowA, int colA,
                                           int *h_count);
swift_status swift_ref_formatTransform_f64(float *ms, swift_slide_matrix_f64 *m,
                                           const int *sortrowidx_tmp, const double *sortval_tmp,
                                           const int *sortnnz_tmp, int nnz, int rowA, int colA,
                                           int *h_count);
/* src/block_catgory.h:1-160.  shuffle_ratio may be NULL. */
swift_status swift_ref_block_catgory_f32(swift_slide_matrix_f32 *m, double *shuffle_ratio);
swift_status swift_ref_block_catgory_f64(swift_slide_matrix_f64 *m, double *shuffle_ratio);
/* src/balance.h:1-69 */
swift_status swift_ref_balance_f32(swift_slide_matrix_f32 *m, int m_rows, int n_reside,
                                   int reside_nnz, const int *cscptr, const int *cscrowidx);
swift_status swift_ref_balance_f64(swift_slide_matrix_f64 *m, int m_rows, int n_reside,
                                   int reside_nnz, const int *cscptr, const int *cscrowidx);
/* src/back_process.h:23-229.  blockratio may be NULL. */
swift_status swift_ref_row_idx_sort_f32(swift_slide_matrix_f32 *m, int rowA, int colA,
                                        int width, float *blockratio);
swift_status swift_ref_row_idx_sort_f64(swift_slide_matrix_f64 *m, int rowA, int colA,
                                        int width, float *blockratio);
/* Swift_GPU (variant 0), Swift_gpu1 (1), Swift_gpu2 (2), Swift_GPU_3 (3), Swift_GPU_4 (4):
 * C = A * B from a host slide_matrix.  B is the column-sorted dense operand, column-major
 * (K x N, leading dimension K) for every variant except 2, which takes it row-major
 * (K x N, leading dimension N); C is returned in the same layout (M x N).  The reference
 * wrappers' timing window (kernels only) is reported in *ms. */
swift_status swift_ref_spmm_f32(int variant, const swift_slide_matrix_f32 *m, int rowA,
                                int colA, int width, int nnz, const float *h_B_sorted,
                                float *h_C, float *ms);
swift_status swift_ref_spmm_f64(int variant, const swift_slide_matrix_f64 *m, int rowA,
                                int colA, int width, int nnz, const double *h_B_sorted,
                                double *h_C, float *ms);

#if defined(__GNUC__)
#pragma GCC visibility pop
#endif

#ifdef __cplusplus
}
#endif
#endif /* SWIFT_B200_H */
