// common.cuh -- internal declarations shared by the Swift B200 library's translation units.
#pragma once

#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <cstdint>
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "swift_b200.h"

namespace swift {

constexpr int kTile = 32;  // slidesize / TILESIZE of the reference (src/format.h:76-78)

// ---------------------------------------------------------------- errors
void set_last_error(const char *where, const char *what);

#define SW_CHECK_CUDA(expr)                                                                  \
  do {                                                                                       \
    cudaError_t e__ = (expr);                                                                \
    if (e__ != cudaSuccess) {                                                                \
      ::swift::set_last_error(#expr, cudaGetErrorString(e__));                               \
      return e__ == cudaErrorMemoryAllocation ? SWIFT_ERR_ALLOC : SWIFT_ERR_CUDA;            \
    }                                                                                        \
  } while (0)

#define SW_CHECK_LAUNCH() SW_CHECK_CUDA(cudaGetLastError())

#define SW_TRY(expr)                                                                         \
  do {                                                                                       \
    swift_status s__ = (expr);                                                               \
    if (s__ != SWIFT_OK) return s__;                                                         \
  } while (0)

inline cudaStream_t S(swift_stream_t s) { return reinterpret_cast<cudaStream_t>(s); }

// ---------------------------------------------------------------- device buffers
// Device allocations come from the device's default memory pool, on a private per-device
// stream (alloc_stream) that is synchronised before the buffer is handed out, so a buffer is
// ready for any stream.  A buffer is returned to the pool either stream-ordered on
// release_stream() -- set by swift_plan_destroy / swift_batch_destroy while they delete a plan
// or batch, to a stream that waits for that object's own work, so destruction neither blocks
// the host nor stalls other streams -- or, when a buffer is replaced or freed elsewhere, after a
// device-wide synchronisation (the ordering a plain cudaFree gives).
// Id of the CUDA context current on this thread (cuCtxGetId through the runtime's driver entry
// points): tells a reset device's new context from the destroyed one.
swift_status current_context_id(unsigned long long *id);
cudaStream_t alloc_stream();
cudaStream_t &release_stream();  // thread-local; null outside the destroy paths
// A private stream (of the current device) that waits for the work recorded in `uses` -- after
// a device-wide synchronisation when that record is incomplete -- for a destroy path to release
// buffers on; null when no stream can be made (buffers are then freed after a device
// synchronisation).
cudaStream_t release_stream_after(const std::vector<std::pair<cudaStream_t, cudaEvent_t>> &uses,
                                  bool sync_device);
// Deletes a plan or batch on its own device with its buffers released on `fs`.
template <class Obj>
void delete_releasing(Obj *o, int device, cudaStream_t fs) {
  int prev = -1;
  cudaGetDevice(&prev);
  if (prev != device) cudaSetDevice(device);
  release_stream() = fs;
  delete o;
  release_stream() = nullptr;
  if (fs) cudaStreamDestroy(fs);  // its frees still run, after the waited-for work
  if (prev >= 0 && prev != device) cudaSetDevice(prev);
}

// Owning device allocation (plan lifetime).  Size in bytes; never shared.
struct DevBuf {
  void *p = nullptr;
  size_t bytes = 0;
  DevBuf() = default;
  DevBuf(const DevBuf &) = delete;
  DevBuf &operator=(const DevBuf &) = delete;
  DevBuf(DevBuf &&o) noexcept : p(o.p), bytes(o.bytes) { o.p = nullptr; o.bytes = 0; }
  DevBuf &operator=(DevBuf &&o) noexcept {
    if (this != &o) { reset(); p = o.p; bytes = o.bytes; o.p = nullptr; o.bytes = 0; }
    return *this;
  }
  ~DevBuf() { reset(); }
  void reset() {
    if (p) {
      if (cudaStream_t rs = release_stream()) {
        cudaFreeAsync(p, rs);
      } else {
        cudaDeviceSynchronize();
        cudaFreeAsync(p, alloc_stream());
      }
    }
    p = nullptr;
    bytes = 0;
  }
  swift_status alloc(size_t n) {
    reset();
    if (n == 0) n = 16;  // keep every pointer valid and 16-byte aligned
    cudaStream_t s = alloc_stream();
    cudaError_t e = s ? cudaMallocAsync(&p, n, s) : cudaErrorInvalidResourceHandle;
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) {
      if (p) cudaFreeAsync(p, s);
      p = nullptr;
      set_last_error("cudaMallocAsync", cudaGetErrorString(e));
      return SWIFT_ERR_ALLOC;
    }
    bytes = n;
    return SWIFT_OK;
  }
  template <class T> T *as() const { return static_cast<T *>(p); }
};

// Stream-ordered temporary (cudaMallocAsync / cudaFreeAsync on the same stream), so it may
// go out of scope while kernels that use it are still queued.
struct TmpBuf {
  void *p = nullptr;
  cudaStream_t st = nullptr;
  TmpBuf() = default;
  TmpBuf(const TmpBuf &) = delete;
  TmpBuf &operator=(const TmpBuf &) = delete;
  ~TmpBuf() {
    if (p) cudaFreeAsync(p, st);
  }
  swift_status alloc(size_t n, cudaStream_t s) {
    if (p) cudaFreeAsync(p, st);
    p = nullptr;
    st = s;
    if (n == 0) n = 16;
    cudaError_t e = cudaMallocAsync(&p, n, s);
    if (e != cudaSuccess) {
      p = nullptr;
      set_last_error("cudaMallocAsync", cudaGetErrorString(e));
      return SWIFT_ERR_ALLOC;
    }
    return SWIFT_OK;
  }
  template <class T> T *as() const { return static_cast<T *>(p); }
};

// ---------------------------------------------------------------- plan
struct RowLayout {
  // Row-ordered execution of a CSR-shaped operand (A itself, or A^T = the sorted CSC).
  int rows = 0, cols = 0, nnz = 0;
  const int *ptr = nullptr;     // rows+1 (points into a plan buffer)
  const int *idx = nullptr;     // nnz column (gather) indices
  const void *val = nullptr;    // nnz values
  const int *out_row = nullptr; // optional: output row of layout row r (NULL = r)
  // long rows: rows with more than `split` nonzeros are cut into pieces of `split`
  int split = 128;
  int long_rows = 0, pieces = 0;
  DevBuf piece_row;      // [pieces] layout row of each piece
  DevBuf piece_idx;      // [pieces] index of the piece within its row
  DevBuf long_first;     // [long_rows] first scratch slot / piece of each long row
  DevBuf long_count;     // [long_rows] pieces of each long row
  DevBuf long_of_row;    // [rows] long-row ordinal or -1
  DevBuf counters;       // [long_rows] arrival counters (self-resetting)
  DevBuf scratch;        // partial sums, grown on demand: pieces * N * 8 bytes
  size_t scratch_bytes = 0;
  bool built = false;
  // merge-path tasks (spmm_merge.cu): U positions of the merged nonzero/row-end sequence each
  int merge_U = 0, ntasks = 0, nsplit = 0;
  bool merge_built = false;
  DevBuf task_row;                    // [ntasks+1] row holding each task's first position
  DevBuf head_split, tail_split;      // [ntasks] split-row id of the task's first / last row or -1
  DevBuf task_hdr;                    // [ntasks] int4 packing of the three arrays above
  DevBuf eidx;                        // [nnz] gather indices, bit 31 set on each row's first
  DevBuf split_row, split_first, split_last, split_cnt;  // [nsplit]
  DevBuf mscratch;                    // [2*ntasks][N] partial rows ([2*ntasks][2N] for [Y | dX])
  // SDDMM alone needs no split-row bookkeeping, so it walks its own finer tasks
  int sdd_U = 0, sdd_ntasks = 0;
  DevBuf sdd_hdr;                     // [sdd_ntasks] int4 (first row, last row, -1, -1)
};

// Parameters of the merge-path row engine (autotuned per (N, dtype); overridable).
struct MergeOpts {
  int U = 512;      // merged positions per task
  int unroll = 4;   // B-row loads in flight per lane and batch (4, 8 or 16)
  int vbytes = 0;   // vector bytes per lane: 0 = widest the operands allow, 32, 16 or 4
  int kernel = 0;   // 0 choose, 1 lean walk, 2 flagged-index walk, 3 general walk, 4 staged walk
};

struct Plan {
  int M = 0, K = 0, nnz = 0;
  int device = 0;
  int sm_count = 148;
  swift_dtype val_type = SWIFT_F32;
  size_t vsz = 4;  // bytes per value
  bool has_csr = false;  // false for plans made from a host slide_matrix (compat path)

  // CSR copy
  DevBuf rowptr, colidx, val;
  // column sort
  DevBuf cnt;       // [K] nonzeros per original column
  DevBuf perm;      // [K] sorted position -> original column
  DevBuf invperm;   // [K]
  DevBuf sortnnz;   // [K+1] counts in sorted order
  DevBuf sptr;      // [K+1] sorted CSC pointer
  DevBuf srow;      // [nnz] sorted CSC row indices
  DevBuf sval;      // [nnz] sorted CSC values
  DevBuf spos;      // [nnz] CSR position of each sorted CSC entry
  // steps
  int nsteps = 0;
  DevBuf step_col, step_base, step_tall;  // [nsteps]
  DevBuf step_tile_off;                   // [nsteps+1] first tile of each step
  // regular tiles
  int tilenum = 0;
  int nstrips = 0;     // tiled-engine work items
  DevBuf item_tile;    // [nstrips+1] first tile of each work item
  DevBuf tile_colidx, tile_depth, tile_tall, tile_format;  // [tilenum]
  DevBuf sortrowidx, sortval;                              // [32*tilenum]
  int fmt_count[3] = {0, 0, 0};
  // reside
  int reside_col = 0, reside_nnz = 0;
  DevBuf reside_ptr, reside_row, reside_val;  // [reside_col+1], [reside_nnz]
  int numblk = 0;
  DevBuf colorblk, blkstart, blkstop, blkptr;
  // stats
  int max_col = 0, max_row = 0, empty_cols = 0;
  double build_ms = 0;
  // row-ordered layouts
  RowLayout fwd;  // A
  RowLayout bwd;  // A^T (sorted CSC rows, output through perm)
  int long_row_split = 128;
  // autotuned choice per (N, dtype)
  std::map<std::pair<int, int>, swift_engine> tuned;
  std::map<std::pair<int, int>, MergeOpts> tuned_merge;
  bool merge_override = false;
  MergeOpts merge_opts;  // used when set explicitly, and as the default otherwise
  // A == A^T including values (square plans): -1 not yet checked, 0 no, 1 yes; the fused
  // backward then computes dX = A dY in the same pass.  use_symmetry = 0 disables that.
  int symmetric = -1;
  int use_symmetry = 1;
  // row-major copies of column-major dense operands for the row walk (grown on demand)
  DevBuf rowcopy_b, rowcopy_c;
  // grouped tiled engine: the regular slots of every 8-tile group in row-sorted order -- C row,
  // sorted column and value per sorted slot (built on first use; new values invalidate it)
  DevBuf g_row, g_col, g_val;
  bool grouped_built = false;
  // band engine (spmm_band.cu): |col - row| profile, the chosen half-width (-2 not profiled
  // yet, -1 no width pays), and the split of A into dense diagonal tiles + the rest (built on
  // first use; new values are scattered through band_dst)
  int band_w = -2, band_used_w = -1, band_rest_nnz = 0;
  long long band_hist[129] = {};
  bool band_built = false;
  DevBuf band_tiles, band_ptr, band_idx, band_val, band_dst;
  // the tiles in the tensor-core kernel's A-fragment order, one layout per 16-bit type of B
  // (index 0 BF16, 1 FP16): 16-row windows, each row scaled by a power of two and split into
  // hi + lo parts of that type, then the rows' inverse factors; built on the first product of
  // that type after a build or a refill (a buffer per type, so that alternating BF16 and FP16
  // products rebuild nothing)
  DevBuf band_mma[2];
  bool band_mma_built[2] = {false, false};
  RowLayout band_rest;
  std::mutex mu;  // guards lazily built layouts and scratch growth
  // Streams this plan's work was enqueued on, each with an event recorded after its latest
  // call, so that destroying the plan waits for its own work only.  Work captured into a CUDA
  // graph (and streams beyond kMaxUses) can run later on any stream: then destruction waits
  // for the whole device.
  static constexpr int kMaxUses = 16;
  std::mutex use_mu;
  std::vector<std::pair<cudaStream_t, cudaEvent_t>> uses;
  bool sync_device_on_destroy = false;
  ~Plan();
};

// Records that `st` holds work on this plan; UseNote does it when an entry point returns.
void note_use(Plan &p, cudaStream_t st);
struct UseNote {
  Plan &p;
  cudaStream_t st;
  ~UseNote();
};

size_t plan_device_bytes(const Plan &p);

// ---------------------------------------------------------------- primitives (primitives.cu)
// Exclusive scan of n int32 values into out (n+1 entries: out[n] = total).  `in` may alias
// `out`.  Scratch is allocated stream-ordered.
swift_status scan_exclusive_i32(const int *in, int *out, int64_t n, cudaStream_t st);
// Stable LSD radix sort of (key, value) pairs by the low `bits` bits of key.  Results in
// keys_out / vals_out.  keys_in / vals_in are clobbered.
swift_status radix_sort_pairs(uint32_t *keys_in, uint32_t *vals_in, uint32_t *keys_out,
                              uint32_t *vals_out, int64_t n, int bits, cudaStream_t st);
// max over n int32 (n >= 0) into *dev_out (single int on device)
swift_status reduce_max_i32(const int *in, int64_t n, int *dev_out, cudaStream_t st);
// out[r * ld_out + c] = in[r + c * ld_in] for r < rows, c < cols: a column-major matrix
// rewritten row-major (with rows and cols swapped, the reverse).  esz = 2, 4 or 8 bytes.
swift_status transpose_dense(const void *in, int rows, int cols, int64_t ld_in, void *out,
                             int64_t ld_out, size_t esz, cudaStream_t st);

// ---------------------------------------------------------------- format build (format_build.cu)
swift_status build_from_csr(Plan &p, const swift_csr &A, const swift_plan_opts *opts,
                            cudaStream_t st);
// Steps, tiles, reside and balance from a device-resident sorted CSC already in the plan
// (p.sortnnz, p.sptr, p.srow, p.sval).
swift_status build_tiles(Plan &p, cudaStream_t st);
// New CSR-order values already in p.val: refills the sorted CSC values, tile slots, reside part.
swift_status refresh_values(Plan &p, cudaStream_t st);
// Tiled-engine work items from tile_colidx (also used for plans made from a slide_matrix).
swift_status build_items(Plan &p, cudaStream_t st);
// Balance blocks from p.reside_ptr (device) and its host copy.
swift_status build_balance(Plan &p, const int *h_reside_ptr, cudaStream_t st);
// Tile formats (and fmt_count) from p.sortrowidx.
swift_status classify_tiles(Plan &p, cudaStream_t st);
swift_status stable_column_order(const int *d_cnt, int K, int *d_perm, int *d_invperm,
                                 int *d_sortnnz, int *max_count, cudaStream_t st);
swift_status csr_to_csc_device(const int *d_rowptr, const int *d_colidx, const void *d_val,
                               bool f64, int M, int K, int nnz, int *d_colptr, int *d_rowidx,
                               void *d_cscval, int *d_cnt, cudaStream_t st);
swift_status build_row_layout(Plan &p, RowLayout &L, bool transpose, cudaStream_t st);
// Segment arrays of block_catgory on device (countrow[tilenum+1], segmentoffset[segsum+1],
// sortrowindex[32*tilenum]); segsum returned on host.
swift_status build_segments(const Plan &p, DevBuf &countrow, DevBuf &segmentoffset,
                            DevBuf &sortrowindex, int *segsum, cudaStream_t st);
// Per-8-tile row sort (back_process.h) on device into separate arrays.
swift_status build_row_sort(const Plan &p, DevBuf &sorted_rows, DevBuf &val_position,
                            DevBuf &val_offset, float *blockratio, cudaStream_t st);

// ---------------------------------------------------------------- kernels (spmm_*.cu)
struct DenseArgs {
  int N = 0;
  swift_dtype dtype = SWIFT_F32;
  const void *B = nullptr;
  int64_t ldb = 0;
  swift_layout b_layout = SWIFT_ROW_MAJOR;
  bool b_presorted = false;
  void *C = nullptr;
  int64_t ldc = 0;
  swift_layout c_layout = SWIFT_ROW_MAJOR;
  // 16-bit operands with per-row scales (row walk only): B row k holds B_true[k] / b_scale[k]
  // (b_scale may be null: all 1); C row r is written as C_true[r] / c_scale[r], c_scale[r] a
  // power of two chosen per row
  const float *b_scale = nullptr;
  float *c_scale = nullptr;
};
// variant 1 = reside per column without balance blocks (Swift_gpu1's kernel)
swift_status run_tiled(const Plan &p, const DenseArgs &a, int reside_variant, cudaStream_t st,
                       bool grouped = false);
// The grouped engine's slots (p.g_row, p.g_col, p.g_val) from the regular tiles.  keys and
// vpos: the per-group sorted rows and each original slot's sorted position, as row_idx_sort
// leaves them (src/back_process.h:23-229); both null to sort p.sortrowidx here.  A vpos that is
// not a permutation of each group returns SWIFT_ERR_INVALID_ARG.
swift_status build_grouped(Plan &p, const int *keys, const int *vpos, cudaStream_t st);

// band engine (spmm_band.cu)
swift_status band_profile(Plan &p, cudaStream_t st);  // p.mu held
swift_status band_refill(Plan &p, cudaStream_t st);   // p.mu held
bool band_operands_ok(const Plan &p, const DenseArgs &d);
swift_status run_band(Plan &p, const DenseArgs &d, const MergeOpts &o, cudaStream_t st);
swift_status band_timeout_flag(int *flag, int reset);
swift_status run_rowwise(Plan &p, RowLayout &L, const DenseArgs &a, cudaStream_t st);
swift_status run_merge(Plan &p, RowLayout &L, const DenseArgs &d, const MergeOpts &o,
                       cudaStream_t st);
swift_status build_merge_tasks(RowLayout &L, int U, cudaStream_t st);
// One merge-path pass over A for any of Y = A X, dA = SDDMM(dY, X) and (A symmetric)
// dX = A dY; dtype must equal the plan's value type.  SWIFT_ERR_UNSUPPORTED when the shape
// is not covered (the caller then uses the piece-based kernels).
swift_status run_bwd_merge(Plan &p, int N, swift_dtype dt, const void *X, int64_t ldx,
                           const void *dY, int64_t lddy, void *Y, int64_t ldy, void *dX,
                           int64_t lddx, void *dA, cudaStream_t st);
// Checks (once) whether A == A^T with equal values; result cached in p.symmetric.
swift_status check_symmetric(Plan &p, cudaStream_t st);
swift_status run_f64_reference(const Plan &p, int N, const double *B, int64_t ldb, double *C,
                               int64_t ldc, cudaStream_t st);
swift_status run_sddmm(Plan &p, int N, swift_dtype dt, const void *U, int64_t ldu,
                       const void *V, int64_t ldv, void *out, cudaStream_t st);
swift_status run_fused_fwd_sddmm(Plan &p, int N, swift_dtype dt, const void *X, int64_t ldx,
                                 const void *dY, int64_t lddy, void *Y, int64_t ldy, void *dA,
                                 cudaStream_t st);
swift_status zero_dense(void *C, int rows, int N, int64_t ld, swift_layout layout, size_t esz,
                        cudaStream_t st);

// ---------------------------------------------------------------- device helpers
__device__ __forceinline__ unsigned lanemask_lt() {
  unsigned m;
  asm volatile("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
  return m;
}

__device__ __forceinline__ int lane_id() { return threadIdx.x & 31; }

swift_status run_rowwise_external(Plan &p, RowLayout &L, const DenseArgs &d, void *scratch,
                                  int *counters, cudaStream_t st);

// Batched products (spmm_merge.cu): one launch record per member, a persistent grid.
size_t merge_args_size();
swift_status merge_batch_member(const Plan &p, RowLayout &L, int U, int N, const void *B, int64_t ldb,
                                void *C, int64_t ldc, void *args_out, int *shape, int64_t *items,
                                cudaStream_t st);
swift_status merge_batch_grid(int device, int *grid);
swift_status launch_merge_batch(const void *d_args, const int *d_shape, const int64_t *d_item_off,
                                int count, int grid, cudaStream_t st);

}  // namespace swift

// The opaque handle of the C ABI.
struct swift_plan {
  swift::Plan p;
};
