// capi.cu -- extern "C" entry points of libswiftb200.so (declared in include/swift_b200.h).
#include <algorithm>
#include <chrono>
#include <cstdlib>

#include "common.cuh"

namespace swift {

template <class VAL_T, class SLIDE>
swift_status export_slide(const Plan &p, SLIDE *out, int with_row_sort, float *blockratio,
                          cudaStream_t st);

namespace {
thread_local std::string g_last_error;
}

void set_last_error(const char *where, const char *what) {
  g_last_error = std::string(where) + ": " + what;
}

size_t plan_device_bytes(const Plan &p) {
  const DevBuf *bufs[] = {&p.rowptr, &p.colidx, &p.val, &p.cnt, &p.perm, &p.invperm, &p.sortnnz,
                          &p.sptr, &p.srow, &p.sval, &p.spos, &p.step_col, &p.step_base,
                          &p.step_tall, &p.step_tile_off, &p.item_tile, &p.tile_colidx,
                          &p.tile_depth, &p.tile_tall, &p.tile_format, &p.sortrowidx, &p.sortval,
                          &p.reside_ptr, &p.reside_row, &p.reside_val, &p.colorblk, &p.blkstart,
                          &p.blkstop, &p.blkptr, &p.rowcopy_b, &p.rowcopy_c, &p.g_row, &p.g_col,
                          &p.g_val, &p.band_tiles, &p.band_ptr, &p.band_idx, &p.band_val, &p.band_dst,
                          &p.band_mma[0], &p.band_mma[1]};
  size_t s = 0;
  for (const DevBuf *b : bufs) s += b->bytes;
  for (const RowLayout *L : {&p.fwd, &p.bwd, &p.band_rest}) {
    const DevBuf *lb[] = {&L->piece_row, &L->piece_idx, &L->long_first, &L->long_count,
                          &L->long_of_row, &L->counters, &L->scratch, &L->task_row,
                          &L->head_split, &L->tail_split, &L->split_row, &L->split_first,
                          &L->split_last, &L->split_cnt, &L->mscratch, &L->task_hdr, &L->eidx,
                          &L->sdd_hdr};
    for (const DevBuf *b : lb) s += b->bytes;
  }
  return s;
}

static swift_status check_device(int *sm_count) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) { set_last_error("cudaGetDevice", cudaGetErrorString(e)); return SWIFT_ERR_NO_DEVICE; }
  cudaDeviceProp prop;
  e = cudaGetDeviceProperties(&prop, dev);
  if (e != cudaSuccess) { set_last_error("cudaGetDeviceProperties", cudaGetErrorString(e)); return SWIFT_ERR_NO_DEVICE; }
  if (prop.major != 10) {
    set_last_error("device", "libswiftb200 is built for sm_100a (compute capability 10.x) only");
    return SWIFT_ERR_NO_DEVICE;
  }
  if (sm_count) *sm_count = prop.multiProcessorCount;
  return SWIFT_OK;
}

static size_t dtype_size(swift_dtype d) {
  switch (d) {
    case SWIFT_F32: return 4;
    case SWIFT_F64: return 8;
    case SWIFT_BF16:
    case SWIFT_F16: return 2;
  }
  return 0;
}

// Untuned row-walk parameters for layout L and dense width N: the default walk with tasks of
// the largest power of two up to 512 positions that still leaves about `waves` waves of 32
// warps per SM (narrow rows pack several tasks into a warp, so they want smaller tasks).
// Measured best: six for A's rows, three for the rows of A^T.
MergeOpts default_merge_opts(const Plan &p, const RowLayout &L, int N, swift_dtype dt, int waves) {
  MergeOpts o;
  const int esz = dt == SWIFT_F64 ? 8 : (dt == SWIFT_F32 ? 4 : 2);
  const int lanes = std::max(1, (N * esz + 15) / 16);
  int SG = 2;
  while (SG < lanes && SG < 32) SG <<= 1;
  const int64_t want = ((int64_t)L.nnz + L.rows) / ((int64_t)p.sm_count * 32 * (32 / SG) * waves);
  o.U = 64;
  while (o.U < 512 && 2 * o.U <= want) o.U *= 2;
  return o;
}

MergeOpts merge_opts_for(Plan &p, int N, swift_dtype dt) {
  std::lock_guard<std::mutex> g(p.mu);
  if (p.merge_override) return p.merge_opts;
  auto it = p.tuned_merge.find({N, (int)dt});
  return it != p.tuned_merge.end() ? it->second : default_merge_opts(p, p.fwd, N, dt, 6);
}

swift_status ensure_bwd(Plan &p, cudaStream_t st) {
  std::lock_guard<std::mutex> g(p.mu);
  if (p.bwd.built) return SWIFT_OK;
  return build_row_layout(p, p.bwd, true, st);
}

}  // namespace swift

using namespace swift;

namespace swift {
void note_use(Plan &p, cudaStream_t st) {
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  std::lock_guard<std::mutex> g(p.use_mu);
  if (cudaStreamIsCapturing(st, &cs) != cudaSuccess || cs != cudaStreamCaptureStatusNone) {
    p.sync_device_on_destroy = true;  // replayed later, on whatever stream the graph runs on
    return;
  }
  for (auto &u : p.uses)
    if (u.first == st) {
      cudaEventRecord(u.second, st);
      return;
    }
  cudaEvent_t ev = nullptr;
  if ((int)p.uses.size() >= Plan::kMaxUses ||
      cudaEventCreateWithFlags(&ev, cudaEventDisableTiming) != cudaSuccess) {
    p.sync_device_on_destroy = true;
    return;
  }
  cudaEventRecord(ev, st);
  p.uses.emplace_back(st, ev);
}

UseNote::~UseNote() { note_use(p, st); }

// The current device's allocation stream, made once per device and CUDA context: after a
// cudaDeviceReset the old stream died with its context, and a new one is made in the new one.
cudaStream_t alloc_stream() {
  static std::mutex mu;
  struct Entry {
    unsigned long long ctx = 0;
    cudaStream_t s = nullptr;
  };
  static Entry streams[128];
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 128) return nullptr;
  if (cudaSetDevice(dev) != cudaSuccess) return nullptr;  // the device's primary context current
  unsigned long long id = 0;
  if (current_context_id(&id) != SWIFT_OK) return nullptr;
  std::lock_guard<std::mutex> g(mu);
  Entry &e = streams[dev];
  if (!e.s || e.ctx != id) {
    e.s = nullptr;
    if (cudaStreamCreateWithFlags(&e.s, cudaStreamNonBlocking) != cudaSuccess) e.s = nullptr;
    e.ctx = id;
  }
  return e.s;
}

cudaStream_t &release_stream() {
  thread_local cudaStream_t s = nullptr;
  return s;
}

cudaStream_t release_stream_after(const std::vector<std::pair<cudaStream_t, cudaEvent_t>> &uses,
                                  bool sync_device) {
  if (sync_device) cudaDeviceSynchronize();
  cudaStream_t fs = nullptr;
  if (cudaStreamCreateWithFlags(&fs, cudaStreamNonBlocking) != cudaSuccess) return nullptr;
  for (auto &u : uses) cudaStreamWaitEvent(fs, u.second, 0);
  return fs;
}

Plan::~Plan() {
  // swift_plan_destroy has ordered the buffers' release after the plan's own work
  for (auto &u : uses) cudaEventDestroy(u.second);
}
}  // namespace swift

extern "C" {

const char *swift_status_string(swift_status s) {
  switch (s) {
    case SWIFT_OK: return "ok";
    case SWIFT_ERR_INVALID_ARG: return "invalid argument";
    case SWIFT_ERR_BAD_CSR: return "malformed CSR input";
    case SWIFT_ERR_BAD_PERM: return "column permutation does not sort the column counts";
    case SWIFT_ERR_UNSUPPORTED: return "unsupported dtype / layout / engine combination";
    case SWIFT_ERR_CUDA: return "CUDA error";
    case SWIFT_ERR_ALLOC: return "allocation failed";
    case SWIFT_ERR_OVERFLOW: return "size exceeds the int32 index range";
    case SWIFT_ERR_TIMEOUT: return "bounded device wait timed out";
    case SWIFT_ERR_NO_DEVICE: return "no sm_100 CUDA device";
    case SWIFT_ERR_VERIFY: return "result differs from the golden product";
    case SWIFT_ERR_IO: return "file cannot be opened or read";
    case SWIFT_ERR_FORMAT: return "malformed MatrixMarket file";
  }
  return "unknown status";
}

const char *swift_version(void) { return SWIFT_B200_VERSION; }

const char *swift_last_error(void) { return g_last_error.c_str(); }

swift_status swift_device_check(int *sm_count, int *cc_major, int *cc_minor) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) { set_last_error("cudaGetDevice", cudaGetErrorString(e)); return SWIFT_ERR_NO_DEVICE; }
  cudaDeviceProp prop;
  e = cudaGetDeviceProperties(&prop, dev);
  if (e != cudaSuccess) return SWIFT_ERR_NO_DEVICE;
  if (sm_count) *sm_count = prop.multiProcessorCount;
  if (cc_major) *cc_major = prop.major;
  if (cc_minor) *cc_minor = prop.minor;
  return prop.major == 10 ? SWIFT_OK : SWIFT_ERR_NO_DEVICE;
}

swift_status swift_plan_create(const swift_csr *A, const swift_plan_opts *opts,
                               swift_stream_t stream, swift_plan **out) {
  if (!A || !out) return SWIFT_ERR_INVALID_ARG;
  *out = nullptr;
  if (A->rows < 0 || A->cols < 0 || A->nnz < 0 || !A->rowptr) return SWIFT_ERR_INVALID_ARG;
  if (A->nnz > 0 && (!A->colidx || !A->val)) return SWIFT_ERR_INVALID_ARG;
  if (A->val_type != SWIFT_F32 && A->val_type != SWIFT_F64) return SWIFT_ERR_UNSUPPORTED;
  if (A->mem != SWIFT_HOST && A->mem != SWIFT_DEVICE) return SWIFT_ERR_INVALID_ARG;
  if (A->mem == SWIFT_HOST) {
    // cheap host-side validation before anything is uploaded
    if (A->rowptr[0] != 0 || A->rowptr[A->rows] != A->nnz) return SWIFT_ERR_BAD_CSR;
    for (int i = 0; i < A->rows; ++i)
      if (A->rowptr[i] > A->rowptr[i + 1]) return SWIFT_ERR_BAD_CSR;
    for (int i = 0; i < A->nnz; ++i)
      if (A->colidx[i] < 0 || A->colidx[i] >= A->cols) return SWIFT_ERR_BAD_CSR;
  }
  int sms = 0;
  SW_TRY(check_device(&sms));
  cudaStream_t st = S(stream);
  swift_plan *h = new (std::nothrow) swift_plan;
  if (!h) return SWIFT_ERR_ALLOC;
  Plan &p = h->p;
  p.M = A->rows; p.K = A->cols; p.nnz = A->nnz;
  cudaGetDevice(&p.device);
  p.sm_count = sms;
  p.val_type = A->val_type;
  p.vsz = dtype_size(A->val_type);
  p.long_row_split = (opts && opts->long_row_split > 0) ? opts->long_row_split : 128;
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  cudaEventRecord(e0, st);
  swift_status rc = build_from_csr(p, *A, opts, st);
  if (rc == SWIFT_OK) rc = build_row_layout(p, p.fwd, false, st);
  if (rc == SWIFT_OK && opts && opts->build_transpose) rc = ensure_bwd(p, st);
  cudaEventRecord(e1, st);
  if (rc == SWIFT_OK) {
    cudaError_t e = cudaEventSynchronize(e1);
    if (e != cudaSuccess) { set_last_error("plan build", cudaGetErrorString(e)); rc = SWIFT_ERR_CUDA; }
    float ms = 0;
    cudaEventElapsedTime(&ms, e0, e1);
    p.build_ms = ms;
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (rc != SWIFT_OK) {
    cudaStreamSynchronize(st);
    delete h;
    return rc;
  }
  *out = h;
  return SWIFT_OK;
}


swift_status swift_plan_destroy(swift_plan *plan) {
  if (!plan) return SWIFT_ERR_INVALID_ARG;
  Plan &p = plan->p;
  int prev = -1;
  cudaGetDevice(&prev);
  if (prev != p.device) cudaSetDevice(p.device);
  cudaStream_t fs;
  {
    std::lock_guard<std::mutex> g(p.use_mu);
    fs = release_stream_after(p.uses, p.sync_device_on_destroy);
  }
  if (prev >= 0 && prev != p.device) cudaSetDevice(prev);
  // the buffers go back to the pool once the plan's own streams reach this point (every stream
  // when a captured graph holds the plan); the host does not wait
  delete_releasing(plan, p.device, fs);
  return SWIFT_OK;
}

swift_status swift_plan_get_stats(const swift_plan *plan, swift_plan_stats *o) {
  if (!plan || !o) return SWIFT_ERR_INVALID_ARG;
  const Plan &p = plan->p;
  memset(o, 0, sizeof(*o));
  o->rows = p.M; o->cols = p.K; o->nnz = p.nnz;
  o->nsteps = p.nsteps; o->tilenum = p.tilenum; o->regular_nnz = p.tilenum * kTile;
  o->reside_col = p.reside_col; o->reside_nnz = p.reside_nnz; o->numblk = p.numblk;
  for (int i = 0; i < 3; ++i) o->fmt_count[i] = p.fmt_count[i];
  o->max_col_nnz = p.max_col; o->max_row_nnz = p.max_row; o->empty_cols = p.empty_cols;
  o->long_rows = p.fwd.long_rows; o->long_pieces = p.fwd.pieces; o->long_row_split = p.fwd.split;
  o->build_ms = p.build_ms;
  o->device_bytes = plan_device_bytes(p);
  return SWIFT_OK;
}

swift_status swift_plan_set_values(swift_plan *plan, const void *val, swift_memspace mem,
                                   swift_stream_t stream) {
  if (!plan || (mem != SWIFT_HOST && mem != SWIFT_DEVICE)) return SWIFT_ERR_INVALID_ARG;
  Plan &p = plan->p;
  if (!p.has_csr) return SWIFT_ERR_UNSUPPORTED;
  if (p.nnz > 0 && !val) return SWIFT_ERR_INVALID_ARG;
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  UseNote use_note{p, st};
  std::lock_guard<std::mutex> g(p.mu);
  p.grouped_built = false;  // rebuilt from the new slot values on its next use
  if (p.nnz > 0)
    SW_CHECK_CUDA(cudaMemcpyAsync(p.val.p, val, p.vsz * (size_t)p.nnz,
                                  mem == SWIFT_HOST ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToDevice, st));
  SW_TRY(band_refill(p, st));  // the band split's tiles and rest take the new values in place
  return refresh_values(p, st);
}

swift_status swift_plan_export_f32(const swift_plan *plan, swift_slide_matrix_f32 *out,
                                   int with_row_sort, float *blockratio) {
  if (!plan || !out) return SWIFT_ERR_INVALID_ARG;
  if (plan->p.val_type != SWIFT_F32) return SWIFT_ERR_UNSUPPORTED;
  return export_slide<float>(plan->p, out, with_row_sort, blockratio, nullptr);
}

swift_status swift_plan_export_f64(const swift_plan *plan, swift_slide_matrix_f64 *out,
                                   int with_row_sort, float *blockratio) {
  if (!plan || !out) return SWIFT_ERR_INVALID_ARG;
  if (plan->p.val_type != SWIFT_F64) return SWIFT_ERR_UNSUPPORTED;
  return export_slide<double>(plan->p, out, with_row_sort, blockratio, nullptr);
}

#define SWIFT_SLIDE_FREE(m)                                                                   \
  do {                                                                                        \
    void *ps[] = {m->sortval, m->sortrowidx, m->tile_ptr, m->tile_len, m->tile_colidx,        \
                  m->tile_tall, m->tile_format, m->countrow, m->segmentoffset, m->segptr,     \
                  m->seginfo, m->seglength, m->sortrowindex, m->val_position, m->val_offset,  \
                  m->reside_cscptr, m->reside_cscrowidx, m->reside_val, m->colorblk,          \
                  m->blkstart, m->blkstop, m->blkptr};                                        \
    for (void *q : ps) free(q);                                                               \
    memset(m, 0, sizeof(*m));                                                                 \
  } while (0)

void swift_slide_free_f32(swift_slide_matrix_f32 *m) { if (m) SWIFT_SLIDE_FREE(m); }
void swift_slide_free_f64(swift_slide_matrix_f64 *m) { if (m) SWIFT_SLIDE_FREE(m); }

swift_status swift_plan_export_sorted(const swift_plan *plan, int *perm, int *sortnnz,
                                      int *sortrowidx_tmp, void *sortval_tmp) {
  if (!plan) return SWIFT_ERR_INVALID_ARG;
  const Plan &p = plan->p;
  if (!p.has_csr) return SWIFT_ERR_UNSUPPORTED;
  if (perm) SW_CHECK_CUDA(cudaMemcpy(perm, p.perm.p, sizeof(int) * (size_t)p.K, cudaMemcpyDeviceToHost));
  if (sortnnz) SW_CHECK_CUDA(cudaMemcpy(sortnnz, p.sortnnz.p, sizeof(int) * (size_t)p.K, cudaMemcpyDeviceToHost));
  if (sortrowidx_tmp) SW_CHECK_CUDA(cudaMemcpy(sortrowidx_tmp, p.srow.p, sizeof(int) * (size_t)p.nnz, cudaMemcpyDeviceToHost));
  if (sortval_tmp) SW_CHECK_CUDA(cudaMemcpy(sortval_tmp, p.sval.p, p.vsz * (size_t)p.nnz, cudaMemcpyDeviceToHost));
  return SWIFT_OK;
}

static swift_status check_dense(const swift_plan *plan, int N, swift_dtype dt, const void *B,
                                int64_t ldb, swift_layout bl, int brows, const void *C,
                                int64_t ldc, swift_layout cl, int crows) {
  if (!plan || N < 0) return SWIFT_ERR_INVALID_ARG;
  if (dtype_size(dt) == 0) return SWIFT_ERR_INVALID_ARG;
  if ((bl != SWIFT_ROW_MAJOR && bl != SWIFT_COL_MAJOR) || (cl != SWIFT_ROW_MAJOR && cl != SWIFT_COL_MAJOR))
    return SWIFT_ERR_INVALID_ARG;
  if (N == 0) return SWIFT_OK;
  if ((brows > 0 && !B) || (crows > 0 && !C)) return SWIFT_ERR_INVALID_ARG;
  if (ldb < (bl == SWIFT_ROW_MAJOR ? N : std::max(brows, 1))) return SWIFT_ERR_INVALID_ARG;
  if (ldc < (cl == SWIFT_ROW_MAJOR ? N : std::max(crows, 1))) return SWIFT_ERR_INVALID_ARG;
  const Plan &p = plan->p;
  if (p.val_type == SWIFT_F64 && dt != SWIFT_F64) return SWIFT_ERR_UNSUPPORTED;
  if (p.val_type == SWIFT_F32 && dt == SWIFT_F64) return SWIFT_ERR_UNSUPPORTED;
  return SWIFT_OK;
}

swift_status swift_spmm(const swift_plan *plan, swift_engine engine, int N, swift_dtype dtype,
                        const void *B, int64_t ldb, swift_layout b_layout, int b_presorted,
                        void *C, int64_t ldc, swift_layout c_layout, swift_stream_t stream) {
  SW_TRY(check_dense(plan, N, dtype, B, ldb, b_layout, plan ? plan->p.K : 0, C, ldc, c_layout,
                     plan ? plan->p.M : 0));
  Plan &p = const_cast<Plan &>(plan->p);
  DenseArgs d;
  d.N = N; d.dtype = dtype; d.B = B; d.ldb = ldb; d.b_layout = b_layout; d.b_presorted = b_presorted != 0;
  d.C = C; d.ldc = ldc; d.c_layout = c_layout;
  cudaStream_t st = S(stream);
  UseNote use_note{p, st};
  const bool row_ok = p.has_csr && b_layout == SWIFT_ROW_MAJOR && c_layout == SWIFT_ROW_MAJOR && !b_presorted;
  // Column-major operands: in that layout each nonzero's N contributions land M elements apart,
  // so the row walk runs on row-major copies instead (B transposed in, C transposed out through
  // plan-held buffers, like the plan's other scratch); the tiled engine keeps the direct
  // column-major kernel.
  const bool via_rows = p.has_csr && !b_presorted && !row_ok && p.M > 0 && N > 0 &&
                        (engine == SWIFT_ENGINE_ROWWISE || (engine == SWIFT_ENGINE_AUTO && [&] {
                           std::lock_guard<std::mutex> g(p.mu);
                           auto it = p.tuned.find({N, (int)dtype});
                           return it == p.tuned.end() || it->second == SWIFT_ENGINE_ROWWISE ||
                                  it->second == SWIFT_ENGINE_BAND;
                         }()));
  if (via_rows) {
    const size_t esz = dtype == SWIFT_F64 ? 8 : (dtype == SWIFT_F32 ? 4 : 2);
    DenseArgs r = d;
    r.b_layout = r.c_layout = SWIFT_ROW_MAJOR;
    {
      std::lock_guard<std::mutex> g(p.mu);
      const size_t nb = esz * (size_t)p.K * N, nc = esz * (size_t)p.M * N;
      if (b_layout == SWIFT_COL_MAJOR && p.rowcopy_b.bytes < nb) SW_TRY(p.rowcopy_b.alloc(nb));
      if (c_layout == SWIFT_COL_MAJOR && p.rowcopy_c.bytes < nc) SW_TRY(p.rowcopy_c.alloc(nc));
    }
    if (b_layout == SWIFT_COL_MAJOR) {
      SW_TRY(transpose_dense(B, p.K, N, ldb, p.rowcopy_b.p, N, esz, st));
      r.B = p.rowcopy_b.p;
      r.ldb = N;
    }
    if (c_layout == SWIFT_COL_MAJOR) {
      r.C = p.rowcopy_c.p;
      r.ldc = N;
    }
    SW_TRY(run_merge(p, p.fwd, r, merge_opts_for(p, N, dtype), st));
    if (c_layout == SWIFT_COL_MAJOR) SW_TRY(transpose_dense(p.rowcopy_c.p, N, p.M, N, C, ldc, esz, st));
    return SWIFT_OK;
  }
  if (engine == SWIFT_ENGINE_AUTO) {
    engine = row_ok ? SWIFT_ENGINE_ROWWISE : SWIFT_ENGINE_TILED;
    std::lock_guard<std::mutex> g(p.mu);
    auto it = p.tuned.find({N, (int)dtype});
    if (it != p.tuned.end() && (it->second == SWIFT_ENGINE_TILED || row_ok)) engine = it->second;
    if (engine == SWIFT_ENGINE_BAND && !band_operands_ok(p, d)) engine = SWIFT_ENGINE_ROWWISE;
  }
  if (engine == SWIFT_ENGINE_BAND) return run_band(p, d, merge_opts_for(p, N, dtype), st);
  if (engine == SWIFT_ENGINE_ROWWISE) {
    if (!row_ok) return SWIFT_ERR_UNSUPPORTED;
    if (p.M == 0) return SWIFT_OK;
    return run_merge(p, p.fwd, d, merge_opts_for(p, N, dtype), st);
  }
  if (engine == SWIFT_ENGINE_TILED) return run_tiled(p, d, 0, st);
  if (engine == SWIFT_ENGINE_TILED_GROUPED) {
    if (b_layout != SWIFT_ROW_MAJOR || c_layout != SWIFT_ROW_MAJOR) return SWIFT_ERR_UNSUPPORTED;
    if (dtype == SWIFT_BF16 || dtype == SWIFT_F16) return SWIFT_ERR_UNSUPPORTED;
    {
      std::lock_guard<std::mutex> g(p.mu);
      if (!p.grouped_built) SW_TRY(build_grouped(p, nullptr, nullptr, st));
    }
    return run_tiled(p, d, 0, st, true);
  }
  return SWIFT_ERR_INVALID_ARG;
}

swift_status swift_spmm_scaled(const swift_plan *plan, int N, swift_dtype dtype, const void *B, int64_t ldb,
                               const float *b_scale, void *C, int64_t ldc, float *c_scale,
                               swift_stream_t stream) {
  SW_TRY(check_dense(plan, N, dtype, B, ldb, SWIFT_ROW_MAJOR, plan ? plan->p.K : 0, C, ldc, SWIFT_ROW_MAJOR,
                     plan ? plan->p.M : 0));
  if (dtype != SWIFT_BF16 && dtype != SWIFT_F16) return SWIFT_ERR_UNSUPPORTED;
  Plan &p = const_cast<Plan &>(plan->p);
  if (!p.has_csr) return SWIFT_ERR_UNSUPPORTED;
  if (N == 0 || p.M == 0) return SWIFT_OK;
  if (!c_scale) return SWIFT_ERR_INVALID_ARG;
  DenseArgs d;
  d.N = N; d.dtype = dtype; d.B = B; d.ldb = ldb; d.C = C; d.ldc = ldc;
  d.b_scale = b_scale;
  d.c_scale = c_scale;
  UseNote use_note{p, S(stream)};
  return run_merge(p, p.fwd, d, merge_opts_for(p, N, dtype), S(stream));
}

swift_status swift_spmm_transposed(const swift_plan *plan, int N, swift_dtype dtype,
                                   const void *Y, int64_t ldy, void *X, int64_t ldx,
                                   swift_stream_t stream) {
  SW_TRY(check_dense(plan, N, dtype, Y, ldy, SWIFT_ROW_MAJOR, plan ? plan->p.M : 0, X, ldx,
                     SWIFT_ROW_MAJOR, plan ? plan->p.K : 0));
  Plan &p = const_cast<Plan &>(plan->p);
  if (!p.has_csr) return SWIFT_ERR_UNSUPPORTED;
  cudaStream_t st = S(stream);
  UseNote use_note{p, st};
  SW_TRY(ensure_bwd(p, st));
  if (p.K == 0 || N == 0) return SWIFT_OK;
  DenseArgs d;
  d.N = N; d.dtype = dtype; d.B = Y; d.ldb = ldy; d.C = X; d.ldc = ldx;
  return run_merge(p, p.bwd, d, default_merge_opts(p, p.bwd, N, dtype, 3), st);
}

swift_status swift_sddmm(const swift_plan *plan, int N, swift_dtype dtype, const void *U,
                         int64_t ldu, const void *V, int64_t ldv, void *out,
                         swift_stream_t stream) {
  SW_TRY(check_dense(plan, N, dtype, V, ldv, SWIFT_ROW_MAJOR, plan ? plan->p.K : 0, U, ldu,
                     SWIFT_ROW_MAJOR, plan ? plan->p.M : 0));
  Plan &p = const_cast<Plan &>(plan->p);
  if (!p.has_csr) return SWIFT_ERR_UNSUPPORTED;
  if (p.nnz > 0 && !out) return SWIFT_ERR_INVALID_ARG;
  if (p.nnz == 0) return SWIFT_OK;
  cudaStream_t st = S(stream);
  UseNote use_note{p, st};
  if (N == 0) {
    SW_CHECK_CUDA(cudaMemsetAsync(out, 0, p.vsz * (size_t)p.nnz, st));
    return SWIFT_OK;
  }
  const swift_status rc = run_bwd_merge(p, N, dtype, V, ldv, U, ldu, nullptr, 0, nullptr, 0, out, st);
  if (rc != SWIFT_ERR_UNSUPPORTED) return rc;
  return run_sddmm(p, N, dtype, U, ldu, V, ldv, out, st);
}

swift_status swift_plan_set_symmetry(swift_plan *plan, int use) {
  if (!plan || (use != 0 && use != 1)) return SWIFT_ERR_INVALID_ARG;
  std::lock_guard<std::mutex> g(plan->p.mu);
  plan->p.use_symmetry = use;
  return SWIFT_OK;
}

swift_status swift_plan_is_symmetric(swift_plan *plan, int *symmetric, swift_stream_t stream) {
  if (!plan || !symmetric) return SWIFT_ERR_INVALID_ARG;
  UseNote use_note{plan->p, S(stream)};
  SW_TRY(check_symmetric(plan->p, S(stream)));
  *symmetric = plan->p.symmetric;
  return SWIFT_OK;
}

swift_status swift_fused_forward_backward(const swift_plan *plan, int N, swift_dtype dtype,
                                          const void *X, int64_t ldx, const void *dY,
                                          int64_t lddy, void *Y, int64_t ldy, void *dX,
                                          int64_t lddx, void *dA, swift_stream_t stream) {
  if (!plan || !X || !dY) return SWIFT_ERR_INVALID_ARG;
  Plan &p = const_cast<Plan &>(plan->p);
  if (!p.has_csr) return SWIFT_ERR_UNSUPPORTED;
  if (dtype != SWIFT_F32 && dtype != SWIFT_F64) return SWIFT_ERR_UNSUPPORTED;
  SW_TRY(check_dense(plan, N, dtype, X, ldx, SWIFT_ROW_MAJOR, p.K, dY, lddy, SWIFT_ROW_MAJOR, p.M));
  cudaStream_t st = S(stream);
  UseNote use_note{p, st};
  if (N == 0) return SWIFT_OK;
  if (Y && dA && dX && p.use_symmetry) {
    // A == A^T with equal values: dX = A dY joins the same pass over A
    SW_TRY(check_symmetric(p, st));
    if (p.symmetric == 1) {
      const swift_status rc = run_bwd_merge(p, N, dtype, X, ldx, dY, lddy, Y, ldy, dX, lddx, dA, st);
      if (rc != SWIFT_ERR_UNSUPPORTED) return rc;
    }
  }
  if (Y || dA) {
    swift_status rc = SWIFT_ERR_UNSUPPORTED;
    if (Y && dA) rc = run_bwd_merge(p, N, dtype, X, ldx, dY, lddy, Y, ldy, nullptr, 0, dA, st);
    if (rc != SWIFT_ERR_UNSUPPORTED) SW_TRY(rc);
    else if (Y && dA) SW_TRY(run_fused_fwd_sddmm(p, N, dtype, X, ldx, dY, lddy, Y, ldy, dA, st));
    else if (Y) {
      DenseArgs d;
      d.N = N; d.dtype = dtype; d.B = X; d.ldb = ldx; d.C = Y; d.ldc = ldy;
      SW_TRY(run_rowwise(p, p.fwd, d, st));
    } else SW_TRY(run_sddmm(p, N, dtype, dY, lddy, X, ldx, dA, st));
  }
  if (dX) {
    SW_TRY(ensure_bwd(p, st));
    DenseArgs d;
    d.N = N; d.dtype = dtype; d.B = dY; d.ldb = lddy; d.C = dX; d.ldc = lddx;
    SW_TRY(run_merge(p, p.bwd, d, default_merge_opts(p, p.bwd, N, dtype, 3), st));
  }
  return SWIFT_OK;
}

swift_status swift_spmm_f64_reference(const swift_plan *plan, int N, const double *B,
                                      int64_t ldb, double *C, int64_t ldc,
                                      swift_stream_t stream) {
  if (!plan || N < 0 || (N > 0 && (!B || !C)) || ldb < N || ldc < N) return SWIFT_ERR_INVALID_ARG;
  UseNote use_note{const_cast<Plan &>(plan->p), S(stream)};
  return run_f64_reference(plan->p, N, B, ldb, C, ldc, S(stream));
}

swift_status swift_plan_autotune(swift_plan *plan, int N, swift_dtype dtype, const void *B,
                                 void *C, swift_stream_t stream, double *best_ms,
                                 swift_engine *best_engine) {
  if (!plan || !B || !C || N <= 0) return SWIFT_ERR_INVALID_ARG;
  Plan &p = plan->p;
  cudaStream_t st = S(stream);
  UseNote use_note{p, st};
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  struct Cand {
    swift_engine eng;
    MergeOpts mo;
  };
  std::vector<Cand> cands;
  if (dtype != SWIFT_BF16 && dtype != SWIFT_F16) {
    cands.push_back({SWIFT_ENGINE_TILED, MergeOpts{}});
    cands.push_back({SWIFT_ENGINE_TILED_GROUPED, MergeOpts{}});
  }
  if (p.has_csr && p.val_type == SWIFT_F32 && dtype != SWIFT_F64 && N >= 128 && N % 4 == 0) {
    int w = -1;
    {
      std::lock_guard<std::mutex> g(p.mu);
      if (band_profile(p, st) == SWIFT_OK) w = p.band_w;
    }
    if (w >= 0) {
      // the band engine's rest walk: task size x vector width (the tiles take no parameters)
      for (int U : {256, 512, 1024})
        for (int vb : {16, 32}) {
          MergeOpts mo;
          mo.U = U;
          mo.unroll = 4;
          mo.vbytes = vb;
          mo.kernel = 2;
          cands.push_back({SWIFT_ENGINE_BAND, mo});
        }
    }
  }
  if (p.has_csr) {
    // task size (the work-balance grain) x (loads in flight, vector bytes, kernel variant)
    const int shapes[][3] = {{4, 16, 1}, {8, 16, 1}, {4, 32, 1}, {4, 16, 2}, {4, 32, 2}};
    for (int U : {128, 256, 512, 1024})
      for (const auto &sh : shapes) {
        MergeOpts mo;
        mo.U = U;
        mo.unroll = sh[0];
        mo.vbytes = sh[1];
        mo.kernel = sh[2];
        cands.push_back({SWIFT_ENGINE_ROWWISE, mo});
      }
  }
  const bool saved_override = p.merge_override;
  const MergeOpts saved_opts = p.merge_opts;
  // ms per product of candidate c over `reps` launches (after warm-up), or < 0 if it fails
  auto time_cand = [&](const Cand &c, int warm, int reps) -> double {
    p.merge_override = true;
    p.merge_opts = c.mo;
    swift_status rc = SWIFT_OK;
    for (int w = 0; w < warm && rc == SWIFT_OK; ++w)
      rc = swift_spmm(plan, c.eng, N, dtype, B, N, SWIFT_ROW_MAJOR, 0, C, N, SWIFT_ROW_MAJOR, stream);
    if (rc != SWIFT_OK) return -1.0;
    cudaEventRecord(e0, st);
    for (int r = 0; r < reps; ++r)
      swift_spmm(plan, c.eng, N, dtype, B, N, SWIFT_ROW_MAJOR, 0, C, N, SWIFT_ROW_MAJOR, stream);
    cudaEventRecord(e1, st);
    if (cudaEventSynchronize(e1) != cudaSuccess) return -1.0;
    float ms = 0;
    cudaEventElapsedTime(&ms, e0, e1);
    return ms / reps;
  };
  // a short pass over every candidate, then a longer one over the three fastest (the
  // candidates differ by a few per cent, about the noise of a short pass)
  std::vector<std::pair<double, size_t>> first;
  for (size_t i = 0; i < cands.size(); ++i) {
    const double ms = time_cand(cands[i], 2, 5);
    if (ms >= 0) first.push_back({ms, i});
  }
  std::sort(first.begin(), first.end());
  double best = 1e300;
  Cand win{SWIFT_ENGINE_TILED, MergeOpts{}};
  for (size_t k = 0; k < first.size() && k < 3; ++k) {
    const double ms = time_cand(cands[first[k].second], 1, 20);
    if (ms >= 0 && ms < best) { best = ms; win = cands[first[k].second]; }
  }
  p.merge_override = saved_override;
  p.merge_opts = saved_opts;
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (best >= 1e300) return SWIFT_ERR_UNSUPPORTED;
  {
    std::lock_guard<std::mutex> g(p.mu);
    p.tuned[{N, (int)dtype}] = win.eng;
    if (win.eng == SWIFT_ENGINE_ROWWISE || win.eng == SWIFT_ENGINE_BAND) p.tuned_merge[{N, (int)dtype}] = win.mo;
  }
  if (best_ms) *best_ms = best;
  if (best_engine) *best_engine = win.eng;
  return SWIFT_OK;
}

swift_status swift_plan_band_profile(swift_plan *plan, long long *hist, int *half_width,
                                     swift_stream_t stream) {
  if (!plan) return SWIFT_ERR_INVALID_ARG;
  Plan &p = plan->p;
  if (!p.has_csr) return SWIFT_ERR_UNSUPPORTED;
  cudaStream_t st = S(stream);
  UseNote use_note{p, st};
  std::lock_guard<std::mutex> g(p.mu);
  SW_TRY(band_profile(p, st));
  if (hist)
    for (int d = 0; d <= SWIFT_BAND_PROFILE_MAX; ++d) hist[d] = p.band_hist[d];
  if (half_width) *half_width = p.band_w;
  return SWIFT_OK;
}

swift_status swift_band_timeout_flag(int *flag, int reset) { return band_timeout_flag(flag, reset); }

swift_status swift_plan_set_rowwise_params(swift_plan *plan, int task_size, int loads_in_flight,
                                           int vector_bytes, int kernel) {
  if (!plan || task_size < 0 || kernel < 0 || kernel > 4) return SWIFT_ERR_INVALID_ARG;
  if (vector_bytes != 0 && vector_bytes != 4 && vector_bytes != 16 && vector_bytes != 32)
    return SWIFT_ERR_INVALID_ARG;
  Plan &p = plan->p;
  std::lock_guard<std::mutex> g(p.mu);
  if (task_size == 0) {
    p.merge_override = false;
    p.merge_opts = MergeOpts{};
    return SWIFT_OK;
  }
  p.merge_override = true;
  p.merge_opts.U = task_size;
  p.merge_opts.unroll = loads_in_flight > 0 ? loads_in_flight : 4;
  p.merge_opts.vbytes = vector_bytes;
  p.merge_opts.kernel = kernel;
  return SWIFT_OK;
}

swift_status swift_plan_get_rowwise_params(swift_plan *plan, int N, swift_dtype dtype,
                                           int *task_size, int *loads_in_flight,
                                           int *vector_bytes, int *kernel) {
  if (!plan) return SWIFT_ERR_INVALID_ARG;
  MergeOpts o = merge_opts_for(plan->p, N, dtype);
  if (task_size) *task_size = o.U;
  if (loads_in_flight) *loads_in_flight = o.unroll;
  if (vector_bytes) *vector_bytes = o.vbytes;
  if (kernel) *kernel = o.kernel;
  return SWIFT_OK;
}

}  // extern "C"
