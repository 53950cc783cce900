// compat.cu -- the reference's preprocessing and SpMM functions with its host-buffer calling
// convention (swift_ref_* in swift_b200.h; C++ shims with the exact reference signatures in
// include/swift_compat.h).  Inputs and outputs are host arrays; device buffers live only for
// the call; every stage runs on the GPU with this library's kernels.
//
//   csr_to_csc        src/gpu_csr2csc.h:51-157
//   col_sort/ColSort  src/coo2csc.h:82-134, src/ColSort_cuda.h:48-143
//   formattransation  src/coo2csc.h:137-435      formatTransform src/formatTransform_cuda.h:198-435
//   block_catgory     src/block_catgory.h:1-160  balance src/balance.h:1-69
//   row_idx_sort      src/back_process.h:23-229
//   Swift_GPU (0), Swift_gpu1 (1), Swift_gpu2 (2), Swift_GPU_3 (3), Swift_GPU_4 (4)
//                     src/Swift.h:184, src/Swift_gpu_col_major.h:171,
//                     src/Swift_gpu_row_major.h:136, src/Swift_3.h:216, src/Swift_4.h:305
#include <cstdlib>

#include "common.cuh"

namespace swift {

template <class VAL_T, class SLIDE>
swift_status export_slide(const Plan &p, SLIDE *out, int with_row_sort, float *blockratio,
                          cudaStream_t st);

namespace {

// Sorted CSC gather by column order: one warp per sorted column i copies column perm[i].
template <class T>
__global__ void colsort_gather_kernel(const int *__restrict__ perm, const int *__restrict__ colptr,
                                      const int *__restrict__ sptr, const int *__restrict__ rowidx,
                                      const T *__restrict__ val, int K, int *__restrict__ srow,
                                      T *__restrict__ sval) {
  const int warps = (gridDim.x * blockDim.x) >> 5;
  const int l = threadIdx.x & 31;
  for (int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < K; i += warps) {
    const int c = perm[i], src = colptr[c], len = colptr[c + 1] - src, dst = sptr[i];
    for (int j = l; j < len; j += 32) {
      srow[dst + j] = rowidx[src + j];
      sval[dst + j] = val[src + j];
    }
  }
}

// sort_dense[i, :] = dense[perm[i], :] (row-major K x N), src/ColSort_cuda.h:9-21.
template <class T>
__global__ void dense_row_gather_kernel(const int *__restrict__ perm, const T *__restrict__ B,
                                        int K, int N, T *__restrict__ out) {
  const int warps = (gridDim.x * blockDim.x) >> 5;
  const int l = threadIdx.x & 31;
  for (int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < K; i += warps) {
    const T *src = B + (int64_t)perm[i] * N;
    T *dst = out + (int64_t)i * N;
    for (int j = l; j < N; j += 32) dst[j] = src[j];
  }
}

int grid_warps(int64_t n) {
  return (int)std::max<int64_t>(1, std::min<int64_t>((n * 32 + 255) / 256, 148 * 32));
}

template <class T> swift_status upload(DevBuf &d, const T *h, size_t n, cudaStream_t st) {
  SW_TRY(d.alloc(sizeof(T) * n));
  if (n) SW_CHECK_CUDA(cudaMemcpyAsync(d.p, h, sizeof(T) * n, cudaMemcpyHostToDevice, st));
  return SWIFT_OK;
}
template <class T> swift_status download(T *h, const void *d, size_t n, cudaStream_t st) {
  if (n) SW_CHECK_CUDA(cudaMemcpyAsync(h, d, sizeof(T) * n, cudaMemcpyDeviceToHost, st));
  return SWIFT_OK;
}
template <class T> T *host_array(size_t n) { return static_cast<T *>(calloc(n ? n : 1, sizeof(T))); }

struct Timer {
  cudaEvent_t a = nullptr, b = nullptr;
  cudaStream_t st;
  explicit Timer(cudaStream_t s) : st(s) {
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    cudaEventRecord(a, st);
  }
  float stop() {
    cudaEventRecord(b, st);
    cudaEventSynchronize(b);
    float ms = 0;
    cudaEventElapsedTime(&ms, a, b);
    return ms;
  }
  ~Timer() {
    cudaEventDestroy(a);
    cudaEventDestroy(b);
  }
};

template <class T> swift_dtype dtype_of();
template <> swift_dtype dtype_of<float>() { return SWIFT_F32; }
template <> swift_dtype dtype_of<double>() { return SWIFT_F64; }

swift_status device_ok() {
  int sms = 0, major = 0, minor = 0;
  return swift_device_check(&sms, &major, &minor);
}

// ------------------------------------------------------------------ csr_to_csc
template <class T>
swift_status ref_csr_to_csc(float *ms, int m, int n, int nnz, const T *csr_val, const int *rowptr,
                            const int *colind, T *csc_val, int *csc_row_ind, int *csc_col_ptr,
                            int *nnzpercol) {
  if (m < 0 || n < 0 || nnz < 0 || !rowptr || (nnz && (!colind || !csr_val))) return SWIFT_ERR_INVALID_ARG;
  SW_TRY(device_ok());
  cudaStream_t st = nullptr;
  DevBuf rp, ci, v, cp, ri, cv, cnt;
  SW_TRY(upload(rp, rowptr, (size_t)m + 1, st));
  SW_TRY(upload(ci, colind, (size_t)nnz, st));
  SW_TRY(upload(v, csr_val, (size_t)nnz, st));
  SW_TRY(cp.alloc(sizeof(int) * ((size_t)n + 1)));
  SW_TRY(ri.alloc(sizeof(int) * (size_t)nnz));
  SW_TRY(cv.alloc(sizeof(T) * (size_t)nnz));
  SW_TRY(cnt.alloc(sizeof(int) * (size_t)n));
  Timer tm(st);
  SW_TRY(csr_to_csc_device(rp.as<int>(), ci.as<int>(), v.p, sizeof(T) == 8, m, n, nnz, cp.as<int>(),
                           ri.as<int>(), cv.p, cnt.as<int>(), st));
  const float t = tm.stop();
  if (ms) *ms = t;
  SW_TRY(download(csc_col_ptr, cp.p, (size_t)n + 1, st));
  SW_TRY(download(csc_row_ind, ri.p, (size_t)nnz, st));
  SW_TRY(download(csc_val, cv.p, (size_t)nnz, st));
  if (nnzpercol) SW_TRY(download(nnzpercol, cnt.p, (size_t)n, st));
  SW_CHECK_CUDA(cudaStreamSynchronize(st));
  return SWIFT_OK;
}

// ------------------------------------------------------------------ col_sort / ColSort
template <class T>
swift_status ref_col_sort(float *ms, int colA, int nnz, int width, const int *nnzpercol,
                          const int *csccolptr, const int *cscrowidx, const T *cscval,
                          int *sortrowidx_tmp, T *sortval_tmp, int *sortnnz_tmp, const T *dense,
                          T *sort_dense) {
  if (colA < 0 || nnz < 0 || width < 0 || !nnzpercol || !csccolptr || !sortnnz_tmp) return SWIFT_ERR_INVALID_ARG;
  SW_TRY(device_ok());
  cudaStream_t st = nullptr;
  DevBuf cnt, cp, ri, cv, perm, inv, sn, sp, sr, sv, B, sB;
  SW_TRY(upload(cnt, nnzpercol, (size_t)colA, st));
  SW_TRY(upload(cp, csccolptr, (size_t)colA + 1, st));
  SW_TRY(upload(ri, cscrowidx, (size_t)nnz, st));
  SW_TRY(upload(cv, cscval, (size_t)nnz, st));
  SW_TRY(perm.alloc(sizeof(int) * (size_t)colA));
  SW_TRY(inv.alloc(sizeof(int) * (size_t)colA));
  SW_TRY(sn.alloc(sizeof(int) * ((size_t)colA + 1)));
  SW_TRY(sp.alloc(sizeof(int) * ((size_t)colA + 1)));
  SW_TRY(sr.alloc(sizeof(int) * (size_t)nnz));
  SW_TRY(sv.alloc(sizeof(T) * (size_t)nnz));
  const bool with_dense = dense && sort_dense && width > 0;
  if (with_dense) {
    SW_TRY(upload(B, dense, (size_t)colA * width, st));
    SW_TRY(sB.alloc(sizeof(T) * (size_t)colA * width));
  }
  SW_CHECK_CUDA(cudaMemsetAsync(sn.p, 0, sn.bytes, st));
  Timer tm(st);
  SW_TRY(stable_column_order(cnt.as<int>(), colA, perm.as<int>(), inv.as<int>(), sn.as<int>(), nullptr, st));
  SW_TRY(scan_exclusive_i32(sn.as<int>(), sp.as<int>(), colA, st));
  if (colA > 0)
    colsort_gather_kernel<T><<<grid_warps(colA), 256, 0, st>>>(perm.as<int>(), cp.as<int>(), sp.as<int>(),
                                                               ri.as<int>(), cv.as<T>(), colA, sr.as<int>(),
                                                               sv.as<T>());
  SW_CHECK_LAUNCH();
  if (with_dense && colA > 0)
    dense_row_gather_kernel<T><<<grid_warps(colA), 256, 0, st>>>(perm.as<int>(), B.as<T>(), colA, width, sB.as<T>());
  SW_CHECK_LAUNCH();
  const float t = tm.stop();
  if (ms) *ms = t;
  SW_TRY(download(sortnnz_tmp, sn.p, (size_t)colA, st));
  if (sortrowidx_tmp) SW_TRY(download(sortrowidx_tmp, sr.p, (size_t)nnz, st));
  if (sortval_tmp) SW_TRY(download(sortval_tmp, sv.p, (size_t)nnz, st));
  if (with_dense) SW_TRY(download(sort_dense, sB.p, (size_t)colA * width, st));
  SW_CHECK_CUDA(cudaStreamSynchronize(st));
  return SWIFT_OK;
}

// A format-only plan from the sorted CSC (no CSR on the device).
template <class T>
swift_status plan_from_sorted(Plan &p, const int *sortrowidx_tmp, const T *sortval_tmp,
                              const int *sortnnz_tmp, int nnz, int rowA, int colA, cudaStream_t st) {
  p.M = rowA; p.K = colA; p.nnz = nnz;
  p.val_type = dtype_of<T>();
  p.vsz = sizeof(T);
  p.has_csr = false;
  SW_TRY(p.sortnnz.alloc(sizeof(int) * ((size_t)colA + 1)));
  SW_CHECK_CUDA(cudaMemsetAsync(p.sortnnz.p, 0, p.sortnnz.bytes, st));
  if (colA) SW_CHECK_CUDA(cudaMemcpyAsync(p.sortnnz.p, sortnnz_tmp, sizeof(int) * (size_t)colA, cudaMemcpyHostToDevice, st));
  SW_TRY(p.sptr.alloc(sizeof(int) * ((size_t)colA + 1)));
  SW_TRY(scan_exclusive_i32(p.sortnnz.as<int>(), p.sptr.as<int>(), colA, st));
  SW_TRY(upload(p.srow, sortrowidx_tmp, (size_t)nnz, st));
  SW_TRY(upload(p.sval, sortval_tmp, (size_t)nnz, st));
  return SWIFT_OK;
}

// ------------------------------------------------------------------ formattransation
template <class T, class SLIDE>
swift_status ref_formattransation(float *ms, SLIDE *m, const int *sortrowidx_tmp, const T *sortval_tmp,
                                  const int *sortnnz_tmp, int nnz, int rowA, int colA,
                                  double *reside_ratio, bool regular_only, int *h_count) {
  if (!m || nnz < 0 || colA < 0 || (nnz && (!sortrowidx_tmp || !sortval_tmp)) || (colA && !sortnnz_tmp))
    return SWIFT_ERR_INVALID_ARG;
  SW_TRY(device_ok());
  cudaStream_t st = nullptr;
  Plan p;
  SW_TRY(plan_from_sorted(p, sortrowidx_tmp, sortval_tmp, sortnnz_tmp, nnz, rowA, colA, st));
  Timer tm(st);
  SW_TRY(build_tiles(p, st));
  const float t = tm.stop();
  if (ms) *ms = t;
  const size_t T_ = (size_t)p.tilenum, nreg = T_ * kTile;
  m->tilenum = p.tilenum;
  m->regular_nnz = (int)nreg;
  m->tile_ptr = host_array<int>(T_ + 1);
  m->tile_len = host_array<int>(T_);
  for (size_t i = 0; i <= T_; ++i) m->tile_ptr[i] = (int)(i * kTile);
  for (size_t i = 0; i < T_; ++i) m->tile_len[i] = kTile;
  m->tile_colidx = host_array<int>(T_);
  SW_TRY(download(m->tile_colidx, p.tile_colidx.p, T_, st));
  // the reference's GPU transform sizes the slot arrays by nnz (src/formatTransform_cuda.h:370-380)
  const size_t slots = regular_only ? (size_t)std::max(nnz, (int)nreg) : nreg;
  m->sortrowidx = host_array<int>(slots);
  m->sortval = host_array<T>(slots);
  SW_TRY(download(m->sortrowidx, p.sortrowidx.p, nreg, st));
  SW_TRY(download(m->sortval, p.sortval.p, nreg, st));
  if (!regular_only) {
    m->tile_tall = host_array<int>(T_);
    SW_TRY(download(m->tile_tall, p.tile_tall.p, T_, st));
    m->reside_col = p.reside_col;
    m->reside_nnz = p.reside_nnz;
    m->reside_cscptr = host_array<int>((size_t)p.reside_col + 1);
    m->reside_cscrowidx = host_array<int>((size_t)p.reside_nnz);
    m->reside_val = host_array<T>((size_t)p.reside_nnz);
    SW_TRY(download(m->reside_cscptr, p.reside_ptr.p, (size_t)p.reside_col + 1, st));
    SW_TRY(download(m->reside_cscrowidx, p.reside_row.p, (size_t)p.reside_nnz, st));
    SW_TRY(download(m->reside_val, p.reside_val.p, (size_t)p.reside_nnz, st));
    if (reside_ratio) *reside_ratio = nnz ? (double)p.reside_nnz / (double)nnz : 0.0;
  }
  if (h_count) *h_count = p.nsteps;
  SW_CHECK_CUDA(cudaStreamSynchronize(st));
  return SWIFT_OK;
}

// A plan holding the regular tiles of a host slide_matrix.
template <class T, class SLIDE>
swift_status plan_from_tiles(Plan &p, const SLIDE *m, cudaStream_t st) {
  p.tilenum = m->tilenum;
  p.vsz = sizeof(T);
  p.val_type = dtype_of<T>();
  const size_t nreg = (size_t)m->tilenum * kTile;
  SW_TRY(upload(p.sortrowidx, m->sortrowidx, nreg, st));
  return SWIFT_OK;
}

// ------------------------------------------------------------------ block_catgory
template <class T, class SLIDE>
swift_status ref_block_catgory(SLIDE *m, double *shuffle_ratio) {
  if (!m || m->tilenum < 0 || (m->tilenum && !m->sortrowidx)) return SWIFT_ERR_INVALID_ARG;
  SW_TRY(device_ok());
  cudaStream_t st = nullptr;
  Plan p;
  SW_TRY((plan_from_tiles<T, SLIDE>(p, m, st)));
  SW_TRY(classify_tiles(p, st));
  DevBuf countrow, segoff, sri;
  int segsum = 0;
  SW_TRY(build_segments(p, countrow, segoff, sri, &segsum, st));
  const size_t T_ = (size_t)p.tilenum;
  m->tile_format = host_array<int>(T_);
  m->segsum = segsum;
  m->segmentoffset = host_array<int>((size_t)segsum + 1);
  m->sortrowindex = host_array<int>(T_ * kTile);
  SW_TRY(download(m->tile_format, p.tile_format.p, T_, st));
  SW_TRY(download(m->segmentoffset, segoff.p, (size_t)segsum + 1, st));
  SW_TRY(download(m->sortrowindex, sri.p, T_ * kTile, st));
  SW_CHECK_CUDA(cudaStreamSynchronize(st));
  if (shuffle_ratio) *shuffle_ratio = (double)p.fmt_count[0] / (double)p.tilenum;  // 0/0 like the reference
  return SWIFT_OK;
}

// ------------------------------------------------------------------ balance
template <class T, class SLIDE>
swift_status ref_balance(SLIDE *m, int n_reside, const int *cscptr) {
  if (!m || n_reside < 0 || n_reside > kTile || (n_reside && !cscptr)) return SWIFT_ERR_INVALID_ARG;
  SW_TRY(device_ok());
  cudaStream_t st = nullptr;
  Plan p;
  p.reside_col = n_reside;
  SW_TRY(upload(p.reside_ptr, cscptr, (size_t)n_reside + 1, st));
  SW_TRY(build_balance(p, cscptr, st));
  const size_t nb = (size_t)p.numblk;
  m->numblk = p.numblk;
  m->colorblk = host_array<unsigned>(nb);
  m->blkstart = host_array<int>(nb);
  m->blkstop = host_array<int>(nb);
  m->blkptr = host_array<int>(nb);
  SW_TRY(download(m->colorblk, p.colorblk.p, nb, st));
  SW_TRY(download(m->blkstart, p.blkstart.p, nb, st));
  SW_TRY(download(m->blkstop, p.blkstop.p, nb, st));
  SW_TRY(download(m->blkptr, p.blkptr.p, nb, st));
  SW_CHECK_CUDA(cudaStreamSynchronize(st));
  return SWIFT_OK;
}

// ------------------------------------------------------------------ row_idx_sort
template <class T, class SLIDE>
swift_status ref_row_idx_sort(SLIDE *m, float *blockratio) {
  if (!m || m->tilenum < 0 || (m->tilenum && !m->sortrowidx)) return SWIFT_ERR_INVALID_ARG;
  SW_TRY(device_ok());
  cudaStream_t st = nullptr;
  Plan p;
  SW_TRY((plan_from_tiles<T, SLIDE>(p, m, st)));
  DevBuf sorted, vpos, voff;
  SW_TRY(build_row_sort(p, sorted, vpos, voff, blockratio, st));
  const size_t nreg = (size_t)p.tilenum * kTile;
  m->val_position = host_array<int>(nreg);
  m->val_offset = host_array<int>(nreg);
  SW_TRY(download(m->val_position, vpos.p, nreg, st));
  SW_TRY(download(m->val_offset, voff.p, nreg, st));
  SW_TRY(download(m->sortrowidx, sorted.p, nreg, st));  // overwritten with the sorted keys
  SW_CHECK_CUDA(cudaStreamSynchronize(st));
  return SWIFT_OK;
}

// ------------------------------------------------------------------ Swift_GPU* products
// Every index the tiled kernels will follow, checked on the host before upload: tiles cover
// columns [tile_colidx, tile_colidx + 32) of K, slot rows lie in [0, M), the reside pointer is
// a monotone [0 .. reside_nnz] over at most 32 columns (reside column q is column K-1-q), and
// balance blocks stay inside their column.
template <class SLIDE>
swift_status check_slide(const SLIDE *m, int variant, int M, int K) {
  auto bad = [](const char *what) {
    set_last_error("slide_matrix", what);
    return SWIFT_ERR_INVALID_ARG;
  };
  // Swift_gpu1 runs before balance() in the reference's driver (test/k-32/FP32/main.cu:359-382),
  // so its slide_matrix still holds whatever malloc left in numblk/colorblk: variant 1 reads
  // neither field.
  if (m->tilenum < 0 || m->reside_col < 0 || m->reside_nnz < 0 || (variant != 1 && m->numblk < 0))
    return bad("negative size");
  const size_t nreg = (size_t)m->tilenum * kTile;
  if (m->tilenum > 0 && (!m->tile_colidx || !m->sortrowidx || !m->sortval)) return bad("missing tile arrays");
  for (int t = 0; t < m->tilenum; ++t)
    if (m->tile_colidx[t] < 0 || (int64_t)m->tile_colidx[t] + kTile > K) return bad("tile_colidx out of range");
  for (size_t j = 0; j < nreg; ++j)
    if (m->sortrowidx[j] < 0 || m->sortrowidx[j] >= M) return bad("sortrowidx out of range");
  if (m->reside_col > kTile || m->reside_col > K) return bad("reside_col above 32 or K");
  if (!m->reside_cscptr) {
    if (m->reside_col > 0 || m->reside_nnz > 0) return bad("missing reside_cscptr");
  } else {
    if (m->reside_cscptr[0] != 0 || m->reside_cscptr[m->reside_col] != m->reside_nnz) return bad("reside_cscptr ends");
    for (int q = 0; q < m->reside_col; ++q)
      if (m->reside_cscptr[q + 1] < m->reside_cscptr[q]) return bad("reside_cscptr not monotone");
  }
  if (m->reside_nnz > 0 && (!m->reside_cscrowidx || !m->reside_val)) return bad("missing reside arrays");
  for (int j = 0; j < m->reside_nnz; ++j)
    if (m->reside_cscrowidx[j] < 0 || m->reside_cscrowidx[j] >= M) return bad("reside row out of range");
  if (variant != 1 && m->colorblk && m->numblk > 0) {
    if (!m->blkstart || !m->blkstop) return bad("missing balance arrays");
    for (int b = 0; b < m->numblk; ++b) {
      const unsigned cb = m->colorblk[b];
      const int q = (int)(cb & 0x7fffffffu);
      if (q >= m->reside_col) return bad("balance block column out of range");
      if (cb >> 31) {
        const int lo = m->reside_cscptr[q], hi = m->reside_cscptr[q + 1];
        if (m->blkstart[b] < lo || m->blkstop[b] > hi || m->blkstart[b] > m->blkstop[b])
          return bad("balance block outside its column");
      }
    }
  }
  return SWIFT_OK;
}

template <class T, class SLIDE>
swift_status ref_spmm(int variant, const SLIDE *m, int rowA, int colA, int width, int nnz,
                      const T *h_B, T *h_C, float *ms) {
  if (!m || variant < 0 || variant > 4 || rowA < 0 || colA < 0 || width < 0 || !h_B || !h_C)
    return SWIFT_ERR_INVALID_ARG;
  SW_TRY(check_slide(m, variant, rowA, colA));
  SW_TRY(device_ok());
  cudaStream_t st = nullptr;
  Plan p;
  p.M = rowA; p.K = colA; p.nnz = nnz;
  p.val_type = dtype_of<T>();
  p.vsz = sizeof(T);
  p.tilenum = m->tilenum;
  const size_t nreg = (size_t)m->tilenum * kTile;
  SW_TRY(upload(p.tile_colidx, m->tile_colidx, (size_t)m->tilenum, st));
  SW_TRY(upload(p.sortrowidx, m->sortrowidx, nreg, st));
  SW_TRY(upload(p.sortval, m->sortval, nreg, st));
  // Swift_GPU_4 runs after row_idx_sort: sortrowidx holds each group's sorted rows and
  // val_position maps every original slot to its sorted one (src/back_process.h:23-229); the
  // grouped engine walks exactly that order
  const bool grouped = variant == 4 && m->val_position && nreg > 0;
  if (grouped) {
    DevBuf vpos;
    SW_TRY(upload(vpos, m->val_position, nreg, st));
    const swift_status rc = build_grouped(p, p.sortrowidx.as<int>(), vpos.as<int>(), st);
    if (rc != SWIFT_OK) {
      set_last_error("Swift_GPU_4", "val_position is not a permutation of each group of 8 tiles");
      return rc;
    }
  }
  p.reside_col = m->reside_col;
  p.reside_nnz = m->reside_nnz;
  SW_TRY(upload(p.reside_ptr, m->reside_cscptr, (size_t)m->reside_col + 1, st));
  SW_TRY(upload(p.reside_row, m->reside_cscrowidx, (size_t)m->reside_nnz, st));
  SW_TRY(upload(p.reside_val, m->reside_val, (size_t)m->reside_nnz, st));
  p.numblk = (variant == 1) ? 0 : (m->colorblk ? m->numblk : 0);
  if (p.numblk > 0) {
    SW_TRY(upload(p.colorblk, m->colorblk, (size_t)p.numblk, st));
    SW_TRY(upload(p.blkstart, m->blkstart, (size_t)p.numblk, st));
    SW_TRY(upload(p.blkstop, m->blkstop, (size_t)p.numblk, st));
  }
  SW_TRY(build_items(p, st));
  // Swift_gpu2 takes row-major B and C; the other variants column-major ones with leading
  // dimension = rows (src/main.cu:338-340).  A column-major product scatters every nonzero's
  // contribution over N columns rowA elements apart, so those variants transpose B to row-major,
  // run the row-major kernel and transpose C back; the reported time covers all three.
  const bool colmajor = variant != 2;
  DevBuf B, C, Bt, Ct;
  SW_TRY(upload(B, h_B, (size_t)colA * width, st));
  SW_TRY(C.alloc(sizeof(T) * (size_t)rowA * width));
  if (colmajor) {
    SW_TRY(Bt.alloc(sizeof(T) * (size_t)colA * width));
    SW_TRY(Ct.alloc(sizeof(T) * (size_t)rowA * width));
  }
  DenseArgs d;
  d.N = width; d.dtype = dtype_of<T>(); d.b_presorted = true;
  d.B = colmajor ? Bt.p : B.p;
  d.C = colmajor ? Ct.p : C.p;
  d.b_layout = d.c_layout = SWIFT_ROW_MAJOR;
  d.ldb = d.ldc = std::max(width, 1);
  Timer tm(st);
  if (colmajor) SW_TRY(transpose_dense(B.p, colA, width, colA, Bt.p, width, sizeof(T), st));
  SW_TRY(run_tiled(p, d, variant == 1 ? 1 : 0, st, grouped));
  if (colmajor) SW_TRY(transpose_dense(Ct.p, width, rowA, width, C.p, rowA, sizeof(T), st));
  const float t = tm.stop();
  if (ms) *ms = t;
  SW_TRY(download(h_C, C.p, (size_t)rowA * width, st));
  SW_CHECK_CUDA(cudaStreamSynchronize(st));
  return SWIFT_OK;
}

}  // namespace
}  // namespace swift

using namespace swift;

extern "C" {

swift_status swift_ref_csr_to_csc_f32(float *ms, int m, int n, int nnz, const float *csr_val,
                                      const int *csr_row_ptr, const int *csr_col_ind,
                                      float *csc_val, int *csc_row_ind, int *csc_col_ptr,
                                      int *nnzpercol) {
  return ref_csr_to_csc<float>(ms, m, n, nnz, csr_val, csr_row_ptr, csr_col_ind, csc_val, csc_row_ind,
                               csc_col_ptr, nnzpercol);
}
swift_status swift_ref_csr_to_csc_f64(float *ms, int m, int n, int nnz, const double *csr_val,
                                      const int *csr_row_ptr, const int *csr_col_ind,
                                      double *csc_val, int *csc_row_ind, int *csc_col_ptr,
                                      int *nnzpercol) {
  return ref_csr_to_csc<double>(ms, m, n, nnz, csr_val, csr_row_ptr, csr_col_ind, csc_val, csc_row_ind,
                                csc_col_ptr, nnzpercol);
}

swift_status swift_ref_col_sort_f32(float *ms, int colA, int nnz, int width, const int *nnzpercol,
                                    const int *csccolptr, const int *cscrowidx,
                                    const float *cscval, int *sortrowidx_tmp,
                                    float *sortval_tmp, int *sortnnz_tmp, const float *dense,
                                    float *sort_dense) {
  return ref_col_sort<float>(ms, colA, nnz, width, nnzpercol, csccolptr, cscrowidx, cscval,
                             sortrowidx_tmp, sortval_tmp, sortnnz_tmp, dense, sort_dense);
}
swift_status swift_ref_col_sort_f64(float *ms, int colA, int nnz, int width, const int *nnzpercol,
                                    const int *csccolptr, const int *cscrowidx,
                                    const double *cscval, int *sortrowidx_tmp,
                                    double *sortval_tmp, int *sortnnz_tmp, const double *dense,
                                    double *sort_dense) {
  return ref_col_sort<double>(ms, colA, nnz, width, nnzpercol, csccolptr, cscrowidx, cscval,
                              sortrowidx_tmp, sortval_tmp, sortnnz_tmp, dense, sort_dense);
}

swift_status swift_ref_formattransation_f32(float *ms, swift_slide_matrix_f32 *m,
                                            const int *sortrowidx_tmp, const float *sortval_tmp,
                                            const int *sortnnz_tmp, int nnz, int rowA, int colA,
                                            double *reside_ratio) {
  return ref_formattransation<float>(ms, m, sortrowidx_tmp, sortval_tmp, sortnnz_tmp, nnz, rowA, colA,
                                     reside_ratio, false, nullptr);
}
swift_status swift_ref_formattransation_f64(float *ms, swift_slide_matrix_f64 *m,
                                            const int *sortrowidx_tmp, const double *sortval_tmp,
                                            const int *sortnnz_tmp, int nnz, int rowA, int colA,
                                            double *reside_ratio) {
  return ref_formattransation<double>(ms, m, sortrowidx_tmp, sortval_tmp, sortnnz_tmp, nnz, rowA, colA,
                                      reside_ratio, false, nullptr);
}

swift_status swift_ref_formatTransform_f32(float *ms, swift_slide_matrix_f32 *m,
                                           const int *sortrowidx_tmp, const float *sortval_tmp,
                                           const int *sortnnz_tmp, int nnz, int rowA, int colA,
                                           int *h_count) {
  return ref_formattransation<float>(ms, m, sortrowidx_tmp, sortval_tmp, sortnnz_tmp, nnz, rowA, colA,
                                     nullptr, true, h_count);
}
swift_status swift_ref_formatTransform_f64(float *ms, swift_slide_matrix_f64 *m,
                                           const int *sortrowidx_tmp, const double *sortval_tmp,
                                           const int *sortnnz_tmp, int nnz, int rowA, int colA,
                                           int *h_count) {
  return ref_formattransation<double>(ms, m, sortrowidx_tmp, sortval_tmp, sortnnz_tmp, nnz, rowA, colA,
                                      nullptr, true, h_count);
}

swift_status swift_ref_block_catgory_f32(swift_slide_matrix_f32 *m, double *shuffle_ratio) {
  return ref_block_catgory<float>(m, shuffle_ratio);
}
swift_status swift_ref_block_catgory_f64(swift_slide_matrix_f64 *m, double *shuffle_ratio) {
  return ref_block_catgory<double>(m, shuffle_ratio);
}

swift_status swift_ref_balance_f32(swift_slide_matrix_f32 *m, int m_rows, int n_reside,
                                   int reside_nnz, const int *cscptr, const int *cscrowidx) {
  (void)m_rows; (void)reside_nnz; (void)cscrowidx;
  return ref_balance<float>(m, n_reside, cscptr);
}
swift_status swift_ref_balance_f64(swift_slide_matrix_f64 *m, int m_rows, int n_reside,
                                   int reside_nnz, const int *cscptr, const int *cscrowidx) {
  (void)m_rows; (void)reside_nnz; (void)cscrowidx;
  return ref_balance<double>(m, n_reside, cscptr);
}

swift_status swift_ref_row_idx_sort_f32(swift_slide_matrix_f32 *m, int rowA, int colA,
                                        int width, float *blockratio) {
  (void)rowA; (void)colA; (void)width;
  return ref_row_idx_sort<float>(m, blockratio);
}
swift_status swift_ref_row_idx_sort_f64(swift_slide_matrix_f64 *m, int rowA, int colA,
                                        int width, float *blockratio) {
  (void)rowA; (void)colA; (void)width;
  return ref_row_idx_sort<double>(m, blockratio);
}

swift_status swift_ref_spmm_f32(int variant, const swift_slide_matrix_f32 *m, int rowA,
                                int colA, int width, int nnz, const float *h_B_sorted,
                                float *h_C, float *ms) {
  return ref_spmm<float>(variant, m, rowA, colA, width, nnz, h_B_sorted, h_C, ms);
}
swift_status swift_ref_spmm_f64(int variant, const swift_slide_matrix_f64 *m, int rowA,
                                int colA, int width, int nnz, const double *h_B_sorted,
                                double *h_C, float *ms) {
  return ref_spmm<double>(variant, m, rowA, colA, width, nnz, h_B_sorted, h_C, ms);
}

}  // extern "C"
