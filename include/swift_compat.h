/* swift_compat.h -- the reference's preprocessing and SpMM functions under their own names and
 * signatures, as inline C++ over the C ABI of swift_b200.h.  A program written against the
 * reference's headers (src/ for FP64, test/k-32/FP32/ for FP32) includes this file instead and
 * links -lswiftb200; every stage then runs on the GPU with this library's kernels.
 *
 * `slide_matrix` is the FP64 layout unless SWIFT_COMPAT_FP32 is defined before inclusion (the
 * reference picks one value type per build, src/format.h:6-39 and test/k-32/FP32/format.h).
 * Both flavours' functions are overloads, so a program may use both structures explicitly.
 *
 * Behaviour kept from the reference:
 *   - timings are written through the same reference parameters (milliseconds);
 *   - a failed call prints to stderr and carries on, like the reference's CHECK_CUDA_ERROR
 *     (src/Swift_gpu_row_major.h:5-16); SpMM wrappers then report time -1;
 *   - the SpMM wrappers check C against h_golden_resultmtx (row-major M x N) with the reference
 *     test |golden - C| > 1e-2 (src/auxiliary.h:156-165) and print "... Check NO PASS! error = n"
 *     and set the time to -1 on a mismatch (src/Swift.h:396-402);
 *   - h_resultmtx receives C in the wrapper's own layout (column-major M x N, leading dimension
 *     M, for every wrapper but Swift_gpu2, which is row-major).
 * Difference: gflops_Swift_gpu is set to 2 * nnz * width / time (the reference leaves it 0).
 */
#ifndef SWIFT_COMPAT_H
#define SWIFT_COMPAT_H

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <vector>

#include "swift_b200.h"

#ifdef SWIFT_COMPAT_FP32
typedef swift_slide_matrix_f32 slide_matrix;
#else
typedef swift_slide_matrix_f64 slide_matrix;
#endif

namespace swift_compat_detail {

inline bool report(swift_status s, const char *what) {
  if (s == SWIFT_OK) return true;
  std::fprintf(stderr, "swift_b200 %s failed: %s (%s)\n", what, swift_status_string(s),
               swift_last_error());
  return false;
}

/* C (layout of the wrapper) against a row-major golden result; counts |diff| > 1e-2. */
template <class T>
int verify(const T *C, const T *golden, int rowA, int width, bool col_major) {
  if (!golden) return 0;
  int errors = 0;
  for (int i = 0; i < rowA; ++i)
    for (int j = 0; j < width; ++j) {
      const T c = col_major ? C[(size_t)j * rowA + i] : C[(size_t)i * width + j];
      if (std::fabs(golden[(size_t)i * width + j] - c) > 1e-2) ++errors;
    }
  return errors;
}

template <class T, class SLIDE, class G>
void spmm(int variant, const char *name, float &time, G &gflops, SLIDE *matrix, int rowA, int colA,
          int width, int nnz, T *h_densemtx, T *h_resultmtx, T *h_golden_resultmtx) {
  float ms = 0.f;
  swift_status s;
  if (sizeof(T) == 8)
    s = swift_ref_spmm_f64(variant, reinterpret_cast<const swift_slide_matrix_f64 *>(matrix), rowA,
                           colA, width, nnz, reinterpret_cast<const double *>(h_densemtx),
                           reinterpret_cast<double *>(h_resultmtx), &ms);
  else
    s = swift_ref_spmm_f32(variant, reinterpret_cast<const swift_slide_matrix_f32 *>(matrix), rowA,
                           colA, width, nnz, reinterpret_cast<const float *>(h_densemtx),
                           reinterpret_cast<float *>(h_resultmtx), &ms);
  if (!report(s, name)) {
    time = -1.f;
    return;
  }
  time = ms;
  gflops = ms > 0.f ? (G)(2.0 * (double)nnz * (double)width / ((double)ms * 1e6)) : (G)0;
  const int errors = verify(h_resultmtx, h_golden_resultmtx, rowA, width, variant != 2);
  if (errors != 0) {
    std::printf("%s Check NO PASS! error = %d \n", name, errors);
    time = -1.f;
  }
}

}  // namespace swift_compat_detail

/* ---------------------------------------------------------------- CSR -> CSC
 * src/gpu_csr2csc.h:51 (FP64), test/k-32/FP32/gpu_csr2csc.h:51 (FP32) */
inline void csr_to_csc(double &time_csr2csc, int m, int n, int nnz, const double *csr_val,
                       const int *csr_row_ptr, const int *csr_col_ind, double *csc_val,
                       int *csc_row_ind, int *csc_col_ptr, int *nnzpercol) {
  float ms = 0.f;
  swift_compat_detail::report(swift_ref_csr_to_csc_f64(&ms, m, n, nnz, csr_val, csr_row_ptr,
                                                       csr_col_ind, csc_val, csc_row_ind,
                                                       csc_col_ptr, nnzpercol),
                              "csr_to_csc");
  time_csr2csc = ms;
}
inline void csr_to_csc(float &time_csr2csc, int m, int n, int nnz, const float *csr_val,
                       const int *csr_row_ptr, const int *csr_col_ind, float *csc_val,
                       int *csc_row_ind, int *csc_col_ptr, int *nnzpercol) {
  float ms = 0.f;
  swift_compat_detail::report(swift_ref_csr_to_csc_f32(&ms, m, n, nnz, csr_val, csr_row_ptr,
                                                       csr_col_ind, csc_val, csc_row_ind,
                                                       csc_col_ptr, nnzpercol),
                              "csr_to_csc");
  time_csr2csc = ms;
}

/* ---------------------------------------------------------------- column sort
 * col_sort: src/coo2csc.h:82 (FP64), test/k-32/FP32/coo2csc.h:82 (FP32).  The nonzero count is
 * csccolptr[colA].  Column order: stable ascending by count (ties by column index), the order
 * of the reference's GPU sort (src/ColSort_cuda.h:108). */
inline void col_sort(int colA, int width_dense_mtx, int *nnzpercol, int *csccolptr, int *cscrowidx,
                     double *cscval, int *sortrowidx_tmp, double *sortval_tmp, int *sortnnz_tmp,
                     double *dense_mtx, double *sort_dense_mtx) {
  swift_compat_detail::report(
      swift_ref_col_sort_f64(nullptr, colA, colA > 0 ? csccolptr[colA] : 0, width_dense_mtx,
                             nnzpercol, csccolptr, cscrowidx, cscval, sortrowidx_tmp, sortval_tmp,
                             sortnnz_tmp, dense_mtx, sort_dense_mtx),
      "col_sort");
}
inline void col_sort(int colA, int width_dense_mtx, int *nnzpercol, int *csccolptr, int *cscrowidx,
                     float *cscval, int *sortrowidx_tmp, float *sortval_tmp, int *sortnnz_tmp,
                     float *dense_mtx, float *sort_dense_mtx) {
  swift_compat_detail::report(
      swift_ref_col_sort_f32(nullptr, colA, colA > 0 ? csccolptr[colA] : 0, width_dense_mtx,
                             nnzpercol, csccolptr, cscrowidx, cscval, sortrowidx_tmp, sortval_tmp,
                             sortnnz_tmp, dense_mtx, sort_dense_mtx),
      "col_sort");
}
/* src/ColSort_cuda.h:48 (also test/k-32/FP32/ColSort_cuda.h:51, which takes double too) */
inline void ColSort(double &timeForSort, int colA, int nnz, int width, int *nnzPerCol,
                    int *cscColPtr, int *cscRowIdx, double *cscVal, int *sortrowidxTmp,
                    double *sortvalTmp, int *sortnnzTmp, double *densemtx, double *sort_densemtx) {
  float ms = 0.f;
  swift_compat_detail::report(
      swift_ref_col_sort_f64(&ms, colA, nnz, width, nnzPerCol, cscColPtr, cscRowIdx, cscVal,
                             sortrowidxTmp, sortvalTmp, sortnnzTmp, densemtx, sort_densemtx),
      "ColSort");
  timeForSort = ms;
}
inline void ColSort(double &timeForSort, int colA, int nnz, int width, int *nnzPerCol,
                    int *cscColPtr, int *cscRowIdx, float *cscVal, int *sortrowidxTmp,
                    float *sortvalTmp, int *sortnnzTmp, float *densemtx, float *sort_densemtx) {
  float ms = 0.f;
  swift_compat_detail::report(
      swift_ref_col_sort_f32(&ms, colA, nnz, width, nnzPerCol, cscColPtr, cscRowIdx, cscVal,
                             sortrowidxTmp, sortvalTmp, sortnnzTmp, densemtx, sort_densemtx),
      "ColSort");
  timeForSort = ms;
}

/* ---------------------------------------------------------------- tiles + reside part
 * src/coo2csc.h:137 (FP64, with reside_ratio), test/k-32/FP32/coo2csc.h:140 (FP32).  The first
 * argument is a by-value timing slot in the reference and is ignored here as there. */
inline void formattransation(double time_irrpart, swift_slide_matrix_f64 *matrix,
                             int *sortrowidx_tmp, double *sortval_tmp, int *sortnnz_tmp, int nnz,
                             int rowA, int colA, double &reside_ratio) {
  (void)time_irrpart;
  swift_compat_detail::report(
      swift_ref_formattransation_f64(nullptr, matrix, sortrowidx_tmp, sortval_tmp, sortnnz_tmp,
                                     nnz, rowA, colA, &reside_ratio),
      "formattransation");
}
inline void formattransation(float time_irrpart, swift_slide_matrix_f32 *matrix,
                             int *sortrowidx_tmp, float *sortval_tmp, int *sortnnz_tmp, int nnz,
                             int rowA, int colA) {
  (void)time_irrpart;
  swift_compat_detail::report(
      swift_ref_formattransation_f32(nullptr, matrix, sortrowidx_tmp, sortval_tmp, sortnnz_tmp,
                                     nnz, rowA, colA, nullptr),
      "formattransation");
}
/* src/formatTransform_cuda.h:198 -- regular tiles only; h_count = number of steps */
inline void formatTransform(double &timeFormatTran, swift_slide_matrix_f64 *matrix,
                            int *sortrowidx_tmp, double *sortval_tmp, int *sortnnz_tmp, int nnz,
                            int rowA, int colA, int &h_count) {
  float ms = 0.f;
  swift_compat_detail::report(
      swift_ref_formatTransform_f64(&ms, matrix, sortrowidx_tmp, sortval_tmp, sortnnz_tmp, nnz,
                                    rowA, colA, &h_count),
      "formatTransform");
  timeFormatTran = ms;
}
inline void formatTransform(double &timeFormatTran, swift_slide_matrix_f32 *matrix,
                            int *sortrowidx_tmp, float *sortval_tmp, int *sortnnz_tmp, int nnz,
                            int rowA, int colA, int &h_count) {
  float ms = 0.f;
  swift_compat_detail::report(
      swift_ref_formatTransform_f32(&ms, matrix, sortrowidx_tmp, sortval_tmp, sortnnz_tmp, nnz,
                                    rowA, colA, &h_count),
      "formatTransform");
  timeFormatTran = ms;
}

/* ---------------------------------------------------------------- tile classes
 * src/block_catgory.h:1 (FP64, with shuffle_ratio), test/k-32/FP32/block_catgory.h:1 (FP32) */
inline void block_catgory(swift_slide_matrix_f64 *matrix, double &shuffle_ratio) {
  swift_compat_detail::report(swift_ref_block_catgory_f64(matrix, &shuffle_ratio), "block_catgory");
}
inline void block_catgory(swift_slide_matrix_f32 *matrix) {
  swift_compat_detail::report(swift_ref_block_catgory_f32(matrix, nullptr), "block_catgory");
}

/* ---------------------------------------------------------------- reside balance
 * src/balance.h:1 (both flavours): n = number of reside columns, cscptr = reside_cscptr */
inline void balance(swift_slide_matrix_f64 *matrix, int m, int n, int nnz, int *cscptr,
                    int *cscrowidx) {
  swift_compat_detail::report(swift_ref_balance_f64(matrix, m, n, nnz, cscptr, cscrowidx), "balance");
}
inline void balance(swift_slide_matrix_f32 *matrix, int m, int n, int nnz, int *cscptr,
                    int *cscrowidx) {
  swift_compat_detail::report(swift_ref_balance_f32(matrix, m, n, nnz, cscptr, cscrowidx), "balance");
}

/* ---------------------------------------------------------------- per-8-tile row sort
 * src/back_process.h:23 (FP64), test/k-32/FP32/back_process.h:23 (FP32, with blockratio) */
inline void row_idx_sort(swift_slide_matrix_f64 *matrix, double *dense_mtx, int rowA, int colA,
                         int width) {
  (void)dense_mtx;
  swift_compat_detail::report(swift_ref_row_idx_sort_f64(matrix, rowA, colA, width, nullptr),
                              "row_idx_sort");
}
inline void row_idx_sort(swift_slide_matrix_f32 *matrix, float *dense_mtx, int rowA, int colA,
                         int width, float &blockratio) {
  (void)dense_mtx;
  swift_compat_detail::report(swift_ref_row_idx_sort_f32(matrix, rowA, colA, width, &blockratio),
                              "row_idx_sort");
}

/* ---------------------------------------------------------------- SpMM wrappers
 * FP64: src/Swift.h:184, src/Swift_gpu_col_major.h:171, src/Swift_gpu_row_major.h:136,
 *       src/Swift_3.h:216, src/Swift_4.h:305 (gflops double&).
 * FP32: test/k-32/FP32/Swift.h:217, Swift_gpu_col_major.h:209, Swift_gpu_row_major.h:136,
 *       Swift_3.h:208, Swift_4.h:310 (gflops float&). */
#define SWIFT_COMPAT_SPMM(NAME, VARIANT, LABEL)                                                  \
  inline void NAME(char *filename, float &time_Swift_gpu, double &gflops_Swift_gpu,             \
                   swift_slide_matrix_f64 *matrix, int rowA, int colA, int width, int nnz,      \
                   double *h_densemtx, double *h_resultmtx, double *h_golden_resultmtx) {       \
    (void)filename;                                                                             \
    swift_compat_detail::spmm(VARIANT, LABEL, time_Swift_gpu, gflops_Swift_gpu, matrix, rowA,   \
                              colA, width, nnz, h_densemtx, h_resultmtx, h_golden_resultmtx);   \
  }                                                                                             \
  inline void NAME(char *filename, float &time_Swift_gpu, float &gflops_Swift_gpu,              \
                   swift_slide_matrix_f32 *matrix, int rowA, int colA, int width, int nnz,      \
                   float *h_densemtx, float *h_resultmtx, float *h_golden_resultmtx) {          \
    (void)filename;                                                                             \
    swift_compat_detail::spmm(VARIANT, LABEL, time_Swift_gpu, gflops_Swift_gpu, matrix, rowA,   \
                              colA, width, nnz, h_densemtx, h_resultmtx, h_golden_resultmtx);   \
  }

SWIFT_COMPAT_SPMM(Swift_GPU, 0, "Swift GPU SpMM (dense mtx col-major)")
SWIFT_COMPAT_SPMM(Swift_gpu1, 1, "Swift GPU SpMM (dense mtx col-major)")
SWIFT_COMPAT_SPMM(Swift_gpu2, 2, "Swift GPU SpMM (dense mtx row major, opt)")
SWIFT_COMPAT_SPMM(Swift_GPU_3, 3, "Swift GPU (3.0) SpMM")
SWIFT_COMPAT_SPMM(Swift_GPU_4, 4, "Swift GPU (4.0) SpMM")
#undef SWIFT_COMPAT_SPMM

/* ---------------------------------------------------------------- driver helpers
 * src/auxiliary.h:28-50: the best of the three wrapper times, ignoring failed ones (-1).  All
 * three failed: -1.  Exactly one valid: the reference matches none of its cases and leaves
 * time_final as it was; so does this. */
inline void result_check(float time_Swift_gpu, float time_Swift_gpu1, float time_Swift_gpu2,
                         float &time_final) {
  const float t[3] = {time_Swift_gpu, time_Swift_gpu1, time_Swift_gpu2};
  int failed = 0;
  float best = 0.f;
  bool any = false;
  for (float x : t) {
    if (x == -1) {
      ++failed;
    } else {
      best = any ? std::fmin(best, x) : x;
      any = true;
    }
  }
  if (failed == 3) time_final = -1;
  else if (failed <= 1) time_final = best;
}

/* src/auxiliary.h:53-64: targetmtx (cols x rows, row-major) = the transpose of originmtx
 * (rows x cols, row-major); the drivers use it to turn row-major B into the column-major
 * operand of the GPU wrappers and back. */
template <class T>
inline void dense_mtx2dense_mtx_spmm(int rows, int cols, T *originmtx, T *targetmtx) {
  for (int i = 0; i < cols; ++i)
    for (int j = 0; j < rows; ++j) targetmtx[(size_t)i * rows + j] = originmtx[(size_t)j * cols + i];
}

/* src/auxiliary.h:156-165: counts the positions where |resultB - resultA| > 1e-2 into result
 * (added to its current value, as in the reference). */
template <class T>
inline void ResultVerify(T *resultA, T *resultB, int length, int &result) {
  for (int i = 0; i < length; ++i) {
    const T d = resultB[i] - resultA[i];  // difference in the value type, as the reference
    if (std::fabs(d) > 1e-2) ++result;
  }
}

/* ---------------------------------------------------------------- src/auxiliary.h:167-332
 * MatrixMarket coordinate file -> CSR in malloc'd arrays (the caller frees them with free(), as
 * the reference's callers do), through swift_mtx_read.  Returns the reference's codes: 0,
 * -1 (cannot open), -2 (banner; prints the reference's message), -4 (size line); and -5 where
 * the reference would go on with undefined values (an index outside the matrix, a missing
 * or malformed entry, an "array" file). */
namespace swift_compat_detail {
template <class T>
inline int mmio(int *m, int *n, int *nnz, int *isSymmetric, int **csrrowptr, int **csrcolidx,
                T **csrval, const char *filename, swift_dtype dt) {
  int code = 0;
  void *v = nullptr;
  const swift_status s = swift_mtx_read(filename, dt, m, n, nnz, isSymmetric, csrrowptr, csrcolidx, &v, &code);
  if (s != SWIFT_OK) {
    if (code == -2) std::printf("Could not process Matrix Market banner.\n");
    else report(s, "mmio_allinone");
    return code ? code : -5;
  }
  *csrval = static_cast<T *>(v);
  return 0;
}
}  // namespace swift_compat_detail

inline int mmio_allinone(int *m, int *n, int *nnz, int *isSymmetric, int **csrrowptr, int **csrcolidx,
                         double **csrval, char *filename) {
  return swift_compat_detail::mmio(m, n, nnz, isSymmetric, csrrowptr, csrcolidx, csrval, filename, SWIFT_F64);
}
inline int mmio_allinone(int *m, int *n, int *nnz, int *isSymmetric, int **csrrowptr, int **csrcolidx,
                         float **csrval, char *filename) {
  return swift_compat_detail::mmio(m, n, nnz, isSymmetric, csrrowptr, csrcolidx, csrval, filename, SWIFT_F32);
}

/* ---------------------------------------------------------------- driver-level macros
 * What the reference's drivers take from its headers besides functions: the tile size
 * (src/auxiliary.h:6-8), the file the drivers append their result line to (src/auxiliary.h:22;
 * test/k-32/FP32/auxiliary.h:22 for the FP32 flavour), and the two error checks that the
 * reference's cuSPARSE harness (src/gpu_cusparse_spmm.h) expands, defined in its
 * src/gpu_csr2csc.h:4-22: report the failed call with its line and carry on. */
#ifndef TILESIZE
#define TILESIZE 32
#endif
#ifndef RESULT_FILE_PATH
#ifdef SWIFT_COMPAT_FP32
#define RESULT_FILE_PATH "./data/results_Swift_FP32_32.txt"
#else
#define RESULT_FILE_PATH "./data/results_Swift_32.txt"
#endif
#endif
#ifndef CHECK_CUDA
#define CHECK_CUDA(call)                                                                         \
  {                                                                                              \
    const cudaError_t swift_compat_rc_ = (call);                                                 \
    if (swift_compat_rc_ != cudaSuccess)                                                         \
      std::printf("swift_compat: CUDA call at line %d failed: %s (%d)\n", __LINE__,               \
                  cudaGetErrorString(swift_compat_rc_), (int)swift_compat_rc_);                   \
  }
#endif
#ifndef CHECK_CUSPARSE
#define CHECK_CUSPARSE(call)                                                                     \
  {                                                                                              \
    const cusparseStatus_t swift_compat_sp_ = (call);                                            \
    if (swift_compat_sp_ != CUSPARSE_STATUS_SUCCESS)                                             \
      std::printf("swift_compat: cuSPARSE call at line %d failed: %s (%d)\n", __LINE__,           \
                  cusparseGetErrorString(swift_compat_sp_), (int)swift_compat_sp_);               \
  }
#endif

/* ---------------------------------------------------------------- src/format.h:48 */
inline void Tile_destroy(swift_slide_matrix_f64 *matrix) { swift_slide_free_f64(matrix); }
inline void Tile_destroy(swift_slide_matrix_f32 *matrix) { swift_slide_free_f32(matrix); }

#endif /* SWIFT_COMPAT_H */
