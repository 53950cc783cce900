/*
 * swift_oracle.h -- CPU oracle for the Swift SpMM path (TEST INFRASTRUCTURE ONLY).
 *
 * This is a plain-C restatement of the reference's host algorithm for the Swift format
 * and its CPU SpMM.  It exists only to check the CUDA library: tests, the smoke check and
 * the CPU-baseline leg of the benchmark may call it; the library never does.
 *
 * Parity pin: every function here is checked bit-for-bit against the reference's own
 * headers compiled in place (oracle/Makefile builds oracle/_ref/) by tests/test_oracle.py,
 * and the committed fixtures under tests/golden/ were produced by that reference build.
 *
 * Each function is compiled twice, for the reference's FP32 flavour (test/k-32/FP32/) and
 * its FP64 flavour (src/); the suffix _f32 / _f64 names the value type.
 */
#ifndef SWIFT_ORACLE_H
#define SWIFT_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

#define OR_DECLARE(VAL_T, SFX)                                                                 \
  typedef struct {                                                                             \
    /* regular part (src/coo2csc.h:137-300) */                                                 \
    int tilenum, regular_nnz, nsteps;                                                          \
    int *tile_ptr, *tile_len, *tile_colidx, *tile_tall;                                        \
    int *sortrowidx;                                                                           \
    VAL_T *sortval;                                                                            \
    /* irregular ("reside") part (src/coo2csc.h:304-406) */                                    \
    int reside_col, reside_nnz;                                                                \
    int *reside_cscptr, *reside_cscrowidx;                                                     \
    VAL_T *reside_val;                                                                         \
    /* classification (src/block_catgory.h) */                                                 \
    int segsum;                                                                                \
    int *tile_format, *countrow, *segmentoffset, *sortrowindex;                                \
    /* load balance (src/balance.h) */                                                         \
    int numblk;                                                                                \
    unsigned int *colorblk;                                                                    \
    int *blkstart, *blkstop, *blkptr;                                                          \
    /* per-8-tile row sort (src/back_process.h) */                                             \
    int *val_position, *val_offset;                                                            \
  } or_slide##SFX;                                                                             \
                                                                                               \
  int or_csr2csc##SFX(int M, int K, int nnz, const int *rowptr, const int *colidx,             \
                      const VAL_T *val, int *cscrowidx, int *csccolptr, int *nnzpercol,        \
                      VAL_T *cscval);                                                          \
  void or_col_sort##SFX(int K, int N, const int *nnzpercol, const int *perm,                   \
                        const int *csccolptr, const int *cscrowidx, const VAL_T *cscval,       \
                        int *sortrowidx_tmp, VAL_T *sortval_tmp, int *sortnnz_tmp,             \
                        const VAL_T *B, VAL_T *sortB);                                         \
  int or_formattransation##SFX(or_slide##SFX *m, const int *sortrowidx_tmp,                    \
                               const VAL_T *sortval_tmp, const int *sortnnz_tmp, int nnz,      \
                               int M, int K);                                                  \
  int or_block_catgory##SFX(or_slide##SFX *m);                                                 \
  int or_balance##SFX(or_slide##SFX *m);                                                       \
  int or_row_idx_sort##SFX(or_slide##SFX *m, float *blockratio);                               \
  void or_swift_cpu##SFX(const or_slide##SFX *m, int M, int K, int N, const VAL_T *sortB,      \
                         VAL_T *C);                                                            \
  void or_swift_cpu_tiles##SFX(const or_slide##SFX *m, int t0, int t1, int with_reside, int M,  \
                               int K, int N, const VAL_T *sortB, VAL_T *C);                    \
  void or_slide_free##SFX(or_slide##SFX *m);

OR_DECLARE(float, _f32)
OR_DECLARE(double, _f64)

/* Stable ascending column order by nnz count, ties by ascending column index.  This is
 * the order thrust::sort_by_key produces in the reference's GPU column sort
 * (src/ColSort_cuda.h:96-108), and the primary parity contract for the format arrays. */
void or_col_perm_stable(int K, const int *nnzpercol, int *perm);

/* Dense-accumulating golden products in FP64 (the reference's own golden is the naive
 * CSR loop at src/main.cu:145-155; these keep its loop order but accumulate in double). */
void or_csr_spmm_f64(int M, int K, int N, const int *rowptr, const int *colidx,
                     const double *val, const double *B, double *C);
void or_csr_spmm_t_f64(int M, int K, int N, const int *rowptr, const int *colidx,
                       const double *val, const double *dY, double *dX);
/* out[e] = sum_n U[row_e, n] * V[col_e, n] over the CSR pattern (U is M x N, V is K x N). */
void or_sddmm_f64(int M, int K, int N, const int *rowptr, const int *colidx, const double *U,
                  const double *V, double *out);

#ifdef __cplusplus
}
#endif
#endif
