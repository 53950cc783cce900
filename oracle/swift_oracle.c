/*
 * swift_oracle.c -- CPU oracle for the Swift SpMM path (TEST INFRASTRUCTURE ONLY; see
 * swift_oracle.h).  Instantiates swift_oracle_impl.h for the FP32 and FP64 flavours and
 * adds the FP64 golden products used to state errors.
 */
#include "swift_oracle.h"

#include <stdlib.h>
#include <string.h>

#define VAL_T float
#define SFX _f32
#include "swift_oracle_impl.h"
#undef VAL_T
#undef SFX

#define VAL_T double
#define SFX _f64
#include "swift_oracle_impl.h"
#undef VAL_T
#undef SFX

/* (count << 32 | index) keys sort to count-ascending, index-ascending order. */
static int cmp_u64(const void *a, const void *b) {
  unsigned long long x = *(const unsigned long long *)a, y = *(const unsigned long long *)b;
  return (x > y) - (x < y);
}

void or_col_perm_stable(int K, const int *nnzpercol, int *perm) {
  unsigned long long *k = (unsigned long long *)malloc(sizeof(*k) * (size_t)(K > 0 ? K : 1));
  for (int c = 0; c < K; ++c) k[c] = ((unsigned long long)(unsigned)nnzpercol[c] << 32) | (unsigned)c;
  qsort(k, (size_t)K, sizeof(*k), cmp_u64);
  for (int i = 0; i < K; ++i) perm[i] = (int)(k[i] & 0xffffffffu);
  free(k);
}

void or_csr_spmm_f64(int M, int K, int N, const int *rowptr, const int *colidx,
                     const double *val, const double *B, double *C) {
  (void)K;
  for (int i = 0; i < M; ++i) {
    double *c = C + (size_t)i * N;
    for (int n = 0; n < N; ++n) c[n] = 0.0;
    for (int p = rowptr[i]; p < rowptr[i + 1]; ++p) {
      const double *b = B + (size_t)colidx[p] * N;
      for (int n = 0; n < N; ++n) c[n] += val[p] * b[n];
    }
  }
}

void or_csr_spmm_t_f64(int M, int K, int N, const int *rowptr, const int *colidx,
                       const double *val, const double *dY, double *dX) {
  memset(dX, 0, sizeof(double) * (size_t)K * N);
  for (int i = 0; i < M; ++i)
    for (int p = rowptr[i]; p < rowptr[i + 1]; ++p) {
      double *x = dX + (size_t)colidx[p] * N;
      const double *y = dY + (size_t)i * N;
      for (int n = 0; n < N; ++n) x[n] += val[p] * y[n];
    }
}

void or_sddmm_f64(int M, int K, int N, const int *rowptr, const int *colidx, const double *U,
                  const double *V, double *out) {
  (void)K;
  for (int i = 0; i < M; ++i)
    for (int p = rowptr[i]; p < rowptr[i + 1]; ++p) {
      double s = 0.0;
      for (int n = 0; n < N; ++n) s += U[(size_t)i * N + n] * V[(size_t)colidx[p] * N + n];
      out[p] = s;
    }
}
