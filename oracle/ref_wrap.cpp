/*
 * ref_wrap.cpp -- C entry points over the REFERENCE's own host code, compiled in place from
 * the reference tree by oracle/Makefile into oracle/_ref/.  TEST INFRASTRUCTURE ONLY: this
 * pins the CPU oracle (swift_oracle.c) to the reference and provides the reference's CPU
 * SpMM for the benchmark's reference arm.  No reference source is copied here; the headers
 * are included from the reference checkout (-I<ref>/test/k-32/FP32 or -I<ref>/src).
 *
 * Build flavours: -DREF_FP32 (test/k-32/FP32/, value type float) or -DREF_FP64 (src/,
 * value type double).  Exported names carry the flavour suffix.
 */
#include <sys/time.h>

#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "coo2csc.h"  // also brings auxiliary.h, mmio.h and format.h (slide_matrix, cmp)
#include "Swift_cpu.h"
#include "back_process.h"
#include "balance.h"
#include "block_catgory.h"

#include "swift_oracle.h"

#if defined(REF_FP32)
typedef float ref_t;
typedef or_slide_f32 or_slide_t;
#define REFN(name) name##_f32
#elif defined(REF_FP64)
typedef double ref_t;
typedef or_slide_f64 or_slide_t;
#define REFN(name) name##_f64
#else
#error "define REF_FP32 or REF_FP64"
#endif

namespace {
// The reference's std::sort permutation (src/coo2csc.h:96-102), reproduced by running the
// reference's own comparator on the same input.
void std_sort_perm(int K, const int *nnzpercol, int *perm) {
  std::vector<sortA> arr(K);
  for (int i = 0; i < K; ++i) { arr[i].sortnnzpercol = nnzpercol[i]; arr[i].index = i; }
  std::sort(arr.begin(), arr.end(), cmp);
  for (int i = 0; i < K; ++i) perm[i] = arr[i].index;
}

// Copy the reference slide_matrix pointers into the oracle's flat struct (the oracle's
// or_slide_free releases them; both sides use malloc).
void export_slide(const slide_matrix *s, or_slide_t *o) {
  o->tilenum = s->tilenum;
  o->regular_nnz = s->regular_nnz;
  o->tile_ptr = s->tile_ptr;
  o->tile_len = s->tile_len;
  o->tile_colidx = s->tile_colidx;
  o->tile_tall = s->tile_tall;
  o->sortrowidx = s->sortrowidx;
  o->sortval = s->sortval;
  o->reside_col = s->reside_col;
  o->reside_nnz = s->reside_nnz;
  o->reside_cscptr = s->reside_cscptr;
  o->reside_cscrowidx = s->reside_cscrowidx;
  o->reside_val = s->reside_val;
  o->segsum = s->segsum;
  o->tile_format = s->tile_format;
  o->countrow = nullptr;  // local to block_catgory in the reference (not kept in the struct)
  o->segmentoffset = s->segmentoffset;
  o->sortrowindex = s->sortrowindex;
  o->numblk = s->numblk;
  o->colorblk = s->colorblk;
  o->blkstart = s->blkstart;
  o->blkstop = s->blkstop;
  o->blkptr = s->blkptr;
  o->val_position = s->val_position;
  o->val_offset = s->val_offset;
}

void import_slide(const or_slide_t *o, slide_matrix *s) {
  memset(s, 0, sizeof(*s));
  s->tilenum = o->tilenum;
  s->regular_nnz = o->regular_nnz;
  s->tile_ptr = o->tile_ptr;
  s->tile_len = o->tile_len;
  s->tile_colidx = o->tile_colidx;
  s->tile_tall = o->tile_tall;
  s->sortrowidx = o->sortrowidx;
  s->sortval = o->sortval;
  s->reside_col = o->reside_col;
  s->reside_nnz = o->reside_nnz;
  s->reside_cscptr = o->reside_cscptr;
  s->reside_cscrowidx = o->reside_cscrowidx;
  s->reside_val = o->reside_val;
  s->segsum = o->segsum;
  s->tile_format = o->tile_format;
  s->segmentoffset = o->segmentoffset;
  s->sortrowindex = o->sortrowindex;
  s->numblk = o->numblk;
  s->colorblk = o->colorblk;
  s->blkstart = o->blkstart;
  s->blkstop = o->blkstop;
  s->blkptr = o->blkptr;
  s->val_position = o->val_position;
  s->val_offset = o->val_offset;
}
}  // namespace

extern "C" {

// src/coo2csc.h:11-79
int REFN(ref_csr2csc)(int M, int K, int nnz, const int *rowptr, const int *colidx,
                      const ref_t *val, int *cscrowidx, int *csccolptr, int *nnzpercol,
                      ref_t *cscval) {
  int *r = nullptr, *p = nullptr, *cnt = nullptr;
  ref_t *v = nullptr;
  csr2csc(nnz, M, K, const_cast<int *>(colidx), const_cast<int *>(rowptr),
          const_cast<ref_t *>(val), &r, &p, &cnt, &v);
  memcpy(cscrowidx, r, sizeof(int) * (size_t)nnz);
  memcpy(csccolptr, p, sizeof(int) * (size_t)(K + 1));
  memcpy(nnzpercol, cnt, sizeof(int) * (size_t)K);
  memcpy(cscval, v, sizeof(ref_t) * (size_t)nnz);
  free(r); free(p); free(cnt); free(v);
  return 0;
}

// The reference's column permutation as its host col_sort computes it (std::sort).
void REFN(ref_std_sort_perm)(int K, const int *nnzpercol, int *perm) { std_sort_perm(K, nnzpercol, perm); }

// src/coo2csc.h:82-134 with a given permutation.  The reference's col_sort is run on keys
// equal to each column's rank in `perm`; those keys are unique, so its std::sort yields
// exactly `perm`, and its own gather code produces the sorted CSC and sorted B.  The sorted
// counts are then restored from the real counts.
void REFN(ref_col_sort)(int K, int N, const int *nnzpercol, const int *perm,
                        const int *csccolptr, const int *cscrowidx, const ref_t *cscval,
                        int *sortrowidx_tmp, ref_t *sortval_tmp, int *sortnnz_tmp,
                        const ref_t *B, ref_t *sortB) {
  std::vector<int> rank(K);
  for (int i = 0; i < K; ++i) rank[perm[i]] = i;
  std::vector<ref_t> Bdummy, sBdummy;
  const ref_t *Bp = B;
  ref_t *sBp = sortB;
  if (!B || !sortB) {
    Bdummy.assign((size_t)K * (N > 0 ? N : 1), ref_t(0));
    sBdummy.assign(Bdummy.size(), ref_t(0));
    Bp = Bdummy.data();
    sBp = sBdummy.data();
  }
  col_sort(K, N, rank.data(), const_cast<int *>(csccolptr), const_cast<int *>(cscrowidx),
           const_cast<ref_t *>(cscval), sortrowidx_tmp, sortval_tmp, sortnnz_tmp,
           const_cast<ref_t *>(Bp), sBp);
  for (int i = 0; i < K; ++i) sortnnz_tmp[i] = nnzpercol[perm[i]];
}

// src/coo2csc.h:82-134 run as-is (its own std::sort on the real counts).
void REFN(ref_col_sort_native)(int K, int N, const int *nnzpercol, const int *csccolptr,
                               const int *cscrowidx, const ref_t *cscval, int *sortrowidx_tmp,
                               ref_t *sortval_tmp, int *sortnnz_tmp, const ref_t *B,
                               ref_t *sortB) {
  col_sort(K, N, const_cast<int *>(nnzpercol), const_cast<int *>(csccolptr),
           const_cast<int *>(cscrowidx), const_cast<ref_t *>(cscval), sortrowidx_tmp,
           sortval_tmp, sortnnz_tmp, const_cast<ref_t *>(B), sortB);
}

// src/coo2csc.h:137-435, then src/block_catgory.h and src/balance.h, exactly as the
// reference driver sequences them (src/main.cu:279-291, 367-370).
int REFN(ref_build)(or_slide_t *out, const int *sortrowidx_tmp, const ref_t *sortval_tmp,
                    const int *sortnnz_tmp, int nnz, int M, int K) {
  slide_matrix *s = (slide_matrix *)calloc(1, sizeof(slide_matrix));
  std::vector<int> cnt(sortnnz_tmp, sortnnz_tmp + K);
  cnt.push_back(0);  // formattransation scans colA+1 entries of its own copy only
#if defined(REF_FP32)
  formattransation(0.f, s, const_cast<int *>(sortrowidx_tmp), const_cast<ref_t *>(sortval_tmp),
                   cnt.data(), nnz, M, K);
  block_catgory(s);
#else
  double reside_ratio = 0, shuffle_ratio = 0;
  formattransation(0.0, s, const_cast<int *>(sortrowidx_tmp), const_cast<ref_t *>(sortval_tmp),
                   cnt.data(), nnz, M, K, reside_ratio);
  block_catgory(s, shuffle_ratio);
#endif
  balance(s, M, s->reside_col, s->reside_nnz, s->reside_cscptr, s->reside_cscrowidx);
  memset(out, 0, sizeof(*out));
  export_slide(s, out);
  // The reference fills tile_tall but never the step count; recount steps for the caller.
  int ns = 0;
  for (int c = 0; c < K; ++c) ns += (sortnnz_tmp[c] != (c ? sortnnz_tmp[c - 1] : 0));
  out->nsteps = ns;
  // The reference leaves segptr/seginfo/seglength/val_* unallocated at this point.
  free(s);
  return 0;
}

// src/back_process.h:23-229 (FP32 flavour adds blockratio).
int REFN(ref_row_idx_sort)(or_slide_t *io, int M, int K, int N, float *blockratio) {
  slide_matrix s;
  import_slide(io, &s);
  std::vector<ref_t> dense((size_t)K * (N > 0 ? N : 1), ref_t(0));
#if defined(REF_FP32)
  float br = 0.f;
  row_idx_sort(&s, dense.data(), M, K, N, br);
  if (blockratio) *blockratio = br;
#else
  row_idx_sort(&s, dense.data(), M, K, N);
  if (blockratio) *blockratio = 0.f;
#endif
  io->val_position = s.val_position;
  io->val_offset = s.val_offset;
  return 0;
}

// src/Swift_cpu.h:2-78; returns the reference's own elapsed time in ms.
double REFN(ref_swift_cpu)(const or_slide_t *m, int M, int K, int N, const ref_t *sortB,
                           ref_t *C) {
  slide_matrix s;
  import_slide(m, &s);
  ref_t t = 0;
  Swift_cpu(t, &s, 0, M, K, N, const_cast<ref_t *>(sortB), C);
  return (double)t;
}

// Swift_cpu unchanged, run on a view of tiles [t0, t1) (and the reside part if
// with_reside): the tile arrays of the view start at tile t0 while slot indices stay
// absolute, which is how Swift_cpu indexes them (src/Swift_cpu.h:31-50).  Used to time
// bounded samples of a large workload.  Returns wall ms (steady clock).
double REFN(ref_swift_cpu_tiles)(const or_slide_t *m, int t0, int t1, int with_reside, int M,
                                 int K, int N, const ref_t *sortB, ref_t *C) {
  slide_matrix s;
  import_slide(m, &s);
  s.tilenum = t1 - t0;
  s.tile_ptr = m->tile_ptr + t0;
  s.tile_len = m->tile_len + t0;
  s.tile_colidx = m->tile_colidx + t0;
  if (!with_reside) s.reside_col = 0;
  ref_t t = 0;
  timeval a, b;
  gettimeofday(&a, nullptr);
  Swift_cpu(t, &s, 0, M, K, N, const_cast<ref_t *>(sortB), C);
  gettimeofday(&b, nullptr);
  return (b.tv_sec - a.tv_sec) * 1000.0 + (b.tv_usec - a.tv_usec) / 1000.0;
}

#if defined(REF_FP64)
// The reference's MatrixMarket reader (src/auxiliary.h:167-332) as it stands.  FP64 build only:
// the FP32 copy passes a float to "%lg" (test/k-32/FP32/auxiliary.h:65), which writes a double
// into it.  Callers feed it well-formed files, a missing file or a bad banner only: on other
// malformed input its size-line loop does not end (src/mmio.h:162-167).
int ref_mmio_allinone_f64(const char *path, int *m, int *n, int *nnz, int *is_symmetric, int **rowptr,
                          int **colidx, double **val) {
  return mmio_allinone(m, n, nnz, is_symmetric, rowptr, colidx, val, const_cast<char *>(path));
}
void ref_host_free(void *p) { free(p); }
#endif

}  // extern "C"
