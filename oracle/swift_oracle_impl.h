/*
 * swift_oracle_impl.h -- body of the CPU oracle, instantiated once per value type by
 * swift_oracle.c (VAL_T = float / double, SFX = _f32 / _f64).  TEST INFRASTRUCTURE ONLY.
 *
 * The formulation is this project's own (flags, scans and per-column lists rather than the
 * reference's in-place pointer walks), but every output array is defined to be bit-identical
 * to the reference's.  Line citations name the reference code each function must reproduce.
 */
#define CAT_(a, b) a##b
#define CAT(a, b) CAT_(a, b)
#define FN(name) CAT(name, SFX)
#define SLIDE CAT(or_slide, SFX)

#define OR_TILE 32 /* slidesize / TILESIZE: src/format.h:76-78, src/auxiliary.h:6-8 */

/* CSR -> CSC by counting sort; within a column the rows ascend because rows are visited in
 * order.  src/coo2csc.h:11-79 (host) and src/gpu_csr2csc.h:51-157 (cuSPARSE csr2cscEx2,
 * same arrays).  Returns 0, or -1 if the CSR is malformed. */
int FN(or_csr2csc)(int M, int K, int nnz, const int *rowptr, const int *colidx,
                   const VAL_T *val, int *cscrowidx, int *csccolptr, int *nnzpercol,
                   VAL_T *cscval) {
  if (rowptr[0] != 0 || rowptr[M] != nnz) return -1;
  for (int c = 0; c < K; ++c) nnzpercol[c] = 0;
  for (int p = 0; p < nnz; ++p) {
    if (colidx[p] < 0 || colidx[p] >= K) return -1;
    nnzpercol[colidx[p]]++;
  }
  csccolptr[0] = 0;
  for (int c = 0; c < K; ++c) csccolptr[c + 1] = csccolptr[c] + nnzpercol[c];
  int *fill = (int *)malloc(sizeof(int) * (size_t)(K > 0 ? K : 1));
  for (int c = 0; c < K; ++c) fill[c] = csccolptr[c];
  for (int i = 0; i < M; ++i)
    for (int p = rowptr[i]; p < rowptr[i + 1]; ++p) {
      int q = fill[colidx[p]]++;
      cscrowidx[q] = i;
      cscval[q] = val[p];
    }
  free(fill);
  return 0;
}

/* Column sort given the permutation: sorted counts, the concatenated sorted CSC and the
 * row-permuted dense operand.  src/coo2csc.h:104-133 (host col_sort after its std::sort)
 * and src/ColSort_cuda.h:9-45 (Pre4sortedx / Pre4SortIdxVal). */
void FN(or_col_sort)(int K, int N, const int *nnzpercol, const int *perm,
                     const int *csccolptr, const int *cscrowidx, const VAL_T *cscval,
                     int *sortrowidx_tmp, VAL_T *sortval_tmp, int *sortnnz_tmp, const VAL_T *B,
                     VAL_T *sortB) {
  long out = 0;
  for (int i = 0; i < K; ++i) {
    int c = perm[i];
    sortnnz_tmp[i] = nnzpercol[c];
    if (B && sortB)
      for (int n = 0; n < N; ++n) sortB[(size_t)i * N + n] = B[(size_t)c * N + n];
    for (int q = csccolptr[c]; q < csccolptr[c + 1]; ++q, ++out) {
      sortrowidx_tmp[out] = cscrowidx[q];
      sortval_tmp[out] = cscval[q];
    }
  }
}

static void *FN(or_alloc)(size_t n, size_t sz) {
  void *p = calloc(n ? n : 1, sz);
  return p;
}

/* Regular tiles and the irregular remainder from the sorted CSC.  Reproduces
 * src/coo2csc.h:137-435 (formattransation):
 *   steps   = sorted columns c whose count differs from column c-1 (first differences,
 *             src/auxiliary.h:100-113, src/coo2csc.h:165-182);
 *   tiles   = for each step (col i, base s[i-1], tall d[i]), for each full group j of 32
 *             columns starting at i, for each depth base..base+tall-1 (src/coo2csc.h:220-242);
 *             lane l of a tile holds depth `depth` of sorted column tile_colidx+l
 *             (src/coo2csc.h:263-278);
 *   reside  = the last r=(K-i)%32 columns of each step at its depths, stored column-wise
 *             under the reversed index q=K-1-c in step order (src/coo2csc.h:304-406). */
int FN(or_formattransation)(SLIDE *m, const int *R, const VAL_T *V, const int *s, int nnz,
                            int M, int K) {
  (void)M;
  memset(m, 0, sizeof(*m));
  long *ptr = (long *)FN(or_alloc)((size_t)K + 1, sizeof(long));
  for (int c = 0; c < K; ++c) ptr[c + 1] = ptr[c] + s[c];
  if (ptr[K] != nnz) { free(ptr); return -1; }

  /* steps */
  int *st_col = (int *)FN(or_alloc)((size_t)K, sizeof(int));
  int *st_base = (int *)FN(or_alloc)((size_t)K, sizeof(int));
  int *st_tall = (int *)FN(or_alloc)((size_t)K, sizeof(int));
  int ns = 0;
  for (int c = 0; c < K; ++c) {
    int prev = c ? s[c - 1] : 0;
    if (s[c] != prev) { st_col[ns] = c; st_base[ns] = prev; st_tall[ns] = s[c] - prev; ++ns; }
  }
  m->nsteps = ns;

  long tilenum = 0, reside_nnz = 0;
  int reside_col = 0;
  for (int k = 0; k < ns; ++k) {
    int groups = (K - st_col[k]) / OR_TILE, r = (K - st_col[k]) % OR_TILE;
    tilenum += (long)groups * st_tall[k];
    if (r) { reside_nnz += (long)r * st_tall[k]; if (r > reside_col) reside_col = r; }
  }
  m->tilenum = (int)tilenum;
  m->regular_nnz = (int)(tilenum * OR_TILE);
  m->reside_col = reside_col;
  m->reside_nnz = (int)reside_nnz;

  m->tile_ptr = (int *)FN(or_alloc)((size_t)tilenum + 1, sizeof(int));
  m->tile_len = (int *)FN(or_alloc)((size_t)tilenum, sizeof(int));
  m->tile_colidx = (int *)FN(or_alloc)((size_t)tilenum, sizeof(int));
  m->tile_tall = (int *)FN(or_alloc)((size_t)tilenum, sizeof(int));
  m->sortrowidx = (int *)FN(or_alloc)((size_t)m->regular_nnz, sizeof(int));
  m->sortval = (VAL_T *)FN(or_alloc)((size_t)m->regular_nnz, sizeof(VAL_T));
  long t = 0;
  for (int k = 0; k < ns; ++k) {
    int groups = (K - st_col[k]) / OR_TILE;
    for (int j = 0; j < groups; ++j)
      for (int jx = 0; jx < st_tall[k]; ++jx, ++t) {
        int col0 = st_col[k] + OR_TILE * j, depth = st_base[k] + jx;
        m->tile_ptr[t] = (int)(t * OR_TILE);
        m->tile_len[t] = OR_TILE;
        m->tile_colidx[t] = col0;
        m->tile_tall[t] = st_tall[k];
        for (int l = 0; l < OR_TILE; ++l) {
          long src = ptr[col0 + l] + depth;
          m->sortrowidx[t * OR_TILE + l] = R[src];
          m->sortval[t * OR_TILE + l] = V[src];
        }
      }
  }
  m->tile_ptr[tilenum] = (int)(tilenum * OR_TILE);

  /* reside: column q (sorted column K-1-q) collects, in step order, the depths of every step
   * whose remainder r exceeds q. */
  m->reside_cscptr = (int *)FN(or_alloc)((size_t)reside_col + 1, sizeof(int));
  m->reside_cscrowidx = (int *)FN(or_alloc)((size_t)reside_nnz, sizeof(int));
  m->reside_val = (VAL_T *)FN(or_alloc)((size_t)reside_nnz, sizeof(VAL_T));
  for (int k = 0; k < ns; ++k) {
    int r = (K - st_col[k]) % OR_TILE;
    for (int q = 0; q < r; ++q) m->reside_cscptr[q + 1] += st_tall[k];
  }
  for (int q = 0; q < reside_col; ++q) m->reside_cscptr[q + 1] += m->reside_cscptr[q];
  int *fill = (int *)FN(or_alloc)((size_t)reside_col + 1, sizeof(int));
  for (int q = 0; q < reside_col; ++q) fill[q] = m->reside_cscptr[q];
  for (int k = 0; k < ns; ++k) {
    int r = (K - st_col[k]) % OR_TILE;
    for (int jx = 0; jx < st_tall[k]; ++jx)
      for (int q = 0; q < r; ++q) {
        long src = ptr[K - 1 - q] + st_base[k] + jx;
        int dst = fill[q]++;
        m->reside_cscrowidx[dst] = R[src];
        m->reside_val[dst] = V[src];
      }
  }
  free(fill);
  free(st_col); free(st_base); free(st_tall); free(ptr);
  return (m->regular_nnz + m->reside_nnz == nnz) ? 0 : -2;
}

/* Tile classification and per-tile row segments.  src/block_catgory.h:1-160:
 *   format 0 = all 32 rows equal, 2 = 1..15 adjacent row changes, 1 = 16 or more;
 *   countrow = exclusive scan of (changes+1) per tile, segsum its total;
 *   segmentoffset[seg] = run length - 1 (length segsum+1, last 0);
 *   sortrowindex[first slot of each run] = run length - 1, other slots 0. */
int FN(or_block_catgory)(SLIDE *m) {
  int T = m->tilenum;
  m->tile_format = (int *)FN(or_alloc)((size_t)T, sizeof(int));
  m->countrow = (int *)FN(or_alloc)((size_t)T + 1, sizeof(int));
  for (int t = 0; t < T; ++t) {
    const int *r = m->sortrowidx + (long)t * OR_TILE;
    int changes = 0;
    for (int l = 1; l < OR_TILE; ++l) changes += (r[l] != r[l - 1]);
    m->tile_format[t] = changes == 0 ? 0 : (changes < 16 ? 2 : 1);
    m->countrow[t + 1] = m->countrow[t] + changes + 1;
  }
  m->segsum = m->countrow[T];
  m->segmentoffset = (int *)FN(or_alloc)((size_t)m->segsum + 1, sizeof(int));
  m->sortrowindex = (int *)FN(or_alloc)((size_t)m->regular_nnz, sizeof(int));
  for (int t = 0; t < T; ++t) {
    const int *r = m->sortrowidx + (long)t * OR_TILE;
    int seg = m->countrow[t], start = 0;
    for (int l = 1; l <= OR_TILE; ++l) {
      if (l == OR_TILE || r[l] != r[l - 1]) {
        m->segmentoffset[seg] = l - start - 1;
        m->sortrowindex[(long)t * OR_TILE + start] = l - start - 1;
        ++seg;
        start = l;
      }
    }
  }
  return 0;
}

/* Load balance of the reside columns.  src/balance.h:1-69: a column with <= 32 entries is
 * one block tagged with its index q; a longer one is cut into ceil(len/32) blocks of
 * ceil(len/nblk) entries (the last takes the rest), tagged q | 0x80000000 with absolute
 * [blkstart, blkstop).  blkptr[q] = first block of column q (array length numblk). */
int FN(or_balance)(SLIDE *m) {
  int n = m->reside_col, nb = 0;
  const int *p = m->reside_cscptr;
  for (int q = 0; q < n; ++q) {
    int len = p[q + 1] - p[q];
    nb += len <= OR_TILE ? 1 : (len + OR_TILE - 1) / OR_TILE;
  }
  m->numblk = nb;
  m->colorblk = (unsigned int *)FN(or_alloc)((size_t)nb, sizeof(unsigned int));
  m->blkstart = (int *)FN(or_alloc)((size_t)nb, sizeof(int));
  m->blkstop = (int *)FN(or_alloc)((size_t)nb, sizeof(int));
  m->blkptr = (int *)FN(or_alloc)((size_t)nb, sizeof(int));
  int b = 0;
  for (int q = 0; q < n; ++q) {
    int len = p[q + 1] - p[q];
    m->blkptr[q] = b;
    if (len <= OR_TILE) {
      m->colorblk[b++] = (unsigned int)q;
    } else {
      int nblk = (len + OR_TILE - 1) / OR_TILE, lenblk = (len + nblk - 1) / nblk;
      for (int j = 0; j < nblk; ++j, ++b) {
        m->colorblk[b] = (unsigned int)q | 0x80000000u;
        m->blkstart[b] = p[q] + j * lenblk;
        m->blkstop[b] = (j == nblk - 1) ? p[q] + len : p[q] + (j + 1) * lenblk;
      }
    }
  }
  return 0;
}

/* Per-group row sort for the segmented-reduce kernel.  src/back_process.h:23-229:
 * groups of 8 tiles (256 slots) plus one remainder group; the row keys of each group are
 * sorted ascending and written back over sortrowidx (sortval is NOT permuted);
 * val_position[orig slot] = sorted slot (ties by ascending original slot here -- the
 * reference's std::sort leaves tie order unspecified); val_offset marks runs of equal
 * sorted keys: run head = run length-1, singleton = -1, other members 0 -- except that in
 * the remainder group a singleton in the last slot that follows a run keeps 0
 * (src/back_process.h:172-205 has no branch for it).  blockratio is the FP32 flavour's
 * statistic (test/k-32/FP32/back_process.h:205-249): fraction of groups whose slots are
 * all singletons. */
static int FN(or_cmp_pair)(const void *a, const void *b) {
  const long *x = (const long *)a, *y = (const long *)b;
  return (*x > *y) - (*x < *y);
}
int FN(or_row_idx_sort)(SLIDE *m, float *blockratio) {
  int T = m->tilenum, nr = m->regular_nnz;
  m->val_position = (int *)FN(or_alloc)((size_t)nr, sizeof(int));
  m->val_offset = (int *)FN(or_alloc)((size_t)nr, sizeof(int));
  int ngroups = (T + 7) / 8;
  long *key = (long *)FN(or_alloc)(256, sizeof(long));
  int nonsame = 0;
  for (int g = 0; g < ngroups; ++g) {
    int t0 = g * 8, t1 = t0 + 8 < T ? t0 + 8 : T;
    int base = t0 * OR_TILE, cnt = (t1 - t0) * OR_TILE;
    int last_group = (T % 8 != 0) && (g == ngroups - 1);
    /* (row key << 9 | original slot): ascending order = stable sort by row */
    for (int i = 0; i < cnt; ++i) key[i] = ((long)m->sortrowidx[base + i] << 9) | i;
    qsort(key, (size_t)cnt, sizeof(long), FN(or_cmp_pair));
    for (int i = 0; i < cnt; ++i) {
      m->sortrowidx[base + i] = (int)(key[i] >> 9);
      m->val_position[base + (int)(key[i] & 511)] = i;
    }
    int *k = m->sortrowidx + base, *off = m->val_offset + base;
    int start = 0;
    for (int i = 1; i <= cnt; ++i) {
      if (i == cnt || k[i] != k[i - 1]) {
        int len = i - start;
        /* a last-slot singleton of the remainder group that follows a run of >= 2 */
        int quirk = last_group && start == cnt - 1 && start >= 2 && k[start - 1] == k[start - 2];
        if (len > 1)
          off[start] = len - 1;
        else if (!quirk)
          off[start] = -1;
        start = i;
      }
    }
    int all_single = 1;
    for (int i = 0; i < cnt; ++i) if (off[i] != -1) { all_single = 0; break; }
    nonsame += all_single;
  }
  free(key);
  if (blockratio) *blockratio = (float)nonsame / (float)ngroups;
  return 0;
}

/* CPU SpMM over the format, accumulating in the value type in the reference's exact order:
 * tiles in order, slots in order, dense columns in order; then reside columns q = 0.. .
 * src/Swift_cpu.h:2-78 (FP32: test/k-32/FP32/Swift_cpu.h:2-65).  C must be zeroed. */
void FN(or_swift_cpu)(const SLIDE *m, int M, int K, int N, const VAL_T *sortB, VAL_T *C) {
  (void)M;
  for (int t = 0; t < m->tilenum; ++t)
    for (int l = 0; l < OR_TILE; ++l) {
      long j = (long)t * OR_TILE + l;
      int col = m->tile_colidx[t] + l, row = m->sortrowidx[j];
      VAL_T v = m->sortval[j];
      for (int n = 0; n < N; ++n) C[(size_t)row * N + n] += v * sortB[(size_t)col * N + n];
    }
  for (int q = 0; q < m->reside_col; ++q) {
    int col = K - q - 1;
    for (int j = m->reside_cscptr[q]; j < m->reside_cscptr[q + 1]; ++j) {
      int row = m->reside_cscrowidx[j];
      VAL_T v = m->reside_val[j];
      for (int n = 0; n < N; ++n) C[(size_t)row * N + n] += v * sortB[(size_t)col * N + n];
    }
  }
}

/* The same product restricted to tiles [t0, t1) (plus the reside part if with_reside), for
 * timing bounded samples of large workloads. */
void FN(or_swift_cpu_tiles)(const SLIDE *m, int t0, int t1, int with_reside, int M, int K,
                            int N, const VAL_T *sortB, VAL_T *C) {
  SLIDE v = *m;
  (void)M;
  for (int t = t0; t < t1; ++t)
    for (int l = 0; l < OR_TILE; ++l) {
      long j = (long)t * OR_TILE + l;
      int col = m->tile_colidx[t] + l, row = m->sortrowidx[j];
      VAL_T w = m->sortval[j];
      for (int n = 0; n < N; ++n) C[(size_t)row * N + n] += w * sortB[(size_t)col * N + n];
    }
  if (with_reside) {
    v.tilenum = 0;
    FN(or_swift_cpu)(&v, M, K, N, sortB, C);
  }
}

void FN(or_slide_free)(SLIDE *m) {
  void *ps[] = {m->tile_ptr, m->tile_len, m->tile_colidx, m->tile_tall, m->sortrowidx,
                m->sortval, m->reside_cscptr, m->reside_cscrowidx, m->reside_val,
                m->tile_format, m->countrow, m->segmentoffset, m->sortrowindex, m->colorblk,
                m->blkstart, m->blkstop, m->blkptr, m->val_position, m->val_offset};
  for (size_t i = 0; i < sizeof(ps) / sizeof(ps[0]); ++i) free(ps[i]);
  memset(m, 0, sizeof(*m));
}

#undef SLIDE
#undef FN
