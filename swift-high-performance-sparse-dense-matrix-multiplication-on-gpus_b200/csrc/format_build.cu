// format_build.cu -- builds the Swift format on the GPU in O(nnz + K) work.
//
// Reference host pipeline reproduced array for array (src/main.cu:207-385):
//   csr_to_csc        src/gpu_csr2csc.h:51-157, host twin src/coo2csc.h:11-79
//   col_sort/ColSort  src/coo2csc.h:82-134, src/ColSort_cuda.h:48-143
//   formattransation  src/coo2csc.h:137-435 (regular tiles + reside)
//   block_catgory     src/block_catgory.h:1-160 (tile formats; segments on export)
//   balance           src/balance.h:1-69
// The reference's GPU variant of the transform (src/formatTransform_cuda.h) counts step
// ranks and per-column prefixes with O(K^2) loops; here every stage is a flag/scan/scatter
// or a stable radix sort, so the 1M-column workloads build in milliseconds.
//
// Layout in HBM (all int32 unless noted, owned by the plan):
//   perm[K], invperm[K], sortnnz[K+1], sptr[K+1]            column sort
//   srow[nnz], sval[nnz], spos[nnz]                          sorted CSC (= A^T in CSR form)
//   step_col/base/tall[nsteps], step_tile_off[nsteps+1]      staircase of sorted counts
//   item_tile[nitems+1]                                     tiled-engine work items
//   tile_colidx/depth/tall/format[tilenum]                   regular tile headers
//   sortrowidx[32*tilenum], sortval[32*tilenum]              regular tile slots (lane-major)
//   reside_ptr[reside_col+1], reside_row/val[reside_nnz]     irregular remainder (q = K-1-c)
//   colorblk/blkstart/blkstop/blkptr[numblk]                 balanced reside blocks
#include <cmath>

#include "common.cuh"

namespace swift {

namespace {

constexpr int kStripTiles = 16;  // max regular tiles per tiled-engine work item

template <class T> __global__ void validate_csr_kernel(const int *__restrict__ rowptr,
                                                       const int *__restrict__ colidx, int M,
                                                       int K, int nnz, int *err) {
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t r = i; r < M; r += stride)
    if (rowptr[r] > rowptr[r + 1]) atomicOr(err, 1);
  if (i == 0 && (rowptr[0] != 0 || rowptr[M] != nnz)) atomicOr(err, 1);
  for (int64_t p = i; p < nnz; p += stride) {
    int c = colidx[p];
    if (c < 0 || c >= K) atomicOr(err, 2);
  }
}

__global__ void col_count_kernel(const int *__restrict__ colidx, int nnz, int *__restrict__ cnt) {
  for (int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p < nnz;
       p += (int64_t)gridDim.x * blockDim.x)
    atomicAdd(&cnt[colidx[p]], 1);
}

__global__ void iota_kernel(uint32_t *a, int n) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    a[i] = (uint32_t)i;
}

__global__ void copy_i32_to_u32(const int *__restrict__ a, uint32_t *__restrict__ b, int n) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    b[i] = (uint32_t)a[i];
}

// perm / invperm / sorted counts (src/ColSort_cuda.h:96-108, src/coo2csc.h:104-116).
__global__ void perm_finish_kernel(const uint32_t *__restrict__ sorted_cols,
                                   const int *__restrict__ cnt, int K, int *__restrict__ perm,
                                   int *__restrict__ invperm, int *__restrict__ sortnnz) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < K;
       i += (int64_t)gridDim.x * blockDim.x) {
    int c = (int)sorted_cols[i];
    perm[i] = c;
    invperm[c] = (int)i;
    sortnnz[i] = cnt[c];
  }
}

// An injected order must be a permutation that sorts the counts ascending.
__global__ void perm_check_kernel(const int *__restrict__ perm, const int *__restrict__ cnt,
                                  int K, int *__restrict__ seen, int *err) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < K;
       i += (int64_t)gridDim.x * blockDim.x) {
    int c = perm[i];
    if (c < 0 || c >= K) { atomicOr(err, 4); continue; }
    if (atomicAdd(&seen[c], 1) != 0) atomicOr(err, 4);
    if (i > 0) {
      int cp = perm[i - 1];
      if (cp >= 0 && cp < K && cnt[cp] > cnt[c]) atomicOr(err, 4);
    }
  }
}

__global__ void nnz_keys_kernel(const int *__restrict__ colidx, const int *__restrict__ invperm,
                                int nnz, uint32_t *__restrict__ key, uint32_t *__restrict__ val) {
  for (int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p < nnz;
       p += (int64_t)gridDim.x * blockDim.x) {
    key[p] = (uint32_t)invperm[colidx[p]];
    val[p] = (uint32_t)p;
  }
}

// Largest i in [0, n) with a[i] <= x (a non-decreasing, a[0] <= x).
__device__ __forceinline__ int last_le(const int *__restrict__ a, int n, int x) {
  int lo = 0, hi = n - 1;
  while (lo < hi) {
    int mid = (lo + hi + 1) >> 1;
    if (__ldg(a + mid) <= x) lo = mid; else hi = mid - 1;
  }
  return lo;
}

// Sorted CSC gather: entry q of the sorted CSC is CSR entry p = sorted_p[q]; its row is
// the row whose range holds p.  Rows ascend within a column because the radix sort is
// stable over CSR order (the counting sort of src/coo2csc.h:44-56 has the same property).
template <class T>
__global__ void sorted_csc_gather_kernel(const uint32_t *__restrict__ sorted_p,
                                         const int *__restrict__ rowptr, int M,
                                         const T *__restrict__ val, int nnz,
                                         int *__restrict__ srow, T *__restrict__ sval,
                                         int *__restrict__ spos) {
  for (int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; q < nnz;
       q += (int64_t)gridDim.x * blockDim.x) {
    int p = (int)sorted_p[q];
    srow[q] = last_le(rowptr, M, p);
    sval[q] = val[p];
    spos[q] = p;
  }
}

// First differences of the sorted counts mark the steps (src/coo2csc.h:155-182).
__global__ void step_flags_kernel(const int *__restrict__ s, int K, int *__restrict__ flag) {
  for (int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; c < K;
       c += (int64_t)gridDim.x * blockDim.x)
    flag[c] = s[c] != (c ? s[c - 1] : 0);
}

__global__ void step_fill_kernel(const int *__restrict__ s, const int *__restrict__ pos, int K,
                                 int *__restrict__ step_col, int *__restrict__ step_base,
                                 int *__restrict__ step_tall) {
  for (int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; c < K;
       c += (int64_t)gridDim.x * blockDim.x) {
    int prev = c ? s[c - 1] : 0;
    if (s[c] != prev) {
      int k = pos[c];
      step_col[k] = (int)c;
      step_base[k] = prev;
      step_tall[k] = s[c] - prev;
    }
  }
}

// info layout written by step_scan_kernel
enum { kInfoSteps = 0, kInfoTiles, kInfoResideCol, kInfoResideNnz, kInfoLen };

// One block: per-step tile offsets, reside column lengths and pointer
// (src/coo2csc.h:185-197 tilenum; :304-321 reside sizes; :355-380 reside_cscptr).
__global__ void step_scan_kernel(const int *__restrict__ nsteps_p, int K,
                                 const int *__restrict__ step_col, const int *__restrict__ step_tall,
                                 int *__restrict__ tile_off, int *__restrict__ reside_ptr,
                                 int *__restrict__ info) {
  __shared__ int rlen[kTile];
  __shared__ int carry_t, tot_t;
  __shared__ int wsum_t[32];
  const int ns = *nsteps_p;
  if (threadIdx.x < kTile) rlen[threadIdx.x] = 0;
  if (threadIdx.x == 0) carry_t = 0;
  __syncthreads();
  int rmax = 0;
  for (int base = 0; base < ns; base += blockDim.x) {
    int k = base + threadIdx.x;
    int tiles = 0;
    if (k < ns) {
      int col = step_col[k], tall = step_tall[k];
      int groups = (K - col) / kTile, r = (K - col) % kTile;
      tiles = groups * tall;
      if (r) {
        rmax = max(rmax, r);
        for (int q = 0; q < r; ++q) atomicAdd(&rlen[q], tall);
      }
    }
    // block exclusive scan of tiles (blockDim.x = 1024)
    int it = tiles;
    for (int o = 1; o < 32; o <<= 1) {
      int a = __shfl_up_sync(0xffffffffu, it, o);
      if ((threadIdx.x & 31) >= o) it += a;
    }
    int w = threadIdx.x >> 5;
    if ((threadIdx.x & 31) == 31) wsum_t[w] = it;
    __syncthreads();
    if (w == 0) {
      int a = wsum_t[threadIdx.x], ia = a;
      for (int o = 1; o < 32; o <<= 1) {
        int x = __shfl_up_sync(0xffffffffu, ia, o);
        if (threadIdx.x >= o) ia += x;
      }
      wsum_t[threadIdx.x] = ia - a;
      if (threadIdx.x == 31) tot_t = ia;
    }
    __syncthreads();
    if (k < ns) tile_off[k] = carry_t + wsum_t[w] + it - tiles;
    __syncthreads();
    if (threadIdx.x == 0) carry_t += tot_t;
    __syncthreads();
  }
  // max remainder over the block
  for (int o = 16; o > 0; o >>= 1) rmax = max(rmax, __shfl_down_sync(0xffffffffu, rmax, o));
  __shared__ int rmax_s;
  if (threadIdx.x == 0) rmax_s = 0;
  __syncthreads();
  if ((threadIdx.x & 31) == 0) atomicMax(&rmax_s, rmax);
  __syncthreads();
  if (threadIdx.x == 0) {
    tile_off[ns] = carry_t;
    int acc = 0;
    reside_ptr[0] = 0;
    for (int q = 0; q < rmax_s; ++q) { acc += rlen[q]; reside_ptr[q + 1] = acc; }
    for (int q = rmax_s + 1; q <= kTile; ++q) reside_ptr[q] = acc;
    info[kInfoSteps] = ns;
    info[kInfoTiles] = carry_t;
    info[kInfoResideCol] = rmax_s;
    info[kInfoResideNnz] = acc;
  }
}

// One warp per regular tile: headers, lane-major slots, and the classification of
// src/block_catgory.h:11-72 (0: all rows equal, 2: 1..15 adjacent changes, 1: more).
template <class T>
__global__ void tile_fill_kernel(int tilenum, int nsteps, const int *__restrict__ tile_off,
                                 const int *__restrict__ step_col, const int *__restrict__ step_base,
                                 const int *__restrict__ step_tall, const int *__restrict__ sptr,
                                 const int *__restrict__ srow, const T *__restrict__ sval,
                                 int *__restrict__ tile_colidx, int *__restrict__ tile_depth,
                                 int *__restrict__ tile_tall, int *__restrict__ tile_format,
                                 int *__restrict__ sortrowidx, T *__restrict__ sortval,
                                 int *__restrict__ fmt_count) {
  const int warps = (gridDim.x * blockDim.x) >> 5;
  const int l = threadIdx.x & 31;
  int f0 = 0, f1 = 0, f2 = 0;
  for (int t = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; t < tilenum; t += warps) {
    const int k = last_le(tile_off, nsteps, t);
    const int tall = step_tall[k];
    const int local = t - tile_off[k];
    const int j = local / tall, jx = local - j * tall;
    const int col0 = step_col[k] + kTile * j;
    const int depth = step_base[k] + jx;
    const int src = sptr[col0 + l] + depth;
    const int r = srow[src];
    const T v = sval[src];
    sortrowidx[(int64_t)t * kTile + l] = r;
    sortval[(int64_t)t * kTile + l] = v;
    const int up = __shfl_up_sync(0xffffffffu, r, 1);
    const int changes = __popc(__ballot_sync(0xffffffffu, l > 0 && up != r));
    const int fmt = changes == 0 ? 0 : (changes < 16 ? 2 : 1);
    if (l == 0) {
      tile_colidx[t] = col0;
      tile_depth[t] = depth;
      tile_tall[t] = tall;
      tile_format[t] = fmt;
      f0 += fmt == 0; f1 += fmt == 1; f2 += fmt == 2;
    }
  }
  if (l == 0) {
    if (f0) atomicAdd(&fmt_count[0], f0);
    if (f1) atomicAdd(&fmt_count[1], f1);
    if (f2) atomicAdd(&fmt_count[2], f2);
  }
}

// One block per reside column q (sorted column c = K-1-q): keep the depths whose step
// leaves column c in its remainder (q < r_step), in depth order (src/coo2csc.h:384-400).
template <class T>
__global__ void reside_fill_kernel(int K, int nsteps, const int *__restrict__ sortnnz,
                                   const int *__restrict__ sptr, const int *__restrict__ srow,
                                   const T *__restrict__ sval, const int *__restrict__ step_col,
                                   const int *__restrict__ step_base,
                                   const int *__restrict__ reside_ptr, int *__restrict__ rrow,
                                   T *__restrict__ rval) {
  __shared__ int wsum[32];
  __shared__ int carry_s, tot_s;
  const int q = blockIdx.x;
  const int c = K - 1 - q;
  const int len = sortnnz[c];
  const int base = sptr[c];
  const int dst0 = reside_ptr[q];
  if (threadIdx.x == 0) carry_s = 0;
  __syncthreads();
  for (int d0 = 0; d0 < len; d0 += blockDim.x) {
    const int d = d0 + threadIdx.x;
    int keep = 0;
    if (d < len) {
      const int k = last_le(step_base, nsteps, d);
      keep = ((K - step_col[k]) % kTile) > q;
    }
    int incl = keep;
    for (int o = 1; o < 32; o <<= 1) {
      int a = __shfl_up_sync(0xffffffffu, incl, o);
      if ((threadIdx.x & 31) >= o) incl += a;
    }
    const int w = threadIdx.x >> 5;
    if ((threadIdx.x & 31) == 31) wsum[w] = incl;
    __syncthreads();
    if (w == 0) {
      int nw = blockDim.x >> 5;
      int a = threadIdx.x < nw ? wsum[threadIdx.x] : 0, ia = a;
      for (int o = 1; o < 32; o <<= 1) {
        int x = __shfl_up_sync(0xffffffffu, ia, o);
        if (threadIdx.x >= o) ia += x;
      }
      if (threadIdx.x < nw) wsum[threadIdx.x] = ia - a;
      if (threadIdx.x == nw - 1) tot_s = ia;
    }
    __syncthreads();
    const int dst = dst0 + carry_s + wsum[w] + incl - 1;
    if (keep && dst < reside_ptr[q + 1]) {  // the step scan sized this column's range
      rrow[dst] = srow[base + d];
      rval[dst] = sval[base + d];
    }
    __syncthreads();
    if (threadIdx.x == 0) carry_s += tot_s;
    __syncthreads();
  }
}

// src/balance.h:1-69.  One thread per reside column; blocks numbered in column order.
__global__ void balance_kernel(int n, const int *__restrict__ reside_ptr,
                               unsigned *__restrict__ colorblk, int *__restrict__ blkstart,
                               int *__restrict__ blkstop, int *__restrict__ blkptr) {
  const int q = threadIdx.x;
  if (q >= n) return;
  int first = 0;
  for (int i = 0; i < q; ++i) {
    int len = reside_ptr[i + 1] - reside_ptr[i];
    first += len <= kTile ? 1 : (len + kTile - 1) / kTile;
  }
  const int p0 = reside_ptr[q], len = reside_ptr[q + 1] - p0;
  blkptr[q] = first;
  if (len <= kTile) {
    colorblk[first] = (unsigned)q;
    return;
  }
  const int nblk = (len + kTile - 1) / kTile, lenblk = (len + nblk - 1) / nblk;
  for (int j = 0; j < nblk; ++j) {
    colorblk[first + j] = (unsigned)q | 0x80000000u;
    blkstart[first + j] = p0 + j * lenblk;
    blkstop[first + j] = (j == nblk - 1) ? p0 + len : p0 + (j + 1) * lenblk;
  }
}

// Row layout: rows longer than `split` are cut into ceil(len/split) pieces of `split`
// nonzeros (the last takes the rest) -- the balance rule of src/balance.h:48-66 applied to
// the rows of A (or of A^T) so that no warp walks a power-law row alone.
__global__ void long_flags_kernel(const int *__restrict__ ptr, int rows, int split,
                                  int *__restrict__ isl, int *__restrict__ npieces,
                                  int *__restrict__ maxlen) {
  int m = 0;
  for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < rows;
       r += (int64_t)gridDim.x * blockDim.x) {
    int len = ptr[r + 1] - ptr[r];
    m = max(m, len);
    bool l = len > split;
    isl[r] = l;
    npieces[r] = l ? (len + split - 1) / split : 0;
  }
  for (int o = 16; o > 0; o >>= 1) m = max(m, __shfl_down_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0) atomicMax(maxlen, m);
}

__global__ void long_fill_kernel(const int *__restrict__ ptr, int rows, int split,
                                 const int *__restrict__ lpos, const int *__restrict__ ppos,
                                 int *__restrict__ long_of_row, int *__restrict__ long_first,
                                 int *__restrict__ long_count, int *__restrict__ piece_row,
                                 int *__restrict__ piece_idx) {
  for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < rows;
       r += (int64_t)gridDim.x * blockDim.x) {
    int len = ptr[r + 1] - ptr[r];
    if (len <= split) { long_of_row[r] = -1; continue; }
    int o = lpos[r], first = ppos[r], n = (len + split - 1) / split;
    long_of_row[r] = o;
    long_first[o] = first;
    long_count[o] = n;
    for (int j = 0; j < n; ++j) { piece_row[first + j] = (int)r; piece_idx[first + j] = j; }
  }
}

// src/block_catgory.h:11-72 on an existing tile array: one warp per tile.
__global__ void classify_kernel(const int *__restrict__ rows, int T, int *__restrict__ fmt_out,
                                int *__restrict__ fmt_count) {
  const int warps = (gridDim.x * blockDim.x) >> 5;
  const int l = threadIdx.x & 31;
  int f0 = 0, f1 = 0, f2 = 0;
  for (int t = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; t < T; t += warps) {
    const int r = rows[(int64_t)t * kTile + l];
    const int up = __shfl_up_sync(0xffffffffu, r, 1);
    const int changes = __popc(__ballot_sync(0xffffffffu, l > 0 && up != r));
    const int fmt = changes == 0 ? 0 : (changes < 16 ? 2 : 1);
    if (l == 0) {
      fmt_out[t] = fmt;
      f0 += fmt == 0; f1 += fmt == 1; f2 += fmt == 2;
    }
  }
  if (l == 0) {
    if (f0) atomicAdd(&fmt_count[0], f0);
    if (f1) atomicAdd(&fmt_count[1], f1);
    if (f2) atomicAdd(&fmt_count[2], f2);
  }
}

__global__ void item_flags_kernel(const int *__restrict__ colidx, int T, int *__restrict__ flag) {
  for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < T;
       t += (int64_t)gridDim.x * blockDim.x)
    flag[t] = t == 0 || colidx[t] != colidx[t - 1] || (t % kStripTiles) == 0;
}

__global__ void item_fill_kernel(const int *__restrict__ colidx, int T, const int *__restrict__ pos,
                                 int *__restrict__ item_tile) {
  for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t <= T;
       t += (int64_t)gridDim.x * blockDim.x) {
    if (t == T) item_tile[pos[T]] = T;
    else if (t == 0 || colidx[t] != colidx[t - 1] || (t % kStripTiles) == 0) item_tile[pos[t]] = (int)t;
  }
}

int grid_for(int64_t n, int threads = 256, int cap = 148 * 16) {
  int64_t b = (n + threads - 1) / threads;
  if (b < 1) b = 1;
  return (int)std::min<int64_t>(b, cap);
}

int bitlen(uint32_t x) {
  int b = 0;
  while (x) { ++b; x >>= 1; }
  return b;
}

}  // namespace

// ---------------------------------------------------------------------------------------------
// Tiled-engine work items: maximal runs of consecutive tiles with equal tile_colidx (one
// step and group at successive depths), cut at every multiple of kStripTiles tiles.
swift_status build_items(Plan &p, cudaStream_t st) {
  const int T = p.tilenum;
  TmpBuf flags;
  SW_TRY(flags.alloc(sizeof(int) * ((size_t)T + 1), st));
  if (T > 0) item_flags_kernel<<<grid_for(T), 256, 0, st>>>(p.tile_colidx.as<int>(), T, flags.as<int>());
  SW_CHECK_LAUNCH();
  SW_TRY(scan_exclusive_i32(flags.as<int>(), flags.as<int>(), T, st));
  int n = 0;
  SW_CHECK_CUDA(cudaMemcpyAsync(&n, flags.as<int>() + T, sizeof(int), cudaMemcpyDeviceToHost, st));
  SW_CHECK_CUDA(cudaStreamSynchronize(st));
  p.nstrips = n;
  SW_TRY(p.item_tile.alloc(sizeof(int) * ((size_t)n + 1)));
  item_fill_kernel<<<grid_for(T + 1), 256, 0, st>>>(p.tile_colidx.as<int>(), T, flags.as<int>(),
                                                     p.item_tile.as<int>());
  SW_CHECK_LAUNCH();
  return SWIFT_OK;
}

// Balance blocks of the reside part (src/balance.h:1-69): the block count comes from the
// host-visible reside pointer, the arrays are filled on the device from p.reside_ptr.
swift_status build_balance(Plan &p, const int *h_reside_ptr, cudaStream_t st) {
  int nb = 0;
  for (int q = 0; q < p.reside_col; ++q) {
    int len = h_reside_ptr[q + 1] - h_reside_ptr[q];
    nb += len <= kTile ? 1 : (len + kTile - 1) / kTile;
  }
  p.numblk = nb;
  SW_TRY(p.colorblk.alloc(sizeof(unsigned) * (size_t)nb));
  SW_TRY(p.blkstart.alloc(sizeof(int) * (size_t)nb));
  SW_TRY(p.blkstop.alloc(sizeof(int) * (size_t)nb));
  SW_TRY(p.blkptr.alloc(sizeof(int) * (size_t)nb));
  if (nb > 0) {
    SW_CHECK_CUDA(cudaMemsetAsync(p.blkstart.p, 0, sizeof(int) * nb, st));
    SW_CHECK_CUDA(cudaMemsetAsync(p.blkstop.p, 0, sizeof(int) * nb, st));
    SW_CHECK_CUDA(cudaMemsetAsync(p.blkptr.p, 0, sizeof(int) * nb, st));
    balance_kernel<<<1, 32, 0, st>>>(p.reside_col, p.reside_ptr.as<int>(), p.colorblk.as<unsigned>(),
                                     p.blkstart.as<int>(), p.blkstop.as<int>(), p.blkptr.as<int>());
    SW_CHECK_LAUNCH();
  }
  return SWIFT_OK;
}

// Tile formats from p.sortrowidx alone (block_catgory on a format built elsewhere).
swift_status classify_tiles(Plan &p, cudaStream_t st) {
  SW_TRY(p.tile_format.alloc(sizeof(int) * ((size_t)p.tilenum + 3)));
  TmpBuf fmt;
  SW_TRY(fmt.alloc(sizeof(int) * 4, st));
  SW_CHECK_CUDA(cudaMemsetAsync(fmt.p, 0, sizeof(int) * 4, st));
  if (p.tilenum > 0)
    classify_kernel<<<grid_for((int64_t)p.tilenum * 32, 256, 148 * 32), 256, 0, st>>>(
        p.sortrowidx.as<int>(), p.tilenum, p.tile_format.as<int>(), fmt.as<int>());
  SW_CHECK_LAUNCH();
  int hf[4];
  SW_CHECK_CUDA(cudaMemcpyAsync(hf, fmt.p, sizeof(int) * 4, cudaMemcpyDeviceToHost, st));
  SW_CHECK_CUDA(cudaStreamSynchronize(st));
  for (int i = 0; i < 3; ++i) p.fmt_count[i] = hf[i];
  return SWIFT_OK;
}

// Stable ascending order of K columns by count (ties by index): perm, invperm, sorted counts.
swift_status stable_column_order(const int *d_cnt, int K, int *d_perm, int *d_invperm,
                                 int *d_sortnnz, int *max_count, cudaStream_t st) {
  if (K == 0) return SWIFT_OK;
  TmpBuf k0, v0, k1, v1, mx;
  SW_TRY(k0.alloc(sizeof(uint32_t) * (size_t)K, st));
  SW_TRY(v0.alloc(sizeof(uint32_t) * (size_t)K, st));
  SW_TRY(k1.alloc(sizeof(uint32_t) * (size_t)K, st));
  SW_TRY(v1.alloc(sizeof(uint32_t) * (size_t)K, st));
  SW_TRY(mx.alloc(sizeof(int) * 4, st));
  SW_TRY(reduce_max_i32(d_cnt, K, mx.as<int>(), st));
  int hmax = 0;
  SW_CHECK_CUDA(cudaMemcpyAsync(&hmax, mx.p, sizeof(int), cudaMemcpyDeviceToHost, st));
  SW_CHECK_CUDA(cudaStreamSynchronize(st));
  if (max_count) *max_count = hmax;
  copy_i32_to_u32<<<grid_for(K), 256, 0, st>>>(d_cnt, k0.as<uint32_t>(), K);
  iota_kernel<<<grid_for(K), 256, 0, st>>>(v0.as<uint32_t>(), K);
  SW_TRY(radix_sort_pairs(k0.as<uint32_t>(), v0.as<uint32_t>(), k1.as<uint32_t>(), v1.as<uint32_t>(),
                          K, bitlen((uint32_t)hmax), st));
  perm_finish_kernel<<<grid_for(K), 256, 0, st>>>(v1.as<uint32_t>(), d_cnt, K, d_perm, d_invperm, d_sortnnz);
  SW_CHECK_LAUNCH();
  return SWIFT_OK;
}

// CSR -> CSC on the device (src/gpu_csr2csc.h:51-157 semantics): counts, column pointer, and
// entries in column order with rows ascending within a column.
swift_status csr_to_csc_device(const int *d_rowptr, const int *d_colidx, const void *d_val,
                               bool f64, int M, int K, int nnz, int *d_colptr, int *d_rowidx,
                               void *d_cscval, int *d_cnt, cudaStream_t st) {
  SW_CHECK_CUDA(cudaMemsetAsync(d_cnt, 0, sizeof(int) * (size_t)std::max(K, 1), st));
  if (nnz) col_count_kernel<<<grid_for(nnz), 256, 0, st>>>(d_colidx, nnz, d_cnt);
  SW_CHECK_LAUNCH();
  SW_TRY(scan_exclusive_i32(d_cnt, d_colptr, K, st));
  if (nnz == 0) return SWIFT_OK;
  TmpBuf k0, v0, k1, v1, pos;
  SW_TRY(k0.alloc(sizeof(uint32_t) * (size_t)nnz, st));
  SW_TRY(v0.alloc(sizeof(uint32_t) * (size_t)nnz, st));
  SW_TRY(k1.alloc(sizeof(uint32_t) * (size_t)nnz, st));
  SW_TRY(v1.alloc(sizeof(uint32_t) * (size_t)nnz, st));
  SW_TRY(pos.alloc(sizeof(int) * (size_t)nnz, st));
  copy_i32_to_u32<<<grid_for(nnz), 256, 0, st>>>(d_colidx, k0.as<uint32_t>(), nnz);
  iota_kernel<<<grid_for(nnz), 256, 0, st>>>(v0.as<uint32_t>(), nnz);
  SW_TRY(radix_sort_pairs(k0.as<uint32_t>(), v0.as<uint32_t>(), k1.as<uint32_t>(), v1.as<uint32_t>(),
                          nnz, bitlen((uint32_t)(K - 1)), st));
  if (f64)
    sorted_csc_gather_kernel<double><<<grid_for(nnz), 256, 0, st>>>(
        v1.as<uint32_t>(), d_rowptr, M, static_cast<const double *>(d_val), nnz, d_rowidx,
        static_cast<double *>(d_cscval), pos.as<int>());
  else
    sorted_csc_gather_kernel<float><<<grid_for(nnz), 256, 0, st>>>(
        v1.as<uint32_t>(), d_rowptr, M, static_cast<const float *>(d_val), nnz, d_rowidx,
        static_cast<float *>(d_cscval), pos.as<int>());
  SW_CHECK_LAUNCH();
  return SWIFT_OK;
}

swift_status build_tiles(Plan &p, cudaStream_t st) {
  const int K = p.K;
  const size_t vsz = p.vsz;
  // steps
  const int cap = (int)std::min<int64_t>(K, (int64_t)std::sqrt(2.0 * (double)p.nnz) + 2);
  SW_TRY(p.step_col.alloc(sizeof(int) * cap));
  SW_TRY(p.step_base.alloc(sizeof(int) * cap));
  SW_TRY(p.step_tall.alloc(sizeof(int) * cap));
  SW_TRY(p.step_tile_off.alloc(sizeof(int) * (cap + 1)));
  SW_TRY(p.reside_ptr.alloc(sizeof(int) * (kTile + 1)));
  TmpBuf flags, info;
  SW_TRY(flags.alloc(sizeof(int) * ((size_t)K + 1), st));
  SW_TRY(info.alloc(sizeof(int) * (kInfoLen + kTile + 1), st));
  if (K > 0) {
    step_flags_kernel<<<grid_for(K), 256, 0, st>>>(p.sortnnz.as<int>(), K, flags.as<int>());
    SW_TRY(scan_exclusive_i32(flags.as<int>(), flags.as<int>(), K, st));
    step_fill_kernel<<<grid_for(K), 256, 0, st>>>(p.sortnnz.as<int>(), flags.as<int>(), K,
                                                   p.step_col.as<int>(), p.step_base.as<int>(),
                                                   p.step_tall.as<int>());
  } else {
    SW_CHECK_CUDA(cudaMemsetAsync(flags.p, 0, sizeof(int), st));
  }
  step_scan_kernel<<<1, 1024, 0, st>>>(flags.as<int>() + K, K, p.step_col.as<int>(),
                                       p.step_tall.as<int>(), p.step_tile_off.as<int>(),
                                       p.reside_ptr.as<int>(), info.as<int>());
  SW_CHECK_LAUNCH();
  int h[kInfoLen + kTile + 1];
  SW_CHECK_CUDA(cudaMemcpyAsync(h, info.p, sizeof(int) * kInfoLen, cudaMemcpyDeviceToHost, st));
  SW_CHECK_CUDA(cudaMemcpyAsync(h + kInfoLen, p.reside_ptr.p, sizeof(int) * (kTile + 1),
                                cudaMemcpyDeviceToHost, st));
  SW_CHECK_CUDA(cudaStreamSynchronize(st));
  p.nsteps = h[kInfoSteps];
  p.tilenum = h[kInfoTiles];
  p.reside_col = h[kInfoResideCol];
  p.reside_nnz = h[kInfoResideNnz];
  const int *rptr = h + kInfoLen;
  if ((int64_t)p.tilenum * kTile + p.reside_nnz != p.nnz) {
    set_last_error("build_tiles", "regular + reside != nnz");
    return SWIFT_ERR_CUDA;
  }
  // regular tiles
  const int64_t nreg = (int64_t)p.tilenum * kTile;
  SW_TRY(p.tile_colidx.alloc(sizeof(int) * (size_t)p.tilenum));
  SW_TRY(p.tile_depth.alloc(sizeof(int) * (size_t)p.tilenum));
  SW_TRY(p.tile_tall.alloc(sizeof(int) * (size_t)p.tilenum));
  SW_TRY(p.tile_format.alloc(sizeof(int) * ((size_t)p.tilenum + 3)));
  SW_TRY(p.sortrowidx.alloc(sizeof(int) * (size_t)nreg));
  SW_TRY(p.sortval.alloc(vsz * (size_t)nreg));
  TmpBuf fmt;
  SW_TRY(fmt.alloc(sizeof(int) * 4, st));
  SW_CHECK_CUDA(cudaMemsetAsync(fmt.p, 0, sizeof(int) * 4, st));
  if (p.tilenum > 0) {
    const int blocks = grid_for((int64_t)p.tilenum * 32, 256, 148 * 32);
    if (p.val_type == SWIFT_F64)
      tile_fill_kernel<double><<<blocks, 256, 0, st>>>(
          p.tilenum, p.nsteps, p.step_tile_off.as<int>(), p.step_col.as<int>(),
          p.step_base.as<int>(), p.step_tall.as<int>(), p.sptr.as<int>(), p.srow.as<int>(),
          p.sval.as<double>(), p.tile_colidx.as<int>(), p.tile_depth.as<int>(),
          p.tile_tall.as<int>(), p.tile_format.as<int>(), p.sortrowidx.as<int>(),
          p.sortval.as<double>(), fmt.as<int>());
    else
      tile_fill_kernel<float><<<blocks, 256, 0, st>>>(
          p.tilenum, p.nsteps, p.step_tile_off.as<int>(), p.step_col.as<int>(),
          p.step_base.as<int>(), p.step_tall.as<int>(), p.sptr.as<int>(), p.srow.as<int>(),
          p.sval.as<float>(), p.tile_colidx.as<int>(), p.tile_depth.as<int>(),
          p.tile_tall.as<int>(), p.tile_format.as<int>(), p.sortrowidx.as<int>(),
          p.sortval.as<float>(), fmt.as<int>());
    SW_CHECK_LAUNCH();
  }
  // reside
  SW_TRY(p.reside_row.alloc(sizeof(int) * (size_t)p.reside_nnz));
  SW_TRY(p.reside_val.alloc(vsz * (size_t)p.reside_nnz));
  if (p.reside_col > 0) {
    if (p.val_type == SWIFT_F64)
      reside_fill_kernel<double><<<p.reside_col, 256, 0, st>>>(
          K, p.nsteps, p.sortnnz.as<int>(), p.sptr.as<int>(), p.srow.as<int>(),
          p.sval.as<double>(), p.step_col.as<int>(), p.step_base.as<int>(),
          p.reside_ptr.as<int>(), p.reside_row.as<int>(), p.reside_val.as<double>());
    else
      reside_fill_kernel<float><<<p.reside_col, 256, 0, st>>>(
          K, p.nsteps, p.sortnnz.as<int>(), p.sptr.as<int>(), p.srow.as<int>(),
          p.sval.as<float>(), p.step_col.as<int>(), p.step_base.as<int>(),
          p.reside_ptr.as<int>(), p.reside_row.as<int>(), p.reside_val.as<float>());
    SW_CHECK_LAUNCH();
  }
  SW_TRY(build_balance(p, rptr, st));
  SW_TRY(build_items(p, st));
  int hf[4];
  SW_CHECK_CUDA(cudaMemcpyAsync(hf, fmt.p, sizeof(int) * 4, cudaMemcpyDeviceToHost, st));
  SW_CHECK_CUDA(cudaStreamSynchronize(st));
  p.fmt_count[0] = hf[0];
  p.fmt_count[1] = hf[1];
  p.fmt_count[2] = hf[2];
  return SWIFT_OK;
}

// ---------------------------------------------------------------------------------------------
swift_status build_from_csr(Plan &p, const swift_csr &A, const swift_plan_opts *opts,
                            cudaStream_t st) {
  const int M = A.rows, K = A.cols, nnz = A.nnz;
  const size_t vsz = p.vsz;
  // device copy of the CSR
  SW_TRY(p.rowptr.alloc(sizeof(int) * ((size_t)M + 1)));
  SW_TRY(p.colidx.alloc(sizeof(int) * (size_t)nnz));
  SW_TRY(p.val.alloc(vsz * (size_t)nnz));
  const cudaMemcpyKind kind = A.mem == SWIFT_HOST ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToDevice;
  SW_CHECK_CUDA(cudaMemcpyAsync(p.rowptr.p, A.rowptr, sizeof(int) * ((size_t)M + 1), kind, st));
  if (nnz) {
    SW_CHECK_CUDA(cudaMemcpyAsync(p.colidx.p, A.colidx, sizeof(int) * (size_t)nnz, kind, st));
    SW_CHECK_CUDA(cudaMemcpyAsync(p.val.p, A.val, vsz * (size_t)nnz, kind, st));
  }
  p.has_csr = true;

  TmpBuf err;
  SW_TRY(err.alloc(sizeof(int) * 4, st));
  SW_CHECK_CUDA(cudaMemsetAsync(err.p, 0, sizeof(int) * 4, st));
  validate_csr_kernel<int><<<grid_for(std::max(M, nnz)), 256, 0, st>>>(p.rowptr.as<int>(), p.colidx.as<int>(),
                                                                       M, K, nnz, err.as<int>());
  SW_CHECK_LAUNCH();

  // column counts (src/gpu_csr2csc.h:24-32,110)
  SW_TRY(p.cnt.alloc(sizeof(int) * (size_t)K));
  SW_CHECK_CUDA(cudaMemsetAsync(p.cnt.p, 0, sizeof(int) * (size_t)K, st));
  int herr = 0;
  SW_CHECK_CUDA(cudaMemcpyAsync(&herr, err.p, sizeof(int), cudaMemcpyDeviceToHost, st));
  SW_CHECK_CUDA(cudaStreamSynchronize(st));
  if (herr) return SWIFT_ERR_BAD_CSR;
  if (nnz) col_count_kernel<<<grid_for(nnz), 256, 0, st>>>(p.colidx.as<int>(), nnz, p.cnt.as<int>());
  SW_CHECK_LAUNCH();

  // column order
  SW_TRY(p.perm.alloc(sizeof(int) * (size_t)K));
  SW_TRY(p.invperm.alloc(sizeof(int) * (size_t)K));
  SW_TRY(p.sortnnz.alloc(sizeof(int) * ((size_t)K + 1)));
  SW_TRY(p.sptr.alloc(sizeof(int) * ((size_t)K + 1)));
  SW_CHECK_CUDA(cudaMemsetAsync(p.sortnnz.p, 0, sizeof(int) * ((size_t)K + 1), st));
  {
    TmpBuf k0, v0, k1, v1;
    SW_TRY(k0.alloc(sizeof(uint32_t) * (size_t)K, st));
    SW_TRY(v0.alloc(sizeof(uint32_t) * (size_t)K, st));
    SW_TRY(k1.alloc(sizeof(uint32_t) * (size_t)K, st));
    SW_TRY(v1.alloc(sizeof(uint32_t) * (size_t)K, st));
    if (opts && opts->col_perm) {
      const cudaMemcpyKind pk = opts->col_perm_mem == SWIFT_HOST ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToDevice;
      SW_CHECK_CUDA(cudaMemcpyAsync(p.perm.p, opts->col_perm, sizeof(int) * (size_t)K, pk, st));
      TmpBuf seen;
      SW_TRY(seen.alloc(sizeof(int) * (size_t)K, st));
      SW_CHECK_CUDA(cudaMemsetAsync(seen.p, 0, sizeof(int) * (size_t)K, st));
      if (K) perm_check_kernel<<<grid_for(K), 256, 0, st>>>(p.perm.as<int>(), p.cnt.as<int>(), K,
                                                            seen.as<int>(), err.as<int>());
      SW_CHECK_CUDA(cudaMemcpyAsync(&herr, err.p, sizeof(int), cudaMemcpyDeviceToHost, st));
      SW_CHECK_CUDA(cudaStreamSynchronize(st));
      if (herr) return SWIFT_ERR_BAD_PERM;
      if (K) copy_i32_to_u32<<<grid_for(K), 256, 0, st>>>(p.perm.as<int>(), v1.as<uint32_t>(), K);
      if (K) perm_finish_kernel<<<grid_for(K), 256, 0, st>>>(v1.as<uint32_t>(), p.cnt.as<int>(), K,
                                                             p.perm.as<int>(), p.invperm.as<int>(),
                                                             p.sortnnz.as<int>());
      SW_CHECK_LAUNCH();
    } else {
      // stable ascending sort of (count, column): thrust::sort_by_key order
      SW_TRY(stable_column_order(p.cnt.as<int>(), K, p.perm.as<int>(), p.invperm.as<int>(),
                                 p.sortnnz.as<int>(), &p.max_col, st));
    }
  }
  SW_TRY(scan_exclusive_i32(p.sortnnz.as<int>(), p.sptr.as<int>(), K, st));

  // sorted CSC: stable radix sort of CSR entries by sorted column position
  SW_TRY(p.srow.alloc(sizeof(int) * (size_t)nnz));
  SW_TRY(p.sval.alloc(vsz * (size_t)nnz));
  SW_TRY(p.spos.alloc(sizeof(int) * (size_t)nnz));
  if (nnz) {
    TmpBuf k0, v0, k1, v1;
    SW_TRY(k0.alloc(sizeof(uint32_t) * (size_t)nnz, st));
    SW_TRY(v0.alloc(sizeof(uint32_t) * (size_t)nnz, st));
    SW_TRY(k1.alloc(sizeof(uint32_t) * (size_t)nnz, st));
    SW_TRY(v1.alloc(sizeof(uint32_t) * (size_t)nnz, st));
    nnz_keys_kernel<<<grid_for(nnz), 256, 0, st>>>(p.colidx.as<int>(), p.invperm.as<int>(), nnz,
                                                   k0.as<uint32_t>(), v0.as<uint32_t>());
    SW_TRY(radix_sort_pairs(k0.as<uint32_t>(), v0.as<uint32_t>(), k1.as<uint32_t>(),
                            v1.as<uint32_t>(), nnz, bitlen((uint32_t)(K - 1)), st));
    if (p.val_type == SWIFT_F64)
      sorted_csc_gather_kernel<double><<<grid_for(nnz), 256, 0, st>>>(
          v1.as<uint32_t>(), p.rowptr.as<int>(), M, p.val.as<double>(), nnz, p.srow.as<int>(),
          p.sval.as<double>(), p.spos.as<int>());
    else
      sorted_csc_gather_kernel<float><<<grid_for(nnz), 256, 0, st>>>(
          v1.as<uint32_t>(), p.rowptr.as<int>(), M, p.val.as<float>(), nnz, p.srow.as<int>(),
          p.sval.as<float>(), p.spos.as<int>());
    SW_CHECK_LAUNCH();
  }
  return build_tiles(p, st);
}

namespace {
template <class T>
__global__ void value_gather_kernel(const int *__restrict__ spos, const T *__restrict__ val, int64_t nnz,
                                    T *__restrict__ sval) {
  for (int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; q < nnz;
       q += (int64_t)gridDim.x * blockDim.x)
    sval[q] = val[spos[q]];
}

template <class T>
swift_status refresh_typed(Plan &p, cudaStream_t st) {
  if (p.nnz > 0) {
    value_gather_kernel<T><<<grid_for(p.nnz), 256, 0, st>>>(p.spos.as<int>(), p.val.as<T>(), p.nnz,
                                                             p.sval.as<T>());
    SW_CHECK_LAUNCH();
  }
  if (p.tilenum > 0) {
    TmpBuf fmt;
    SW_TRY(fmt.alloc(sizeof(int) * 4, st));
    SW_CHECK_CUDA(cudaMemsetAsync(fmt.p, 0, sizeof(int) * 4, st));
    tile_fill_kernel<T><<<grid_for((int64_t)p.tilenum * 32, 256, 148 * 32), 256, 0, st>>>(
        p.tilenum, p.nsteps, p.step_tile_off.as<int>(), p.step_col.as<int>(), p.step_base.as<int>(),
        p.step_tall.as<int>(), p.sptr.as<int>(), p.srow.as<int>(), p.sval.as<T>(), p.tile_colidx.as<int>(),
        p.tile_depth.as<int>(), p.tile_tall.as<int>(), p.tile_format.as<int>(), p.sortrowidx.as<int>(),
        p.sortval.as<T>(), fmt.as<int>());
    SW_CHECK_LAUNCH();
  }
  if (p.reside_col > 0) {
    reside_fill_kernel<T><<<p.reside_col, 256, 0, st>>>(
        p.K, p.nsteps, p.sortnnz.as<int>(), p.sptr.as<int>(), p.srow.as<int>(), p.sval.as<T>(),
        p.step_col.as<int>(), p.step_base.as<int>(), p.reside_ptr.as<int>(), p.reside_row.as<int>(),
        p.reside_val.as<T>());
    SW_CHECK_LAUNCH();
  }
  return SWIFT_OK;
}
}  // namespace

// New values for the plan's fixed pattern (CSR order, already in p.val): the sorted CSC
// values, the tile slots and the reside part are refilled from it; pattern arrays, the
// column order and every row layout stay as built.
swift_status refresh_values(Plan &p, cudaStream_t st) {
  if (!p.has_csr) return SWIFT_ERR_UNSUPPORTED;
  return p.val_type == SWIFT_F64 ? refresh_typed<double>(p, st) : refresh_typed<float>(p, st);
}

// ---------------------------------------------------------------------------------------------
swift_status build_row_layout(Plan &p, RowLayout &L, bool transpose, cudaStream_t st) {
  if (!p.has_csr) return SWIFT_ERR_UNSUPPORTED;
  if (!transpose) {
    L.rows = p.M; L.cols = p.K; L.ptr = p.rowptr.as<int>(); L.idx = p.colidx.as<int>();
    L.val = p.val.p; L.out_row = nullptr;
  } else {
    L.rows = p.K; L.cols = p.M; L.ptr = p.sptr.as<int>(); L.idx = p.srow.as<int>();
    L.val = p.sval.p; L.out_row = p.perm.as<int>();
  }
  L.nnz = p.nnz;
  L.split = p.long_row_split > 0 ? p.long_row_split : 128;
  const int R = L.rows;
  TmpBuf isl, np, lpos, ppos, mx;
  SW_TRY(isl.alloc(sizeof(int) * ((size_t)R + 1), st));
  SW_TRY(np.alloc(sizeof(int) * ((size_t)R + 1), st));
  SW_TRY(lpos.alloc(sizeof(int) * ((size_t)R + 1), st));
  SW_TRY(ppos.alloc(sizeof(int) * ((size_t)R + 1), st));
  SW_TRY(mx.alloc(sizeof(int) * 4, st));
  SW_CHECK_CUDA(cudaMemsetAsync(mx.p, 0, sizeof(int) * 4, st));
  if (R > 0)
    long_flags_kernel<<<grid_for(R), 256, 0, st>>>(L.ptr, R, L.split, isl.as<int>(), np.as<int>(),
                                                   mx.as<int>());
  SW_CHECK_LAUNCH();
  SW_TRY(scan_exclusive_i32(isl.as<int>(), lpos.as<int>(), R, st));
  SW_TRY(scan_exclusive_i32(np.as<int>(), ppos.as<int>(), R, st));
  int h[3];
  SW_CHECK_CUDA(cudaMemcpyAsync(&h[0], lpos.as<int>() + R, sizeof(int), cudaMemcpyDeviceToHost, st));
  SW_CHECK_CUDA(cudaMemcpyAsync(&h[1], ppos.as<int>() + R, sizeof(int), cudaMemcpyDeviceToHost, st));
  SW_CHECK_CUDA(cudaMemcpyAsync(&h[2], mx.p, sizeof(int), cudaMemcpyDeviceToHost, st));
  SW_CHECK_CUDA(cudaStreamSynchronize(st));
  L.long_rows = h[0];
  L.pieces = h[1];
  if (!transpose) p.max_row = h[2]; else p.max_col = h[2];
  SW_TRY(L.long_of_row.alloc(sizeof(int) * (size_t)R));
  SW_TRY(L.long_first.alloc(sizeof(int) * (size_t)L.long_rows));
  SW_TRY(L.long_count.alloc(sizeof(int) * (size_t)L.long_rows));
  SW_TRY(L.counters.alloc(sizeof(int) * (size_t)L.long_rows));
  SW_TRY(L.piece_row.alloc(sizeof(int) * (size_t)L.pieces));
  SW_TRY(L.piece_idx.alloc(sizeof(int) * (size_t)L.pieces));
  SW_CHECK_CUDA(cudaMemsetAsync(L.counters.p, 0, sizeof(int) * (size_t)std::max(L.long_rows, 1), st));
  if (R > 0)
    long_fill_kernel<<<grid_for(R), 256, 0, st>>>(L.ptr, R, L.split, lpos.as<int>(), ppos.as<int>(),
                                                  L.long_of_row.as<int>(), L.long_first.as<int>(),
                                                  L.long_count.as<int>(), L.piece_row.as<int>(),
                                                  L.piece_idx.as<int>());
  SW_CHECK_LAUNCH();
  L.built = true;
  return SWIFT_OK;
}

}  // namespace swift
