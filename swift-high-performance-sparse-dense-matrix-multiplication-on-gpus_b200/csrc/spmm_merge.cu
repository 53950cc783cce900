// spmm_merge.cu -- row-ordered SpMM with merge-path work balance.
//
// The merged sequence of a CSR operand interleaves its nonzeros with one end marker per row
// (row r occupies positions ptr[r]+r .. ptr[r+1]+r, the last being its end marker).  A task
// is a fixed slice of U positions; a sub-warp walks its slice, keeping the current C row in
// registers across nonzeros and storing it when it passes the row's end marker, so it never
// waits on a row's metadata before issuing the next row's B loads, empty rows cost one
// store, and power-law rows need no special casing.  A row whose positions straddle task
// boundaries is "split": each task touching it stores its partial row to scratch and counts
// its arrival; the last task to arrive adds the partials in task order and writes C, so the
// result does not depend on scheduling.
//
// Memory-level parallelism: each lane keeps UNR independent B-row vectors in flight per batch
// (16 for one vector per lane) and the next chunk of (index, value) pairs is fetched while
// the current one is consumed.  Vectors are 32 bytes (sm_100 256-bit accesses) when the
// operands allow, which halves the load instructions per byte against 16-byte vectors.
#include <cstring>

#include "common.cuh"
#include "vec.cuh"

namespace swift {

struct MergeArgs {
  int rows, N, U, ntasks;
  int64_t total;  // nnz + rows
  const int *ptr, *idx;
  const void *val;
  const int *out_row;
  const void *B;
  int64_t ldb;
  void *C;
  int64_t ldc;
  const int *task_row, *head_split, *tail_split;
  const int *task_hdr;  // [ntasks] int4 (task_row[t], task_row[t+1], head_split, tail_split)
  const int *split_row, *split_first, *split_last;
  int *split_cnt;
  void *scratch;  // [2 * ntasks][N] partial rows
  const float *b_scale;  // per-B-row scales (scaled 16-bit walk): folded into the values
  float *c_scale;        // per-C-row scales (scaled 16-bit walk): written with each row
};

namespace {

// B vectors in flight per lane: 8 (16 when deep), capped so the batch holds at most 256 bytes
// of accumulator-type values per lane (64 registers).
constexpr int unroll_for(int VB, int VPL, bool deep, int acc_bytes) {
  const int lim = 256 / (VB * VPL * acc_bytes) > 0 ? 256 / (VB * VPL * acc_bytes) : 1;
  const int base = deep ? 16 : 8;
  return base < lim ? base : lim;
}

// Per-row scale of 16-bit C: the power of two s that puts the row's largest magnitude m in
// [2^14, 2^15) (well inside FP16's range and BF16's), 1 for an all-zero row.  Every lane of the
// sub-warp returns the same s; dividing by a power of two is exact.
template <int SG>
__device__ __forceinline__ float row_scale(float m, unsigned sgmask) {
#pragma unroll
  for (int o = SG / 2; o >= 1; o >>= 1) m = fmaxf(m, __shfl_xor_sync(sgmask, m, o, SG));
  if (!(m > 0.f) || !(m < 3.0e38f)) return 1.f;
  const int e = (int)((__float_as_uint(m) >> 23) & 0xffu) - 127;  // floor(log2 m), normal m
  const int se = min(max(e - 14, -126), 127);
  return __uint_as_float((unsigned)(se + 127) << 23);
}

// Writes a finished row of the scaled walk: divided by its scale, which lane 0 records.
template <class T, class ACC, int VB, int SG>
__device__ __forceinline__ void store_scaled_row(const MergeArgs &a, int orow, int sl, unsigned sgmask,
                                                 ACC (&acc)[VB], bool inb) {
  float m = 0.f;
#pragma unroll
  for (int e = 0; e < VB; ++e) m = fmaxf(m, fabsf((float)acc[e]));
  const float s = row_scale<SG>(m, sgmask);
  const float inv = 1.f / s;  // exact: s is a power of two
#pragma unroll
  for (int e = 0; e < VB; ++e) acc[e] = (ACC)((float)acc[e] * inv);
  if (sl == 0) a.c_scale[orow] = s;
  if (inb) vstore<T, ACC, VB>(static_cast<T *>(a.C) + (int64_t)orow * a.ldc + sl * VB, acc);
}

template <class T, class ACC, int VB, int SG, int VPL>
__device__ __forceinline__ void store_c(const MergeArgs &a, int row, int col0, int sl,
                                        const ACC (&acc)[VPL][VB]) {
  const int orow = a.out_row ? __ldg(a.out_row + row) : row;
  T *dst = static_cast<T *>(a.C) + (int64_t)orow * a.ldc + col0 + sl * VB;
#pragma unroll
  for (int v = 0; v < VPL; ++v)
    if (col0 + v * SG * VB + sl * VB < a.N) vstore<T, ACC, VB>(dst + v * SG * VB, acc[v]);
}

template <class ACC, int VB, int SG, int VPL>
__device__ __forceinline__ void store_partial(const MergeArgs &a, int slot, int col0, int sl,
                                              const ACC (&acc)[VPL][VB]) {
  ACC *dst = static_cast<ACC *>(a.scratch) + (int64_t)slot * a.N + col0 + sl * VB;
#pragma unroll
  for (int v = 0; v < VPL; ++v)
#pragma unroll
    for (int e = 0; e < VB; ++e)
      if (col0 + v * SG * VB + sl * VB + e < a.N) __stcg(dst + v * SG * VB + e, acc[v][e]);
}

// Counts this task's arrival for split row s; the last task adds the partials in task order.
template <class T, class ACC, int VB, int SG, int VPL, bool SCALE = false>
__device__ __forceinline__ void arrive(const MergeArgs &a, int s, int sl, unsigned sgmask) {
  __threadfence();
  __syncwarp(sgmask);
  int old = 0;
  if (sl == 0) old = atomicAdd(a.split_cnt + s, 1);
  old = __shfl_sync(sgmask, old, 0, SG);
  const int ta = a.split_first[s], tb = a.split_last[s];
  if (old != tb - ta) return;
  __threadfence();
  constexpr int CW = SG * VB * VPL;
  const ACC *scr = static_cast<const ACC *>(a.scratch);
  for (int col0 = 0; col0 < a.N; col0 += CW) {
    ACC acc[VPL][VB];
#pragma unroll
    for (int v = 0; v < VPL; ++v)
#pragma unroll
      for (int e = 0; e < VB; ++e) acc[v][e] = ACC(0);
    for (int t = ta; t <= tb; ++t) {
      const int slot = t == ta ? 2 * t + 1 : 2 * t;
      const ACC *src = scr + (int64_t)slot * a.N + col0 + sl * VB;
#pragma unroll
      for (int v = 0; v < VPL; ++v)
#pragma unroll
        for (int e = 0; e < VB; ++e)
          if (col0 + v * SG * VB + sl * VB + e < a.N) acc[v][e] += __ldcg(src + v * SG * VB + e);
    }
    if constexpr (SCALE) {  // the scaled walk's rows fit one chunk (N <= SG * VB, VPL == 1)
      const int row = a.split_row[s];
      store_scaled_row<T, ACC, VB, SG>(a, a.out_row ? __ldg(a.out_row + row) : row, sl, sgmask, acc[0],
                                       col0 + sl * VB < a.N);
    } else {
      store_c<T, ACC, VB, SG, VPL>(a, a.split_row[s], col0, sl, acc);
    }
  }
  __syncwarp(sgmask);
  if (sl == 0) a.split_cnt[s] = 0;  // ready for the next product
}

template <class T, class TA, class ACC, int VB, int SG, int VPL, int UNR, int MINB>
__global__ void __launch_bounds__(256, MINB) merge_spmm_kernel(const MergeArgs a) {
  constexpr int G = 32 / SG;
  constexpr int CW = SG * VB * VPL;
  const int lane = threadIdx.x & 31, sg = lane / SG, sl = lane % SG;
  const unsigned sgmask = SG == 32 ? 0xffffffffu : (((1u << SG) - 1u) << (sg * SG));
  const int t = (int)((blockIdx.x * (unsigned)blockDim.x + threadIdx.x) >> 5) * G + sg;
  if (t >= a.ntasks) return;
  const int64_t d0 = (int64_t)t * a.U;
  const int64_t d1 = d0 + a.U < a.total ? d0 + a.U : a.total;
  const int r = __ldg(a.task_row + t), rn = __ldg(a.task_row + t + 1);
  const int p = (int)(d0 - r), pn = (int)(d1 - rn);
  const int hs = __ldg(a.head_split + t), ts = __ldg(a.tail_split + t);
  const T *__restrict__ B = static_cast<const T *>(a.B);
  const TA *__restrict__ val = static_cast<const TA *>(a.val);
  for (int col0 = 0; col0 < a.N; col0 += CW) {
    bool inb[VPL];
#pragma unroll
    for (int v = 0; v < VPL; ++v) inb[v] = col0 + v * SG * VB + sl * VB < a.N;
    ACC acc[VPL][VB];
#pragma unroll
    for (int v = 0; v < VPL; ++v)
#pragma unroll
      for (int e = 0; e < VB; ++e) acc[v][e] = ACC(0);
    int cur = r;
    int rbase = cur;
    int myend = rbase + 1 + sl <= a.rows ? __ldg(a.ptr + rbase + 1 + sl) : 0x7fffffff;
    int pe = __shfl_sync(sgmask, myend, 0, SG);
    // stores row `cur` (or its head partial) and advances to the next row
    auto finish_and_advance = [&]() {
      if (cur == r && hs >= 0) store_partial<ACC, VB, SG, VPL>(a, 2 * t, col0, sl, acc);
      else store_c<T, ACC, VB, SG, VPL>(a, cur, col0, sl, acc);
#pragma unroll
      for (int v = 0; v < VPL; ++v)
#pragma unroll
        for (int e = 0; e < VB; ++e) acc[v][e] = ACC(0);
      ++cur;
      if (cur - rbase >= SG) {
        rbase = cur;
        myend = rbase + 1 + sl <= a.rows ? __ldg(a.ptr + rbase + 1 + sl) : 0x7fffffff;
      }
      pe = __shfl_sync(sgmask, myend, cur - rbase, SG);
    };
    // (index, value) pairs are fetched one chunk ahead of their use
    int nxc = 0;
    ACC nxv = ACC(0);
    if (p + sl < pn) {
      nxc = __ldcs(a.idx + p + sl);
      nxv = (ACC)__ldcs(val + p + sl);
    }
    for (int q0 = p; q0 < pn; q0 += SG) {
      const int m = min(SG, pn - q0);
      const int myc = nxc;
      const ACC myv = nxv;
      if (q0 + SG + sl < pn) {
        nxc = __ldcs(a.idx + q0 + SG + sl);
        nxv = (ACC)__ldcs(val + q0 + SG + sl);
      }
      for (int k = 0; k < m; k += UNR) {
        ACC b[UNR][VPL][VB];
#pragma unroll
        for (int u = 0; u < UNR; ++u) {
          const int c = __shfl_sync(sgmask, myc, (k + u) & (SG - 1), SG);
          const bool ok = k + u < m;
          const T *row = B + (int64_t)c * a.ldb + col0 + sl * VB;
#pragma unroll
          for (int v = 0; v < VPL; ++v) {
            if (ok && inb[v]) vload<T, ACC, VB>(row + v * SG * VB, b[u][v]);
            else {
#pragma unroll
              for (int e = 0; e < VB; ++e) b[u][v][e] = ACC(0);
            }
          }
        }
#pragma unroll
        for (int u = 0; u < UNR; ++u) {
          if (k + u >= m) break;
          const int q = q0 + k + u;
          while (q == pe) finish_and_advance();
          const ACC w = __shfl_sync(sgmask, myv, (k + u) & (SG - 1), SG);
#pragma unroll
          for (int v = 0; v < VPL; ++v)
#pragma unroll
            for (int e = 0; e < VB; ++e) acc[v][e] = fma(w, b[u][v][e], acc[v][e]);
        }
      }
    }
    while (cur < rn) finish_and_advance();
    if (ts >= 0) store_partial<ACC, VB, SG, VPL>(a, (hs >= 0 && r == rn) ? 2 * t : 2 * t + 1, col0, sl, acc);
  }
  if (hs >= 0 && r < rn) arrive<T, ACC, VB, SG, VPL>(a, hs, sl, sgmask);
  if (ts >= 0) arrive<T, ACC, VB, SG, VPL>(a, ts, sl, sgmask);
}

// Lean variant for the common case where one vector per lane spans the whole C row slice
// (N <= SG * VB): the same walk with the least live state, so that up to 64 warps fit on an
// SM -- for this gather pattern occupancy, not loads per warp, sets the throughput.
template <class T, class TA, class ACC, int VB, int SG, int UNR, int MINB>
__global__ void __launch_bounds__(256, MINB) merge_lean_kernel(const MergeArgs a) {
  constexpr int G = 32 / SG;
  const int lane = threadIdx.x & 31, sg = lane / SG, sl = lane % SG;
  const unsigned sgmask = SG == 32 ? 0xffffffffu : (((1u << SG) - 1u) << (sg * SG));
  const int t = (int)((blockIdx.x * (unsigned)blockDim.x + threadIdx.x) >> 5) * G + sg;
  if (t >= a.ntasks) return;
  const int4 hdr = __ldg(reinterpret_cast<const int4 *>(a.task_hdr) + t);  // r, rn, hs, ts
  const int64_t d0 = (int64_t)t * a.U;
  const int p = (int)(d0 - hdr.x);
  const int pn = (int)((d0 + a.U < a.total ? d0 + a.U : a.total) - hdr.y);
  const bool inb = sl * VB < a.N;
  ACC acc[VB];
#pragma unroll
  for (int e = 0; e < VB; ++e) acc[e] = ACC(0);
  // row ends of the next SG rows, one per lane; the block after it is fetched one block ahead
  // so that crossing into it never waits on memory
  int cur = hdr.x, rbase = cur;
  auto rowend = [&](int r) { return r <= a.rows ? __ldg(a.ptr + r) : 0x7fffffff; };
  int myend = rowend(rbase + 1 + sl);
  int myend2 = rowend(rbase + SG + 1 + sl);
  int pe = __shfl_sync(sgmask, myend, 0, SG);
  auto finish_and_advance = [&]() {
    if (cur == hdr.x && hdr.z >= 0) {
      ACC *dst = static_cast<ACC *>(a.scratch) + (int64_t)(2 * t) * a.N + sl * VB;
      if (inb) {
#pragma unroll
        for (int e = 0; e < VB; ++e) __stcg(dst + e, acc[e]);
      }
    } else if (inb) {
      const int orow = a.out_row ? __ldg(a.out_row + cur) : cur;
      vstore<T, ACC, VB>(static_cast<T *>(a.C) + (int64_t)orow * a.ldc + sl * VB, acc);
    }
#pragma unroll
    for (int e = 0; e < VB; ++e) acc[e] = ACC(0);
    ++cur;
    if (cur - rbase >= SG) {
      rbase += SG;
      myend = myend2;
      myend2 = rowend(rbase + SG + 1 + sl);
    }
    pe = __shfl_sync(sgmask, myend, cur - rbase, SG);
  };
  const T *__restrict__ Bl = static_cast<const T *>(a.B) + sl * VB;
  for (int q0 = p; q0 < pn; q0 += SG) {
    const int m = min(SG, pn - q0);
    int myc = 0;
    ACC myv = ACC(0);
    if (sl < m) {
      myc = __ldcs(a.idx + q0 + sl);
      myv = (ACC)__ldcs(static_cast<const TA *>(a.val) + q0 + sl);
    }
    for (int k = 0; k < m; k += UNR) {
      ACC b[UNR][VB];
#pragma unroll
      for (int u = 0; u < UNR; ++u) {
        const int c = __shfl_sync(sgmask, myc, (k + u) & (SG - 1), SG);
        if (k + u < m && inb) vload<T, ACC, VB>(Bl + (int64_t)c * a.ldb, b[u]);
        else {
#pragma unroll
          for (int e = 0; e < VB; ++e) b[u][e] = ACC(0);
        }
      }
#pragma unroll
      for (int u = 0; u < UNR; ++u) {
        if (k + u >= m) break;
        while (q0 + k + u == pe) finish_and_advance();
        const ACC w = __shfl_sync(sgmask, myv, (k + u) & (SG - 1), SG);
#pragma unroll
        for (int e = 0; e < VB; ++e) acc[e] = fma(w, b[u][e], acc[e]);
      }
    }
  }
  while (cur < hdr.y) finish_and_advance();
  if (hdr.w >= 0 && inb) {
    ACC *dst = static_cast<ACC *>(a.scratch) + (int64_t)((hdr.z >= 0 && hdr.x == hdr.y) ? 2 * t : 2 * t + 1) * a.N + sl * VB;
#pragma unroll
    for (int e = 0; e < VB; ++e) __stcg(dst + e, acc[e]);
  }
  if (hdr.z >= 0 && hdr.x < hdr.y) arrive<T, ACC, VB, SG, 1>(a, hdr.z, sl, sgmask);
  if (hdr.w >= 0) arrive<T, ACC, VB, SG, 1>(a, hdr.w, sl, sgmask);
}

// Streamlined walk: the execution copy of the gather indices carries bit 31 on the first
// nonzero of every row, so the end-of-row bookkeeping is skipped unless a batch holds a row
// start; (index, value) pairs of a 32-nonzero chunk are staged in shared memory and read back
// with one broadcast load per nonzero; full chunks run fully unrolled.
// One task of the flagged walk by one sub-warp (sl = lane within the sub-warp, stage = its
// 32-entry staging buffer).
// SCALE (16-bit B and C only): values multiplied by their column's b_scale as they are staged,
// each finished row divided by its power-of-two scale and the scale written to c_scale.
template <class T, class TA, class ACC, int VB, int SG, bool FULL = false, bool SCALE = false>
__device__ __forceinline__ void flag_walk(const MergeArgs &a, int t, int sl, unsigned sgmask,
                                          int2 *stage, ACC *vstage) {
  static_assert(!SCALE || (sizeof(T) == 2 && sizeof(TA) == 4), "scaled walk: 16-bit B and C, FP32 values");
  // FP32 values ride in stage[].y; FP64 values are staged in vstage
  constexpr int UNR = 4;
  const int4 hdr = __ldg(reinterpret_cast<const int4 *>(a.task_hdr) + t);  // r, rn, hs, ts
  const int64_t d0 = (int64_t)t * a.U;
  const int p = (int)(d0 - hdr.x);
  const int pn = (int)((d0 + a.U < a.total ? d0 + a.U : a.total) - hdr.y);
  const bool inb = FULL || sl * VB < a.N;
  ACC acc[VB];
#pragma unroll
  for (int e = 0; e < VB; ++e) acc[e] = ACC(0);
  // row ends of the next SG rows, one per lane; the block after it is fetched one block ahead
  // so that crossing into it never waits on memory
  int cur = hdr.x, rbase = cur;
  auto rowend = [&](int r) { return r <= a.rows ? __ldg(a.ptr + r) : 0x7fffffff; };
  int myend = rowend(rbase + 1 + sl);
  int myend2 = rowend(rbase + SG + 1 + sl);
  int pe = __shfl_sync(sgmask, myend, 0, SG);
  auto finish_and_advance = [&]() {
    if (cur == hdr.x && hdr.z >= 0) {
      ACC *dst = static_cast<ACC *>(a.scratch) + (int64_t)(2 * t) * a.N + sl * VB;
      if (inb) {
#pragma unroll
        for (int e = 0; e < VB; ++e) __stcg(dst + e, acc[e]);
      }
    } else if constexpr (SCALE) {
      store_scaled_row<T, ACC, VB, SG>(a, a.out_row ? __ldg(a.out_row + cur) : cur, sl, sgmask, acc, inb);
    } else if (inb) {
      const int orow = a.out_row ? __ldg(a.out_row + cur) : cur;
      vstore<T, ACC, VB>(static_cast<T *>(a.C) + (int64_t)orow * a.ldc + sl * VB, acc);
    }
#pragma unroll
    for (int e = 0; e < VB; ++e) acc[e] = ACC(0);
    ++cur;
    if (cur - rbase >= SG) {
      rbase += SG;
      myend = myend2;
      myend2 = rowend(rbase + SG + 1 + sl);
    }
    pe = __shfl_sync(sgmask, myend, cur - rbase, SG);
  };
  auto accumulate = [&](ACC w, const BVec<T, ACC, VB> &b) { b.template fma_into<true>(acc, w); };
  auto value_at = [&](int j) -> ACC {
    if constexpr (sizeof(TA) == 8) return vstage[j];
    else return (ACC)__int_as_float(stage[j].y);
  };
  const char *Bl = reinterpret_cast<const char *>(static_cast<const T *>(a.B) + sl * VB);
  const uint32_t ldb_bytes = (uint32_t)(a.ldb * (int64_t)sizeof(T));  // < 2^32 (checked at launch)
  const TA *val = static_cast<const TA *>(a.val);
  for (int q0 = p; q0 < pn; q0 += 32) {
    const int m = min(32, pn - q0);
    __syncwarp(sgmask);
#pragma unroll
    for (int j = sl; j < 32; j += SG) {
      int2 e = make_int2(0, 0);
      if (j < m) {
        e.x = __ldcs(a.idx + q0 + j);
        if constexpr (sizeof(TA) == 8) {
          vstage[j] = (ACC)__ldcs(val + q0 + j);
        } else if constexpr (SCALE) {  // B_true = b_scale * B (b_scale may be null)
          const float bs = a.b_scale ? __ldg(a.b_scale + (e.x & 0x7fffffff)) : 1.f;
          e.y = __float_as_int((float)__ldcs(val + q0 + j) * bs);
        } else {
          e.y = __float_as_int((float)__ldcs(val + q0 + j));
        }
      }
      stage[j] = e;
    }
    __syncwarp(sgmask);
    if (m == 32) {
#pragma unroll 1
      for (int k = 0; k < 32; k += UNR) {
        BVec<T, ACC, VB> b[UNR];
        int flags = 0;
#pragma unroll
        for (int u = 0; u < UNR; ++u) {
          const int c = stage[k + u].x;
          flags |= c;
          if (inb) b[u].load(reinterpret_cast<const T *>(Bl + (uint64_t)(uint32_t)(c & 0x7fffffff) * ldb_bytes));
          else b[u].zero();
        }
        if (flags < 0) {
#pragma unroll
          for (int u = 0; u < UNR; ++u) {
            while (q0 + k + u == pe) finish_and_advance();
            accumulate(value_at(k + u), b[u]);
          }
        } else {
#pragma unroll
          for (int u = 0; u < UNR; ++u) accumulate(value_at(k + u), b[u]);
        }
      }
    } else {
      for (int k = 0; k < m; ++k) {
        const int c = stage[k].x;
        BVec<T, ACC, VB> b;
        if (inb) b.load(reinterpret_cast<const T *>(Bl + (uint64_t)(uint32_t)(c & 0x7fffffff) * ldb_bytes));
        else b.zero();
        while (q0 + k == pe) finish_and_advance();
        accumulate(value_at(k), b);
      }
    }
  }
  while (cur < hdr.y) finish_and_advance();
  if (hdr.w >= 0 && inb) {
    ACC *dst = static_cast<ACC *>(a.scratch) + (int64_t)((hdr.z >= 0 && hdr.x == hdr.y) ? 2 * t : 2 * t + 1) * a.N + sl * VB;
#pragma unroll
    for (int e = 0; e < VB; ++e) __stcg(dst + e, acc[e]);
  }
  if (hdr.z >= 0 && hdr.x < hdr.y) arrive<T, ACC, VB, SG, 1, SCALE>(a, hdr.z, sl, sgmask);
  if (hdr.w >= 0) arrive<T, ACC, VB, SG, 1, SCALE>(a, hdr.w, sl, sgmask);
}

template <class T, class TA, class ACC, int VB, int SG, int MINB, bool FULL, bool SCALE = false>
__global__ void __launch_bounds__(256, MINB) merge_flag_kernel(const MergeArgs a) {
  constexpr int G = 32 / SG;
  // one staging row per sub-warp, padded by one element: the sub-warps of a warp read their
  // rows with broadcast loads in the same instruction, and unpadded 256-byte rows would put
  // those reads on the same banks
  __shared__ int2 stage_all[8 * G][33];
  __shared__ ACC vstage_all[sizeof(TA) == 8 ? 8 * G : 1][33];
  const int lane = threadIdx.x & 31, sg = lane / SG, sl = lane % SG;
  const unsigned sgmask = SG == 32 ? 0xffffffffu : (((1u << SG) - 1u) << (sg * SG));
  const int t = (int)((blockIdx.x * (unsigned)blockDim.x + threadIdx.x) >> 5) * G + sg;
  if (t >= a.ntasks) return;
  const int w = (threadIdx.x >> 5) * G + sg;
  flag_walk<T, TA, ACC, VB, SG, FULL, SCALE>(a, t, sl, sgmask, stage_all[w], vstage_all[sizeof(TA) == 8 ? w : 0]);
}

// ---------------------------------------------------------------- staged walk
// cp.async (16 bytes per lane, completion tracked per thread in commit order).
__device__ __forceinline__ void cp_async16(void *smem, const void *gmem) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int NPEND>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;" ::"n"(NPEND) : "memory");
}

// Shared memory of the staged walk per 256-thread block: every lane's ring of D 16-byte
// slots, then per sub-warp a ring of NCH chunks of 32 (index, value) pairs.
constexpr int staged_nch(int D) { return D / 4 - 1 <= 4 ? 2 : 4; }
constexpr int staged_smem(int SG, int D) { return 8 * 32 * D * 16 + 8 * (32 / SG) * staged_nch(D) * 32 * 8; }
constexpr int staged_minb(int SG, int D) {
  const int b = (227 * 1024) / (staged_smem(SG, D) + 1024);
  return b < 1 ? 1 : (b > 6 ? 6 : b);
}

// Staged walk (FP32 values, B and C; N == SG * 4, so every lane holds one 16-byte slice of a
// row).  Nonzeros go in groups of four (aligned to multiples of 4 in the nonzero order); each
// lane keeps its slices of the next D / 4 - 1 groups' B rows in flight in a lane-private ring
// of D slots of shared memory, filled by cp.async -- so the bytes in flight per SM are bounded
// by shared memory rather than by registers, and one wait, one commit and two 16-byte reads of
// (indices, values) serve four nonzeros.  Chunks of 32 (index, value) pairs ride the same copy
// groups into a ring one or two chunks ahead.  Copies complete in commit order: waiting until
// at most D / 4 - 2 groups are pending makes the current group's slices visible to the lane,
// and a __syncwarp after the wait that covers a staging copy makes the staged chunk visible to
// every lane.  The partial groups at the ends of a task take plain loads.  Row bookkeeping,
// split rows and results are those of the flagged walk.
template <int SG, int D, int MINB>
__global__ void __launch_bounds__(256, MINB) merge_staged_kernel(const MergeArgs a) {
  constexpr int G = 32 / SG;
  constexpr int LAG = D / 4 - 1;  // groups in flight per lane
  constexpr int NCH = staged_nch(D);
  constexpr int SMASK = NCH * 32 - 1;
  static_assert((D & (D - 1)) == 0 && LAG >= 1 && LAG <= 8, "ring depth");
  extern __shared__ float4 staged_dyn[];
  const int lane = threadIdx.x & 31, sg = lane / SG, sl = lane % SG;
  const unsigned sgmask = SG == 32 ? 0xffffffffu : (((1u << SG) - 1u) << (sg * SG));
  const int t = (int)((blockIdx.x * (unsigned)blockDim.x + threadIdx.x) >> 5) * G + sg;
  if (t >= a.ntasks) return;
  const int w = (threadIdx.x >> 5) * G + sg;
  float4 *ring = staged_dyn + (threadIdx.x >> 5) * 32 * D;  // [D][32 lanes] per warp
  int *sidx = reinterpret_cast<int *>(staged_dyn + 8 * 32 * D) + w * (NCH * 64);
  float *sval = reinterpret_cast<float *>(sidx + NCH * 32);
  const int4 hdr = __ldg(reinterpret_cast<const int4 *>(a.task_hdr) + t);  // r, rn, hs, ts
  const int64_t d0 = (int64_t)t * a.U;
  const int p = (int)(d0 - hdr.x);
  const int pn = (int)((d0 + a.U < a.total ? d0 + a.U : a.total) - hdr.y);
  const int nnz = (int)(a.total - a.rows);
  float acc[4] = {0.f, 0.f, 0.f, 0.f};
  int cur = hdr.x, rbase = cur;
  auto rowend = [&](int r) { return r <= a.rows ? __ldg(a.ptr + r) : 0x7fffffff; };
  int myend = rowend(rbase + 1 + sl);
  int myend2 = rowend(rbase + SG + 1 + sl);
  int pe = __shfl_sync(sgmask, myend, 0, SG);
  auto finish_and_advance = [&]() {
    if (cur == hdr.x && hdr.z >= 0) {
      float *dst = static_cast<float *>(a.scratch) + (int64_t)(2 * t) * a.N + sl * 4;
#pragma unroll
      for (int e = 0; e < 4; ++e) __stcg(dst + e, acc[e]);
    } else {
      const int orow = a.out_row ? __ldg(a.out_row + cur) : cur;
      vstore<float, float, 4>(static_cast<float *>(a.C) + (int64_t)orow * a.ldc + sl * 4, acc);
    }
#pragma unroll
    for (int e = 0; e < 4; ++e) acc[e] = 0.f;
    ++cur;
    if (cur - rbase >= SG) {
      rbase += SG;
      myend = myend2;
      myend2 = rowend(rbase + SG + 1 + sl);
    }
    pe = __shfl_sync(sgmask, myend, cur - rbase, SG);
  };
  auto accumulate = [&](float wv, const float4 &b) {
    const float bv[4] = {b.x, b.y, b.z, b.w};
    fma_vec<float, 4>(acc, wv, bv);
  };
  const char *Bl = reinterpret_cast<const char *>(static_cast<const float *>(a.B) + sl * 4);
  const uint32_t ldb_bytes = (uint32_t)(a.ldb * (int64_t)sizeof(float));  // < 2^32 (checked at launch)
  const int *vbits = static_cast<const int *>(a.val);
  // one nonzero without the pipeline (the partial groups at a task's ends)
  auto single = [&](int x) {
    const int c = __ldg(a.idx + x);
    const float wv = __int_as_float(__ldg(vbits + x));
    const float4 b = __ldg(reinterpret_cast<const float4 *>(Bl + (uint64_t)(uint32_t)(c & 0x7fffffff) * ldb_bytes));
    if (c < 0) {
      while (x == pe) finish_and_advance();
    }
    accumulate(wv, b);
  };
  const int g0 = (p + 3) >> 2, g1 = pn >> 2;  // full groups [g0, g1)
  if (g0 >= g1) {
    for (int x = p; x < pn; ++x) single(x);
  } else {
    for (int x = p; x < 4 * g0; ++x) single(x);
    // chunk k = nonzeros [32k, 32k + 32): 8 pieces of 4 indices, 8 pieces of 4 values
    auto stage = [&](int k) {
      for (int pc = sl; pc < 16; pc += SG) {
        const int part = pc & 7, e0 = 32 * k + part * 4;
        int *dst = (pc < 8 ? sidx : reinterpret_cast<int *>(sval)) + ((32 * k) & SMASK) + part * 4;
        const int *src = (pc < 8 ? a.idx : vbits) + e0;
        if (e0 + 4 <= nnz) {
          cp_async16(dst, src);
        } else {
#pragma unroll
          for (int i = 0; i < 4; ++i) dst[i] = e0 + i < nnz ? __ldg(src + i) : 0;
        }
      }
    };
    auto issue = [&](int g) {
      const int4 c = *reinterpret_cast<const int4 *>(sidx + ((4 * g) & SMASK));
      float4 *slot = ring + ((4 * g) & (D - 1)) * 32 + lane;
      cp_async16(slot, Bl + (uint64_t)((uint32_t)c.x & 0x7fffffffu) * ldb_bytes);
      cp_async16(slot + 32, Bl + (uint64_t)((uint32_t)c.y & 0x7fffffffu) * ldb_bytes);
      cp_async16(slot + 64, Bl + (uint64_t)((uint32_t)c.z & 0x7fffffffu) * ldb_bytes);
      cp_async16(slot + 96, Bl + (uint64_t)((uint32_t)c.w & 0x7fffffffu) * ldb_bytes);
    };
    // the ring holds NCH chunks: the current one and the NCH - 1 after it
    const int k0 = g0 >> 3;
#pragma unroll 1
    for (int k = k0; k < k0 + NCH; ++k)
      if (32 * k < 4 * g1) stage(k);
    cp_async_commit();
    cp_async_wait<0>();
    __syncwarp(sgmask);
#pragma unroll 1
    for (int i = 0; i < LAG; ++i) {
      if (g0 + i < g1) issue(g0 + i);
      cp_async_commit();
    }
#pragma unroll 1
    for (int g = g0; g < g1; ++g) {
      cp_async_wait<LAG - 1>();
      if ((g & 7) == (LAG & 7)) __syncwarp(sgmask);  // the chunk staged LAG groups ago
      const int x0 = 4 * g;
      const int4 c = *reinterpret_cast<const int4 *>(sidx + (x0 & SMASK));
      const float4 wv = *reinterpret_cast<const float4 *>(sval + (x0 & SMASK));
      const float4 *slot = ring + (x0 & (D - 1)) * 32 + lane;
      const float4 b0 = slot[0], b1 = slot[32], b2 = slot[64], b3 = slot[96];
      if ((c.x | c.y | c.z | c.w) < 0) {
        if (c.x < 0) { while (x0 == pe) finish_and_advance(); }
        accumulate(wv.x, b0);
        if (c.y < 0) { while (x0 + 1 == pe) finish_and_advance(); }
        accumulate(wv.y, b1);
        if (c.z < 0) { while (x0 + 2 == pe) finish_and_advance(); }
        accumulate(wv.z, b2);
        if (c.w < 0) { while (x0 + 3 == pe) finish_and_advance(); }
        accumulate(wv.w, b3);
      } else {
        accumulate(wv.x, b0);
        accumulate(wv.y, b1);
        accumulate(wv.z, b2);
        accumulate(wv.w, b3);
      }
      if ((g & 7) == 0 && g != g0) {
        const int k = (g >> 3) + NCH - 1;  // into the slot of chunk (g >> 3) - 1, now consumed
        if (32 * k < 4 * g1) {
          __syncwarp(sgmask);  // the slots being refilled were read by every lane
          stage(k);
        }
      }
      if (g + LAG < g1) issue(g + LAG);
      cp_async_commit();
    }
    cp_async_wait<0>();
    for (int x = 4 * g1; x < pn; ++x) single(x);
  }
  while (cur < hdr.y) finish_and_advance();
  if (hdr.w >= 0) {
    float *dst = static_cast<float *>(a.scratch) + (int64_t)((hdr.z >= 0 && hdr.x == hdr.y) ? 2 * t : 2 * t + 1) * a.N + sl * 4;
#pragma unroll
    for (int e = 0; e < 4; ++e) __stcg(dst + e, acc[e]);
  }
  if (hdr.z >= 0 && hdr.x < hdr.y) arrive<float, float, 4, SG, 1>(a, hdr.z, sl, sgmask);
  if (hdr.w >= 0) arrive<float, float, 4, SG, 1>(a, hdr.w, sl, sgmask);
}

// ---------------------------------------------------------------- backward walks
// One pass over A in row order for any of: Y = A X (DOY); dA_e = dY[row_e] . X[col_e] (DODA);
// and, for A == A^T with equal values, dX = A^T dY = A dY (DODX: dY rows are gathered like
// X rows).  A gathered X row serves both Y and dA; the current row's dY slice stays in
// registers.  dA is reduced across the sub-warp four nonzeros at a time (5 shuffles per 4).
struct BwdArgs {
  MergeArgs m;     // X in m.B / m.ldb, Y in m.C / m.ldc, Y partials in m.scratch
  const void *dY;  // M x N: per-row operand of dA, gathered operand of dX
  int64_t lddy;
  void *dX;
  int64_t lddx;
  void *dA;        // nnz values in CSR order
};

// Sum over the SG lanes of a sub-warp of four per-lane values; every lane returns the total
// of value (2 * h1 + h2), h1 = lane bit SG/2, h2 = lane bit SG/4.  Needs SG >= 4.
template <class T, int SG>
__device__ __forceinline__ T reduce4(T p0, T p1, T p2, T p3, int sl, unsigned m) {
  const bool h1 = sl & (SG / 2), h2 = sl & (SG / 4);
  T k0 = h1 ? p2 : p0, k1 = h1 ? p3 : p1;
  const T s0 = h1 ? p0 : p2, s1 = h1 ? p1 : p3;
  k0 += __shfl_xor_sync(m, s0, SG / 2, SG);
  k1 += __shfl_xor_sync(m, s1, SG / 2, SG);
  T k = h2 ? k1 : k0;
  const T s = h2 ? k0 : k1;
  k += __shfl_xor_sync(m, s, SG / 4, SG);
#pragma unroll
  for (int o = SG / 8; o >= 1; o >>= 1) k += __shfl_xor_sync(m, k, o, SG);
  return k;
}

template <class T, int SG>
__device__ __forceinline__ T reduce1(T v, unsigned m) {
#pragma unroll
  for (int o = SG / 2; o >= 1; o >>= 1) v += __shfl_xor_sync(m, v, o, SG);
  return v;
}

// Last-arriving task of split row s adds the partials in task order.  Scratch rows hold
// W = N values, or 2N when [Y | dX] are produced together (lanes of the second half of the
// sub-warp own dX).
template <class T, int VB, int SG, bool DODX>
__device__ __forceinline__ void arrive_bwd(const BwdArgs &ba, int s, int sl, unsigned sgmask) {
  const MergeArgs &a = ba.m;
  __threadfence();
  __syncwarp(sgmask);
  int old = 0;
  if (sl == 0) old = atomicAdd(a.split_cnt + s, 1);
  old = __shfl_sync(sgmask, old, 0, SG);
  const int ta = a.split_first[s], tb = a.split_last[s];
  if (old != tb - ta) return;
  __threadfence();
  constexpr int H = DODX ? SG / 2 : SG;
  const int row = a.split_row[s];
  const int role = DODX ? sl / H : 0, lsl = sl % H;
  const int64_t W = DODX ? 2 * (int64_t)a.N : a.N;
  if (lsl * VB < a.N) {
    T y[VB];
#pragma unroll
    for (int e = 0; e < VB; ++e) y[e] = T(0);
    const T *s1 = static_cast<const T *>(a.scratch);
    for (int t = ta; t <= tb; ++t) {
      const int64_t off = (int64_t)(t == ta ? 2 * t + 1 : 2 * t) * W + role * a.N + lsl * VB;
#pragma unroll
      for (int e = 0; e < VB; ++e) y[e] += __ldcg(s1 + off + e);
    }
    T *dst = role ? static_cast<T *>(ba.dX) + (int64_t)row * ba.lddx : static_cast<T *>(a.C) + (int64_t)row * a.ldc;
    vstore<T, T, VB>(dst + lsl * VB, y);
  }
  __syncwarp(sgmask);
  if (sl == 0) a.split_cnt[s] = 0;
}

// With DODX the sub-warp splits in two halves: lanes [0, SG/2) gather X rows and accumulate
// Y, lanes [SG/2, SG) gather dY rows and accumulate dX -- the product with [X | dY] of twice
// the width -- so each lane keeps one gathered vector per nonzero.
template <class T, int VB, int SG, bool DOY, bool DODA, bool DODX, int MINB>
__global__ void __launch_bounds__(256, MINB) merge_bwd_kernel(const BwdArgs ba) {
  static_assert(SG >= 4, "the four-value reduction needs sub-warps of 4 or more lanes");
  constexpr int G = 32 / SG;
  constexpr int UNR = 4;
  constexpr int H = DODX ? SG / 2 : SG;
  constexpr bool F64 = sizeof(T) == 8;
  __shared__ int2 stage_all[8 * G][33];  // padded as in merge_flag_kernel
  __shared__ T vstage_all[F64 ? 8 * G : 1][33];
  const MergeArgs &a = ba.m;
  const int lane = threadIdx.x & 31, sg = lane / SG, sl = lane % SG;
  const unsigned sgmask = SG == 32 ? 0xffffffffu : (((1u << SG) - 1u) << (sg * SG));
  const int t = (int)((blockIdx.x * (unsigned)blockDim.x + threadIdx.x) >> 5) * G + sg;
  if (t >= a.ntasks) return;
  int2 *stage = stage_all[(threadIdx.x >> 5) * G + sg];
  T *vstage = vstage_all[F64 ? (threadIdx.x >> 5) * G + sg : 0];
  const int role = DODX ? sl / H : 0, lsl = sl % H;
  const int64_t W = DODX ? 2 * (int64_t)a.N : a.N;
  const int4 hdr = __ldg(reinterpret_cast<const int4 *>(a.task_hdr) + t);  // r, rn, hs, ts
  const int64_t d0 = (int64_t)t * a.U;
  const int p = (int)(d0 - hdr.x);
  const int pn = (int)((d0 + a.U < a.total ? d0 + a.U : a.total) - hdr.y);
  const bool inb = lsl * VB < a.N;
  const bool full_lanes = a.N == H * VB;  // every lane of the sub-warp in range (warp-uniform)
  // dY rows are consumed in row order.  For SDDMM alone (registers to spare) the next row's
  // vector is fetched when the walk enters a row, so its latency overlaps the current row's
  // gathers; the fused passes load it on entry.
  constexpr bool PREU = DODA && !DOY && !DODX;
  T acc[VB], urow[VB], unext[PREU ? VB : 1];
#pragma unroll
  for (int e = 0; e < VB; ++e) acc[e] = urow[e] = T(0);
  const T *dYp = static_cast<const T *>(ba.dY);
  auto fetch_u = [&](int row, auto &dst) {
    if (DODA) {
      if (role == 0 && inb && row < a.rows) vload<T, T, VB>(dYp + (int64_t)row * ba.lddy + lsl * VB, dst);
      else {
#pragma unroll
        for (int e = 0; e < VB; ++e) dst[e] = T(0);
      }
    }
  };
  int cur = hdr.x, rbase = cur;
  int myend = rbase + 1 + sl <= a.rows ? __ldg(a.ptr + rbase + 1 + sl) : 0x7fffffff;
  int pe = __shfl_sync(sgmask, myend, 0, SG);
  fetch_u(cur, urow);
  if constexpr (PREU) fetch_u(cur + 1, unext);
  auto finish_and_advance = [&]() {
    if (DOY || DODX) {
      if (cur == hdr.x && hdr.z >= 0) {
        if (inb) {
          T *dst = static_cast<T *>(a.scratch) + (int64_t)(2 * t) * W + role * a.N + lsl * VB;
#pragma unroll
          for (int e = 0; e < VB; ++e) __stcg(dst + e, acc[e]);
        }
      } else if (inb) {
        T *dst = role ? static_cast<T *>(ba.dX) + (int64_t)cur * ba.lddx : static_cast<T *>(a.C) + (int64_t)cur * a.ldc;
        vstore<T, T, VB>(dst + lsl * VB, acc);
      }
#pragma unroll
      for (int e = 0; e < VB; ++e) acc[e] = T(0);
    }
    ++cur;
    if (cur - rbase >= SG) {
      rbase = cur;
      myend = rbase + 1 + sl <= a.rows ? __ldg(a.ptr + rbase + 1 + sl) : 0x7fffffff;
    }
    pe = __shfl_sync(sgmask, myend, cur - rbase, SG);
    if constexpr (PREU) {
#pragma unroll
      for (int e = 0; e < VB; ++e) urow[e] = unext[e];
      fetch_u(cur + 1, unext);
    } else {
      fetch_u(cur, urow);
    }
  };
  const char *Gl = role ? reinterpret_cast<const char *>(dYp + lsl * VB)
                        : reinterpret_cast<const char *>(static_cast<const T *>(a.B) + lsl * VB);
  // 32 x 32 -> 64-bit row offsets (the launch guarantees ld * sizeof(T) < 2^32)
  const uint32_t g_ld = (uint32_t)((role ? ba.lddy : a.ldb) * (int64_t)sizeof(T));
  constexpr unsigned LOW = SG == 32 ? 0xffffffffu : ((1u << SG) - 1u);
  const T *val = static_cast<const T *>(a.val);
  T *dA = static_cast<T *>(ba.dA);
  // SDDMM alone: a slot past the chunk's end holds column 0, so its gather stays in bounds and
  // its dot product is never stored -- the loads need no slot predicate, and lanes past N keep
  // the zeros set here (their loads are predicated off).
  BVec<T, T, VB> x[UNR];
#pragma unroll
  for (int u = 0; u < UNR; ++u) x[u].zero();
  for (int q0 = p; q0 < pn; q0 += 32) {
    const int m = min(32, pn - q0);
    unsigned rs = 0;
    __syncwarp(sgmask);
#pragma unroll
    for (int i = 0; i < 32 / SG; ++i) {
      const int j = sl + i * SG;
      int2 e = make_int2(0, 0);
      if (j < m) {
        e.x = __ldcs(a.idx + q0 + j);
        if (DOY || DODX) {
          if (F64) vstage[j] = __ldcs(val + q0 + j);
          else e.y = __float_as_int((float)__ldcs(val + q0 + j));
        }
      }
      rs |= ((__ballot_sync(sgmask, e.x < 0) >> (sg * SG)) & LOW) << (i * SG);
      e.x &= 0x7fffffff;
      stage[j] = e;
    }
    __syncwarp(sgmask);
    if (!PREU && m == 32 && full_lanes) {
      // a full chunk with every lane in range: unconditional loads, no per-slot checks
#pragma unroll 1
      for (int k = 0; k < 32; k += UNR) {
        T part[UNR];
#pragma unroll
        for (int u = 0; u < UNR; ++u) x[u].load(reinterpret_cast<const T *>(Gl + (uint64_t)(uint32_t)stage[k + u].x * g_ld));
        auto slot = [&](int u) {
          if (DOY || DODX) {
            const T w = F64 ? vstage[k + u] : (T)__int_as_float(stage[k + u].y);
            x[u].template fma_into<true>(acc, w);
          }
          if (DODA) {
            T d = T(0);
#pragma unroll
            for (int e = 0; e < VB; ++e) d = fma(urow[e], x[u].v[e], d);
            part[u] = d;
          }
        };
        if ((rs >> k) & 0xFu) {  // a row starts in this group: look for row ends slot by slot
#pragma unroll
          for (int u = 0; u < UNR; ++u) {
            while (q0 + k + u == pe) finish_and_advance();
            slot(u);
          }
        } else {
#pragma unroll
          for (int u = 0; u < UNR; ++u) slot(u);
        }
        if (DODA) {
          constexpr bool HALF = DODX && H >= 4;
          constexpr int RW = HALF ? H : SG;
          const int rl = HALF ? lsl : sl;
          const T r = reduce4<T, RW>(part[0], part[1], part[2], part[3], rl, sgmask);
          const int idx = ((rl & (RW / 2)) ? 2 : 0) + ((rl & (RW / 4)) ? 1 : 0);
          if ((!HALF || role == 0) && (rl & (RW / 4 - 1)) == 0) dA[q0 + k + idx] = r;
        }
      }
      continue;
    }
    for (int k = 0; k < m; k += UNR) {
      T part[UNR];
#pragma unroll
      for (int u = 0; u < UNR; ++u) {
        if constexpr (PREU) {
          if (inb) x[u].load(reinterpret_cast<const T *>(Gl + (uint64_t)(uint32_t)stage[k + u].x * g_ld));
        } else {
          const bool ok = k + u < m;
          const uint32_t c = ok ? (uint32_t)stage[k + u].x : 0u;
          if (inb && ok) x[u].load(reinterpret_cast<const T *>(Gl + (uint64_t)c * g_ld));
          else x[u].zero();
        }
        part[u] = T(0);
      }
      const bool starts = (rs >> k) & 0xFu;
#pragma unroll
      for (int u = 0; u < UNR; ++u) {
        if (k + u >= m) break;
        if (starts) {
          while (q0 + k + u == pe) finish_and_advance();
        }
        if (DOY || DODX) {
          const T w = F64 ? vstage[k + u] : (T)__int_as_float(stage[k + u].y);
          x[u].template fma_into<true>(acc, w);
        }
        if (DODA) {
          T d = T(0);
#pragma unroll
          for (int e = 0; e < VB; ++e) d = fma(urow[e], x[u].v[e], d);
          part[u] = d;
        }
      }
      if (DODA) {
        // with DODX only the X half holds partial dot products: reduce over it alone when it has
        // the four lanes the four-value reduction needs
        constexpr bool HALF = DODX && H >= 4;
        constexpr int RW = HALF ? H : SG;
        const int rl = HALF ? lsl : sl;
        const T r = reduce4<T, RW>(part[0], part[1], part[2], part[3], rl, sgmask);
        const int idx = ((rl & (RW / 2)) ? 2 : 0) + ((rl & (RW / 4)) ? 1 : 0);
        if ((!HALF || role == 0) && (rl & (RW / 4 - 1)) == 0 && k + idx < m) dA[q0 + k + idx] = r;
      }
    }
  }
  while (cur < hdr.y) finish_and_advance();
  if (DOY || DODX) {
    if (hdr.w >= 0 && inb) {
      T *dst = static_cast<T *>(a.scratch) + (int64_t)((hdr.z >= 0 && hdr.x == hdr.y) ? 2 * t : 2 * t + 1) * W +
               role * a.N + lsl * VB;
#pragma unroll
      for (int e = 0; e < VB; ++e) __stcg(dst + e, acc[e]);
    }
    if (hdr.z >= 0 && hdr.x < hdr.y) arrive_bwd<T, VB, SG, DODX>(ba, hdr.z, sl, sgmask);
    if (hdr.w >= 0) arrive_bwd<T, VB, SG, DODX>(ba, hdr.w, sl, sgmask);
  }
}

template <class T>
__global__ void sym_check_kernel(int M, const int *__restrict__ rowptr, const int *__restrict__ colidx,
                                 const T *__restrict__ val, const int *__restrict__ invperm,
                                 const int *__restrict__ sptr, const int *__restrict__ srow,
                                 const T *__restrict__ sval, int *__restrict__ bad) {
  const int warps = (gridDim.x * blockDim.x) >> 5, lane = threadIdx.x & 31;
  for (int r = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; r < M; r += warps) {
    const int i = invperm[r];
    const int a0 = rowptr[r], len = rowptr[r + 1] - a0, b0 = sptr[i];
    if (len != sptr[i + 1] - b0) {
      if (lane == 0) *bad = 1;
      continue;
    }
    for (int j = lane; j < len; j += 32)
      if (colidx[a0 + j] != srow[b0 + j] || !(val[a0 + j] == sval[b0 + j])) *bad = 1;
  }
}

// Batched products in one persistent launch: matrix i owns warp items
// [item_off[i], item_off[i+1]), each item G_i = 32 / SG_i consecutive tasks of its plan; the
// sub-warp width follows that matrix's N (16-byte vectors for N <= 128, or scalars for
// N <= 32).  Warps stride over the items of all matrices; every matrix's split rows are
// combined by its own counters exactly as in a single product.
__global__ void __launch_bounds__(256, 4) merge_batch_kernel(const MergeArgs *__restrict__ args,
                                                             const int *__restrict__ shape,
                                                             const int64_t *__restrict__ item_off,
                                                             int count) {
  __shared__ int2 stage_all[8 * 4][33];  // padded as in merge_flag_kernel
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int64_t total = __ldg(item_off + count);
  const int64_t nw = (int64_t)gridDim.x * 8;
  for (int64_t w = (int64_t)blockIdx.x * 8 + warp; w < total; w += nw) {
    __syncwarp();
    int lo = 0, hi = count;
    while (hi - lo > 1) {
      const int mid = (lo + hi) >> 1;
      if (__ldg(item_off + mid) <= w) lo = mid; else hi = mid;
    }
    const MergeArgs &a = args[lo];
    const int item = (int)(w - __ldg(item_off + lo));
    switch (__ldg(shape + lo)) {
#define SW_BATCH_SHAPE(CODE, VB_, SG_, FULL_)                                                          \
  case CODE: {                                                                                  \
    const int sg = lane / SG_, sl = lane % SG_;                                                 \
    const unsigned m = SG_ == 32 ? 0xffffffffu : (((1u << SG_) - 1u) << (sg * SG_));            \
    const int t = item * (32 / SG_) + sg;                                                       \
    if (t < a.ntasks) flag_walk<float, float, float, VB_, SG_, FULL_>(a, t, sl, m, stage_all[warp * 4 + sg], nullptr); \
    break;                                                                                      \
  }
      SW_BATCH_SHAPE(0, 4, 8, false)
      SW_BATCH_SHAPE(1, 4, 16, false)
      SW_BATCH_SHAPE(2, 4, 32, false)
      SW_BATCH_SHAPE(3, 1, 32, false)
      SW_BATCH_SHAPE(4, 4, 8, true)
      SW_BATCH_SHAPE(5, 4, 16, true)
      SW_BATCH_SHAPE(6, 4, 32, true)
#undef SW_BATCH_SHAPE
      default: break;
    }
  }
}

// Execution copy of the gather indices with bit 31 on the first nonzero of every row.
__global__ void row_start_set_kernel(const int *__restrict__ ptr, int rows, int *__restrict__ eidx) {
  for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < rows;
       r += (int64_t)gridDim.x * blockDim.x)
    if (ptr[r + 1] > ptr[r]) eidx[ptr[r]] |= (int)0x80000000u;
}

// ------------------------------------------------------------------ plan-time task build
// Packs (task_row[t], task_row[t+1], head_split[t], tail_split[t]) for the lean kernel.
__global__ void task_hdr_kernel(const int *__restrict__ task_row, const int *__restrict__ hs,
                                const int *__restrict__ ts, int ntasks, int4 *__restrict__ hdr) {
  for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < ntasks;
       t += (int64_t)gridDim.x * blockDim.x)
    hdr[t] = make_int4(task_row[t], task_row[t + 1], hs[t], ts[t]);
}

__global__ void sdd_hdr_kernel(const int *__restrict__ task_row, int ntasks, int4 *__restrict__ hdr) {
  for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < ntasks;
       t += (int64_t)gridDim.x * blockDim.x)
    hdr[t] = make_int4(task_row[t], task_row[t + 1], -1, -1);
}

// task_row[t] = smallest row whose span reaches position t*U (rows for t = ntasks).
__global__ void task_row_kernel(const int *__restrict__ ptr, int rows, int64_t total, int U,
                                int ntasks, int *__restrict__ task_row) {
  for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t <= ntasks;
       t += (int64_t)gridDim.x * blockDim.x) {
    const int64_t d = t * (int64_t)U < total ? t * (int64_t)U : total;
    int lo = 0, hi = rows;  // answer in [0, rows]
    while (lo < hi) {
      const int mid = (lo + hi) >> 1;
      if ((int64_t)__ldg(ptr + mid + 1) + mid >= d) hi = mid; else lo = mid + 1;
    }
    task_row[t] = (t == ntasks) ? rows : lo;
  }
}

__global__ void split_flag_kernel(const int *__restrict__ ptr, int rows, int U, int *__restrict__ flag) {
  for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < rows;
       r += (int64_t)gridDim.x * blockDim.x) {
    const int64_t first = (int64_t)ptr[r] + r, last = (int64_t)ptr[r + 1] + r;
    flag[r] = (first / U) != (last / U);
  }
}

__global__ void split_fill_kernel(const int *__restrict__ ptr, int rows, int U,
                                  const int *__restrict__ pos, int *__restrict__ split_row,
                                  int *__restrict__ split_first, int *__restrict__ split_last,
                                  int *__restrict__ head_split, int *__restrict__ tail_split) {
  for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < rows;
       r += (int64_t)gridDim.x * blockDim.x) {
    const int64_t first = (int64_t)ptr[r] + r, last = (int64_t)ptr[r + 1] + r;
    const int ta = (int)(first / U), tb = (int)(last / U);
    if (ta == tb) continue;
    const int s = pos[r];
    split_row[s] = (int)r;
    split_first[s] = ta;
    split_last[s] = tb;
    tail_split[ta] = s;
    head_split[tb] = s;
    for (int t = ta + 1; t < tb; ++t) { head_split[t] = s; tail_split[t] = s; }
  }
}

int grid_n(int64_t n) { return (int)std::max<int64_t>(1, std::min<int64_t>((n + 255) / 256, 148 * 16)); }

}  // namespace

swift_status build_merge_tasks(RowLayout &L, int U, cudaStream_t st) {
  if (L.merge_U == U && L.merge_built) return SWIFT_OK;
  const int rows = L.rows;
  const int64_t total = (int64_t)L.nnz + rows;
  const int64_t nt = (total + U - 1) / U;
  if (nt >= INT32_MAX / 2) return SWIFT_ERR_OVERFLOW;
  L.ntasks = (int)nt;
  SW_TRY(L.task_row.alloc(sizeof(int) * ((size_t)nt + 1)));
  SW_TRY(L.head_split.alloc(sizeof(int) * (size_t)std::max<int64_t>(nt, 1)));
  SW_TRY(L.tail_split.alloc(sizeof(int) * (size_t)std::max<int64_t>(nt, 1)));
  SW_CHECK_CUDA(cudaMemsetAsync(L.head_split.p, 0xff, L.head_split.bytes, st));
  SW_CHECK_CUDA(cudaMemsetAsync(L.tail_split.p, 0xff, L.tail_split.bytes, st));
  task_row_kernel<<<grid_n(nt + 1), 256, 0, st>>>(L.ptr, rows, total, U, (int)nt, L.task_row.as<int>());
  SW_CHECK_LAUNCH();
  TmpBuf flag;
  SW_TRY(flag.alloc(sizeof(int) * ((size_t)rows + 1), st));
  if (rows > 0) split_flag_kernel<<<grid_n(rows), 256, 0, st>>>(L.ptr, rows, U, flag.as<int>());
  SW_CHECK_LAUNCH();
  SW_TRY(scan_exclusive_i32(flag.as<int>(), flag.as<int>(), rows, st));
  int ns = 0;
  SW_CHECK_CUDA(cudaMemcpyAsync(&ns, flag.as<int>() + rows, sizeof(int), cudaMemcpyDeviceToHost, st));
  SW_CHECK_CUDA(cudaStreamSynchronize(st));
  L.nsplit = ns;
  SW_TRY(L.split_row.alloc(sizeof(int) * (size_t)ns));
  SW_TRY(L.split_first.alloc(sizeof(int) * (size_t)ns));
  SW_TRY(L.split_last.alloc(sizeof(int) * (size_t)ns));
  SW_TRY(L.split_cnt.alloc(sizeof(int) * (size_t)ns));
  SW_CHECK_CUDA(cudaMemsetAsync(L.split_cnt.p, 0, L.split_cnt.bytes, st));
  if (rows > 0)
    split_fill_kernel<<<grid_n(rows), 256, 0, st>>>(L.ptr, rows, U, flag.as<int>(), L.split_row.as<int>(),
                                                    L.split_first.as<int>(), L.split_last.as<int>(),
                                                    L.head_split.as<int>(), L.tail_split.as<int>());
  SW_CHECK_LAUNCH();
  SW_TRY(L.task_hdr.alloc(sizeof(int4) * (size_t)std::max<int64_t>(nt, 1)));
  if (nt > 0)
    task_hdr_kernel<<<grid_n(nt), 256, 0, st>>>(L.task_row.as<int>(), L.head_split.as<int>(),
                                                L.tail_split.as<int>(), (int)nt, L.task_hdr.as<int4>());
  SW_CHECK_LAUNCH();
  if (!L.eidx.p) {
    SW_TRY(L.eidx.alloc(sizeof(int) * (size_t)L.nnz));
    if (L.nnz > 0) {
      SW_CHECK_CUDA(cudaMemcpyAsync(L.eidx.p, L.idx, sizeof(int) * (size_t)L.nnz, cudaMemcpyDeviceToDevice, st));
      if (rows > 0) row_start_set_kernel<<<grid_n(rows), 256, 0, st>>>(L.ptr, rows, L.eidx.as<int>());
      SW_CHECK_LAUNCH();
    }
  }
  L.merge_U = U;
  L.merge_built = true;
  return SWIFT_OK;
}

namespace {

template <class T, class TA, class ACC, int VB, int SG, int VPL, int UNR, int MINB = 4>
swift_status launch_merge(const MergeArgs &a, cudaStream_t st) {
  constexpr int G = 32 / SG;
  const int64_t warps = ((int64_t)a.ntasks + G - 1) / G;
  if (warps == 0) return SWIFT_OK;
  merge_spmm_kernel<T, TA, ACC, VB, SG, VPL, UNR, MINB><<<(unsigned)((warps + 7) / 8), 256, 0, st>>>(a);
  SW_CHECK_LAUNCH();
  return SWIFT_OK;
}

// Lean-kernel shape: at most `want` loads in flight, no more than 256 bytes of batch per lane;
// blocks per SM from an estimate of 28 registers of walk state plus batch and accumulators.
constexpr int lean_unr(int VB, int AB, int want) {
  const int lim = 256 / (VB * AB) > 0 ? 256 / (VB * AB) : 1;
  return want < lim ? want : lim;
}
constexpr int lean_minb(int VB, int AB, int UNR) {
  const int regs = 28 + (UNR + 1) * VB * AB / 4;
  const int b = 65536 / (256 * regs);
  return b < 1 ? 1 : (b > 8 ? 8 : b);
}

// The flagged walk keeps 4 gathered vectors in their stored width (TB bytes per element) and
// the accumulators in AB bytes per element.
constexpr int flag_minb(int VB, int AB, int TB) {
  const int regs = 28 + VB * AB / 4 + 4 * ((VB * TB + 3) / 4);
  const int b = 65536 / (256 * regs);
  return b < 1 ? 1 : (b > 8 ? 8 : b);
}

template <class T, class TA, class ACC, int VB, int SG, int MINB, bool FULL, bool SCALE = false>
swift_status launch_flag(MergeArgs a, const int *eidx, cudaStream_t st) {
  constexpr int G = 32 / SG;
  const int64_t warps = ((int64_t)a.ntasks + G - 1) / G;
  if (warps == 0) return SWIFT_OK;
  a.idx = eidx;
  merge_flag_kernel<T, TA, ACC, VB, SG, MINB, FULL, SCALE><<<(unsigned)((warps + 7) / 8), 256, 0, st>>>(a);
  SW_CHECK_LAUNCH();
  return SWIFT_OK;
}

template <int SG, int D>
swift_status launch_staged(MergeArgs a, const int *eidx, cudaStream_t st) {
  constexpr int G = 32 / SG;
  constexpr int SMEM = staged_smem(SG, D);
  const int64_t warps = ((int64_t)a.ntasks + G - 1) / G;
  if (warps == 0) return SWIFT_OK;
  a.idx = eidx;
  auto k = merge_staged_kernel<SG, D, staged_minb(SG, D)>;
  SW_CHECK_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, SMEM));
  k<<<(unsigned)((warps + 7) / 8), 256, SMEM, st>>>(a);
  SW_CHECK_LAUNCH();
  return SWIFT_OK;
}

template <class T, class TA, class ACC, int VB, int SG, int UNR, int MINB>
swift_status launch_lean(const MergeArgs &a, cudaStream_t st) {
  constexpr int G = 32 / SG;
  const int64_t warps = ((int64_t)a.ntasks + G - 1) / G;
  if (warps == 0) return SWIFT_OK;
  merge_lean_kernel<T, TA, ACC, VB, SG, UNR, MINB><<<(unsigned)((warps + 7) / 8), 256, 0, st>>>(a);
  SW_CHECK_LAUNCH();
  return SWIFT_OK;
}

// unr = loads in flight per lane and batch: 4 or 8 (lean kernel when one vector per lane
// covers N), 16 ("deep", general kernel), else the shape's default
template <class T, class TA, class ACC>
swift_status merge_shape(const MergeArgs &a, int VB, int SG, int VPL, int unr, int kernel,
                         const int *eidx, cudaStream_t st) {
  constexpr int V = VecWidth<T>::value;
  constexpr int W = WideWidth<T>::value;
  constexpr int AB = (int)sizeof(ACC);
  // per-row scales (16-bit B and C): the flagged walk with 16- or 32-byte vectors, one slice
  // per lane
  if (a.b_scale || a.c_scale) {
    if constexpr (sizeof(T) == 2 && sizeof(TA) == 4) {
      if (VPL == 1 && a.N <= SG * VB && a.c_scale && a.ldb * (int64_t)sizeof(T) < (int64_t(1) << 32)) {
#define SW_SCALED(VB_, SG_)                                                                              \
  if (VB == VB_ && SG == SG_)                                                                            \
    return a.N == SG_ * VB_                                                                              \
               ? launch_flag<T, TA, ACC, VB_, SG_, flag_minb(VB_, AB, (int)sizeof(T)), true, true>(a, eidx, st) \
               : launch_flag<T, TA, ACC, VB_, SG_, flag_minb(VB_, AB, (int)sizeof(T)), false, true>(a, eidx, st);
        SW_SCALED(V, 2)
        SW_SCALED(V, 4)
        SW_SCALED(V, 8)
        SW_SCALED(V, 16)
        SW_SCALED(V, 32)
        SW_SCALED(W, 2)
        SW_SCALED(W, 4)
        SW_SCALED(W, 8)
        SW_SCALED(W, 16)
        SW_SCALED(W, 32)
#undef SW_SCALED
      }
    }
    return SWIFT_ERR_UNSUPPORTED;
  }
  // staged walk (kernel 4): FP32 values, B and C, one 16-byte slice per lane covering N;
  // unr selects the ring depth (16 slots = 3 groups of 4 rows in flight, or 32 = 7 groups)
  if constexpr (sizeof(T) == 4 && sizeof(TA) == 4 && sizeof(ACC) == 4) {
    if (kernel == 4 && VB == V && VPL == 1 && a.N == SG * V && a.ldb * (int64_t)sizeof(T) < (int64_t(1) << 32) &&
        (uintptr_t)eidx % 16 == 0 && (uintptr_t)a.val % 16 == 0) {
      const bool deep = unr >= 16;
      switch (SG) {
        case 8: return deep ? launch_staged<8, 32>(a, eidx, st) : launch_staged<8, 16>(a, eidx, st);
        case 16: return deep ? launch_staged<16, 32>(a, eidx, st) : launch_staged<16, 16>(a, eidx, st);
        case 32: return deep ? launch_staged<32, 32>(a, eidx, st) : launch_staged<32, 16>(a, eidx, st);
      }
    }
  }
  // flagged-index kernel (FP32-valued plans): 4 loads in flight
  // (FP64 values double the staging; 2-lane sub-warps would exceed 48 KB of static shared memory)
#define SW_MCASE_FLAG(VB_, SG_)                                                                 \
  if constexpr (sizeof(TA) == 4 || SG_ >= 4) {                                                  \
    if (VB == VB_ && SG == SG_ && VPL == 1 && a.N <= SG_ * VB_) {                               \
      if (a.N == SG_ * VB_) return launch_flag<T, TA, ACC, VB_, SG_, flag_minb(VB_, AB, (int)sizeof(T)), true>(a, eidx, st); \
      return launch_flag<T, TA, ACC, VB_, SG_, flag_minb(VB_, AB, (int)sizeof(T)), false>(a, eidx, st); \
    }                                                                                           \
  }
  {
    if ((kernel == 2 || (kernel == 0 && unr <= 4)) &&
        a.ldb * (int64_t)sizeof(T) < (int64_t(1) << 32)) {
      SW_MCASE_FLAG(W, 2)
      SW_MCASE_FLAG(W, 4)
      SW_MCASE_FLAG(W, 8)
      SW_MCASE_FLAG(W, 16)
      SW_MCASE_FLAG(W, 32)
      SW_MCASE_FLAG(V, 2)
      SW_MCASE_FLAG(V, 4)
      SW_MCASE_FLAG(V, 8)
      SW_MCASE_FLAG(V, 16)
      SW_MCASE_FLAG(V, 32)
      SW_MCASE_FLAG(1, 32)
    }
  }
#undef SW_MCASE_FLAG
#define SW_MCASE(VB_, SG_, VPL_)                                                              \
  if (VB == VB_ && SG == SG_ && VPL == VPL_)                                                    \
    return launch_merge<T, TA, ACC, VB_, SG_, VPL_, unroll_for(VB_, VPL_, false, AB)>(a, st);
#define SW_MCASE_DEEP(VB_, SG_)                                                                 \
  if (VB == VB_ && SG == SG_ && VPL == 1 && unr >= 16 &&                                        \
      unroll_for(VB_, 1, true, AB) > unroll_for(VB_, 1, false, AB))                             \
    return launch_merge<T, TA, ACC, VB_, SG_, 1, unroll_for(VB_, 1, true, AB), 2>(a, st);
  // lean kernel: one vector per lane; 4 (or 8) loads in flight, with the blocks per SM the
  // register estimate of the walk allows
#define SW_MCASE_LEAN(VB_, SG_)                                                                 \
  if (kernel != 3 && VB == VB_ && SG == SG_ && VPL == 1 && a.N <= SG_ * VB_ && unr <= 4)        \
    return launch_lean<T, TA, ACC, VB_, SG_, lean_unr(VB_, AB, 4), lean_minb(VB_, AB, lean_unr(VB_, AB, 4))>(a, st); \
  if (kernel != 3 && VB == VB_ && SG == SG_ && VPL == 1 && a.N <= SG_ * VB_ && unr <= 8)        \
    return launch_lean<T, TA, ACC, VB_, SG_, lean_unr(VB_, AB, 8), lean_minb(VB_, AB, lean_unr(VB_, AB, 8))>(a, st);
  SW_MCASE_LEAN(W, 2)
  SW_MCASE_LEAN(W, 4)
  SW_MCASE_LEAN(W, 8)
  SW_MCASE_LEAN(W, 16)
  SW_MCASE_LEAN(W, 32)
  SW_MCASE_LEAN(V, 2)
  SW_MCASE_LEAN(V, 4)
  SW_MCASE_LEAN(V, 8)
  SW_MCASE_LEAN(V, 16)
  SW_MCASE_LEAN(V, 32)
  SW_MCASE_LEAN(1, 32)
  SW_MCASE(W, 2, 1)
  SW_MCASE(W, 4, 1)
  SW_MCASE(W, 8, 1)
  SW_MCASE(W, 16, 1)
  SW_MCASE(W, 32, 1)
  SW_MCASE(W, 32, 2)
  SW_MCASE_DEEP(V, 16)
  SW_MCASE_DEEP(V, 32)
  SW_MCASE(V, 2, 1)
  SW_MCASE(V, 4, 1)
  SW_MCASE(V, 8, 1)
  SW_MCASE(V, 16, 1)
  SW_MCASE(V, 32, 1)
  SW_MCASE(V, 32, 2)
  SW_MCASE(V, 32, 4)
  SW_MCASE(1, 32, 1)
#undef SW_MCASE
#undef SW_MCASE_DEEP
#undef SW_MCASE_LEAN
  return SWIFT_ERR_UNSUPPORTED;
}

}  // namespace

swift_status run_merge(Plan &p, RowLayout &L, const DenseArgs &d, const MergeOpts &o,
                       cudaStream_t st) {
  {
    std::lock_guard<std::mutex> g(p.mu);
    SW_TRY(build_merge_tasks(L, o.U > 0 ? o.U : 256, st));
    const size_t acc = (p.val_type == SWIFT_F64) ? 8 : 4;
    const size_t need = (size_t)2 * L.ntasks * (size_t)d.N * acc;
    if (need > L.mscratch.bytes) SW_TRY(L.mscratch.alloc(need));
  }
  MergeArgs a{};
  a.rows = L.rows; a.N = d.N; a.U = L.merge_U; a.ntasks = L.ntasks;
  a.total = (int64_t)L.nnz + L.rows;
  a.ptr = L.ptr; a.idx = L.idx; a.val = L.val; a.out_row = L.out_row;
  a.B = d.B; a.ldb = d.ldb; a.C = d.C; a.ldc = d.ldc;
  a.task_row = L.task_row.as<int>(); a.head_split = L.head_split.as<int>(); a.tail_split = L.tail_split.as<int>();
  a.task_hdr = L.task_hdr.as<int>();
  a.split_row = L.split_row.as<int>(); a.split_first = L.split_first.as<int>();
  a.split_last = L.split_last.as<int>(); a.split_cnt = L.split_cnt.as<int>();
  a.scratch = L.mscratch.p;
  a.b_scale = d.b_scale;
  a.c_scale = d.c_scale;
  const size_t esz = d.dtype == SWIFT_F64 ? 8 : (d.dtype == SWIFT_F32 ? 4 : 2);
  auto aligned = [&](int bytes) {
    return ((uintptr_t)d.B % bytes == 0) && ((uintptr_t)d.C % bytes == 0) &&
           ((d.ldb * (int64_t)esz) % bytes == 0) && ((d.ldc * (int64_t)esz) % bytes == 0) &&
           (d.N % (int)(bytes / esz) == 0);
  };
  // vector width: 32 bytes when aligned and at most two vectors per lane cover the row slice,
  // else 16 bytes, else scalar
  int VB = 1;
  const bool scaled = d.b_scale || d.c_scale;  // 16- or 32-byte vectors (merge_shape checks the rest)
  if (scaled && (esz != 2 || !aligned(16))) return SWIFT_ERR_UNSUPPORTED;
  if (o.vbytes != 16 && o.vbytes != 4 && aligned(32) && d.N / (int)(32 / esz) <= (scaled ? 32 : 64))
    VB = (int)(32 / esz);
  else if ((scaled || o.vbytes != 4) && aligned(16)) VB = (int)(16 / esz);
  const int lanes = (d.N + VB - 1) / VB;
  int SG = 32, VPL = 1;
  if (VB > 1) {
    SG = 2;
    while (SG < lanes && SG < 32) SG <<= 1;
    if (lanes > 32) VPL = lanes > 64 ? 4 : 2;
  }
#define SW_MDISPATCH(T, TA, ACC) return merge_shape<T, TA, ACC>(a, VB, SG, VPL, o.unroll, o.kernel, L.eidx.as<int>(), st);
  if (p.val_type == SWIFT_F64) {
    if (d.dtype != SWIFT_F64) return SWIFT_ERR_UNSUPPORTED;
    SW_MDISPATCH(double, double, double)
  }
  switch (d.dtype) {
    case SWIFT_F32: SW_MDISPATCH(float, float, float)
    case SWIFT_BF16: SW_MDISPATCH(__nv_bfloat16, float, float)
    case SWIFT_F16: SW_MDISPATCH(__half, float, float)
    default: return SWIFT_ERR_UNSUPPORTED;
  }
#undef SW_MDISPATCH
}

namespace {

constexpr int bwd_minb(int VB, int AB, int SG, bool DOY, bool DODX) {
  // The FP32 fused passes with 16-byte vectors at N = 64 -- [Y | dX] in 32-lane sub-warps and
  // Y + dA in 16-lane ones -- run five blocks per SM (48 registers, 16-44 bytes of spill): that
  // hides more gather latency than the estimate's four.  Measured on the 262,144-node graph:
  // [Y | dX] 0.447 ms against 0.467 at four blocks and 0.686 at six (160 bytes spilled); Y + dA
  // 0.573 against 0.585 ms.
  if (VB == 4 && AB == 4 && DOY && ((DODX && SG == 32) || (!DODX && SG == 16))) return 5;
  const int regs = 32 + (VB * AB / 4) * 6 + 4 * AB / 4 + (DODX ? 4 : 0);
  const int b = 65536 / (256 * regs);
  return b < 1 ? 1 : (b > 8 ? 8 : b);
}

template <class T, int VB, int SG, bool DOY, bool DODA, bool DODX>
swift_status launch_bwd(const BwdArgs &ba, cudaStream_t st) {
  constexpr int G = 32 / SG;
  const int64_t warps = ((int64_t)ba.m.ntasks + G - 1) / G;
  if (warps == 0) return SWIFT_OK;
  merge_bwd_kernel<T, VB, SG, DOY, DODA, DODX, bwd_minb(VB, (int)sizeof(T), SG, DOY, DODX)>
      <<<(unsigned)((warps + 7) / 8), 256, 0, st>>>(ba);
  SW_CHECK_LAUNCH();
  return SWIFT_OK;
}

template <class T, int VB, bool DOY, bool DODA, bool DODX>
swift_status bwd_by_sg(const BwdArgs &ba, int SG, cudaStream_t st) {
  switch (SG) {
    case 4: return launch_bwd<T, VB, 4, DOY, DODA, DODX>(ba, st);
    case 8: return launch_bwd<T, VB, 8, DOY, DODA, DODX>(ba, st);
    case 16: return launch_bwd<T, VB, 16, DOY, DODA, DODX>(ba, st);
    case 32: return launch_bwd<T, VB, 32, DOY, DODA, DODX>(ba, st);
  }
  return SWIFT_ERR_UNSUPPORTED;
}

template <class T, bool DOY, bool DODA, bool DODX>
swift_status bwd_by_vb(const BwdArgs &ba, int VB, int SG, cudaStream_t st) {
  constexpr int V = VecWidth<T>::value;
  constexpr int W = WideWidth<T>::value;
  // 32-byte vectors for SDDMM alone: half the lanes per row, so a warp walks twice the tasks
  if constexpr (!DOY && !DODX) {
    if (VB == W) return bwd_by_sg<T, W, DOY, DODA, DODX>(ba, SG, st);
  }
  if (VB == V) return bwd_by_sg<T, V, DOY, DODA, DODX>(ba, SG, st);
  if (VB == 1) return bwd_by_sg<T, 1, DOY, DODA, DODX>(ba, SG, st);
  return SWIFT_ERR_UNSUPPORTED;
}

template <class T>
swift_status bwd_dispatch(const BwdArgs &ba, int VB, int SG, bool y, bool da, bool dx, cudaStream_t st) {
  if (y && da && dx) return bwd_by_vb<T, true, true, true>(ba, VB, SG, st);
  if (y && da) return bwd_by_vb<T, true, true, false>(ba, VB, SG, st);
  if (da && !y && !dx) return bwd_by_vb<T, false, true, false>(ba, VB, SG, st);
  return SWIFT_ERR_UNSUPPORTED;
}

}  // namespace

swift_status check_symmetric(Plan &p, cudaStream_t st) {
  if (p.symmetric >= 0) return SWIFT_OK;
  if (!p.has_csr || p.M != p.K) {
    p.symmetric = 0;
    return SWIFT_OK;
  }
  TmpBuf bad;
  SW_TRY(bad.alloc(sizeof(int), st));
  SW_CHECK_CUDA(cudaMemsetAsync(bad.p, 0, sizeof(int), st));
  if (p.M > 0) {
    const int blocks = (int)std::min<int64_t>(((int64_t)p.M * 32 + 255) / 256, 148 * 32);
    if (p.val_type == SWIFT_F64)
      sym_check_kernel<double><<<blocks, 256, 0, st>>>(p.M, p.rowptr.as<int>(), p.colidx.as<int>(),
                                                        p.val.as<double>(), p.invperm.as<int>(), p.sptr.as<int>(),
                                                        p.srow.as<int>(), p.sval.as<double>(), bad.as<int>());
    else
      sym_check_kernel<float><<<blocks, 256, 0, st>>>(p.M, p.rowptr.as<int>(), p.colidx.as<int>(),
                                                       p.val.as<float>(), p.invperm.as<int>(), p.sptr.as<int>(),
                                                       p.srow.as<int>(), p.sval.as<float>(), bad.as<int>());
    SW_CHECK_LAUNCH();
  }
  int h = 0;
  SW_CHECK_CUDA(cudaMemcpyAsync(&h, bad.p, sizeof(int), cudaMemcpyDeviceToHost, st));
  SW_CHECK_CUDA(cudaStreamSynchronize(st));
  p.symmetric = h ? 0 : 1;
  return SWIFT_OK;
}

swift_status run_bwd_merge(Plan &p, int N, swift_dtype dt, const void *X, int64_t ldx,
                           const void *dY, int64_t lddy, void *Y, int64_t ldy, void *dX,
                           int64_t lddx, void *dA, cudaStream_t st) {
  if (!p.has_csr || dt != p.val_type || (dt != SWIFT_F32 && dt != SWIFT_F64)) return SWIFT_ERR_UNSUPPORTED;
  if (dX && (p.M != p.K || p.symmetric != 1)) return SWIFT_ERR_UNSUPPORTED;
  if (N <= 0 || p.M == 0) return SWIFT_ERR_UNSUPPORTED;
  const size_t esz = dt == SWIFT_F64 ? 8 : 4;
  if (ldx * (int64_t)esz >= (int64_t(1) << 32) || lddy * (int64_t)esz >= (int64_t(1) << 32))
    return SWIFT_ERR_UNSUPPORTED;
  const int V = (int)(16 / esz);
  auto al = [&](const void *q, int64_t ld) {
    return !q || (((uintptr_t)q % 16 == 0) && ((ld * (int64_t)esz) % 16 == 0));
  };
  auto al32 = [&](const void *q, int64_t ld) {
    return ((uintptr_t)q % 32 == 0) && ((ld * (int64_t)esz) % 32 == 0);
  };
  int VB = 1;
  if (N % V == 0 && N / V <= 32 && al(X, ldx) && al(dY, lddy) && al(Y, ldy) && al(dX, lddx)) VB = V;
  // SDDMM alone on rows of 8+ wide vectors: 32-byte vectors (N=128 FP32: 0.96 -> 0.91 ms; at
  // N=32 the 4-lane sub-warps lose, 0.42 -> 0.45 ms)
  if (!Y && !dX && N % (2 * V) == 0 && N / (2 * V) >= 8 && N / (2 * V) <= 32 && al32(X, ldx) && al32(dY, lddy))
    VB = 2 * V;
  const int lanes = ((N + VB - 1) / VB) * (dX ? 2 : 1);
  if (lanes > 32) return SWIFT_ERR_UNSUPPORTED;
  int SG = 4;
  while (SG < lanes) SG <<= 1;
  RowLayout &L = p.fwd;
  const bool sdd_only = !Y && !dX;
  // largest power of two in [lo, 512] that leaves about `waves` waves of 32 warps per SM
  auto wave_size = [&](int lo, int waves) {
    const int64_t want = ((int64_t)L.nnz + L.rows) / ((int64_t)p.sm_count * 32 * (32 / SG) * waves);
    int U = lo;
    while (U < 512 && 2 * U <= want) U *= 2;
    return U;
  };
  int sdd_U = 0;
  {
    std::lock_guard<std::mutex> g(p.mu);
    // tasks shared with the forward walk when it ran (its tuned size), else about six waves
    SW_TRY(build_merge_tasks(L, L.merge_built ? L.merge_U : wave_size(64, 6), st));
    const size_t need = (size_t)2 * L.ntasks * (size_t)N * (dX ? 2 : 1) * esz;
    if ((Y || dX) && need > L.mscratch.bytes) SW_TRY(L.mscratch.alloc(need));
    if (sdd_only) {
      // SDDMM alone: no partial rows to combine, so many small tasks cost nothing extra and
      // shorten the tail (measured best near 24 waves: 32 positions at N=32, 128 at N=128)
      sdd_U = wave_size(32, 24);
      if (L.sdd_U != sdd_U || !L.sdd_hdr.p) {
        const int64_t total = (int64_t)L.nnz + L.rows;
        const int64_t nt = (total + sdd_U - 1) / sdd_U;
        if (nt >= INT32_MAX / 2) return SWIFT_ERR_OVERFLOW;
        TmpBuf tr;
        SW_TRY(tr.alloc(sizeof(int) * ((size_t)nt + 1), st));
        task_row_kernel<<<grid_n(nt + 1), 256, 0, st>>>(L.ptr, L.rows, total, sdd_U, (int)nt, tr.as<int>());
        SW_CHECK_LAUNCH();
        SW_TRY(L.sdd_hdr.alloc(sizeof(int4) * (size_t)std::max<int64_t>(nt, 1)));
        if (nt > 0) sdd_hdr_kernel<<<grid_n(nt), 256, 0, st>>>(tr.as<int>(), (int)nt, L.sdd_hdr.as<int4>());
        SW_CHECK_LAUNCH();
        L.sdd_U = sdd_U;
        L.sdd_ntasks = (int)nt;
      }
    }
  }
  BwdArgs ba{};
  MergeArgs &a = ba.m;
  a.rows = L.rows; a.N = N; a.U = L.merge_U; a.ntasks = L.ntasks;
  a.total = (int64_t)L.nnz + L.rows;
  a.ptr = L.ptr; a.idx = L.eidx.as<int>(); a.val = L.val; a.out_row = nullptr;
  a.B = X; a.ldb = ldx; a.C = Y; a.ldc = ldy;
  a.task_row = L.task_row.as<int>(); a.head_split = L.head_split.as<int>(); a.tail_split = L.tail_split.as<int>();
  a.task_hdr = L.task_hdr.as<int>();
  a.split_row = L.split_row.as<int>(); a.split_first = L.split_first.as<int>();
  a.split_last = L.split_last.as<int>(); a.split_cnt = L.split_cnt.as<int>();
  a.scratch = L.mscratch.p;
  if (sdd_only) {
    a.U = sdd_U;
    a.ntasks = L.sdd_ntasks;
    a.task_hdr = L.sdd_hdr.as<int>();
  }
  ba.dY = dY; ba.lddy = lddy; ba.dX = dX; ba.lddx = lddx; ba.dA = dA;
  const bool y = Y != nullptr, da = dA != nullptr, dx = dX != nullptr;
  return dt == SWIFT_F64 ? bwd_dispatch<double>(ba, VB, SG, y, da, dx, st)
                         : bwd_dispatch<float>(ba, VB, SG, y, da, dx, st);
}

size_t merge_args_size() { return sizeof(MergeArgs); }

// One member of a batch: tasks of U positions over the member's own layout L (which points at
// the plan's CSR), scratch for N columns, and its launch record (FP32 plan, FP32 row-major B
// and C).  shape selects the sub-warp width of merge_batch_kernel; items = warp items.
swift_status merge_batch_member(const Plan &p, RowLayout &L, int U, int N, const void *B, int64_t ldb,
                                void *C, int64_t ldc, void *args_out, int *shape, int64_t *items,
                                cudaStream_t st) {
  if (p.val_type != SWIFT_F32 || !p.has_csr || N < 0) return SWIFT_ERR_UNSUPPORTED;
  const bool v16 = ((uintptr_t)B % 16 == 0) && ((uintptr_t)C % 16 == 0) && (ldb % 4 == 0) &&
                   (ldc % 4 == 0) && (N % 4 == 0);
  int sh, G;
  if (ldb * (int64_t)sizeof(float) >= (int64_t(1) << 32)) return SWIFT_ERR_UNSUPPORTED;
  if (v16 && N <= 128) {
    sh = N <= 32 ? 0 : (N <= 64 ? 1 : 2);
    G = sh == 0 ? 4 : (sh == 1 ? 2 : 1);
    if (N == 32 || N == 64 || N == 128) sh += 4;  // every lane in range: no bounds predicate
  } else if (N <= 32) {
    sh = 3;
    G = 1;
  } else {
    set_last_error("swift_batch", "N above 128, or above 32 without 16-byte aligned operands");
    return SWIFT_ERR_UNSUPPORTED;
  }
  L.rows = p.M; L.cols = p.K; L.nnz = p.nnz;
  L.ptr = p.rowptr.as<int>(); L.idx = p.colidx.as<int>(); L.val = p.val.p; L.out_row = nullptr;
  SW_TRY(build_merge_tasks(L, U, st));
  const size_t need = (size_t)2 * L.ntasks * (size_t)N * sizeof(float);
  if (need > L.mscratch.bytes) SW_TRY(L.mscratch.alloc(need));
  MergeArgs a{};
  a.rows = L.rows; a.N = N; a.U = L.merge_U; a.ntasks = (N == 0 || p.M == 0) ? 0 : L.ntasks;
  a.total = (int64_t)L.nnz + L.rows;
  a.ptr = L.ptr; a.idx = L.eidx.as<int>(); a.val = L.val; a.out_row = nullptr;
  a.B = B; a.ldb = ldb; a.C = C; a.ldc = ldc;
  a.task_row = L.task_row.as<int>(); a.head_split = L.head_split.as<int>(); a.tail_split = L.tail_split.as<int>();
  a.task_hdr = L.task_hdr.as<int>();
  a.split_row = L.split_row.as<int>(); a.split_first = L.split_first.as<int>();
  a.split_last = L.split_last.as<int>(); a.split_cnt = L.split_cnt.as<int>();
  a.scratch = L.mscratch.p;
  std::memcpy(args_out, &a, sizeof(MergeArgs));
  *shape = sh;
  *items = ((int64_t)a.ntasks + G - 1) / G;
  return SWIFT_OK;
}

// Persistent grid: every SM filled with as many 256-thread blocks as fit.
swift_status merge_batch_grid(int device, int *grid) {
  int sms = 0, per = 0;
  SW_CHECK_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
  SW_CHECK_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, merge_batch_kernel, 256, 0));
  *grid = sms * std::max(per, 1);
  return SWIFT_OK;
}

swift_status launch_merge_batch(const void *d_args, const int *d_shape, const int64_t *d_item_off,
                                int count, int grid, cudaStream_t st) {
  if (count <= 0 || grid <= 0) return SWIFT_OK;
  merge_batch_kernel<<<grid, 256, 0, st>>>(static_cast<const MergeArgs *>(d_args), d_shape, d_item_off,
                                           count);
  SW_CHECK_LAUNCH();
  return SWIFT_OK;
}

}  // namespace swift
