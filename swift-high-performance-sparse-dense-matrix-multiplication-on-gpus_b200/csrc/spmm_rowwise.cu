// spmm_rowwise.cu -- row-ordered execution engine (C = A B, X = A^T Y, SDDMM, fused).
//
// Why a row-ordered engine next to the Swift tiles: on the 1M-row power-law workloads C is
// 0.5 GB, four times the 126 MB L2.  Swift's column order scatters every product into C
// (nnz * N atomics, src/Swift.h:56,91), so each contribution becomes an HBM read-modify-
// write of a C line.  Here a sub-warp owns one C row, accumulates it in registers across the
// row's nonzeros and writes it once with streaming stores; B rows are gathered with 16-byte
// vector loads (a 512-byte row per warp at N = 128 FP32).  Rows longer than `split` are cut
// into pieces (the balance rule of src/balance.h applied to rows); each piece stores a
// partial row to scratch and the last piece to arrive sums the partials in piece order and
// writes C, so results are deterministic and no C pre-zeroing pass is needed.
//
// The same kernel computes SDDMM (dot products of a register-resident U row with each
// gathered B row) and the fused forward + SDDMM pass that reads each X row once for both.
#include "common.cuh"
#include "vec.cuh"

namespace swift {

namespace {

struct RowKArgs {
  int rows, N, split, pieces, all_short, rows_per_sg, piece_warps;
  const int *ptr, *idx;
  const void *val;
  const int *out_row;
  const void *B;
  int64_t ldb;
  void *C;
  int64_t ldc;
  const void *U;  // SDDMM: row operand (indexed by layout row)
  int64_t ldu;
  void *dout;     // SDDMM output, one value per nonzero (layout order)
  const int *long_of_row, *piece_row, *piece_idx, *long_first, *long_count;
  int *counters;
  void *scratch;
};

template <int VPL> struct Unroll { static constexpr int value = VPL == 1 ? 8 : (VPL == 2 ? 4 : 2); };

// Accumulates nonzeros [p0, p1) of one layout row for the dense columns
// [col0, col0 + SG*VB*VPL).  Lanes of the sub-group load the row's (index, value) pairs SG at
// a time and broadcast them; every lane then issues UNR independent 16-byte loads of B
// before using any of them.
template <class T, class TA, class ACC, int VB, int SG, int VPL, bool SPMM, bool SDDMM>
__device__ __forceinline__ void accumulate_row(const RowKArgs &a, int p0, int p1, int col0,
                                               int sl, unsigned sgmask, ACC (&acc)[VPL][VB],
                                               const ACC (&u)[VPL][VB], bool first_chunk) {
  constexpr int UNR = Unroll<VPL>::value;
  const T *__restrict__ B = static_cast<const T *>(a.B);
  const TA *__restrict__ val = static_cast<const TA *>(a.val);
  TA *__restrict__ dout = static_cast<TA *>(a.dout);
  bool inb[VPL];
#pragma unroll
  for (int v = 0; v < VPL; ++v) inb[v] = col0 + v * SG * VB + sl * VB < a.N;
  for (int base = p0; base < p1; base += SG) {
    const int m = min(SG, p1 - base);
    int myc = 0;
    ACC myv = ACC(0);
    if (sl < m) {
      myc = __ldcs(a.idx + base + sl);
      myv = (ACC)__ldcs(val + base + sl);
    }
    int k = 0;
    for (; k + UNR <= m; k += UNR) {
      ACC b[UNR][VPL][VB];
#pragma unroll
      for (int uu = 0; uu < UNR; ++uu) {
        const int c = __shfl_sync(sgmask, myc, k + uu, SG);
        const T *row = B + (int64_t)c * a.ldb + col0 + sl * VB;
#pragma unroll
        for (int v = 0; v < VPL; ++v) {
          if (inb[v]) vload<T, ACC, VB>(row + v * SG * VB, b[uu][v]);
          else {
#pragma unroll
            for (int e = 0; e < VB; ++e) b[uu][v][e] = ACC(0);
          }
        }
      }
#pragma unroll
      for (int uu = 0; uu < UNR; ++uu) {
        const ACC w = __shfl_sync(sgmask, myv, k + uu, SG);
        if constexpr (SPMM) {
#pragma unroll
          for (int v = 0; v < VPL; ++v)
#pragma unroll
            for (int e = 0; e < VB; ++e) acc[v][e] = fma(w, b[uu][v][e], acc[v][e]);
        }
        if constexpr (SDDMM) {
          ACC d = ACC(0);
#pragma unroll
          for (int v = 0; v < VPL; ++v)
#pragma unroll
            for (int e = 0; e < VB; ++e) d = fma(u[v][e], b[uu][v][e], d);
#pragma unroll
          for (int o = SG / 2; o > 0; o >>= 1) d += __shfl_xor_sync(sgmask, d, o, SG);
          if (sl == 0) {
            const int p = base + k + uu;
            dout[p] = first_chunk ? (TA)d : (TA)((ACC)dout[p] + d);
          }
        }
      }
    }
    for (; k < m; ++k) {
      const int c = __shfl_sync(sgmask, myc, k, SG);
      const ACC w = __shfl_sync(sgmask, myv, k, SG);
      const T *row = B + (int64_t)c * a.ldb + col0 + sl * VB;
      ACC b[VPL][VB];
#pragma unroll
      for (int v = 0; v < VPL; ++v) {
        if (inb[v]) vload<T, ACC, VB>(row + v * SG * VB, b[v]);
        else {
#pragma unroll
          for (int e = 0; e < VB; ++e) b[v][e] = ACC(0);
        }
      }
      if constexpr (SPMM) {
#pragma unroll
        for (int v = 0; v < VPL; ++v)
#pragma unroll
          for (int e = 0; e < VB; ++e) acc[v][e] = fma(w, b[v][e], acc[v][e]);
      }
      if constexpr (SDDMM) {
        ACC d = ACC(0);
#pragma unroll
        for (int v = 0; v < VPL; ++v)
#pragma unroll
          for (int e = 0; e < VB; ++e) d = fma(u[v][e], b[v][e], d);
#pragma unroll
        for (int o = SG / 2; o > 0; o >>= 1) d += __shfl_xor_sync(sgmask, d, o, SG);
        if (sl == 0) {
          const int p = base + k;
          dout[p] = first_chunk ? (TA)d : (TA)((ACC)dout[p] + d);
        }
      }
    }
  }
}

template <class T, class ACC, int VB, int SG, int VPL, bool SDDMM>
__device__ __forceinline__ void load_urow(const RowKArgs &a, int r, int col0, int sl,
                                          ACC (&u)[VPL][VB]) {
#pragma unroll
  for (int v = 0; v < VPL; ++v)
#pragma unroll
    for (int e = 0; e < VB; ++e) u[v][e] = ACC(0);
  if constexpr (SDDMM) {
    const T *row = static_cast<const T *>(a.U) + (int64_t)r * a.ldu + col0 + sl * VB;
#pragma unroll
    for (int v = 0; v < VPL; ++v)
      if (col0 + v * SG * VB + sl * VB < a.N) vload<T, ACC, VB>(row + v * SG * VB, u[v]);
  }
}

template <class T, class ACC, int VB, int SG, int VPL>
__device__ __forceinline__ void store_row(const RowKArgs &a, int orow, int col0, int sl,
                                          const ACC (&acc)[VPL][VB]) {
  T *row = static_cast<T *>(a.C) + (int64_t)orow * a.ldc + col0 + sl * VB;
#pragma unroll
  for (int v = 0; v < VPL; ++v)
    if (col0 + v * SG * VB + sl * VB < a.N) vstore<T, ACC, VB>(row + v * SG * VB, acc[v]);
}

template <class T, class TA, class ACC, int VB, int SG, int VPL, bool SPMM, bool SDDMM>
__global__ void __launch_bounds__(256) rowwise_kernel(const RowKArgs a) {
  constexpr int G = 32 / SG;
  constexpr int CW = SG * VB * VPL;
  const int lane = threadIdx.x & 31, sg = lane / SG, sl = lane % SG;
  const unsigned sgmask = SG == 32 ? 0xffffffffu : (((1u << SG) - 1u) << (sg * SG));
  const int gw = (int)((blockIdx.x * (unsigned)blockDim.x + threadIdx.x) >> 5);
  const int nchunks = (a.N + CW - 1) / CW;
  ACC acc[VPL][VB], u[VPL][VB];

  if (gw < a.piece_warps) {
    // ---------------- a piece of a long row
    const int pc = gw * G + sg;
    if (pc >= a.pieces) return;
    const int r = a.piece_row[pc], j = a.piece_idx[pc];
    const int rs = a.ptr[r], re = a.ptr[r + 1];
    const int p0 = rs + j * a.split, p1 = min(p0 + a.split, re);
    ACC *scr = static_cast<ACC *>(a.scratch) + (int64_t)pc * a.N;
    for (int ch = 0; ch < nchunks; ++ch) {
      const int col0 = ch * CW;
#pragma unroll
      for (int v = 0; v < VPL; ++v)
#pragma unroll
        for (int e = 0; e < VB; ++e) acc[v][e] = ACC(0);
      load_urow<T, ACC, VB, SG, VPL, SDDMM>(a, r, col0, sl, u);
      accumulate_row<T, TA, ACC, VB, SG, VPL, SPMM, SDDMM>(a, p0, p1, col0, sl, sgmask, acc, u, ch == 0);
      if constexpr (SPMM) {
#pragma unroll
        for (int v = 0; v < VPL; ++v)
#pragma unroll
          for (int e = 0; e < VB; ++e) {
            const int col = col0 + v * SG * VB + sl * VB + e;
            if (col < a.N) scr[col] = acc[v][e];
          }
      }
    }
    if constexpr (SPMM) {
      // publish the partial, count arrivals; the last piece reduces in piece order
      __threadfence();
      __syncwarp(sgmask);
      const int o = a.long_of_row[r];
      int old = 0;
      if (sl == 0) old = atomicAdd(&a.counters[o], 1);
      old = __shfl_sync(sgmask, old, 0, SG);
      const int cnt = a.long_count[o];
      if (old == cnt - 1) {
        __threadfence();
        const ACC *first = static_cast<const ACC *>(a.scratch) + (int64_t)a.long_first[o] * a.N;
        const int orow = a.out_row ? a.out_row[r] : r;
        for (int ch = 0; ch < nchunks; ++ch) {
          const int col0 = ch * CW;
#pragma unroll
          for (int v = 0; v < VPL; ++v)
#pragma unroll
            for (int e = 0; e < VB; ++e) acc[v][e] = ACC(0);
          for (int jj = 0; jj < cnt; ++jj) {
            const ACC *s = first + (int64_t)jj * a.N;
#pragma unroll
            for (int v = 0; v < VPL; ++v)
#pragma unroll
              for (int e = 0; e < VB; ++e) {
                const int col = col0 + v * SG * VB + sl * VB + e;
                if (col < a.N) acc[v][e] += __ldcg(s + col);
              }
          }
          store_row<T, ACC, VB, SG, VPL>(a, orow, col0, sl, acc);
        }
        __syncwarp(sgmask);
        if (sl == 0) a.counters[o] = 0;  // ready for the next product
      }
    }
    return;
  }
  // ---------------- consecutive short rows
  const int w2 = gw - a.piece_warps;
  const int r0 = (w2 * G + sg) * a.rows_per_sg;
  for (int i = 0; i < a.rows_per_sg; ++i) {
    const int r = r0 + i;
    if (r >= a.rows) break;
    const int p0 = a.ptr[r], p1 = a.ptr[r + 1];
    if (!a.all_short && p1 - p0 > a.split) continue;  // written by its last piece
    const int orow = a.out_row ? a.out_row[r] : r;
    for (int ch = 0; ch < nchunks; ++ch) {
      const int col0 = ch * CW;
#pragma unroll
      for (int v = 0; v < VPL; ++v)
#pragma unroll
        for (int e = 0; e < VB; ++e) acc[v][e] = ACC(0);
      load_urow<T, ACC, VB, SG, VPL, SDDMM>(a, r, col0, sl, u);
      accumulate_row<T, TA, ACC, VB, SG, VPL, SPMM, SDDMM>(a, p0, p1, col0, sl, sgmask, acc, u, ch == 0);
      if constexpr (SPMM) store_row<T, ACC, VB, SG, VPL>(a, orow, col0, sl, acc);
    }
  }
}

// ---------------------------------------------------------------- dispatch
struct Shape {
  int VB, SG, VPL;
};

template <class T> Shape pick_shape(int N, bool vec_ok) {
  Shape s;
  s.VB = vec_ok ? VecWidth<T>::value : 1;
  const int lanes = (N + s.VB - 1) / s.VB;
  if (s.VB == 1) { s.SG = 32; s.VPL = 1; return s; }
  int sg = 2;
  while (sg < lanes && sg < 32) sg <<= 1;
  s.SG = sg;
  s.VPL = 1;
  if (lanes > 32) s.VPL = lanes > 64 ? 4 : 2;
  return s;
}

template <class T, class TA, class ACC, int VB, int SG, int VPL, bool SPMM, bool SDDMM>
swift_status launch_one(const RowKArgs &a, cudaStream_t st) {
  constexpr int G = 32 / SG;
  const int64_t short_warps = ((int64_t)a.rows + (int64_t)G * a.rows_per_sg - 1) / ((int64_t)G * a.rows_per_sg);
  const int64_t warps = a.piece_warps + short_warps;
  if (warps == 0) return SWIFT_OK;
  const int64_t blocks = (warps + 7) / 8;
  if (blocks > INT32_MAX) return SWIFT_ERR_OVERFLOW;
  rowwise_kernel<T, TA, ACC, VB, SG, VPL, SPMM, SDDMM><<<(unsigned)blocks, 256, 0, st>>>(a);
  SW_CHECK_LAUNCH();
  return SWIFT_OK;
}

template <class T, class TA, class ACC, bool SPMM, bool SDDMM>
swift_status launch_shape(RowKArgs a, Shape s, cudaStream_t st) {
  const int G = 32 / s.SG;
  a.piece_warps = (a.pieces + G - 1) / G;
#define SW_ROW_CASE(VB_, SG_, VPL_)                                                            \
  if (s.VB == VB_ && s.SG == SG_ && s.VPL == VPL_)                                            \
    return launch_one<T, TA, ACC, VB_, SG_, VPL_, SPMM, SDDMM>(a, st);
  constexpr int V = VecWidth<T>::value;
  SW_ROW_CASE(V, 2, 1)
  SW_ROW_CASE(V, 4, 1)
  SW_ROW_CASE(V, 8, 1)
  SW_ROW_CASE(V, 16, 1)
  SW_ROW_CASE(V, 32, 1)
  SW_ROW_CASE(V, 32, 2)
  SW_ROW_CASE(V, 32, 4)
  SW_ROW_CASE(1, 32, 1)
#undef SW_ROW_CASE
  return SWIFT_ERR_UNSUPPORTED;
}

bool aligned16(const void *p, int64_t ld, size_t esz) {
  return ((uintptr_t)p % 16 == 0) && ((ld * (int64_t)esz) % 16 == 0);
}

swift_status ensure_scratch(Plan &p, RowLayout &L, int N, size_t acc_bytes) {
  const size_t need = (size_t)L.pieces * (size_t)N * acc_bytes;
  std::lock_guard<std::mutex> g(p.mu);
  if (need > L.scratch.bytes) SW_TRY(L.scratch.alloc(need));
  return SWIFT_OK;
}

}  // namespace

// Shared entry for SpMM / SDDMM / fused over a row layout.
static swift_status run_layout(Plan &p, RowLayout &L, int N, swift_dtype dt, const void *B,
                               int64_t ldb, void *C, int64_t ldc, const void *U, int64_t ldu,
                               void *dout, bool spmm, bool sddmm, bool all_short,
                               int rows_per_sg, cudaStream_t st) {
  RowKArgs a{};
  a.rows = L.rows; a.N = N; a.split = L.split;
  a.pieces = all_short ? 0 : L.pieces;
  a.all_short = all_short;
  a.rows_per_sg = rows_per_sg > 0 ? rows_per_sg : 1;
  a.ptr = L.ptr; a.idx = L.idx; a.val = L.val; a.out_row = L.out_row;
  a.B = B; a.ldb = ldb; a.C = C; a.ldc = ldc; a.U = U; a.ldu = ldu; a.dout = dout;
  a.long_of_row = L.long_of_row.as<int>(); a.piece_row = L.piece_row.as<int>();
  a.piece_idx = L.piece_idx.as<int>(); a.long_first = L.long_first.as<int>();
  a.long_count = L.long_count.as<int>(); a.counters = L.counters.as<int>();
  const bool f64 = dt == SWIFT_F64;
  if (spmm && a.pieces > 0) SW_TRY(ensure_scratch(p, L, N, f64 || p.val_type == SWIFT_F64 ? 8 : 4));
  a.scratch = L.scratch.p;
  const size_t esz = dt == SWIFT_F64 ? 8 : (dt == SWIFT_F32 ? 4 : 2);
  bool vec_ok = aligned16(B, ldb, esz) && (N % (int)(16 / esz) == 0);
  if (spmm) vec_ok = vec_ok && aligned16(C, ldc, esz);
  if (sddmm) vec_ok = vec_ok && aligned16(U, ldu, esz);
#define SW_DISPATCH(T, TA, ACC)                                                                \
  {                                                                                            \
    Shape s = pick_shape<T>(N, vec_ok);                                                        \
    if (spmm && sddmm) return launch_shape<T, TA, ACC, true, true>(a, s, st);                  \
    if (spmm) return launch_shape<T, TA, ACC, true, false>(a, s, st);                          \
    return launch_shape<T, TA, ACC, false, true>(a, s, st);                                    \
  }
  if (p.val_type == SWIFT_F64) {
    if (dt != SWIFT_F64) return SWIFT_ERR_UNSUPPORTED;
    SW_DISPATCH(double, double, double)
  }
  switch (dt) {
    case SWIFT_F32: SW_DISPATCH(float, float, float)
    case SWIFT_BF16: SW_DISPATCH(__nv_bfloat16, float, float)
    case SWIFT_F16: SW_DISPATCH(__half, float, float)
    default: return SWIFT_ERR_UNSUPPORTED;
  }
#undef SW_DISPATCH
}

// The row kernel with caller-provided scratch for the long-row partials and arrival counters
// (pieces * N accumulator values, long_rows counters that must be zero on entry).  Used by
// the entry point that allocates nothing (spmm_noalloc.cu).
swift_status run_rowwise_external(Plan &p, RowLayout &L, const DenseArgs &d, void *scratch,
                                  int *counters, cudaStream_t st) {
  if (d.b_layout != SWIFT_ROW_MAJOR || d.c_layout != SWIFT_ROW_MAJOR || d.b_presorted)
    return SWIFT_ERR_UNSUPPORTED;
  RowKArgs a{};
  a.rows = L.rows; a.N = d.N; a.split = L.split; a.pieces = L.pieces; a.all_short = 0;
  a.rows_per_sg = 2;
  a.ptr = L.ptr; a.idx = L.idx; a.val = L.val; a.out_row = L.out_row;
  a.B = d.B; a.ldb = d.ldb; a.C = d.C; a.ldc = d.ldc;
  a.long_of_row = L.long_of_row.as<int>(); a.piece_row = L.piece_row.as<int>();
  a.piece_idx = L.piece_idx.as<int>(); a.long_first = L.long_first.as<int>();
  a.long_count = L.long_count.as<int>();
  a.counters = counters;
  a.scratch = scratch;
  const size_t esz = d.dtype == SWIFT_F64 ? 8 : (d.dtype == SWIFT_F32 ? 4 : 2);
  const bool vec_ok = aligned16(d.B, d.ldb, esz) && aligned16(d.C, d.ldc, esz) && (d.N % (int)(16 / esz) == 0);
  if (p.val_type == SWIFT_F64) {
    if (d.dtype != SWIFT_F64) return SWIFT_ERR_UNSUPPORTED;
    return launch_shape<double, double, double, true, false>(a, pick_shape<double>(d.N, vec_ok), st);
  }
  switch (d.dtype) {
    case SWIFT_F32: return launch_shape<float, float, float, true, false>(a, pick_shape<float>(d.N, vec_ok), st);
    case SWIFT_BF16: return launch_shape<__nv_bfloat16, float, float, true, false>(a, pick_shape<__nv_bfloat16>(d.N, vec_ok), st);
    case SWIFT_F16: return launch_shape<__half, float, float, true, false>(a, pick_shape<__half>(d.N, vec_ok), st);
    default: return SWIFT_ERR_UNSUPPORTED;
  }
}

swift_status run_rowwise(Plan &p, RowLayout &L, const DenseArgs &d, cudaStream_t st) {
  if (d.b_layout != SWIFT_ROW_MAJOR || d.c_layout != SWIFT_ROW_MAJOR || d.b_presorted)
    return SWIFT_ERR_UNSUPPORTED;
  return run_layout(p, L, d.N, d.dtype, d.B, d.ldb, d.C, d.ldc, nullptr, 0, nullptr, true, false,
                    false, 2, st);
}

swift_status run_sddmm(Plan &p, int N, swift_dtype dt, const void *U, int64_t ldu, const void *V,
                       int64_t ldv, void *out, cudaStream_t st) {
  return run_layout(p, p.fwd, N, dt, V, ldv, nullptr, 0, U, ldu, out, false, true, false, 2, st);
}

swift_status run_fused_fwd_sddmm(Plan &p, int N, swift_dtype dt, const void *X, int64_t ldx,
                                 const void *dY, int64_t lddy, void *Y, int64_t ldy, void *dA,
                                 cudaStream_t st) {
  return run_layout(p, p.fwd, N, dt, X, ldx, Y, ldy, dY, lddy, dA, true, true, false, 2, st);
}

// Deterministic FP64 reference: every row summed by one sub-warp in CSR order.
namespace {
struct F64RefArgs {
  int rows, N;
  const int *ptr, *idx;
  const void *val;
  int val_f64;
  const double *B;
  int64_t ldb;
  double *C;
  int64_t ldc;
};
__global__ void f64_reference_kernel(const F64RefArgs a) {
  const int gw = (int)((blockIdx.x * (unsigned)blockDim.x + threadIdx.x) >> 5);
  const int lane = threadIdx.x & 31;
  if (gw >= a.rows) return;
  const int p0 = a.ptr[gw], p1 = a.ptr[gw + 1];
  for (int col = lane; col < a.N; col += 32) {
    double s = 0.0;
    for (int p = p0; p < p1; ++p) {
      const double v = a.val_f64 ? static_cast<const double *>(a.val)[p]
                                 : (double)static_cast<const float *>(a.val)[p];
      s = fma(v, a.B[(int64_t)a.idx[p] * a.ldb + col], s);
    }
    a.C[(int64_t)gw * a.ldc + col] = s;
  }
}
}  // namespace

swift_status run_f64_reference(const Plan &p, int N, const double *B, int64_t ldb, double *C,
                               int64_t ldc, cudaStream_t st) {
  if (!p.has_csr) return SWIFT_ERR_UNSUPPORTED;
  F64RefArgs a{p.M, N, p.rowptr.as<int>(), p.colidx.as<int>(), p.val.p,
               p.val_type == SWIFT_F64, B, ldb, C, ldc};
  if (p.M == 0 || N == 0) return SWIFT_OK;
  const int64_t blocks = ((int64_t)p.M * 32 + 255) / 256;
  f64_reference_kernel<<<(unsigned)blocks, 256, 0, st>>>(a);
  SW_CHECK_LAUNCH();
  return SWIFT_OK;
}

}  // namespace swift
