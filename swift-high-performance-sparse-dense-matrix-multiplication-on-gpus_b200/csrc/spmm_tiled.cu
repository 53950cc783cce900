// spmm_tiled.cu -- the Swift kernels proper, over the regular tiles and the balanced reside
// blocks (reference: Swift_GPU src/Swift.h:15-135, Swift_reside_kernel src/Swift.h:138-181,
// Swift_GPU_3/4 src/Swift_3.h, src/Swift_4.h).
//
// Work item = up to 16 consecutive regular tiles that share their 32 sorted columns (tiles of
// one step and group at successive depths, src/coo2csc.h:220-242), so the 32 B rows of the
// item are fetched once per item and reused from L1 across its depths.
//
// Row-major B and C: a sub-warp spans the dense columns with 16-byte vectors; it walks the
// item's slots in order, keeps a running sum while consecutive slots hit the same C row, and
// issues one 16-byte vector atomic per run (format-0 tiles collapse to one atomic per tile,
// format-2 tiles to one per run -- the segmented reduction of src/Swift_4.h in registers).
//
// Column-major B and C (the reference wrappers' layout): lane l owns slot l, reads
// B[n, col0 + l] (coalesced across the warp when B is pre-sorted) and reduces runs of equal
// rows with a segmented warp scan before a scalar atomic, per dense column n.
//
// Reside blocks (src/balance.h): one warp per block of <= 32 entries of one column; the
// column's B row is loaded once and reused for every entry of the block.
#include "common.cuh"
#include "vec.cuh"

namespace swift {

struct TiledArgs {
  int M, K, N, nitems, tilenum, presorted;
  const int *item_tile;    // [nitems+1] first tile of each work item
  const int *tile_colidx;  // [tilenum]
  const int *sortrowidx;   // [32*tilenum]
  const void *sortval;
  const int *perm;         // sorted position -> B row (ignored when presorted)
  const int *reside_ptr, *reside_row;
  const void *reside_val;
  int reside_col, numblk, balanced;
  const unsigned *colorblk;
  const int *blkstart, *blkstop;
  const void *B;
  int64_t ldb;
  void *C;
  int64_t ldc;
  // grouped engine: regular slots per 8-tile group in row-sorted order
  int64_t nreg;
  const int *g_row, *g_col;
  const void *g_val;
};

namespace {

template <class T, class ACC, int VB, int SG>
__global__ void __launch_bounds__(256) tiled_rowmajor_kernel(const TiledArgs a) {
  constexpr int G = 32 / SG;         // sub-groups per warp
  constexpr int SPG = 32 / G;        // slots per sub-group and tile
  constexpr int CW = SG * VB;
  constexpr int BATCH = SPG < 8 ? SPG : 8;
  const int lane = threadIdx.x & 31, sg = lane / SG, sl = lane % SG;
  const unsigned sgmask = SG == 32 ? 0xffffffffu : (((1u << SG) - 1u) << (sg * SG));
  const int item = (int)((blockIdx.x * (unsigned)blockDim.x + threadIdx.x) >> 5);
  if (item >= a.nitems) return;
  const int t0 = a.item_tile[item], t1 = a.item_tile[item + 1];
  const int col0 = a.tile_colidx[t0] + sg * SPG;
  const T *__restrict__ B = static_cast<const T *>(a.B);
  T *__restrict__ C = static_cast<T *>(a.C);
  const T *__restrict__ sval = static_cast<const T *>(a.sortval);
  // B rows of my slots (lane sl < SPG holds slot sl's row)
  int myb = 0;
  if (sl < SPG) myb = a.presorted ? col0 + sl : __ldg(a.perm + col0 + sl);
  for (int cbase = 0; cbase < a.N; cbase += CW) {
    const int col = cbase + sl * VB;
    const bool inb = col < a.N;
    int cur = -1;
    ACC acc[VB];
#pragma unroll
    for (int e = 0; e < VB; ++e) acc[e] = ACC(0);
    for (int t = t0; t < t1; ++t) {
      int myr = 0;
      ACC myv = ACC(0);
      if (sl < SPG) {
        const int64_t s = (int64_t)t * kTile + sg * SPG + sl;
        myr = __ldg(a.sortrowidx + s);
        myv = (ACC)__ldg(sval + s);
      }
#pragma unroll
      for (int k0 = 0; k0 < SPG; k0 += BATCH) {
        ACC b[BATCH][VB];
#pragma unroll
        for (int u = 0; u < BATCH; ++u) {
          const int brow = __shfl_sync(sgmask, myb, k0 + u, SG);
          if (inb) vload<T, ACC, VB>(B + (int64_t)brow * a.ldb + col, b[u]);
          else {
#pragma unroll
            for (int e = 0; e < VB; ++e) b[u][e] = ACC(0);
          }
        }
#pragma unroll
        for (int u = 0; u < BATCH; ++u) {
          const int r = __shfl_sync(sgmask, myr, k0 + u, SG);
          const ACC w = __shfl_sync(sgmask, myv, k0 + u, SG);
          if (r != cur) {
            if (cur >= 0 && inb) vatomic_add<T, ACC, VB>(C + (int64_t)cur * a.ldc + col, acc);
            cur = r;
#pragma unroll
            for (int e = 0; e < VB; ++e) acc[e] = ACC(0);
          }
#pragma unroll
          for (int e = 0; e < VB; ++e) acc[e] = fma(w, b[u][e], acc[e]);
        }
      }
    }
    if (cur >= 0 && inb) vatomic_add<T, ACC, VB>(C + (int64_t)cur * a.ldc + col, acc);
  }
}

// Grouped engine (the slot order of Swift_GPU_4, src/Swift_4.h:6-76): one warp per group of 8
// tiles (256 slots, the last group shorter), whose slots are stored in row-sorted order; each
// sub-warp takes an equal share of them, sums each run of equal rows in registers and issues
// one vector atomic per run -- one per distinct row of the share, where the slot-ordered engine
// issues one per change of row between neighbouring slots.
template <class T, class ACC, int VB, int SG>
__global__ void __launch_bounds__(256) grouped_rowmajor_kernel(const TiledArgs a) {
  constexpr int G = 32 / SG;
  constexpr int CW = SG * VB;
  constexpr int BATCH = 8;
  const int lane = threadIdx.x & 31, sg = lane / SG, sl = lane % SG;
  const unsigned sgmask = SG == 32 ? 0xffffffffu : (((1u << SG) - 1u) << (sg * SG));
  const int64_t grp = (int64_t)((blockIdx.x * (unsigned)blockDim.x + threadIdx.x) >> 5);
  const int64_t s0 = grp * 256;
  if (s0 >= a.nreg) return;
  const int cnt = (int)(a.nreg - s0 < 256 ? a.nreg - s0 : 256);
  const int per = (cnt + G - 1) / G;
  const int lo = sg * per, hi = min(cnt, lo + per);
  const T *__restrict__ B = static_cast<const T *>(a.B);
  T *__restrict__ C = static_cast<T *>(a.C);
  const T *__restrict__ gval = static_cast<const T *>(a.g_val);
  for (int cbase = 0; cbase < a.N; cbase += CW) {
    const int col = cbase + sl * VB;
    const bool inb = col < a.N;
    int cur = -1;
    ACC acc[VB];
#pragma unroll
    for (int e = 0; e < VB; ++e) acc[e] = ACC(0);
    for (int k0 = lo; k0 < hi; k0 += SG) {
      const int m = min(SG, hi - k0);  // the same for every lane of the sub-warp
      int myr = 0, myb = 0;
      ACC myv = ACC(0);
      if (sl < m) {
        const int64_t s = s0 + k0 + sl;
        myr = __ldg(a.g_row + s);
        const int c = __ldg(a.g_col + s);
        myb = a.presorted ? c : __ldg(a.perm + c);
        myv = (ACC)__ldg(gval + s);
      }
      for (int u0 = 0; u0 < m; u0 += BATCH) {
        ACC b[BATCH][VB];
#pragma unroll
        for (int u = 0; u < BATCH; ++u) {
          const int brow = __shfl_sync(sgmask, myb, (u0 + u) & (SG - 1), SG);
          if (inb && u0 + u < m) vload<T, ACC, VB>(B + (int64_t)brow * a.ldb + col, b[u]);
          else {
#pragma unroll
            for (int e = 0; e < VB; ++e) b[u][e] = ACC(0);
          }
        }
#pragma unroll
        for (int u = 0; u < BATCH; ++u) {
          const int r = __shfl_sync(sgmask, myr, (u0 + u) & (SG - 1), SG);
          const ACC w = __shfl_sync(sgmask, myv, (u0 + u) & (SG - 1), SG);
          if (u0 + u < m) {
            if (r != cur) {
              if (cur >= 0 && inb) vatomic_add<T, ACC, VB>(C + (int64_t)cur * a.ldc + col, acc);
              cur = r;
#pragma unroll
              for (int e = 0; e < VB; ++e) acc[e] = ACC(0);
            }
#pragma unroll
            for (int e = 0; e < VB; ++e) acc[e] = fma(w, b[u][e], acc[e]);
          }
        }
      }
    }
    if (cur >= 0 && inb) vatomic_add<T, ACC, VB>(C + (int64_t)cur * a.ldc + col, acc);
  }
}

template <class T, class ACC, int VB, int SG>
__global__ void __launch_bounds__(256) reside_rowmajor_kernel(const TiledArgs a) {
  constexpr int G = 32 / SG;
  constexpr int CW = SG * VB;
  const int lane = threadIdx.x & 31, sg = lane / SG, sl = lane % SG;
  const int wid = (int)((blockIdx.x * (unsigned)blockDim.x + threadIdx.x) >> 5);
  const int nunits = a.balanced ? a.numblk : a.reside_col;
  if (wid >= nunits) return;
  int q, start, stop;
  if (a.balanced) {
    const unsigned cb = a.colorblk[wid];
    q = (int)(cb & 0x7fffffffu);
    if (cb >> 31) { start = a.blkstart[wid]; stop = a.blkstop[wid]; }
    else { start = a.reside_ptr[q]; stop = a.reside_ptr[q + 1]; }
  } else {
    q = wid;
    start = a.reside_ptr[q];
    stop = a.reside_ptr[q + 1];
  }
  const int c = a.K - 1 - q;  // src/Swift.h:166
  const int brow = a.presorted ? c : __ldg(a.perm + c);
  const T *__restrict__ Brow = static_cast<const T *>(a.B) + (int64_t)brow * a.ldb;
  T *__restrict__ C = static_cast<T *>(a.C);
  const T *__restrict__ rv = static_cast<const T *>(a.reside_val);
  for (int cbase = 0; cbase < a.N; cbase += CW) {
    const int col = cbase + sl * VB;
    if (col >= a.N) continue;
    ACC b[VB];
    vload<T, ACC, VB>(Brow + col, b);
    for (int e = start + sg; e < stop; e += G) {
      const int r = __ldg(a.reside_row + e);
      const ACC w = (ACC)__ldg(rv + e);
      ACC x[VB];
#pragma unroll
      for (int i = 0; i < VB; ++i) x[i] = w * b[i];
      vatomic_add<T, ACC, VB>(C + (int64_t)r * a.ldc + col, x);
    }
  }
}

// ------------------------------------------------------------ column-major (reference layout)
template <class T>
__global__ void __launch_bounds__(256) tiled_colmajor_kernel(const TiledArgs a) {
  constexpr int MAXT = 16;
  const int lane = threadIdx.x & 31;
  const int item = (int)((blockIdx.x * (unsigned)blockDim.x + threadIdx.x) >> 5);
  if (item >= a.nitems) return;
  const int t0 = a.item_tile[item], nt = a.item_tile[item + 1] - t0;
  const int col = a.tile_colidx[t0] + lane;
  const int brow = a.presorted ? col : __ldg(a.perm + col);
  const T *__restrict__ sval = static_cast<const T *>(a.sortval);
  int r[MAXT];
  T v[MAXT];
  unsigned first[MAXT];  // lane of the run start, per tile
  bool last[MAXT];
#pragma unroll
  for (int i = 0; i < MAXT; ++i) {
    r[i] = -1; v[i] = T(0); first[i] = 0; last[i] = false;
    if (i < nt) {
      const int64_t s = (int64_t)(t0 + i) * kTile + lane;
      r[i] = __ldg(a.sortrowidx + s);
      v[i] = __ldg(sval + s);
      const int up = __shfl_up_sync(0xffffffffu, r[i], 1);
      const int dn = __shfl_down_sync(0xffffffffu, r[i], 1);
      const unsigned heads = __ballot_sync(0xffffffffu, lane == 0 || up != r[i]);
      first[i] = 31 - __clz(heads & ((2u << lane) - 1u));
      last[i] = lane == 31 || dn != r[i];
    }
  }
  const T *__restrict__ B = static_cast<const T *>(a.B);
  T *__restrict__ C = static_cast<T *>(a.C);
  for (int n = 0; n < a.N; ++n) {
    const T b = __ldg(B + (int64_t)n * a.ldb + brow);
#pragma unroll
    for (int i = 0; i < MAXT; ++i) {
      if (i >= nt) break;
      T x = v[i] * b;
      // segmented inclusive scan over runs of equal rows
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const T y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane - o >= (int)first[i]) x += y;
      }
      if (last[i]) atomicAdd(C + (int64_t)n * a.ldc + r[i], x);
    }
  }
}

template <class T>
__global__ void __launch_bounds__(256) reside_colmajor_kernel(const TiledArgs a) {
  const int lane = threadIdx.x & 31;
  const int wid = (int)((blockIdx.x * (unsigned)blockDim.x + threadIdx.x) >> 5);
  const int nunits = a.balanced ? a.numblk : a.reside_col;
  if (wid >= nunits) return;
  int q, start, stop;
  if (a.balanced) {
    const unsigned cb = a.colorblk[wid];
    q = (int)(cb & 0x7fffffffu);
    if (cb >> 31) { start = a.blkstart[wid]; stop = a.blkstop[wid]; }
    else { start = a.reside_ptr[q]; stop = a.reside_ptr[q + 1]; }
  } else {
    q = wid;
    start = a.reside_ptr[q];
    stop = a.reside_ptr[q + 1];
  }
  const int c = a.K - 1 - q;
  const int brow = a.presorted ? c : __ldg(a.perm + c);
  const T *__restrict__ B = static_cast<const T *>(a.B);
  T *__restrict__ C = static_cast<T *>(a.C);
  const T *__restrict__ rv = static_cast<const T *>(a.reside_val);
  for (int e = start + lane; e < stop; e += 32) {
    const int r = __ldg(a.reside_row + e);
    const T w = __ldg(rv + e);
    for (int n = 0; n < a.N; ++n)
      atomicAdd(C + (int64_t)n * a.ldc + r, w * __ldg(B + (int64_t)n * a.ldb + brow));
  }
}

template <class T, class ACC, int VB, int SG>
swift_status launch_rowmajor(const TiledArgs &a, cudaStream_t st) {
  if (a.g_row) {
    const int64_t groups = (a.nreg + 255) / 256;
    if (groups > 0) {
      const int64_t blocks = (groups * 32 + 255) / 256;
      grouped_rowmajor_kernel<T, ACC, VB, SG><<<(unsigned)blocks, 256, 0, st>>>(a);
      SW_CHECK_LAUNCH();
    }
  } else if (a.nitems > 0) {
    const int64_t blocks = ((int64_t)a.nitems * 32 + 255) / 256;
    tiled_rowmajor_kernel<T, ACC, VB, SG><<<(unsigned)blocks, 256, 0, st>>>(a);
    SW_CHECK_LAUNCH();
  }
  const int units = a.balanced ? a.numblk : a.reside_col;
  if (units > 0) {
    const int64_t blocks = ((int64_t)units * 32 + 255) / 256;
    reside_rowmajor_kernel<T, ACC, VB, SG><<<(unsigned)blocks, 256, 0, st>>>(a);
    SW_CHECK_LAUNCH();
  }
  return SWIFT_OK;
}

template <class T, class ACC>
swift_status dispatch_rowmajor(const TiledArgs &a, bool vec_ok, cudaStream_t st) {
  constexpr int V = VecWidth<T>::value;
  if (!vec_ok) return launch_rowmajor<T, ACC, 1, 32>(a, st);
  const int lanes = (a.N + V - 1) / V;
  if (lanes <= 2) return launch_rowmajor<T, ACC, V, 2>(a, st);
  if (lanes <= 4) return launch_rowmajor<T, ACC, V, 4>(a, st);
  if (lanes <= 8) return launch_rowmajor<T, ACC, V, 8>(a, st);
  if (lanes <= 16) return launch_rowmajor<T, ACC, V, 16>(a, st);
  return launch_rowmajor<T, ACC, V, 32>(a, st);
}

template <class T>
swift_status launch_colmajor(const TiledArgs &a, cudaStream_t st) {
  if (a.nitems > 0) {
    const int64_t blocks = ((int64_t)a.nitems * 32 + 255) / 256;
    tiled_colmajor_kernel<T><<<(unsigned)blocks, 256, 0, st>>>(a);
    SW_CHECK_LAUNCH();
  }
  const int units = a.balanced ? a.numblk : a.reside_col;
  if (units > 0) {
    const int64_t blocks = ((int64_t)units * 32 + 255) / 256;
    reside_colmajor_kernel<T><<<(unsigned)blocks, 256, 0, st>>>(a);
    SW_CHECK_LAUNCH();
  }
  return SWIFT_OK;
}

}  // namespace

swift_status zero_dense(void *C, int rows, int N, int64_t ld, swift_layout layout, size_t esz,
                        cudaStream_t st) {
  const int outer = layout == SWIFT_ROW_MAJOR ? rows : N;
  const int inner = layout == SWIFT_ROW_MAJOR ? N : rows;
  if (outer == 0 || inner == 0) return SWIFT_OK;
  SW_CHECK_CUDA(cudaMemset2DAsync(C, (size_t)ld * esz, 0, (size_t)inner * esz, (size_t)outer, st));
  return SWIFT_OK;
}

swift_status run_tiled(const Plan &p, const DenseArgs &d, int reside_variant, cudaStream_t st, bool grouped) {
  if (d.b_layout != d.c_layout) return SWIFT_ERR_UNSUPPORTED;
  if (grouped && (d.c_layout != SWIFT_ROW_MAJOR || !p.grouped_built)) return SWIFT_ERR_UNSUPPORTED;
  if (d.dtype == SWIFT_BF16 || d.dtype == SWIFT_F16) return SWIFT_ERR_UNSUPPORTED;
  if ((d.dtype == SWIFT_F64) != (p.val_type == SWIFT_F64)) return SWIFT_ERR_UNSUPPORTED;
  const size_t esz = d.dtype == SWIFT_F64 ? 8 : 4;
  SW_TRY(zero_dense(d.C, p.M, d.N, d.ldc, d.c_layout, esz, st));
  if (d.N == 0) return SWIFT_OK;
  TiledArgs a{};
  a.M = p.M; a.K = p.K; a.N = d.N; a.nitems = p.nstrips; a.tilenum = p.tilenum;
  a.presorted = d.b_presorted;
  a.item_tile = p.item_tile.as<int>();
  a.tile_colidx = p.tile_colidx.as<int>();
  a.sortrowidx = p.sortrowidx.as<int>();
  a.sortval = p.sortval.p;
  a.perm = p.perm.as<int>();
  a.reside_ptr = p.reside_ptr.as<int>();
  a.reside_row = p.reside_row.as<int>();
  a.reside_val = p.reside_val.p;
  a.reside_col = p.reside_col;
  a.numblk = p.numblk;
  a.balanced = reside_variant == 0 && p.numblk > 0;
  a.colorblk = p.colorblk.as<unsigned>();
  a.blkstart = p.blkstart.as<int>();
  a.blkstop = p.blkstop.as<int>();
  a.B = d.B; a.ldb = d.ldb; a.C = d.C; a.ldc = d.ldc;
  a.nreg = (int64_t)p.tilenum * kTile;
  if (grouped) {
    a.g_row = p.g_row.as<int>();
    a.g_col = p.g_col.as<int>();
    a.g_val = p.g_val.p;
  }
  if (!d.b_presorted && !p.perm.p) return SWIFT_ERR_INVALID_ARG;
  if (d.c_layout == SWIFT_COL_MAJOR)
    return d.dtype == SWIFT_F64 ? launch_colmajor<double>(a, st) : launch_colmajor<float>(a, st);
  const bool vec_ok = ((uintptr_t)d.B % 16 == 0) && ((uintptr_t)d.C % 16 == 0) &&
                      ((d.ldb * (int64_t)esz) % 16 == 0) && ((d.ldc * (int64_t)esz) % 16 == 0) &&
                      (d.N % (int)(16 / esz) == 0);
  return d.dtype == SWIFT_F64 ? dispatch_rowmajor<double, double>(a, vec_ok, st)
                              : dispatch_rowmajor<float, float>(a, vec_ok, st);
}

}  // namespace swift
