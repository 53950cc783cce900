// export.cu -- the reference arrays that the SpMM kernels do not need, built on the GPU on
// demand, and the host export of a plan as a reference slide_matrix (src/format.h:6-39).
//
//   block_catgory segments  src/block_catgory.h:79-159 (countrow, segsum, segmentoffset,
//                           sortrowindex: per-tile runs of equal rows)
//   row_idx_sort            src/back_process.h:23-229 (per-8-tile row sort: sorted keys,
//                           val_position, val_offset; FP32 flavour's blockratio)
#include <cstdlib>

#include "common.cuh"

namespace swift {

namespace {

__global__ void seg_count_kernel(const int *__restrict__ rows, int T, int *__restrict__ cnt) {
  const int l = threadIdx.x & 31;
  const int warps = (gridDim.x * blockDim.x) >> 5;
  for (int t = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; t < T; t += warps) {
    const int r = rows[(int64_t)t * kTile + l];
    const int up = __shfl_up_sync(0xffffffffu, r, 1);
    const int changes = __popc(__ballot_sync(0xffffffffu, l > 0 && up != r));
    if (l == 0) cnt[t] = changes + 1;
  }
}

__global__ void seg_fill_kernel(const int *__restrict__ rows, int T, const int *__restrict__ countrow,
                                int *__restrict__ segmentoffset, int *__restrict__ sortrowindex) {
  const int l = threadIdx.x & 31;
  const int warps = (gridDim.x * blockDim.x) >> 5;
  for (int t = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; t < T; t += warps) {
    const int r = rows[(int64_t)t * kTile + l];
    const int up = __shfl_up_sync(0xffffffffu, r, 1);
    const unsigned heads = __ballot_sync(0xffffffffu, l == 0 || up != r);
    const bool head = (heads >> l) & 1u;
    int val = 0;
    if (head) {
      const unsigned later = l == 31 ? 0u : (heads & ~((2u << l) - 1u));
      const int next = later ? __ffs(later) - 1 : 32;
      val = next - l - 1;
      segmentoffset[countrow[t] + __popc(heads & ((1u << l) - 1u))] = val;
    }
    sortrowindex[(int64_t)t * kTile + l] = val;
  }
}

// One block of 256 threads per group of 8 tiles (the last group may be shorter).
__global__ void row_sort_kernel(const int *__restrict__ rows, int T, int *__restrict__ sorted,
                                int *__restrict__ val_position, int *__restrict__ val_offset,
                                int *__restrict__ all_single_groups) {
  __shared__ unsigned long long key[256];
  __shared__ int rk[256];
  __shared__ int non_single;
  const int g = blockIdx.x, i = threadIdx.x;
  const int t0 = g * 8, t1 = min(t0 + 8, T);
  const int cnt = (t1 - t0) * kTile;
  const int64_t base = (int64_t)t0 * kTile;
  const bool last_group = (T % 8 != 0) && (g == (T + 7) / 8 - 1);
  if (i == 0) non_single = 0;
  key[i] = i < cnt ? ((unsigned long long)(unsigned)rows[base + i] << 9) | (unsigned)i : ~0ull;
  __syncthreads();
  for (int k = 2; k <= 256; k <<= 1)
    for (int j = k >> 1; j > 0; j >>= 1) {
      const int x = i ^ j;
      if (x > i) {
        const bool up = (i & k) == 0;
        const unsigned long long a = key[i], b = key[x];
        if ((a > b) == up) { key[i] = b; key[x] = a; }
      }
      __syncthreads();
    }
  if (i < cnt) {
    rk[i] = (int)(key[i] >> 9);
    sorted[base + i] = rk[i];
    val_position[base + (int)(key[i] & 511u)] = i;
  }
  __syncthreads();
  if (i < cnt) {
    int off = 0;
    if (i == 0 || rk[i] != rk[i - 1]) {
      int len = 1;
      while (i + len < cnt && rk[i + len] == rk[i]) ++len;
      if (len > 1) off = len - 1;
      else {
        // src/back_process.h:172-205 has no branch for a last-slot singleton after a run
        const bool quirk = last_group && i == cnt - 1 && i >= 2 && rk[i - 1] == rk[i - 2];
        off = quirk ? 0 : -1;
      }
    }
    val_offset[base + i] = off;
    if (off != -1) atomicOr(&non_single, 1);
  }
  __syncthreads();
  if (i == 0 && !non_single) atomicAdd(all_single_groups, 1);
}

// Grouped-engine slots: original slot o of group g lands at sorted slot g*256 + vpos[o], with
// its sorted column (tile_colidx of its tile + lane) and value; a vpos entry outside its group
// or hit twice sets *bad (with n slots per group and no slot hit twice, every slot is filled).
template <class V>
__global__ void grouped_scatter_kernel(const int *__restrict__ vpos, const int *__restrict__ tile_colidx,
                                       const V *__restrict__ sortval, int64_t nreg, int *__restrict__ col,
                                       V *__restrict__ val, int *__restrict__ hit, int *__restrict__ bad) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t o = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; o < nreg; o += stride) {
    const int64_t g = o & ~(int64_t)255;
    const int64_t glen = nreg - g < 256 ? nreg - g : 256;
    const int v = vpos[o];
    if (v < 0 || v >= glen) { *bad = 1; continue; }
    const int64_t s = g + v;
    if (atomicExch(hit + s, 1) != 0) { *bad = 1; continue; }
    col[s] = tile_colidx[o >> 5] + (int)(o & 31);
    val[s] = sortval[o];
  }
}

int grid_warps(int64_t warps) {
  int64_t b = (warps * 32 + 255) / 256;
  return (int)std::max<int64_t>(1, std::min<int64_t>(b, 148 * 32));
}

template <class T> T *host_copy(const void *dev, size_t n, cudaStream_t st, swift_status *rc) {
  T *h = static_cast<T *>(malloc(sizeof(T) * (n ? n : 1)));
  if (!h) { *rc = SWIFT_ERR_ALLOC; return nullptr; }
  if (n) {
    cudaError_t e = cudaMemcpyAsync(h, dev, sizeof(T) * n, cudaMemcpyDeviceToHost, st);
    if (e != cudaSuccess) { set_last_error("export copy", cudaGetErrorString(e)); *rc = SWIFT_ERR_CUDA; }
  }
  return h;
}

}  // namespace

swift_status build_grouped(Plan &p, const int *keys, const int *vpos, cudaStream_t st) {
  const int T = p.tilenum;
  const int64_t nreg = (int64_t)T * kTile;
  if ((keys == nullptr) != (vpos == nullptr)) return SWIFT_ERR_INVALID_ARG;
  p.grouped_built = false;
  SW_TRY(p.g_row.alloc(sizeof(int) * (size_t)std::max<int64_t>(nreg, 1)));
  SW_TRY(p.g_col.alloc(sizeof(int) * (size_t)std::max<int64_t>(nreg, 1)));
  SW_TRY(p.g_val.alloc(p.vsz * (size_t)std::max<int64_t>(nreg, 1)));
  if (nreg == 0) {
    p.grouped_built = true;
    return SWIFT_OK;
  }
  TmpBuf tvpos, toff, hit, flags;
  SW_TRY(hit.alloc(sizeof(int) * (size_t)nreg, st));
  SW_TRY(flags.alloc(sizeof(int) * 2, st));
  SW_CHECK_CUDA(cudaMemsetAsync(hit.p, 0, sizeof(int) * (size_t)nreg, st));
  SW_CHECK_CUDA(cudaMemsetAsync(flags.p, 0, sizeof(int) * 2, st));
  if (!keys) {
    SW_TRY(tvpos.alloc(sizeof(int) * (size_t)nreg, st));
    SW_TRY(toff.alloc(sizeof(int) * (size_t)nreg, st));
    row_sort_kernel<<<(T + 7) / 8, 256, 0, st>>>(p.sortrowidx.as<int>(), T, p.g_row.as<int>(), tvpos.as<int>(),
                                                  toff.as<int>(), flags.as<int>() + 1);
    SW_CHECK_LAUNCH();
    vpos = tvpos.as<int>();
  } else {
    SW_CHECK_CUDA(cudaMemcpyAsync(p.g_row.p, keys, sizeof(int) * (size_t)nreg, cudaMemcpyDeviceToDevice, st));
  }
  const int grid = grid_warps((nreg + 31) / 32);
  if (p.val_type == SWIFT_F64)
    grouped_scatter_kernel<double><<<grid, 256, 0, st>>>(vpos, p.tile_colidx.as<int>(), p.sortval.as<double>(), nreg,
                                                         p.g_col.as<int>(), p.g_val.as<double>(), hit.as<int>(),
                                                         flags.as<int>());
  else
    grouped_scatter_kernel<float><<<grid, 256, 0, st>>>(vpos, p.tile_colidx.as<int>(), p.sortval.as<float>(), nreg,
                                                        p.g_col.as<int>(), p.g_val.as<float>(), hit.as<int>(),
                                                        flags.as<int>());
  SW_CHECK_LAUNCH();
  int bad = 0;
  SW_CHECK_CUDA(cudaMemcpyAsync(&bad, flags.p, sizeof(int), cudaMemcpyDeviceToHost, st));
  SW_CHECK_CUDA(cudaStreamSynchronize(st));
  if (bad) {
    set_last_error("grouped slots", "val_position is not a permutation of each group of 8 tiles");
    return SWIFT_ERR_INVALID_ARG;
  }
  p.grouped_built = true;
  return SWIFT_OK;
}

swift_status build_segments(const Plan &p, DevBuf &countrow, DevBuf &segmentoffset,
                            DevBuf &sortrowindex, int *segsum, cudaStream_t st) {
  const int T = p.tilenum;
  SW_TRY(countrow.alloc(sizeof(int) * ((size_t)T + 1)));
  SW_TRY(sortrowindex.alloc(sizeof(int) * (size_t)T * kTile));
  TmpBuf cnt;
  SW_TRY(cnt.alloc(sizeof(int) * ((size_t)T + 1), st));
  if (T > 0) seg_count_kernel<<<grid_warps(T), 256, 0, st>>>(p.sortrowidx.as<int>(), T, cnt.as<int>());
  SW_CHECK_LAUNCH();
  SW_TRY(scan_exclusive_i32(cnt.as<int>(), countrow.as<int>(), T, st));
  int h = 0;
  SW_CHECK_CUDA(cudaMemcpyAsync(&h, countrow.as<int>() + T, sizeof(int), cudaMemcpyDeviceToHost, st));
  SW_CHECK_CUDA(cudaStreamSynchronize(st));
  *segsum = h;
  SW_TRY(segmentoffset.alloc(sizeof(int) * ((size_t)h + 1)));
  SW_CHECK_CUDA(cudaMemsetAsync(segmentoffset.p, 0, sizeof(int) * ((size_t)h + 1), st));
  if (T > 0)
    seg_fill_kernel<<<grid_warps(T), 256, 0, st>>>(p.sortrowidx.as<int>(), T, countrow.as<int>(),
                                                   segmentoffset.as<int>(), sortrowindex.as<int>());
  SW_CHECK_LAUNCH();
  return SWIFT_OK;
}

swift_status build_row_sort(const Plan &p, DevBuf &sorted_rows, DevBuf &val_position,
                            DevBuf &val_offset, float *blockratio, cudaStream_t st) {
  const int T = p.tilenum;
  const size_t n = (size_t)T * kTile;
  SW_TRY(sorted_rows.alloc(sizeof(int) * n));
  SW_TRY(val_position.alloc(sizeof(int) * n));
  SW_TRY(val_offset.alloc(sizeof(int) * n));
  TmpBuf cnt;
  SW_TRY(cnt.alloc(sizeof(int), st));
  SW_CHECK_CUDA(cudaMemsetAsync(cnt.p, 0, sizeof(int), st));
  const int groups = (T + 7) / 8;
  if (groups > 0)
    row_sort_kernel<<<groups, 256, 0, st>>>(p.sortrowidx.as<int>(), T, sorted_rows.as<int>(),
                                            val_position.as<int>(), val_offset.as<int>(), cnt.as<int>());
  SW_CHECK_LAUNCH();
  int h = 0;
  SW_CHECK_CUDA(cudaMemcpyAsync(&h, cnt.p, sizeof(int), cudaMemcpyDeviceToHost, st));
  SW_CHECK_CUDA(cudaStreamSynchronize(st));
  if (blockratio) *blockratio = (float)h / (float)groups;  // 0/0 = NaN like the reference
  return SWIFT_OK;
}

template <class VAL_T, class SLIDE>
swift_status export_slide(const Plan &p, SLIDE *out, int with_row_sort, float *blockratio,
                          cudaStream_t st) {
  memset(out, 0, sizeof(*out));
  const int T = p.tilenum;
  const size_t nreg = (size_t)T * kTile;
  swift_status rc = SWIFT_OK;
  DevBuf countrow, segoff, sri, srt, vpos, voff;
  int segsum = 0;
  SW_TRY(build_segments(p, countrow, segoff, sri, &segsum, st));
  if (with_row_sort) SW_TRY(build_row_sort(p, srt, vpos, voff, blockratio, st));
  out->tilenum = T;
  out->regular_nnz = (int)nreg;
  out->segsum = segsum;
  out->reside_col = p.reside_col;
  out->reside_nnz = p.reside_nnz;
  out->numblk = p.numblk;
  out->sortval = host_copy<VAL_T>(p.sortval.p, nreg, st, &rc);
  out->sortrowidx = host_copy<int>(with_row_sort ? srt.p : p.sortrowidx.p, nreg, st, &rc);
  out->tile_colidx = host_copy<int>(p.tile_colidx.p, T, st, &rc);
  out->tile_tall = host_copy<int>(p.tile_tall.p, T, st, &rc);
  out->tile_format = host_copy<int>(p.tile_format.p, T, st, &rc);
  out->countrow = host_copy<int>(countrow.p, (size_t)T + 1, st, &rc);
  out->segmentoffset = host_copy<int>(segoff.p, (size_t)segsum + 1, st, &rc);
  out->sortrowindex = host_copy<int>(sri.p, nreg, st, &rc);
  if (with_row_sort) {
    out->val_position = host_copy<int>(vpos.p, nreg, st, &rc);
    out->val_offset = host_copy<int>(voff.p, nreg, st, &rc);
  }
  out->reside_cscptr = host_copy<int>(p.reside_ptr.p, (size_t)p.reside_col + 1, st, &rc);
  out->reside_cscrowidx = host_copy<int>(p.reside_row.p, p.reside_nnz, st, &rc);
  out->reside_val = host_copy<VAL_T>(p.reside_val.p, p.reside_nnz, st, &rc);
  out->colorblk = host_copy<unsigned>(p.colorblk.p, p.numblk, st, &rc);
  out->blkstart = host_copy<int>(p.blkstart.p, p.numblk, st, &rc);
  out->blkstop = host_copy<int>(p.blkstop.p, p.numblk, st, &rc);
  out->blkptr = host_copy<int>(p.blkptr.p, p.numblk, st, &rc);
  out->tile_ptr = static_cast<int *>(malloc(sizeof(int) * ((size_t)T + 1)));
  out->tile_len = static_cast<int *>(malloc(sizeof(int) * ((size_t)T ? T : 1)));
  if (!out->tile_ptr || !out->tile_len) rc = SWIFT_ERR_ALLOC;
  else {
    // tile_ptr[t] = 32 t and tile_len[t] = 32 (src/coo2csc.h:233-251, 280-284)
    for (int t = 0; t <= T; ++t) out->tile_ptr[t] = t * kTile;
    for (int t = 0; t < T; ++t) out->tile_len[t] = kTile;
  }
  cudaError_t e = cudaStreamSynchronize(st);
  if (e != cudaSuccess && rc == SWIFT_OK) { set_last_error("export", cudaGetErrorString(e)); rc = SWIFT_ERR_CUDA; }
  return rc;
}

template swift_status export_slide<float, swift_slide_matrix_f32>(const Plan &, swift_slide_matrix_f32 *, int, float *, cudaStream_t);
template swift_status export_slide<double, swift_slide_matrix_f64>(const Plan &, swift_slide_matrix_f64 *, int, float *, cudaStream_t);

}  // namespace swift
