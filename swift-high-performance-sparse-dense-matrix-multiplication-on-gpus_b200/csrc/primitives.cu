// primitives.cu -- device-wide scan, stable radix sort and reductions used by the format
// build.  The reference uses cub::DeviceScan and thrust::sort_by_key for these
// (src/formatTransform_cuda.h:296-300, src/ColSort_cuda.h:108); the library carries its own.
#include "common.cuh"

namespace swift {

namespace {

constexpr int kScanThreads = 256;
constexpr int kScanItems = 8;
constexpr int kScanTile = kScanThreads * kScanItems;

__device__ __forceinline__ int warp_inclusive_scan(int v) {
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    int t = __shfl_up_sync(0xffffffffu, v, o);
    if ((threadIdx.x & 31) >= o) v += t;
  }
  return v;
}

// Block-wide exclusive scan of one value per thread (blockDim.x == kScanThreads);
// returns the exclusive prefix and writes the block total to *total.
__device__ int block_exclusive_scan(int v, int *total) {
  __shared__ int warp_sums[kScanThreads / 32];
  int incl = warp_inclusive_scan(v);
  int w = threadIdx.x >> 5;
  if ((threadIdx.x & 31) == 31) warp_sums[w] = incl;
  __syncthreads();
  if (w == 0) {
    int s = (threadIdx.x < kScanThreads / 32) ? warp_sums[threadIdx.x] : 0;
    int si = warp_inclusive_scan(s);
    if (threadIdx.x < kScanThreads / 32) warp_sums[threadIdx.x] = si - s;
    if (threadIdx.x == kScanThreads / 32 - 1) warp_sums[kScanThreads / 32 - 1] = si - s, *total = si;
  }
  __syncthreads();
  int r = warp_sums[w] + incl - v;
  __syncthreads();
  return r;
}

__global__ void scan_reduce_kernel(const int *__restrict__ in, int64_t n, int *__restrict__ part) {
  int64_t base = (int64_t)blockIdx.x * kScanTile;
  int s = 0;
  for (int i = threadIdx.x; i < kScanTile; i += kScanThreads) {
    int64_t g = base + i;
    if (g < n) s += in[g];
  }
  // block reduce
  for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
  __shared__ int ws[kScanThreads / 32];
  if ((threadIdx.x & 31) == 0) ws[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    int t = 0;
    for (int i = 0; i < kScanThreads / 32; ++i) t += ws[i];
    part[blockIdx.x] = t;
  }
}

// Single-block exclusive scan of `part` (nb entries) in place; total stored at *total.
__global__ void scan_partials_kernel(int *part, int64_t nb, int *total) {
  __shared__ int carry_s;
  __shared__ int tot_s;
  if (threadIdx.x == 0) carry_s = 0;
  __syncthreads();
  for (int64_t base = 0; base < nb; base += kScanThreads) {
    int64_t g = base + threadIdx.x;
    int v = g < nb ? part[g] : 0;
    int ex = block_exclusive_scan(v, &tot_s);
    int carry = carry_s;
    if (g < nb) part[g] = carry + ex;
    __syncthreads();
    if (threadIdx.x == 0) carry_s = carry + tot_s;
    __syncthreads();
  }
  if (threadIdx.x == 0) *total = carry_s;
}

__global__ void scan_apply_kernel(const int *__restrict__ in, int *__restrict__ out, int64_t n,
                                  const int *__restrict__ part) {
  __shared__ int tot_s;
  int64_t base = (int64_t)blockIdx.x * kScanTile + (int64_t)threadIdx.x * kScanItems;
  int v[kScanItems];
  int s = 0;
#pragma unroll
  for (int i = 0; i < kScanItems; ++i) {
    int64_t g = base + i;
    v[i] = g < n ? in[g] : 0;
    s += v[i];
  }
  int ex = block_exclusive_scan(s, &tot_s) + part[blockIdx.x];
#pragma unroll
  for (int i = 0; i < kScanItems; ++i) {
    int64_t g = base + i;
    if (g < n) out[g] = ex;
    ex += v[i];
  }
}

// ---------------------------------------------------------------- radix sort
constexpr int kRsThreads = 256;
constexpr int kRsWarps = kRsThreads / 32;
constexpr int kRsItems = 16;                       // per lane
constexpr int kRsSeg = 32 * kRsItems;              // elements per warp segment
constexpr int kRsTile = kRsWarps * kRsSeg;         // 4096 per block
constexpr int kRsBins = 256;

__global__ void rs_upsweep(const uint32_t *__restrict__ keys, int64_t n, int shift, int nb,
                           int *__restrict__ hist) {
  __shared__ int h[kRsBins];
  h[threadIdx.x] = 0;
  __syncthreads();
  int64_t base = (int64_t)blockIdx.x * kRsTile;
  for (int i = threadIdx.x; i < kRsTile; i += kRsThreads) {
    int64_t g = base + i;
    if (g < n) atomicAdd(&h[(keys[g] >> shift) & (kRsBins - 1)], 1);
  }
  __syncthreads();
  hist[(int64_t)threadIdx.x * nb + blockIdx.x] = h[threadIdx.x];
}

// Stable scatter: element order inside a tile is warp segment, then round, then lane.
__global__ void rs_downsweep(const uint32_t *__restrict__ kin, const uint32_t *__restrict__ vin,
                             uint32_t *__restrict__ kout, uint32_t *__restrict__ vout, int64_t n,
                             int shift, int nb, const int *__restrict__ offs) {
  __shared__ int wcnt[kRsWarps][kRsBins];
  __shared__ int boff[kRsBins];
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  for (int i = threadIdx.x; i < kRsWarps * kRsBins; i += kRsThreads) (&wcnt[0][0])[i] = 0;
  boff[threadIdx.x] = offs[(int64_t)threadIdx.x * nb + blockIdx.x];
  __syncthreads();
  const int64_t seg = (int64_t)blockIdx.x * kRsTile + (int64_t)w * kRsSeg;
  uint32_t k[kRsItems], v[kRsItems];
  int r[kRsItems];
  const unsigned lt = lanemask_lt();
#pragma unroll
  for (int it = 0; it < kRsItems; ++it) {
    const int64_t g = seg + it * 32 + l;
    const bool valid = g < n;
    k[it] = valid ? kin[g] : 0u;
    v[it] = valid ? vin[g] : 0u;
    const int d = valid ? (int)((k[it] >> shift) & (kRsBins - 1)) : kRsBins + l;
    const unsigned peers = __match_any_sync(0xffffffffu, d);
    const int leader = __ffs(peers) - 1;
    int cur = valid ? wcnt[w][d] : 0;
    __syncwarp();
    if (valid && l == leader) wcnt[w][d] = cur + __popc(peers);
    __syncwarp();
    r[it] = cur + __popc(peers & lt);
  }
  __syncthreads();
  {
    const int d = threadIdx.x;
    int run = 0;
#pragma unroll
    for (int ww = 0; ww < kRsWarps; ++ww) {
      int c = wcnt[ww][d];
      wcnt[ww][d] = run;
      run += c;
    }
  }
  __syncthreads();
#pragma unroll
  for (int it = 0; it < kRsItems; ++it) {
    const int64_t g = seg + it * 32 + l;
    if (g < n) {
      const int d = (int)((k[it] >> shift) & (kRsBins - 1));
      const int64_t pos = (int64_t)boff[d] + wcnt[w][d] + r[it];
      kout[pos] = k[it];
      vout[pos] = v[it];
    }
  }
}

__global__ void reduce_max_kernel(const int *__restrict__ in, int64_t n, int *out) {
  int m = 0;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    m = max(m, in[i]);
  for (int o = 16; o > 0; o >>= 1) m = max(m, __shfl_down_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0) atomicMax(out, m);
}

}  // namespace

swift_status scan_exclusive_i32(const int *in, int *out, int64_t n, cudaStream_t st) {
  if (n < 0) return SWIFT_ERR_INVALID_ARG;
  int64_t nb = (n + kScanTile - 1) / kScanTile;
  if (nb == 0) {
    SW_CHECK_CUDA(cudaMemsetAsync(out, 0, sizeof(int), st));
    return SWIFT_OK;
  }
  int *part = nullptr;
  SW_CHECK_CUDA(cudaMallocAsync(&part, sizeof(int) * (size_t)nb, st));
  scan_reduce_kernel<<<(unsigned)nb, kScanThreads, 0, st>>>(in, n, part);
  scan_partials_kernel<<<1, kScanThreads, 0, st>>>(part, nb, out + n);
  scan_apply_kernel<<<(unsigned)nb, kScanThreads, 0, st>>>(in, out, n, part);
  cudaError_t e = cudaGetLastError();
  cudaFreeAsync(part, st);
  if (e != cudaSuccess) {
    set_last_error("scan_exclusive_i32", cudaGetErrorString(e));
    return SWIFT_ERR_CUDA;
  }
  return SWIFT_OK;
}

swift_status radix_sort_pairs(uint32_t *keys_in, uint32_t *vals_in, uint32_t *keys_out,
                              uint32_t *vals_out, int64_t n, int bits, cudaStream_t st) {
  if (n <= 0) return SWIFT_OK;
  const int passes = (bits + 7) / 8;
  if (passes == 0) {
    SW_CHECK_CUDA(cudaMemcpyAsync(keys_out, keys_in, sizeof(uint32_t) * n, cudaMemcpyDeviceToDevice, st));
    SW_CHECK_CUDA(cudaMemcpyAsync(vals_out, vals_in, sizeof(uint32_t) * n, cudaMemcpyDeviceToDevice, st));
    return SWIFT_OK;
  }
  const int64_t nb = (n + kRsTile - 1) / kRsTile;
  if (nb * kRsBins >= (int64_t)INT32_MAX) return SWIFT_ERR_OVERFLOW;
  int *hist = nullptr;
  SW_CHECK_CUDA(cudaMallocAsync(&hist, sizeof(int) * (size_t)(nb * kRsBins + 1), st));
  uint32_t *ki = keys_in, *vi = vals_in, *ko = keys_out, *vo = vals_out;
  // with an even number of passes the result would land in the input buffers: start by
  // writing into them so that the last pass writes the output buffers.
  if (passes % 2 == 0) {
    SW_CHECK_CUDA(cudaMemcpyAsync(keys_out, keys_in, sizeof(uint32_t) * n, cudaMemcpyDeviceToDevice, st));
    SW_CHECK_CUDA(cudaMemcpyAsync(vals_out, vals_in, sizeof(uint32_t) * n, cudaMemcpyDeviceToDevice, st));
    ki = keys_out; vi = vals_out; ko = keys_in; vo = vals_in;
  }
  swift_status rc = SWIFT_OK;
  for (int p = 0; p < passes && rc == SWIFT_OK; ++p) {
    const int shift = 8 * p;
    rs_upsweep<<<(unsigned)nb, kRsThreads, 0, st>>>(ki, n, shift, (int)nb, hist);
    rc = scan_exclusive_i32(hist, hist, nb * kRsBins, st);
    if (rc != SWIFT_OK) break;
    rs_downsweep<<<(unsigned)nb, kRsThreads, 0, st>>>(ki, vi, ko, vo, n, shift, (int)nb, hist);
    std::swap(ki, ko);
    std::swap(vi, vo);
  }
  cudaError_t e = cudaGetLastError();
  cudaFreeAsync(hist, st);
  if (rc != SWIFT_OK) return rc;
  if (e != cudaSuccess) {
    set_last_error("radix_sort_pairs", cudaGetErrorString(e));
    return SWIFT_ERR_CUDA;
  }
  return SWIFT_OK;
}

namespace {
// Tiles of 32 * TR rows x 32 columns through shared memory (one padding element per tile row
// keeps the transposed reads on distinct banks), so both a warp's loads and its stores cover
// 32 consecutive elements and each thread keeps 4 * TR loads in flight; blocks walk the tiles
// down the input's columns.
template <class E, int TR>
__global__ void __launch_bounds__(256) transpose_kernel(const E *__restrict__ in, int rows, int cols,
                                                        int64_t ld_in, E *__restrict__ out, int64_t ld_out) {
  constexpr int R = 32 * TR;
  __shared__ E tile[32][R + 1];
  const int64_t ntr = (rows + R - 1) / R, ntiles = ntr * ((cols + 31) / 32);
  const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
  for (int64_t t = blockIdx.x; t < ntiles; t += gridDim.x) {
    const int64_t r0 = (t % ntr) * R, c0 = (t / ntr) * 32;
#pragma unroll
    for (int j = ty; j < 32; j += 8) {
#pragma unroll
      for (int q = 0; q < TR; ++q) {
        const int64_t r = r0 + 32 * q + tx, c = c0 + j;
        if (r < rows && c < cols) tile[j][32 * q + tx] = in[r + c * ld_in];
      }
    }
    __syncthreads();
#pragma unroll
    for (int j = ty; j < R; j += 8) {
      const int64_t r = r0 + j, c = c0 + tx;
      if (r < rows && c < cols) out[r * ld_out + c] = tile[tx][j];
    }
    __syncthreads();
  }
}

}  // namespace

swift_status transpose_dense(const void *in, int rows, int cols, int64_t ld_in, void *out,
                             int64_t ld_out, size_t esz, cudaStream_t st) {
  const int64_t ntiles = ((int64_t)rows + 31) / 32 * (((int64_t)cols + 31) / 32);
  if (ntiles == 0) return SWIFT_OK;
  constexpr int TR = 4;
  const int64_t ntiles4 = ((int64_t)rows + 32 * TR - 1) / (32 * TR) * (((int64_t)cols + 31) / 32);
  const int grid = (int)std::min<int64_t>(ntiles4, 148 * 8);
  switch (esz) {
    case 2:
      transpose_kernel<uint16_t, TR><<<grid, 256, 0, st>>>(static_cast<const uint16_t *>(in), rows, cols, ld_in,
                                                           static_cast<uint16_t *>(out), ld_out);
      break;
    case 4:
      transpose_kernel<uint32_t, TR><<<grid, 256, 0, st>>>(static_cast<const uint32_t *>(in), rows, cols, ld_in,
                                                           static_cast<uint32_t *>(out), ld_out);
      break;
    case 8:
      transpose_kernel<uint64_t, TR><<<grid, 256, 0, st>>>(static_cast<const uint64_t *>(in), rows, cols, ld_in,
                                                           static_cast<uint64_t *>(out), ld_out);
      break;
    default:
      return SWIFT_ERR_UNSUPPORTED;
  }
  SW_CHECK_LAUNCH();
  return SWIFT_OK;
}

swift_status reduce_max_i32(const int *in, int64_t n, int *dev_out, cudaStream_t st) {
  SW_CHECK_CUDA(cudaMemsetAsync(dev_out, 0, sizeof(int), st));
  if (n <= 0) return SWIFT_OK;
  int blocks = (int)std::min<int64_t>((n + 255) / 256, 148 * 8);
  reduce_max_kernel<<<blocks, 256, 0, st>>>(in, n, dev_out);
  SW_CHECK_LAUNCH();
  return SWIFT_OK;
}

}  // namespace swift
