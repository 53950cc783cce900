// block_stats.cu -- block-density histogram of A, measured on the GPU.
//
// A is cut into blocks of bh consecutive rows x bw consecutive columns, columns taken either in
// A's own order or in the plan's sorted column order (Swift's count order).  Every nonzero gets
// the key (row panel, column block); two stable LSD radix sorts (column block, then row panel)
// bring equal keys together, run starts are flagged and scanned, and each run (one occupied
// block) is binned by its fill f = nonzeros / (bh * bw): bin k holds 2^-(k+1) < f <= 2^-k for
// k < nbins - 1, the last bin everything sparser.  This is the density measurement behind the
// choice of a dense-tile path (the band engine, or tensor cores, pay only where blocks are
// dense); it is not on any product path.
#include <algorithm>

#include "common.cuh"

namespace swift {
namespace {

__global__ void block_keys_kernel(const int *__restrict__ rowptr, const int *__restrict__ colidx, int M, int bh,
                                  int bw, const int *__restrict__ invperm, uint32_t *__restrict__ colblk,
                                  uint32_t *__restrict__ panel) {
  const int lane = threadIdx.x & 31;
  for (int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < M; i += (gridDim.x * blockDim.x) >> 5) {
    const int e1 = __ldg(rowptr + i + 1);
    for (int e = __ldg(rowptr + i) + lane; e < e1; e += 32) {
      const int j = __ldg(colidx + e);
      const int jj = invperm ? __ldg(invperm + j) : j;
      colblk[e] = (uint32_t)(jj / bw);
      panel[e] = (uint32_t)(i / bh);
    }
  }
}

// flag[e] = 1 where (panel, colblk) differs from element e - 1
__global__ void run_start_kernel(const uint32_t *__restrict__ panel, const uint32_t *__restrict__ colblk, int64_t n,
                                 int *__restrict__ flag) {
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (int64_t)gridDim.x * blockDim.x)
    flag[e] = (e == 0 || panel[e] != panel[e - 1] || colblk[e] != colblk[e - 1]) ? 1 : 0;
}

__global__ void run_pos_kernel(const int *__restrict__ flag, const int *__restrict__ run, int64_t n,
                               int *__restrict__ start) {
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (int64_t)gridDim.x * blockDim.x)
    if (flag[e]) start[run[e]] = (int)e;
}

__global__ void bin_runs_kernel(const int *__restrict__ start, int nruns, int64_t n, double cells, int nbins,
                                unsigned long long *__restrict__ blocks, unsigned long long *__restrict__ nnz) {
  for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < nruns; r += gridDim.x * blockDim.x) {
    const int64_t len = (r + 1 < nruns ? (int64_t)start[r + 1] : n) - start[r];
    const double f = (double)len / cells;
    int k = 0;
    double hi = 1.0;
    while (k < nbins - 1 && f <= hi * 0.5) {  // f in (hi/2, hi] -> bin k
      hi *= 0.5;
      ++k;
    }
    atomicAdd(blocks + k, 1ull);
    atomicAdd(nnz + k, (unsigned long long)len);
  }
}

int bits_for(uint32_t maxv) {
  int b = 0;
  while (b < 32 && (maxv >> b) != 0) ++b;
  return b;
}

}  // namespace
}  // namespace swift

using namespace swift;

extern "C" swift_status swift_plan_block_histogram(swift_plan *plan, int bh, int bw, int order, int nbins,
                                                   long long *blocks, long long *nnz, swift_stream_t stream) {
  if (!plan || bh < 1 || bw < 1 || (order != 0 && order != 1) || nbins < 1 || nbins > 64 || !blocks || !nnz)
    return SWIFT_ERR_INVALID_ARG;
  Plan &p = plan->p;
  if (!p.has_csr) return SWIFT_ERR_UNSUPPORTED;
  cudaStream_t st = S(stream);
  UseNote use_note{p, st};
  for (int k = 0; k < nbins; ++k) blocks[k] = nnz[k] = 0;
  const int64_t n = p.nnz;
  if (n == 0) return SWIFT_OK;
  TmpBuf k0, v0, k1, v1, flag, run, hist;
  SW_TRY(k0.alloc(sizeof(uint32_t) * (size_t)n, st));
  SW_TRY(v0.alloc(sizeof(uint32_t) * (size_t)n, st));
  SW_TRY(k1.alloc(sizeof(uint32_t) * (size_t)n, st));
  SW_TRY(v1.alloc(sizeof(uint32_t) * (size_t)n, st));
  const int grid = std::max(1, std::min((p.M + 7) / 8, p.sm_count * 16));
  block_keys_kernel<<<grid, 256, 0, st>>>(p.rowptr.as<int>(), p.colidx.as<int>(), p.M, bh, bw,
                                          order ? p.invperm.as<int>() : nullptr, k0.as<uint32_t>(), v0.as<uint32_t>());
  SW_CHECK_LAUNCH();
  // stable sorts: by column block, then by row panel (LSD order gives (panel, column block))
  SW_TRY(radix_sort_pairs(k0.as<uint32_t>(), v0.as<uint32_t>(), k1.as<uint32_t>(), v1.as<uint32_t>(), n,
                          bits_for((uint32_t)((std::max(p.K, 1) - 1) / bw)), st));
  SW_TRY(radix_sort_pairs(v1.as<uint32_t>(), k1.as<uint32_t>(), v0.as<uint32_t>(), k0.as<uint32_t>(), n,
                          bits_for((uint32_t)((std::max(p.M, 1) - 1) / bh)), st));
  // v0 = panels, k0 = column blocks, in (panel, column block) order
  SW_TRY(flag.alloc(sizeof(int) * ((size_t)n + 1), st));
  SW_TRY(run.alloc(sizeof(int) * ((size_t)n + 1), st));
  const int eg = (int)std::min<int64_t>((n + 255) / 256, (int64_t)p.sm_count * 32);
  run_start_kernel<<<eg, 256, 0, st>>>(v0.as<uint32_t>(), k0.as<uint32_t>(), n, flag.as<int>());
  SW_CHECK_LAUNCH();
  SW_TRY(scan_exclusive_i32(flag.as<int>(), run.as<int>(), n, st));
  int nruns = 0;
  SW_CHECK_CUDA(cudaMemcpyAsync(&nruns, run.as<int>() + n, sizeof(int), cudaMemcpyDeviceToHost, st));
  SW_CHECK_CUDA(cudaStreamSynchronize(st));
  // run starts reuse the column-block buffer (no longer needed)
  int *start = reinterpret_cast<int *>(k1.p);
  run_pos_kernel<<<eg, 256, 0, st>>>(flag.as<int>(), run.as<int>(), n, start);
  SW_CHECK_LAUNCH();
  SW_TRY(hist.alloc(sizeof(unsigned long long) * 2 * (size_t)nbins, st));
  SW_CHECK_CUDA(cudaMemsetAsync(hist.p, 0, sizeof(unsigned long long) * 2 * (size_t)nbins, st));
  unsigned long long *hb = static_cast<unsigned long long *>(hist.p);
  bin_runs_kernel<<<std::max(1, std::min((nruns + 255) / 256, p.sm_count * 16)), 256, 0, st>>>(
      start, nruns, n, (double)bh * (double)bw, nbins, hb, hb + nbins);
  SW_CHECK_LAUNCH();
  std::vector<unsigned long long> h(2 * (size_t)nbins);
  SW_CHECK_CUDA(cudaMemcpyAsync(h.data(), hist.p, sizeof(unsigned long long) * 2 * (size_t)nbins,
                                cudaMemcpyDeviceToHost, st));
  SW_CHECK_CUDA(cudaStreamSynchronize(st));
  for (int k = 0; k < nbins; ++k) {
    blocks[k] = (long long)h[k];
    nnz[k] = (long long)h[nbins + k];
  }
  return SWIFT_OK;
}
