// gather_bound.cu -- the gather ceiling of the row-ordered engines, measured on the GPU.
//
// Every nonzero of the row walk gathers one B row (N elements) through the SM's global-load
// path.  This kernel does only that: the same column stream, the same 16-byte vectors and
// sub-warp widths, four loads in flight per lane, the gathered rows summed in registers and one
// vector per lane written at the end -- no values, no row bookkeeping, no C rows.  Its time is
// the floor any row-ordered SpMM of this operand can reach; a second launch with every column
// folded into 256 rows (the rows stay in L1) separates the load path's own limit from L2 and
// DRAM.  Measurement only; no product path calls it.
#include <algorithm>

#include "common.cuh"

namespace swift {
namespace {

template <int SG>
__global__ void __launch_bounds__(256, 6) gather_bound_kernel(const int *__restrict__ idx, int64_t nnz,
                                                              const float *__restrict__ B, int64_t ldb, int U,
                                                              int fold, float4 *__restrict__ out) {
  constexpr int G = 32 / SG;  // sub-warps per warp, each walking its own slice of U positions
  const int lane = threadIdx.x & 31, sg = lane / SG, sl = lane % SG;
  const unsigned sgmask = SG == 32 ? 0xffffffffu : (((1u << SG) - 1u) << (sg * SG));
  const int64_t t = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) / 32 * G + sg;
  const int64_t p0 = t * U;
  float4 acc = make_float4(0.f, 0.f, 0.f, 0.f);
  if (p0 < nnz) {
    const int64_t p1 = p0 + U < nnz ? p0 + U : nnz;
    const float *Bl = B + sl * 4;
    for (int64_t q0 = p0; q0 < p1; q0 += SG) {
      const int m = (int)(p1 - q0 < SG ? p1 - q0 : SG);
      int myc = sl < m ? __ldcs(idx + q0 + sl) : 0;
      if (fold) myc &= 255;
      for (int k = 0; k < m; k += 4) {
        float4 b[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
          const int c = __shfl_sync(sgmask, myc, (k + u) % SG, SG);
          b[u] = k + u < m ? __ldg(reinterpret_cast<const float4 *>(Bl + (int64_t)c * ldb)) : make_float4(0.f, 0.f, 0.f, 0.f);
        }
#pragma unroll
        for (int u = 0; u < 4; ++u) {
          acc.x += b[u].x; acc.y += b[u].y; acc.z += b[u].z; acc.w += b[u].w;
        }
      }
    }
  }
  out[(int64_t)blockIdx.x * blockDim.x + threadIdx.x] = acc;
}

__global__ void gather_checksum_kernel(const float4 *__restrict__ v, int64_t n, double *__restrict__ sum) {
  double s = 0.0;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    s += (double)v[i].x + (double)v[i].y + (double)v[i].z + (double)v[i].w;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if ((threadIdx.x & 31) == 0) atomicAdd(sum, s);
}

template <int SG>
void launch_gather(const int *idx, int64_t nnz, const float *B, int64_t ldb, int U, int fold, float4 *out,
                   int64_t blocks, cudaStream_t st) {
  gather_bound_kernel<SG><<<(unsigned)blocks, 256, 0, st>>>(idx, nnz, B, ldb, U, fold, out);
}

}  // namespace
}  // namespace swift

using namespace swift;

extern "C" swift_status swift_gather_bound(const swift_plan *plan, int N, const float *B, int64_t ldb, int reps,
                                           swift_stream_t stream, double *ms_stream, double *ms_l1,
                                           double *checksum) {
  if (!plan || !B || (N != 32 && N != 64 && N != 128) || ldb < N || reps < 1) return SWIFT_ERR_INVALID_ARG;
  if ((uintptr_t)B % 16 != 0 || ldb % 4 != 0) return SWIFT_ERR_UNSUPPORTED;
  const Plan &p = plan->p;
  if (!p.has_csr) return SWIFT_ERR_UNSUPPORTED;
  if (p.K < 256) return SWIFT_ERR_UNSUPPORTED;  // the folded launch reads rows 0..255
  cudaStream_t st = S(stream);
  const int SG = N / 4, G = 32 / SG;
  const int U = 512;  // positions per sub-warp, the row walk's default task size
  const int64_t tasks = ((int64_t)p.nnz + U - 1) / U;
  const int64_t blocks = std::max<int64_t>(1, (tasks + 8 * G - 1) / (8 * G));
  TmpBuf out, sum;
  SW_TRY(out.alloc(sizeof(float4) * (size_t)blocks * 256, st));
  SW_TRY(sum.alloc(sizeof(double), st));
  auto run = [&](int fold) {
    switch (SG) {
      case 8: launch_gather<8>(p.colidx.as<int>(), p.nnz, B, ldb, U, fold, out.as<float4>(), blocks, st); break;
      case 16: launch_gather<16>(p.colidx.as<int>(), p.nnz, B, ldb, U, fold, out.as<float4>(), blocks, st); break;
      default: launch_gather<32>(p.colidx.as<int>(), p.nnz, B, ldb, U, fold, out.as<float4>(), blocks, st); break;
    }
  };
  cudaEvent_t e0, e1;
  SW_CHECK_CUDA(cudaEventCreate(&e0));
  SW_CHECK_CUDA(cudaEventCreate(&e1));
  double ms[2] = {0.0, 0.0};
  swift_status rc = SWIFT_OK;
  for (int fold = 0; fold < 2 && rc == SWIFT_OK; ++fold) {
    run(fold);
    run(fold);
    cudaEventRecord(e0, st);
    for (int r = 0; r < reps; ++r) run(fold);
    cudaEventRecord(e1, st);
    const cudaError_t ce = cudaEventSynchronize(e1);
    if (ce != cudaSuccess || cudaGetLastError() != cudaSuccess) {
      set_last_error("swift_gather_bound", cudaGetErrorString(ce));
      rc = SWIFT_ERR_CUDA;
      break;
    }
    float f = 0.f;
    cudaEventElapsedTime(&f, e0, e1);
    ms[fold] = f / reps;
    if (fold == 0 && checksum) {  // sum of every gathered element of the unfolded stream
      cudaMemsetAsync(sum.p, 0, sizeof(double), st);
      gather_checksum_kernel<<<(unsigned)std::min<int64_t>(blocks * 2, (int64_t)p.sm_count * 8), 256, 0, st>>>(
          out.as<float4>(), blocks * 256, sum.as<double>());
      cudaMemcpyAsync(checksum, sum.p, sizeof(double), cudaMemcpyDeviceToHost, st);
      cudaStreamSynchronize(st);
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (rc != SWIFT_OK) return rc;
  if (ms_stream) *ms_stream = ms[0];
  if (ms_l1) *ms_l1 = ms[1];
  return SWIFT_OK;
}
