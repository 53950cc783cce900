// spmm_noalloc.cu -- the product entry point that allocates nothing (swift_spmm_noalloc).
//
// Some callers cannot call cudaMalloc once they are running: real-time or certified
// deployments that forbid device allocation after start-up, and hosts whose device memory is
// owned by another allocator (a framework's caching allocator or a fixed arena), where a
// stray cudaMalloc may fail or fragment that memory and synchronises the whole device.  The
// regular row engine grows its scratch with cudaMalloc when a product needs more of it; this
// entry point runs the same row kernel with its scratch in a fixed device array instead.
#include "common.cuh"

namespace swift {
namespace {

constexpr size_t kNoAllocBytes = SWIFT_NOALLOC_SCRATCH_BYTES;
constexpr int kNoAllocCounters = SWIFT_NOALLOC_MAX_LONG_ROWS;
constexpr size_t kCounterBytes = sizeof(int) * (size_t)kNoAllocCounters;

// Layout: [kNoAllocCounters arrival counters][partial rows of the long-row pieces].  Every GPU
// that loads the library holds this array until the process exits.
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocBytes];

constexpr int kMaxDevices = 64;
std::mutex g_addr_mu;
void *g_addr[kMaxDevices] = {};

// Device address of the array on the current device, looked up once per device (host code
// cannot use the symbol itself: on the host it names a host-side stand-in).
swift_status scratch_address(void **out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) { set_last_error("cudaGetDevice", cudaGetErrorString(e)); return SWIFT_ERR_NO_DEVICE; }
  if (dev < 0 || dev >= kMaxDevices) return SWIFT_ERR_UNSUPPORTED;
  std::lock_guard<std::mutex> g(g_addr_mu);
  if (!g_addr[dev]) {
    void *p = nullptr;
    e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p) {
      set_last_error("cudaGetSymbolAddress", cudaGetErrorString(e));
      return SWIFT_ERR_CUDA;
    }
    g_addr[dev] = p;
  }
  *out = g_addr[dev];
  return SWIFT_OK;
}

}  // namespace
}  // namespace swift

using namespace swift;

extern "C" swift_status swift_spmm_noalloc(const swift_plan *plan, int N, swift_dtype dtype,
                                           const void *B, int64_t ldb, void *C, int64_t ldc,
                                           swift_stream_t stream) {
  if (!plan || N < 0) return SWIFT_ERR_INVALID_ARG;
  Plan &p = const_cast<Plan &>(plan->p);
  if (!p.has_csr || !p.fwd.built) return SWIFT_ERR_UNSUPPORTED;
  if (dtype != SWIFT_F32 && dtype != SWIFT_F64 && dtype != SWIFT_BF16 && dtype != SWIFT_F16)
    return SWIFT_ERR_INVALID_ARG;
  if ((p.val_type == SWIFT_F64) != (dtype == SWIFT_F64)) return SWIFT_ERR_UNSUPPORTED;
  if (N == 0 || p.M == 0) return SWIFT_OK;
  if (!B || !C || ldb < N || ldc < N) return SWIFT_ERR_INVALID_ARG;
  RowLayout &L = p.fwd;
  const size_t acc = p.val_type == SWIFT_F64 ? 8 : 4;
  const size_t need = (size_t)L.pieces * (size_t)N * acc;
  if (L.long_rows > kNoAllocCounters || need > kNoAllocBytes - kCounterBytes) {
    char msg[256];
    snprintf(msg, sizeof(msg),
             "needs %d long-row counters (max %d) and %zu bytes of partial rows (max %zu); "
             "create the plan with a larger long_row_split or use swift_spmm",
             L.long_rows, kNoAllocCounters, need, kNoAllocBytes - kCounterBytes);
    set_last_error("swift_spmm_noalloc", msg);
    return SWIFT_ERR_OVERFLOW;
  }
  void *base = nullptr;
  SW_TRY(scratch_address(&base));
  cudaStream_t st = S(stream);
  // the counters must start at zero; the array keeps whatever the last call left
  if (L.long_rows > 0) SW_CHECK_CUDA(cudaMemsetAsync(base, 0, sizeof(int) * (size_t)L.long_rows, st));
  DenseArgs d;
  d.N = N; d.dtype = dtype; d.B = B; d.ldb = ldb; d.C = C; d.ldc = ldc;
  return run_rowwise_external(p, L, d, static_cast<unsigned char *>(base) + kCounterBytes,
                              static_cast<int *>(base), st);
}
