// spmm_noalloc.cu -- the product entry point that allocates nothing (swift_spmm_noalloc).
//
// Some callers cannot call cudaMalloc once they are running: real-time or certified
// deployments that forbid device allocation after start-up, and hosts whose device memory is
// owned by another allocator (a framework's caching allocator or a fixed arena), where a
// stray cudaMalloc may fail or fragment that memory and synchronises the whole device.  The
// regular row engine grows its scratch with cudaMalloc when a product needs more of it; this
// entry point runs the same row kernel with its scratch in a fixed device array instead.
#include <cuda.h>

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
// Per device: the array's address and the id of the CUDA context it was looked up in.  A
// cudaDeviceReset (or any destruction of the primary context) unloads this module; the next
// call then runs in a new context whose id differs, so the address is looked up again
// instead of reusing one that points into the dead context.
struct ScratchAddr {
  unsigned long long ctx_id = 0;
  void *ptr = nullptr;
};
ScratchAddr g_addr[kMaxDevices];

}  // namespace

// cuCtxGetCurrent / cuCtxGetId through the runtime's driver entry points (no libcuda link).
typedef CUresult (*ctx_get_current_fn)(CUcontext *);
typedef CUresult (*ctx_get_id_fn)(CUcontext, unsigned long long *);

swift_status current_context_id(unsigned long long *id) {
  static ctx_get_current_fn get_current = nullptr;
  static ctx_get_id_fn get_id = nullptr;
  if (!get_current || !get_id) {
    cudaDriverEntryPointQueryResult q1 = cudaDriverEntryPointSymbolNotFound, q2 = q1;
    void *f1 = nullptr, *f2 = nullptr;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f1, cudaEnableDefault, &q1) != cudaSuccess ||
        cudaGetDriverEntryPoint("cuCtxGetId", &f2, cudaEnableDefault, &q2) != cudaSuccess ||
        q1 != cudaDriverEntryPointSuccess || q2 != cudaDriverEntryPointSuccess || !f1 || !f2) {
      set_last_error("cudaGetDriverEntryPoint", "cuCtxGetCurrent / cuCtxGetId not available");
      return SWIFT_ERR_CUDA;
    }
    get_current = reinterpret_cast<ctx_get_current_fn>(f1);
    get_id = reinterpret_cast<ctx_get_id_fn>(f2);
  }
  CUcontext ctx = nullptr;
  if (get_current(&ctx) != CUDA_SUCCESS || !ctx || get_id(ctx, id) != CUDA_SUCCESS) {
    set_last_error("cuCtxGetId", "no current CUDA context");
    return SWIFT_ERR_CUDA;
  }
  return SWIFT_OK;
}

namespace {

// Device address of the array on the current device, looked up once per device and context
// (host code cannot use the symbol itself: on the host it names a host-side stand-in).
swift_status scratch_address(void **out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) { set_last_error("cudaGetDevice", cudaGetErrorString(e)); return SWIFT_ERR_NO_DEVICE; }
  if (dev < 0 || dev >= kMaxDevices) return SWIFT_ERR_UNSUPPORTED;
  // makes the device's primary context current on this thread if no runtime call has yet
  // (since CUDA 12 cudaSetDevice initialises it; a no-op for the current device otherwise)
  e = cudaSetDevice(dev);
  if (e != cudaSuccess) { set_last_error("cudaSetDevice", cudaGetErrorString(e)); return SWIFT_ERR_CUDA; }
  unsigned long long id = 0;
  SW_TRY(current_context_id(&id));
  std::lock_guard<std::mutex> g(g_addr_mu);
  ScratchAddr &a = g_addr[dev];
  if (!a.ptr || a.ctx_id != id) {
    void *p = nullptr;
    e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p) {
      set_last_error("cudaGetSymbolAddress", cudaGetErrorString(e));
      return SWIFT_ERR_CUDA;
    }
    a.ptr = p;
    a.ctx_id = id;
  }
  *out = a.ptr;
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
  UseNote use_note{p, st};
  // the counters must start at zero; the array keeps whatever the last call left
  if (L.long_rows > 0) SW_CHECK_CUDA(cudaMemsetAsync(base, 0, sizeof(int) * (size_t)L.long_rows, st));
  DenseArgs d;
  d.N = N; d.dtype = dtype; d.B = B; d.ldb = ldb; d.C = C; d.ldc = ldc;
  return run_rowwise_external(p, L, d, static_cast<unsigned char *>(base) + kCounterBytes,
                              static_cast<int *>(base), st);
}
