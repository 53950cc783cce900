// spmm_batch.cu -- many independent products C_i = A_i * B_i in one persistent launch.
//
// Each member keeps its own merge-path task layout over its plan's CSR (so a batch never
// shares task arrays, split counters or scratch with the plan's own products); the launch
// records of all members live in one device table that the persistent kernel reads, so
// setting new operands only rewrites the table and a captured CUDA graph stays valid.
#include <algorithm>
#include <memory>
#include <vector>

#include "common.cuh"

struct swift_batch {
  struct Operands {
    std::vector<int> N;
    std::vector<const void *> B;
    std::vector<int64_t> ldb;
    std::vector<void *> C;
    std::vector<int64_t> ldc;
  };
  int device = 0;
  int count = 0;
  // merge-path task size per member class: N <= 32, N <= 64, wider (each class has its own
  // best grain: narrow rows favour small tasks, wide rows large ones)
  int U[3] = {512, 512, 512};
  // N-split per member class: 1 walks a member's N columns at once, 2 walks them as two column
  // halves, each its own table entry (own tasks, split-row scratch and counters), so that each
  // gathered B row is half as wide and the walk over A runs twice.  Members whose half-width is
  // not a multiple of 4 columns stay whole.
  int nsplit[3] = {1, 1, 1};
  int entries = 0;        // table entries (members, or member halves) of the current table
  int graph_entries = -1;  // entries the captured graph was made for
  int grid = 0;
  std::vector<swift_plan *> plans;
  // the order the persistent grid walks the members in: flattest column distribution first
  // (share of nonzeros in the top 1 % of columns, ascending; stable).  Members with a flat
  // distribution gather across their whole B; walking them before the skewed ones measured
  // fastest (batch512: 8.48 ms against 9.7-10.2 ms for shuffled or skewed-first orders).
  std::vector<int> order;
  // layouts[2i + h]: member i's tasks and scratch for column half h (h = 0 also for a whole
  // member).  A layout always serves the same member, so its cached tasks stay valid whatever the
  // N-split (which renumbers the table entries).
  std::vector<std::unique_ptr<swift::RowLayout>> layouts;
  std::vector<unsigned char> h_args;
  std::vector<int> h_shape;
  std::vector<int64_t> h_off;
  swift::DevBuf d_args, d_shape, d_off;
  Operands ops;
  bool ready = false;
  cudaStream_t cap = nullptr;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  // Streams the batch launched on, each with an event recorded after its latest launch, so that
  // destroying the batch waits for its own launches only.  A launch made while the caller's
  // stream is being captured (or beyond kMaxUses streams) can run later on any stream: then
  // destruction waits for the whole device.
  static constexpr int kMaxUses = 16;
  std::vector<std::pair<cudaStream_t, cudaEvent_t>> uses;
  bool sync_device_on_destroy = false;
  ~swift_batch() {
    // swift_batch_destroy has ordered the buffers' release after the batch's own launches
    for (auto &u : uses) cudaEventDestroy(u.second);
    if (exec) cudaGraphExecDestroy(exec);
    if (graph) cudaGraphDestroy(graph);
    if (cap) cudaStreamDestroy(cap);
  }
};

using namespace swift;

namespace {

cudaStream_t to_stream(swift_stream_t s) { return reinterpret_cast<cudaStream_t>(s); }

int member_class(int N) { return N <= 32 ? 0 : (N <= 64 ? 1 : 2); }

swift_status on_device(const swift_batch *b) {
  int dev = -1;
  SW_CHECK_CUDA(cudaGetDevice(&dev));
  if (dev != b->device) {
    set_last_error("swift_batch", "the current device is not the batch's device");
    return SWIFT_ERR_INVALID_ARG;
  }
  return SWIFT_OK;
}

// Column halves member i is walked in under the current N-split (1 or 2).
int member_split(const swift_batch *b, int i) {
  const int N = b->ops.N[i], s = b->nsplit[member_class(N)];
  return (s == 2 && N > 0 && N % 8 == 0) ? 2 : 1;
}

// (Re)builds every member's launch records from the stored operands and uploads the table:
// entries in member order, the halves of a split member side by side.
swift_status build_table(swift_batch *b, cudaStream_t st) {
  const size_t asz = merge_args_size();
  int64_t off = 0;
  int v = 0;
  for (int k = 0; k < b->count; ++k) {
    const int i = b->order[k];
    const int s = member_split(b, i), Nh = b->ops.N[i] / s;
    for (int h = 0; h < s; ++h, ++v) {
      std::unique_ptr<RowLayout> &L = b->layouts[2 * (size_t)i + h];
      if (!L) L.reset(new RowLayout());
      b->h_off[v] = off;
      int64_t items = 0;
      const void *B = b->ops.B[i] ? static_cast<const float *>(b->ops.B[i]) + (size_t)h * Nh : nullptr;
      void *C = b->ops.C[i] ? static_cast<float *>(b->ops.C[i]) + (size_t)h * Nh : nullptr;
      SW_TRY(merge_batch_member(b->plans[i]->p, *L, b->U[member_class(b->ops.N[i])], Nh, B,
                                b->ops.ldb[i], C, b->ops.ldc[i], b->h_args.data() + asz * v, &b->h_shape[v],
                                &items, st));
      off += items;
    }
  }
  b->entries = v;
  b->h_off[v] = off;
  if (v > 0) {
    SW_CHECK_CUDA(cudaMemcpyAsync(b->d_args.p, b->h_args.data(), asz * v, cudaMemcpyHostToDevice, st));
    SW_CHECK_CUDA(cudaMemcpyAsync(b->d_shape.p, b->h_shape.data(), sizeof(int) * v, cudaMemcpyHostToDevice, st));
  }
  SW_CHECK_CUDA(cudaMemcpyAsync(b->d_off.p, b->h_off.data(), sizeof(int64_t) * (v + 1), cudaMemcpyHostToDevice, st));
  SW_CHECK_CUDA(cudaStreamSynchronize(st));  // the host table may change after return
  b->ready = true;
  return SWIFT_OK;
}

swift_status launch(swift_batch *b, cudaStream_t st) {
  return launch_merge_batch(b->d_args.p, b->d_shape.as<int>(), static_cast<const int64_t *>(b->d_off.p),
                            b->entries, b->grid, st);
}

// Records that the batch's work was enqueued on `st` (after the enqueue).
void note_use(swift_batch *b, cudaStream_t st) {
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  if (cudaStreamIsCapturing(st, &cs) != cudaSuccess || cs != cudaStreamCaptureStatusNone) {
    b->sync_device_on_destroy = true;
    return;
  }
  for (auto &u : b->uses)
    if (u.first == st) {
      cudaEventRecord(u.second, st);
      return;
    }
  cudaEvent_t ev = nullptr;
  if ((int)b->uses.size() >= swift_batch::kMaxUses ||
      cudaEventCreateWithFlags(&ev, cudaEventDisableTiming) != cudaSuccess) {
    b->sync_device_on_destroy = true;
    return;
  }
  cudaEventRecord(ev, st);
  b->uses.emplace_back(st, ev);
}

swift_status check_ready(const swift_batch *b, const char *where) {
  if (!b) return SWIFT_ERR_INVALID_ARG;
  if (!b->ready) {
    set_last_error(where, "operands not set");
    return SWIFT_ERR_INVALID_ARG;
  }
  return on_device(b);
}

}  // namespace

extern "C" {

swift_status swift_batch_create(swift_plan *const *plans, int count, swift_stream_t stream,
                                swift_batch **out) {
  (void)stream;
  if (!out || count < 0 || (count > 0 && !plans)) return SWIFT_ERR_INVALID_ARG;
  *out = nullptr;
  int dev = 0;
  SW_CHECK_CUDA(cudaGetDevice(&dev));
  for (int i = 0; i < count; ++i) {
    if (!plans[i]) return SWIFT_ERR_INVALID_ARG;
    const Plan &p = plans[i]->p;
    if (p.device != dev) {
      set_last_error("swift_batch_create", "plans of one batch must live on the current device");
      return SWIFT_ERR_INVALID_ARG;
    }
    if (p.val_type != SWIFT_F32 || !p.has_csr) {
      set_last_error("swift_batch_create", "batches take FP32 plans built from CSR");
      return SWIFT_ERR_UNSUPPORTED;
    }
  }
  std::unique_ptr<swift_batch> b(new (std::nothrow) swift_batch());
  if (!b) return SWIFT_ERR_ALLOC;
  b->device = dev;
  b->count = count;
  b->plans.assign(plans, plans + count);
  {
    std::vector<double> skew((size_t)count, 0.0);
    for (int i = 0; i < count; ++i) {
      const Plan &p = plans[i]->p;
      const int t = std::max(1, p.K / 100);
      if (p.K == 0 || p.nnz == 0) continue;
      std::vector<int> tail((size_t)t);
      SW_CHECK_CUDA(cudaMemcpy(tail.data(), p.sortnnz.as<int>() + (p.K - t), sizeof(int) * (size_t)t,
                               cudaMemcpyDeviceToHost));
      int64_t sum = 0;
      for (int c : tail) sum += c;
      skew[(size_t)i] = (double)sum / (double)p.nnz;
    }
    b->order.resize((size_t)count);
    for (int i = 0; i < count; ++i) b->order[(size_t)i] = i;
    std::stable_sort(b->order.begin(), b->order.end(), [&](int x, int y) { return skew[(size_t)x] < skew[(size_t)y]; });
  }
  const size_t cap = 2 * (size_t)std::max(count, 1);  // table entries: every member split in two at most
  b->layouts.resize(cap);
  b->h_args.assign(merge_args_size() * cap, 0);
  b->h_shape.assign(cap, 0);
  b->h_off.assign(cap + 1, 0);
  SW_TRY(b->d_args.alloc(b->h_args.size()));
  SW_TRY(b->d_shape.alloc(sizeof(int) * b->h_shape.size()));
  SW_TRY(b->d_off.alloc(sizeof(int64_t) * b->h_off.size()));
  SW_TRY(merge_batch_grid(dev, &b->grid));
  *out = b.release();
  return SWIFT_OK;
}

swift_status swift_batch_destroy(swift_batch *batch) {
  if (!batch) return SWIFT_ERR_INVALID_ARG;
  int prev = -1;
  cudaGetDevice(&prev);
  if (prev != batch->device) cudaSetDevice(batch->device);
  cudaStream_t fs = release_stream_after(batch->uses, batch->sync_device_on_destroy);
  if (prev >= 0 && prev != batch->device) cudaSetDevice(prev);
  // the members' layouts go back to the pool once the batch's own launches are done; the host
  // does not wait
  delete_releasing(batch, batch->device, fs);
  return SWIFT_OK;
}

swift_status swift_batch_set_operands(swift_batch *batch, const int *Ns, const void *const *B,
                                      const int64_t *ldb, void *const *C, const int64_t *ldc,
                                      swift_stream_t stream) {
  if (!batch) return SWIFT_ERR_INVALID_ARG;
  const int n = batch->count;
  if (n > 0 && (!Ns || !B || !ldb || !C || !ldc)) return SWIFT_ERR_INVALID_ARG;
  SW_TRY(on_device(batch));
  for (int i = 0; i < n; ++i) {
    const Plan &p = batch->plans[i]->p;
    if (Ns[i] < 0 || ldb[i] < Ns[i] || ldc[i] < Ns[i] || ldb[i] < 1 || ldc[i] < 1) return SWIFT_ERR_INVALID_ARG;
    if (Ns[i] > 0 && ((p.K > 0 && !B[i]) || (p.M > 0 && !C[i]))) return SWIFT_ERR_INVALID_ARG;
  }
  batch->ready = false;
  batch->ops.N.assign(Ns, Ns + n);
  batch->ops.B.assign(B, B + n);
  batch->ops.ldb.assign(ldb, ldb + n);
  batch->ops.C.assign(C, C + n);
  batch->ops.ldc.assign(ldc, ldc + n);
  return build_table(batch, to_stream(stream));
}

swift_status swift_batch_run(swift_batch *batch, swift_stream_t stream) {
  SW_TRY(check_ready(batch, "swift_batch_run"));
  const swift_status rc = launch(batch, to_stream(stream));
  note_use(batch, to_stream(stream));
  return rc;
}

swift_status swift_batch_run_graph(swift_batch *batch, swift_stream_t stream) {
  SW_TRY(check_ready(batch, "swift_batch_run_graph"));
  if (batch->exec && batch->graph_entries != batch->entries) {  // the table's entry count changed
    cudaGraphExecDestroy(batch->exec);
    cudaGraphDestroy(batch->graph);
    batch->exec = nullptr;
    batch->graph = nullptr;
  }
  if (!batch->exec) {
    // captured on a private stream (the legacy default stream cannot be captured)
    if (!batch->cap) SW_CHECK_CUDA(cudaStreamCreateWithFlags(&batch->cap, cudaStreamNonBlocking));
    SW_CHECK_CUDA(cudaStreamBeginCapture(batch->cap, cudaStreamCaptureModeThreadLocal));
    const swift_status rc = launch(batch, batch->cap);
    cudaGraph_t g = nullptr;
    const cudaError_t ce = cudaStreamEndCapture(batch->cap, &g);
    if (rc != SWIFT_OK) {
      if (g) cudaGraphDestroy(g);
      return rc;
    }
    SW_CHECK_CUDA(ce);
    batch->graph = g;
    SW_CHECK_CUDA(cudaGraphInstantiate(&batch->exec, batch->graph, 0));
    batch->graph_entries = batch->entries;
  }
  const cudaError_t le = cudaGraphLaunch(batch->exec, to_stream(stream));
  note_use(batch, to_stream(stream));
  SW_CHECK_CUDA(le);
  return SWIFT_OK;
}

swift_status swift_batch_autotune(swift_batch *batch, swift_stream_t stream, double *best_ms,
                                  int *best_task_size) {
  SW_TRY(check_ready(batch, "swift_batch_autotune"));
  cudaStream_t st = to_stream(stream);
  struct Noted {  // every exit path records the autotune launches
    swift_batch *b;
    cudaStream_t s;
    ~Noted() { note_use(b, s); }
  } noted{batch, st};
  cudaEvent_t e0, e1;
  SW_CHECK_CUDA(cudaEventCreate(&e0));
  SW_CHECK_CUDA(cudaEventCreate(&e1));
  // ms per launch with the task sizes in `U` (and the current N-split), or < 0 on failure
  auto time_sizes = [&](const int (&U)[3], swift_status &rc) -> double {
    for (int c = 0; c < 3; ++c) batch->U[c] = U[c];
    rc = build_table(batch, st);
    for (int w = 0; w < 2 && rc == SWIFT_OK; ++w) rc = launch(batch, st);
    if (rc != SWIFT_OK) return -1.0;
    const int reps = 5;
    cudaEventRecord(e0, st);
    for (int r = 0; r < reps && rc == SWIFT_OK; ++r) rc = launch(batch, st);
    cudaEventRecord(e1, st);
    if (rc != SWIFT_OK) return -1.0;
    cudaEventSynchronize(e1);
    float ms = 0;
    cudaEventElapsedTime(&ms, e0, e1);
    return ms / reps;
  };
  // coordinate descent: the best size for all classes, then each class on its own
  const int cands[] = {128, 256, 512, 1024};
  bool present[3] = {false, false, false};
  for (int i = 0; i < batch->count; ++i) present[member_class(batch->ops.N[i])] = true;
  double best = 1e300;
  int bestU[3] = {batch->U[0], batch->U[1], batch->U[2]};
  swift_status rc = SWIFT_OK;
  for (int u : cands) {
    const int U[3] = {u, u, u};
    const double ms = time_sizes(U, rc);
    if (rc != SWIFT_OK) break;
    if (ms < best) { best = ms; bestU[0] = bestU[1] = bestU[2] = u; }
  }
  for (int c = 0; c < 3 && rc == SWIFT_OK; ++c) {
    if (!present[c]) continue;
    const int keep = bestU[c];
    for (int u : cands) {
      if (u == keep) continue;
      int U[3] = {bestU[0], bestU[1], bestU[2]};
      U[c] = u;
      const double ms = time_sizes(U, rc);
      if (rc != SWIFT_OK) break;
      if (ms < best) { best = ms; bestU[c] = u; }
    }
  }
  // then the N-split of each class present with members that can be halved
  bool splittable[3] = {false, false, false};
  for (int i = 0; i < batch->count; ++i)
    if (batch->ops.N[i] > 0 && batch->ops.N[i] % 8 == 0) splittable[member_class(batch->ops.N[i])] = true;
  for (int c = 0; c < 3 && rc == SWIFT_OK; ++c) {
    if (!splittable[c]) continue;
    const int keep = batch->nsplit[c];
    batch->nsplit[c] = keep == 1 ? 2 : 1;
    const double ms = time_sizes(bestU, rc);
    if (rc != SWIFT_OK) break;
    if (ms < best) best = ms;
    else batch->nsplit[c] = keep;
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  for (int c = 0; c < 3; ++c) batch->U[c] = bestU[c];
  if (rc == SWIFT_OK) rc = build_table(batch, st);
  if (rc != SWIFT_OK) return rc;
  if (best_ms) *best_ms = best;
  if (best_task_size) *best_task_size = bestU[2];
  return SWIFT_OK;
}

swift_status swift_batch_get_task_sizes(const swift_batch *batch, int *sizes) {
  if (!batch || !sizes) return SWIFT_ERR_INVALID_ARG;
  for (int c = 0; c < 3; ++c) sizes[c] = batch->U[c];
  return SWIFT_OK;
}

swift_status swift_batch_set_n_split(swift_batch *batch, const int *splits, swift_stream_t stream) {
  if (!batch || !splits) return SWIFT_ERR_INVALID_ARG;
  for (int c = 0; c < 3; ++c)
    if (splits[c] != 1 && splits[c] != 2) return SWIFT_ERR_INVALID_ARG;
  SW_TRY(on_device(batch));
  for (int c = 0; c < 3; ++c) batch->nsplit[c] = splits[c];
  return batch->ready ? build_table(batch, to_stream(stream)) : SWIFT_OK;
}

swift_status swift_batch_get_n_split(const swift_batch *batch, int *splits) {
  if (!batch || !splits) return SWIFT_ERR_INVALID_ARG;
  for (int c = 0; c < 3; ++c) splits[c] = batch->nsplit[c];
  return SWIFT_OK;
}

}  // extern "C"
