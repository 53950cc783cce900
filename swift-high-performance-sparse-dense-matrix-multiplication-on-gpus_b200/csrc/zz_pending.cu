// temporary: entry points not yet implemented
#include "common.cuh"
extern "C" {
swift_status swift_batch_create(swift_plan *const *, int, swift_stream_t, swift_batch **) { return SWIFT_ERR_UNSUPPORTED; }
swift_status swift_batch_destroy(swift_batch *) { return SWIFT_ERR_UNSUPPORTED; }
swift_status swift_batch_set_operands(swift_batch *, const int *, const void *const *, const int64_t *, void *const *, const int64_t *, swift_stream_t) { return SWIFT_ERR_UNSUPPORTED; }
swift_status swift_batch_run(swift_batch *, swift_stream_t) { return SWIFT_ERR_UNSUPPORTED; }
swift_status swift_batch_run_graph(swift_batch *, swift_stream_t) { return SWIFT_ERR_UNSUPPORTED; }
}
