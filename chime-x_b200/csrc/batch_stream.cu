// batch_stream.cu -- batched ragged launch and streaming loop (in progress).
#include "chimex_internal.h"

using namespace chx;

extern "C" {
int chx_batch_create(chx_batch **, int, const chx_channel_desc *, int, int) {
    return fail(CHX_E_UNSUPPORTED, "batched launch not built yet");
}
int chx_batch_run(chx_batch *, void *, int) { return fail(CHX_E_UNSUPPORTED, "not built"); }
int64_t chx_batch_work_units(const chx_batch *) { return -1; }
double chx_batch_ops(const chx_batch *) { return -1.0; }
int chx_batch_destroy(chx_batch *) { return CHX_OK; }
int chx_autotune(int, int, const uint8_t *, int32_t *, void *, int *, int *, double *) {
    return fail(CHX_E_UNSUPPORTED, "autotuner not built yet");
}
int chx_stream_create(chx_stream **, int, int, int, int64_t, int) {
    return fail(CHX_E_UNSUPPORTED, "streaming not built yet");
}
int chx_stream_admit(chx_stream *, int, int, int *) { return fail(CHX_E_UNSUPPORTED, "not built"); }
int chx_stream_submit(chx_stream *, int, const int *, const uint8_t *const *, const int64_t *,
                      void *) {
    return fail(CHX_E_UNSUPPORTED, "not built");
}
int chx_stream_last_dump(chx_stream *, int, const int32_t **, int64_t *) {
    return fail(CHX_E_UNSUPPORTED, "not built");
}
int chx_stream_stats_get(chx_stream *, chx_stream_stats *) {
    return fail(CHX_E_UNSUPPORTED, "not built");
}
int chx_stream_destroy(chx_stream *) { return CHX_OK; }
}
