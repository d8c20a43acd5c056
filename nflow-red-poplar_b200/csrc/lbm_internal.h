// lbm_internal.h — declarations shared by the host-side translation units.
#pragma once
struct lbm_batch;
namespace lbm {
// Record a formatted message for lbm_last_error() and return `code`.
int set_error(int code, const char* fmt, ...);
void clear_error();
// the batch's CUDA stream (a cudaStream_t) and device ordinal
void* batch_stream(lbm_batch* b);
int batch_device(lbm_batch* b);
}  // namespace lbm
