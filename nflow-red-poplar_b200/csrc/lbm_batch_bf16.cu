// lbm_batch_bf16.cu — the batched kernels for __nv_bfloat16 storage (see
// lbm_batch_kernel.cuh).
#include "lbm_batch_kernel.cuh"

namespace lbm {
namespace batch {
extern const BatchKernels kBatch_bf16 = make_batch_kernels<__nv_bfloat16>();
}  // namespace batch
}  // namespace lbm
