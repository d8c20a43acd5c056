// lbm_batch_f32.cu — the batched kernels for float storage (see
// lbm_batch_kernel.cuh).
#include "lbm_batch_kernel.cuh"

namespace lbm {
namespace batch {
extern const BatchKernels kBatch_f32 = make_batch_kernels<float>();
}  // namespace batch
}  // namespace lbm
