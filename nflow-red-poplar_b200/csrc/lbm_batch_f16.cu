// lbm_batch_f16.cu — the batched kernels for __half storage (see
// lbm_batch_kernel.cuh).
#include "lbm_batch_kernel.cuh"

namespace lbm {
namespace batch {
extern const BatchKernels kBatch_f16 = make_batch_kernels<__half>();
}  // namespace batch
}  // namespace lbm
