// lbm_ops_f16.cu — the single-domain kernels for __half storage (see
// lbm_ops_impl.cuh).
#include "lbm_ops_impl.cuh"

namespace lbm {
extern const StorageOps kOps_f16 = make_ops<__half>();
}  // namespace lbm
