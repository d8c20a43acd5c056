// lbm_ops_f32.cu — the single-domain kernels for float storage (see
// lbm_ops_impl.cuh).
#include "lbm_ops_impl.cuh"

namespace lbm {
extern const StorageOps kOps_f32 = make_ops<float>();
}  // namespace lbm
