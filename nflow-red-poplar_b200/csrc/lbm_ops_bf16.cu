// lbm_ops_bf16.cu — the single-domain kernels for __nv_bfloat16 storage (see
// lbm_ops_impl.cuh).
#include "lbm_ops_impl.cuh"

namespace lbm {
extern const StorageOps kOps_bf16 = make_ops<__nv_bfloat16>();
}  // namespace lbm
