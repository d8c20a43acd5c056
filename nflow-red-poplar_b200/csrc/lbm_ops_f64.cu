// lbm_ops_f64.cu — the single-domain kernels for double storage (see
// lbm_ops_impl.cuh).
#include "lbm_ops_impl.cuh"

namespace lbm {
extern const StorageOps kOps_f64 = make_ops<double>();
}  // namespace lbm
