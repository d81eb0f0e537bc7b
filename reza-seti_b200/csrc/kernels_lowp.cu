// FP32 / FP16 / BF16 storage instantiations (FP32 arithmetic on f - w).
#include "launch_impl.cuh"

namespace lbm {

LBM_INSTANTIATE(float, 19)
LBM_INSTANTIATE(float, 27)
LBM_INSTANTIATE(__half, 19)
LBM_INSTANTIATE(__half, 27)
LBM_INSTANTIATE(__nv_bfloat16, 19)
LBM_INSTANTIATE(__nv_bfloat16, 27)

}  // namespace lbm
