// FP32 kernel instantiations.
#define LBX_KERNEL_TU
#include "lbx_kernels.cuh"

namespace lbx {
LBX_INSTANTIATE(9, float)
LBX_INSTANTIATE(19, float)
LBX_INSTANTIATE(27, float)
}  // namespace lbx
