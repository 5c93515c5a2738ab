// bfloat16 deviation storage (float collision) instantiations.
#define LBX_KERNEL_TU
#include "lbx_kernels.cuh"

namespace lbx {
LBX_INSTANTIATE(9, __nv_bfloat16)
LBX_INSTANTIATE(19, __nv_bfloat16)
LBX_INSTANTIATE(27, __nv_bfloat16)
}  // namespace lbx
