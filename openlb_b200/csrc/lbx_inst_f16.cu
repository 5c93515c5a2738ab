// binary16 deviation storage (float collision) instantiations.
#define LBX_KERNEL_TU
#include "lbx_kernels.cuh"

namespace lbx {
LBX_INSTANTIATE(9, __half)
LBX_INSTANTIATE(19, __half)
LBX_INSTANTIATE(27, __half)
}  // namespace lbx
