// FP64 kernel instantiations (the unit is built like every other without FMA contraction, so
// the operation sequence of lbx_collision.cuh rounds exactly like the reference's CPU build).
#define LBX_KERNEL_TU
#include "lbx_kernels.cuh"

namespace lbx {
LBX_INSTANTIATE(9, double)
LBX_INSTANTIATE(19, double)
LBX_INSTANTIATE(27, double)
}  // namespace lbx
