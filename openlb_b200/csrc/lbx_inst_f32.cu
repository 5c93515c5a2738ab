// FP32 kernel instantiations.
#define LBX_KERNEL_TU
#include "lbx_kernels.cuh"

namespace lbx {
#define LBX_INSTANTIATE(Q, S)                                                                          \
  template cudaError_t launch_step<Q, S>(const LaunchArgs&, cudaStream_t);                            \
  template cudaError_t launch_bouzidi<Q, S>(const LaunchArgs&, const uint32_t*, const uint8_t*,       \
                                            const void*, int64_t, cudaStream_t);                      \
  template cudaError_t launch_transfer<Q, S>(const LaunchArgs&, int, const void*, int, bool, cudaStream_t); \
  template cudaError_t launch_ini_equilibrium<Q, S>(const LaunchArgs&, const double*, const double*, cudaStream_t); \
  template cudaError_t launch_moments<Q, S>(const LaunchArgs&, double*, double*, cudaStream_t);       \
  template cudaError_t launch_mass_momentum<Q, S>(const LaunchArgs&, double*, cudaStream_t);          \
  template cudaError_t launch_link_force<Q, S>(const LaunchArgs&, const uint32_t*, const uint8_t*,    \
                                               int64_t, double*, cudaStream_t);                       \
  template cudaError_t launch_residual<Q, S>(const LaunchArgs&, float*, double*, unsigned long long*, cudaStream_t);

LBX_INSTANTIATE(9, float)
LBX_INSTANTIATE(19, float)
LBX_INSTANTIATE(27, float)
}  // namespace lbx
