// Kernel instantiations for one metric (DK_METRIC_INNER_PRODUCT), all scoring modes; see dk_kernels.cuh.
#include "dk_kernels.cuh"

cudaError_t dk_launch_ip(dk::LaunchPlan& L, int mode, cudaStream_t stream) {
  return dk::launch_modes<DK_METRIC_INNER_PRODUCT>(L, mode, stream);
}
