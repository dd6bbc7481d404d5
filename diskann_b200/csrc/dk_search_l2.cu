// Kernel instantiations for one metric (DK_METRIC_L2), all scoring modes; see dk_kernels.cuh.
#include "dk_kernels.cuh"

cudaError_t dk_launch_l2(dk::LaunchPlan& L, int mode, cudaStream_t stream) {
  return dk::launch_modes<DK_METRIC_L2>(L, mode, stream);
}
