// Kernel instantiations for one metric (DK_METRIC_L2); see dk_kernels.cuh.
#include "dk_kernels.cuh"

cudaError_t dk_launch_l2(dk::LaunchPlan& L, bool pq, cudaStream_t stream) {
  return pq ? dk::launch_dims<DK_METRIC_L2, true>(L, stream) : dk::launch_dims<DK_METRIC_L2, false>(L, stream);
}
