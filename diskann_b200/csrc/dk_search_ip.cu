// Kernel instantiations for one metric (DK_METRIC_INNER_PRODUCT); see dk_kernels.cuh.
#include "dk_kernels.cuh"

cudaError_t dk_launch_ip(dk::LaunchPlan& L, bool pq, cudaStream_t stream) {
  return pq ? dk::launch_dims<DK_METRIC_INNER_PRODUCT, true>(L, stream) : dk::launch_dims<DK_METRIC_INNER_PRODUCT, false>(L, stream);
}
