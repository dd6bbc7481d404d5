// Kernel instantiations for one metric (DK_METRIC_COSINE_NORMALIZED); see dk_kernels.cuh.
#include "dk_kernels.cuh"

cudaError_t dk_launch_cosine_normalized(dk::LaunchPlan& L, bool pq, cudaStream_t stream) {
  return pq ? dk::launch_dims<DK_METRIC_COSINE_NORMALIZED, true>(L, stream) : dk::launch_dims<DK_METRIC_COSINE_NORMALIZED, false>(L, stream);
}
