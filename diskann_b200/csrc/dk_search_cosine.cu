// Kernel instantiations for one metric (DK_METRIC_COSINE); see dk_kernels.cuh.
#include "dk_kernels.cuh"

cudaError_t dk_launch_cosine(dk::LaunchPlan& L, bool pq, cudaStream_t stream) {
  (void)pq;
  return dk::launch_dims<DK_METRIC_COSINE, false>(L, stream);
}
