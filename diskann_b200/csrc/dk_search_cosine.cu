// Kernel instantiations for one metric (DK_METRIC_COSINE), all scoring modes; see dk_kernels.cuh.
#include "dk_kernels.cuh"

cudaError_t dk_launch_cosine(dk::LaunchPlan& L, int mode, cudaStream_t stream) {
  return dk::launch_modes<DK_METRIC_COSINE>(L, mode, stream);
}
