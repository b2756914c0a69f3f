// Wavefront shade kernels: queues 3 (roughDielectric), 4 (roughPlastic).
#include "hk_wf_kernels.cuh"

namespace hk {
template cudaError_t wf_launch_shade_t<3>(const DevScene &, const WfState &, const WfLaunchConfig &, int, cudaStream_t);
template int wf_shade_occupancy_t<3>(int, bool);
template cudaError_t wf_launch_shade_t<4>(const DevScene &, const WfState &, const WfLaunchConfig &, int, cudaStream_t);
template int wf_shade_occupancy_t<4>(int, bool);
}  // namespace hk
