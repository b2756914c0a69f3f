// Wavefront shade kernels: queues 0 (miss), 1 (diffuse), 2 (roughConductor).
#include "hk_wf_kernels.cuh"

namespace hk {
template cudaError_t wf_launch_shade_t<0>(const DevScene &, const WfState &, const WfLaunchConfig &, int, cudaStream_t);
template int wf_shade_occupancy_t<0>(int, bool);
template cudaError_t wf_launch_shade_t<1>(const DevScene &, const WfState &, const WfLaunchConfig &, int, cudaStream_t);
template int wf_shade_occupancy_t<1>(int, bool);
template cudaError_t wf_launch_shade_t<2>(const DevScene &, const WfState &, const WfLaunchConfig &, int, cudaStream_t);
template int wf_shade_occupancy_t<2>(int, bool);
}  // namespace hk
