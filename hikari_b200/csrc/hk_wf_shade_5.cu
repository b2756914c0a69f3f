// Wavefront shade kernels: queues 10 (textured roughPlastic), 11 (textured roughCoating).
#include "hk_wf_kernels.cuh"

namespace hk {
template cudaError_t wf_launch_shade_t<10>(const DevScene &, const WfState &, const WfLaunchConfig &, int, cudaStream_t);
template int wf_shade_occupancy_t<10>(int, bool);
template cudaError_t wf_launch_shade_t<11>(const DevScene &, const WfState &, const WfLaunchConfig &, int, cudaStream_t);
template int wf_shade_occupancy_t<11>(int, bool);
}  // namespace hk
