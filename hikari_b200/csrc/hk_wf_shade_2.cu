// Wavefront shade kernels: queue 5 (roughCoating).
#include "hk_wf_kernels.cuh"

namespace hk {
template cudaError_t wf_launch_shade_t<5>(const DevScene &, const WfState &, const WfLaunchConfig &, int, cudaStream_t);
template int wf_shade_occupancy_t<5>(int, bool);
}  // namespace hk
