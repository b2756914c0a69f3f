// Wavefront traversal kernels (extend, shadow) for the 8-wide tree.
#include "hk_wf_kernels.cuh"

namespace hk {
template cudaError_t wf_launch_extend_t<kAccelBvh8>(const DevScene &, const WfState &, const WfLaunchConfig &, int, cudaStream_t);
template cudaError_t wf_launch_shadow_t<kAccelBvh8>(const DevScene &, const WfState &, const WfLaunchConfig &, cudaStream_t);
template int wf_trace_occupancy_t<kAccelBvh8>(int, int, bool, bool);
}  // namespace hk
