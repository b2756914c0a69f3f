// Wavefront traversal kernels (extend, shadow) for the binary tree.
#include "hk_wf_kernels.cuh"

namespace hk {
template cudaError_t wf_launch_extend_t<kAccelBvh2>(const DevScene &, const WfState &, const WfLaunchConfig &, int, cudaStream_t);
template cudaError_t wf_launch_shadow_t<kAccelBvh2>(const DevScene &, const WfState &, const WfLaunchConfig &, cudaStream_t);
template int wf_trace_occupancy_t<kAccelBvh2>(int, int, bool, bool);
}  // namespace hk
