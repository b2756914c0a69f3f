// Wavefront shade kernels: queue 6 (run-time dispatch (smooth, twoSided, textured)).
#include "hk_wf_kernels.cuh"

namespace hk {
template cudaError_t wf_launch_shade_t<6>(const DevScene &, const WfState &, const WfLaunchConfig &, int, cudaStream_t);
template int wf_shade_occupancy_t<6>(int, bool);
}  // namespace hk
