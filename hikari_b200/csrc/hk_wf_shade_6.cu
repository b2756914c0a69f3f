// Wavefront shade kernels: queues 12 (bumpMap / normalMap over diffuse), 13 (over roughConductor).
#include "hk_wf_kernels.cuh"

namespace hk {
template cudaError_t wf_launch_shade_t<12>(const DevScene &, const WfState &, const WfLaunchConfig &, int, cudaStream_t);
template int wf_shade_occupancy_t<12>(int, bool);
template cudaError_t wf_launch_shade_t<13>(const DevScene &, const WfState &, const WfLaunchConfig &, int, cudaStream_t);
template int wf_shade_occupancy_t<13>(int, bool);
}  // namespace hk
