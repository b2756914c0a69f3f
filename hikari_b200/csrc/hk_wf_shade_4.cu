// Wavefront shade kernels: queues 7 (textured diffuse), 8 (textured roughConductor), 9 (textured roughDielectric).
#include "hk_wf_kernels.cuh"

namespace hk {
template cudaError_t wf_launch_shade_t<7>(const DevScene &, const WfState &, const WfLaunchConfig &, int, cudaStream_t);
template int wf_shade_occupancy_t<7>(int, bool);
template cudaError_t wf_launch_shade_t<8>(const DevScene &, const WfState &, const WfLaunchConfig &, int, cudaStream_t);
template int wf_shade_occupancy_t<8>(int, bool);
template cudaError_t wf_launch_shade_t<9>(const DevScene &, const WfState &, const WfLaunchConfig &, int, cudaStream_t);
template int wf_shade_occupancy_t<9>(int, bool);
}  // namespace hk
