// Wavefront shade kernels: queues 14 (bumpMap / normalMap over roughDielectric), 15 (over roughPlastic), 16 (over roughCoating).
#include "hk_wf_kernels.cuh"

namespace hk {
template cudaError_t wf_launch_shade_t<14>(const DevScene &, const WfState &, const WfLaunchConfig &, int, cudaStream_t);
template int wf_shade_occupancy_t<14>(int, bool);
template cudaError_t wf_launch_shade_t<15>(const DevScene &, const WfState &, const WfLaunchConfig &, int, cudaStream_t);
template int wf_shade_occupancy_t<15>(int, bool);
template cudaError_t wf_launch_shade_t<16>(const DevScene &, const WfState &, const WfLaunchConfig &, int, cudaStream_t);
template int wf_shade_occupancy_t<16>(int, bool);
}  // namespace hk
