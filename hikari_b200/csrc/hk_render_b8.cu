// Megakernel instantiation: 8-wide tree, texture lookups compiled out.
#include "hk_megakernel.cuh"

namespace hk {
template cudaError_t launch_render_t<kAccelBvh8, false>(const DevScene &, const RenderLaunch &, int, cudaStream_t);
template int render_occupancy_t<kAccelBvh8, false>(int, int);
}  // namespace hk
