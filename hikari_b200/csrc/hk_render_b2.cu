// Megakernel instantiation: binary tree, texture lookups compiled out.
#include "hk_megakernel.cuh"

namespace hk {
template cudaError_t launch_render_t<kAccelBvh2, false>(const DevScene &, const RenderLaunch &, int, cudaStream_t);
template int render_occupancy_t<kAccelBvh2, false>(int, int);
}  // namespace hk
