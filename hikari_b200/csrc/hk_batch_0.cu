// BSDF batch instantiations: Diffuse, RoughConductor, Mirror, Conductor.
#include "hk_batch.cuh"

namespace hk {
template cudaError_t launch_bsdf_batch_t<kDiffuse>(const DevScene &, int, uint64_t, const float *, const float *, const float *, const float *, const float *, const float *, float *, float *, float *, int32_t *, float *, float *, int, cudaStream_t);
template cudaError_t launch_bsdf_batch_t<kRoughConductor>(const DevScene &, int, uint64_t, const float *, const float *, const float *, const float *, const float *, const float *, float *, float *, float *, int32_t *, float *, float *, int, cudaStream_t);
template cudaError_t launch_bsdf_batch_t<kMirror>(const DevScene &, int, uint64_t, const float *, const float *, const float *, const float *, const float *, const float *, float *, float *, float *, int32_t *, float *, float *, int, cudaStream_t);
template cudaError_t launch_bsdf_batch_t<kConductor>(const DevScene &, int, uint64_t, const float *, const float *, const float *, const float *, const float *, const float *, float *, float *, float *, int32_t *, float *, float *, int, cudaStream_t);
}  // namespace hk
