// BSDF batch instantiations: RoughDielectric, Dielectric, RoughDiffuse.
#include "hk_batch.cuh"

namespace hk {
template cudaError_t launch_bsdf_batch_t<kRoughDielectric>(const DevScene &, int, uint64_t, const float *, const float *, const float *, const float *, const float *, const float *, float *, float *, float *, int32_t *, float *, float *, int, cudaStream_t);
template cudaError_t launch_bsdf_batch_t<kDielectric>(const DevScene &, int, uint64_t, const float *, const float *, const float *, const float *, const float *, const float *, float *, float *, float *, int32_t *, float *, float *, int, cudaStream_t);
template cudaError_t launch_bsdf_batch_t<kRoughDiffuse>(const DevScene &, int, uint64_t, const float *, const float *, const float *, const float *, const float *, const float *, float *, float *, float *, int32_t *, float *, float *, int, cudaStream_t);
}  // namespace hk
