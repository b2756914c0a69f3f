// BSDF batch instantiations: RoughCoating.
#include "hk_batch.cuh"

namespace hk {
template cudaError_t launch_bsdf_batch_t<kRoughCoating>(const DevScene &, int, uint64_t, const float *, const float *, const float *, const float *, const float *, const float *, float *, float *, float *, int32_t *, float *, float *, int, cudaStream_t);
}  // namespace hk
