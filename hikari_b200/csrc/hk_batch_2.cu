// BSDF batch instantiations: RoughPlastic, Plastic, Coating.
#include "hk_batch.cuh"

namespace hk {
template cudaError_t launch_bsdf_batch_t<kRoughPlastic>(const DevScene &, int, uint64_t, const float *, const float *, const float *, const float *, const float *, const float *, float *, float *, float *, int32_t *, float *, float *, int, cudaStream_t);
template cudaError_t launch_bsdf_batch_t<kPlastic>(const DevScene &, int, uint64_t, const float *, const float *, const float *, const float *, const float *, const float *, float *, float *, float *, int32_t *, float *, float *, int, cudaStream_t);
template cudaError_t launch_bsdf_batch_t<kCoating>(const DevScene &, int, uint64_t, const float *, const float *, const float *, const float *, const float *, const float *, float *, float *, float *, int32_t *, float *, float *, int, cudaStream_t);
}  // namespace hk
