// BSDF batch instantiations: TwoSided, and the run-time dispatch (-1) for
// layers nested deeper than one level.
#include "hk_batch.cuh"

namespace hk {
template cudaError_t launch_bsdf_batch_t<kTwoSided>(const DevScene &, int, uint64_t, const float *, const float *, const float *, const float *, const float *, const float *, float *, float *, float *, int32_t *, float *, float *, int, cudaStream_t);
template cudaError_t launch_bsdf_batch_t<-1>(const DevScene &, int, uint64_t, const float *, const float *, const float *, const float *, const float *, const float *, float *, float *, float *, int32_t *, float *, float *, int, cudaStream_t);
}  // namespace hk
