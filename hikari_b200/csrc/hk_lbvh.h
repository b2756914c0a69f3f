// Tree build on the device (hk_lbvh.cu): the compressed 8-wide tree of
// hk_bvh.h (the same node format the host build writes) over a Morton-ordered
// linear BVH, built in milliseconds.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>

#include "hk_hostutil.h"

namespace hk {

struct GpuBvh8 {
    DevBuf nodes;          // 20 words per 8-wide node
    DevBuf order;          // leaf order -> original triangle index (n words)
    uint32_t nnodes = 0;
    uint32_t depth = 0;    // levels of 8-wide nodes
};

// tris_dev: 9 floats per triangle (v0, v1, v2) in device memory.  Synchronises
// `st` once per tree level.
void build_bvh8_gpu(const float *tris_dev, uint32_t n, cudaStream_t st, GpuBvh8 &out);
// The 48-byte triangle records of the traversal (v0.xyz + original index,
// v1.xyz + mesh id, v2.xyz) in leaf order, gathered on the device.
void gather_tri_records(const float *tris_dev, const int32_t *tmesh_dev, const uint32_t *order_dev, uint32_t n,
                        float *recs_dev, cudaStream_t st);

}  // namespace hk
