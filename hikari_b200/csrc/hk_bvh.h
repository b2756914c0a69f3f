// Host BVH builder: binned-SAH binary BVH over pre-gathered triangles, packed
// into the 64-byte two-child node layout traversed by hk_traverse.cuh.
#pragma once
#include <cstdint>
#include <vector>

namespace hk {

struct Bvh2 {
    std::vector<float> nodes;         // 16 floats per packed node
    std::vector<uint32_t> tri_order;  // leaf order -> original triangle index
    uint32_t depth = 0;
};

// tris: 9 floats per triangle (v0, v1, v2).  Leaves hold at most max_leaf
// triangles; the tree depth is capped below the traversal stack size.
Bvh2 build_bvh2(const float *tris, uint32_t ntris, int max_leaf = 4);

}  // namespace hk
