// Host BVH builder: binned-SAH binary BVH over pre-gathered triangles, packed
// into the 64-byte two-child node layout traversed by hk_traverse.cuh.
#pragma once
#include <cstdint>
#include <string>
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

// Compressed 8-wide BVH (the node format of Ylitie, Karras and Laine,
// "Efficient Incoherent Ray Traversal on GPUs Through Compressed Wide BVHs",
// HPG 2017): 80 bytes = 20 words per node.
//   w0..2  origin p (float bits), w3 = e.x | e.y << 8 | e.z << 16 | imask << 24
//          (child boxes are p + q * 2^(e - 127) per axis, q in 0..255, padded
//          by one step on every side)
//   w4     index of the first internal child node (children are consecutive)
//   w5     index of the node's first triangle (leaf children's triangles are consecutive)
//   w6, w7 meta byte per child slot, bits << 5 | position: a hit sets `bits`
//          at `position` of the node's hit word -- leaf: count ones at its
//          first triangle's offset 0..21 from w5; internal: one bit at 24 +
//          slot (the traversal XORs the slot with the ray octant); 0 = empty
//   w8..19 q_lo.x[8], q_lo.y[8], q_lo.z[8], q_hi.x[8], q_hi.y[8], q_hi.z[8]
// A child in slot s lies on the negative side of axis k when bit k of s is
// set, so a ray visits children in the order s ^ (7 ^ octant) near first.
struct Bvh8 {
    std::vector<uint32_t> nodes;
    uint32_t depth = 0;
};

// One binned-SAH build with leaves of at most 3 triangles, collapsed into the
// 8-wide tree; both trees index one triangle order (tri_order of bvh2).
struct BvhPair {
    Bvh2 bvh2;
    Bvh8 bvh8;
};
BvhPair build_bvh_pair(const float *tris, uint32_t ntris);

// Structural check of a pair built from tris: every triangle is referenced by
// exactly one leaf of each tree, every quantised child box (decoded in double)
// contains its subtree's triangles, child indices are in range.  Returns an
// empty string when the trees are consistent, else the first problem found.
std::string check_bvh_pair(const BvhPair &P, const float *tris, uint32_t ntris);
// The 8-wide part of that check for nodes over the triangle order `order`.
std::string check_bvh8(const std::vector<uint32_t> &nodes, const std::vector<uint32_t> &order, const float *tris,
                       uint32_t ntris);

}  // namespace hk
