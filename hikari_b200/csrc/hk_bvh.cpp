// Binned-SAH BVH2 build (32 bins per axis on centroid bounds, SAH leaf
// termination), subtrees above 64k triangles built on worker threads.
#include "hk_bvh.h"

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstring>
#include <future>
#include <stdexcept>

#include "hk_device.h"

namespace hk {
namespace {

struct Box {
    float lo[3], hi[3];
    void empty() {
        for (int i = 0; i < 3; i++) { lo[i] = INFINITY; hi[i] = -INFINITY; }
    }
    void grow(const Box &b) {
        for (int i = 0; i < 3; i++) { lo[i] = std::min(lo[i], b.lo[i]); hi[i] = std::max(hi[i], b.hi[i]); }
    }
    void grow(const float *p) {
        for (int i = 0; i < 3; i++) { lo[i] = std::min(lo[i], p[i]); hi[i] = std::max(hi[i], p[i]); }
    }
    float area() const {
        float dx = hi[0] - lo[0], dy = hi[1] - lo[1], dz = hi[2] - lo[2];
        if (!(dx >= 0)) return 0.0f;
        return 2.0f * (dx * dy + dy * dz + dz * dx);
    }
};

struct BNode {
    Box box;
    int32_t left = -1, right = -1;   // children (internal)
    uint32_t start = 0, count = 0;   // leaf range
};

constexpr int kBins = 32;
constexpr int kMaxDepth = 60;         // traversal stack holds 64 entries
constexpr uint32_t kParallelMin = 1u << 16;

struct Builder {
    const std::vector<Box> &tb;
    const std::vector<float> &cent;
    std::vector<uint32_t> &order;
    int max_leaf;
    std::atomic<uint32_t> max_depth{0};

    // Builds [b, e) into its own node vector; returns the local root index.
    int32_t build(std::vector<BNode> &nodes, uint32_t b, uint32_t e, uint32_t depth) {
        uint32_t md = max_depth.load();
        while (depth > md && !max_depth.compare_exchange_weak(md, depth)) {}
        int32_t me = (int32_t)nodes.size();
        nodes.emplace_back();
        Box bb, cb;
        bb.empty();
        cb.empty();
        for (uint32_t i = b; i < e; i++) {
            bb.grow(tb[order[i]]);
            cb.grow(&cent[3 * order[i]]);
        }
        nodes[me].box = bb;
        uint32_t n = e - b;
        auto make_leaf = [&]() {
            nodes[me].start = b;
            nodes[me].count = n;
            return me;
        };
        if (n <= 1) return make_leaf();
        int best_axis = -1, best_split = -1;
        float best_cost = INFINITY;
        for (int ax = 0; ax < 3; ax++) {
            float ext = cb.hi[ax] - cb.lo[ax];
            if (!(ext > 0.0f)) continue;
            Box bins[kBins];
            uint32_t cnt[kBins] = {0};
            for (int k = 0; k < kBins; k++) bins[k].empty();
            float scale = kBins / ext;
            for (uint32_t i = b; i < e; i++) {
                int k = std::min(kBins - 1, (int)((cent[3 * order[i] + ax] - cb.lo[ax]) * scale));
                cnt[k]++;
                bins[k].grow(tb[order[i]]);
            }
            float rarea[kBins];
            uint32_t rcnt[kBins];
            Box acc;
            acc.empty();
            uint32_t c = 0;
            for (int k = kBins - 1; k > 0; k--) {
                acc.grow(bins[k]);
                c += cnt[k];
                rarea[k] = acc.area();
                rcnt[k] = c;
            }
            acc.empty();
            c = 0;
            for (int k = 0; k < kBins - 1; k++) {
                acc.grow(bins[k]);
                c += cnt[k];
                if (c == 0 || rcnt[k + 1] == 0) continue;
                float cost = acc.area() * c + rarea[k + 1] * rcnt[k + 1];
                if (cost < best_cost) { best_cost = cost; best_axis = ax; best_split = k; }
            }
        }
        float parent_area = bb.area();
        // SAH: traversal cost 1, intersection cost 1 per triangle
        float split_cost = parent_area > 0.0f ? 1.0f + best_cost / parent_area : INFINITY;
        bool force = n > (uint32_t)max_leaf || depth >= (uint32_t)kMaxDepth - 2;
        if (!force && (best_axis < 0 || (float)n <= split_cost)) return make_leaf();
        uint32_t mid;
        if (best_axis >= 0 && depth < (uint32_t)kMaxDepth - 8) {
            float ext = cb.hi[best_axis] - cb.lo[best_axis], scale = kBins / ext;
            auto it = std::partition(order.begin() + b, order.begin() + e, [&](uint32_t t) {
                int k = std::min(kBins - 1, (int)((cent[3 * t + best_axis] - cb.lo[best_axis]) * scale));
                return k <= best_split;
            });
            mid = (uint32_t)(it - order.begin());
        } else {
            // object median on the widest centroid axis (degenerate bins or deep tree)
            int ax = 0;
            for (int k = 1; k < 3; k++)
                if (cb.hi[k] - cb.lo[k] > cb.hi[ax] - cb.lo[ax]) ax = k;
            mid = b + n / 2;
            std::nth_element(order.begin() + b, order.begin() + mid, order.begin() + e,
                             [&](uint32_t x, uint32_t y) { return cent[3 * x + ax] < cent[3 * y + ax]; });
        }
        if (mid == b || mid == e) mid = b + n / 2;
        if (depth >= (uint32_t)kMaxDepth) throw std::runtime_error("BVH depth limit exceeded");
        int32_t l, r;
        if (n >= kParallelMin) {
            std::vector<BNode> sub;
            auto fut = std::async(std::launch::async, [&] { return build(sub, b, mid, depth + 1); });
            r = build(nodes, mid, e, depth + 1);
            int32_t lr = fut.get();
            // append the left subtree, rebasing its indices
            int32_t base = (int32_t)nodes.size();
            for (auto &nd : sub) {
                if (nd.left >= 0) { nd.left += base; nd.right += base; }
                nodes.push_back(nd);
            }
            l = lr + base;
        } else {
            l = build(nodes, b, mid, depth + 1);
            r = build(nodes, mid, e, depth + 1);
        }
        nodes[me].left = l;
        nodes[me].right = r;
        return me;
    }
};

void put_box(float *dst, const Box &c0, const Box &c1) {
    // a = (c0.lo.x, c0.hi.x, c0.lo.y, c0.hi.y); b = same for c1; c = (c0.lo.z, c0.hi.z, c1.lo.z, c1.hi.z)
    dst[0] = c0.lo[0]; dst[1] = c0.hi[0]; dst[2] = c0.lo[1]; dst[3] = c0.hi[1];
    dst[4] = c1.lo[0]; dst[5] = c1.hi[0]; dst[6] = c1.lo[1]; dst[7] = c1.hi[1];
    dst[8] = c0.lo[2]; dst[9] = c0.hi[2]; dst[10] = c1.lo[2]; dst[11] = c1.hi[2];
}

int32_t leaf_ref(const BNode &n) {
    if (n.count >= 32) throw std::runtime_error("BVH leaf too large");
    uint32_t enc = n.start | (n.count << kLeafCountShift);
    return (int32_t)~enc;
}

}  // namespace

Bvh2 build_bvh2(const float *tris, uint32_t n, int max_leaf) {
    Bvh2 out;
    if (n == 0) return out;
    std::vector<Box> tb(n);
    std::vector<float> cent(3 * (size_t)n);
    out.tri_order.resize(n);
    for (uint32_t t = 0; t < n; t++) {
        tb[t].empty();
        for (int k = 0; k < 3; k++) tb[t].grow(tris + 9 * (size_t)t + 3 * k);
        for (int c = 0; c < 3; c++)
            cent[3 * (size_t)t + c] = (tris[9 * (size_t)t + c] + tris[9 * (size_t)t + 3 + c] + tris[9 * (size_t)t + 6 + c]) * (1.0f / 3.0f);
        out.tri_order[t] = t;
    }
    Builder B{tb, cent, out.tri_order, max_leaf};
    std::vector<BNode> nodes;
    nodes.reserve(2 * (size_t)n / std::max(1, max_leaf / 2) + 16);
    int32_t root = B.build(nodes, 0, n, 0);
    out.depth = B.max_depth.load() + 1;
    // pack internal nodes depth-first (left child directly after its parent)
    std::vector<int32_t> packed(nodes.size(), -1);
    std::vector<int32_t> stack;
    std::vector<int32_t> seq;
    if (nodes[root].left < 0) {
        // single leaf: a root node with the leaf and an empty leaf
        out.nodes.assign(16, 0.0f);
        Box far;
        for (int i = 0; i < 3; i++) { far.lo[i] = far.hi[i] = 1e30f; }
        put_box(out.nodes.data(), nodes[root].box, far);
        int32_t c0 = leaf_ref(nodes[root]), c1 = (int32_t)~0u;
        std::memcpy(&out.nodes[12], &c0, 4);
        std::memcpy(&out.nodes[13], &c1, 4);
        return out;
    }
    stack.push_back(root);
    while (!stack.empty()) {
        int32_t i = stack.back();
        stack.pop_back();
        packed[i] = (int32_t)seq.size();
        seq.push_back(i);
        const BNode &nd = nodes[i];
        if (nodes[nd.right].left >= 0) stack.push_back(nd.right);
        if (nodes[nd.left].left >= 0) stack.push_back(nd.left);
    }
    out.nodes.assign(seq.size() * 16, 0.0f);
    for (size_t k = 0; k < seq.size(); k++) {
        const BNode &nd = nodes[seq[k]];
        const BNode &l = nodes[nd.left], &r = nodes[nd.right];
        float *dst = &out.nodes[16 * k];
        put_box(dst, l.box, r.box);
        int32_t c0 = l.left >= 0 ? packed[nd.left] : leaf_ref(l);
        int32_t c1 = r.left >= 0 ? packed[nd.right] : leaf_ref(r);
        std::memcpy(&dst[12], &c0, 4);
        std::memcpy(&dst[13], &c1, 4);
    }
    return out;
}

}  // namespace hk
