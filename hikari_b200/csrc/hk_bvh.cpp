// Binned-SAH BVH2 build (32 bins per axis on centroid bounds, SAH leaf
// termination), subtrees above 64k triangles built on worker threads.
#include "hk_bvh.h"

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstring>
#include <future>
#include <stdexcept>
#include <thread>
#include <utility>

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

// Centroid bins of the three axes: box and triangle count per bin.
struct Bins {
    Box box[3][kBins];
    uint32_t cnt[3][kBins];
    Bins() {
        for (int a = 0; a < 3; a++)
            for (int k = 0; k < kBins; k++) {
                box[a][k].empty();
                cnt[a][k] = 0;
            }
    }
    void merge(const Bins &o) {
        for (int a = 0; a < 3; a++)
            for (int k = 0; k < kBins; k++) {
                box[a][k].grow(o.box[a][k]);
                cnt[a][k] += o.cnt[a][k];
            }
    }
};

constexpr uint32_t kParallelScan = 1u << 20;   // ranges this long are scanned in parallel chunks

struct Builder {
    const std::vector<Box> &tb;
    const std::vector<float> &cent;
    std::vector<uint32_t> &order;
    int max_leaf;
    std::atomic<uint32_t> max_depth{0};

    static uint32_t chunks_for(uint32_t n) {
        if (n < kParallelScan) return 1;
        const uint32_t hw = std::max(1u, std::thread::hardware_concurrency());
        return std::min(std::min(hw, 16u), n / (kParallelScan / 4));
    }

    Bins bin_range(uint32_t i0, uint32_t i1, const Box &cb) const {
        Bins B;
        float scale[3];
        for (int ax = 0; ax < 3; ax++) {
            const float ext = cb.hi[ax] - cb.lo[ax];
            scale[ax] = ext > 0.0f ? kBins / ext : 0.0f;
        }
        for (uint32_t i = i0; i < i1; i++) {
            const uint32_t t = order[i];
            for (int ax = 0; ax < 3; ax++) {
                if (scale[ax] == 0.0f) continue;
                const int k = std::min(kBins - 1, (int)((cent[3 * t + ax] - cb.lo[ax]) * scale[ax]));
                B.cnt[ax][k]++;
                B.box[ax][k].grow(tb[t]);
            }
        }
        return B;
    }

    // Builds [b, e) into its own node vector; returns the local root index.
    int32_t build(std::vector<BNode> &nodes, uint32_t b, uint32_t e, uint32_t depth) {
        uint32_t md = max_depth.load();
        while (depth > md && !max_depth.compare_exchange_weak(md, depth)) {}
        int32_t me = (int32_t)nodes.size();
        nodes.emplace_back();
        Box bb, cb;
        bb.empty();
        cb.empty();
        const uint32_t nchunks = chunks_for(e - b);
        if (nchunks > 1) {   // large ranges: bounds in parallel chunks (min / max reduce exactly)
            std::vector<std::future<std::pair<Box, Box>>> f;
            for (uint32_t q = 0; q < nchunks; ++q)
                f.push_back(std::async(std::launch::async, [&, q] {
                    Box x, y;
                    x.empty();
                    y.empty();
                    const uint32_t i0 = b + (uint64_t)(e - b) * q / nchunks, i1 = b + (uint64_t)(e - b) * (q + 1) / nchunks;
                    for (uint32_t i = i0; i < i1; i++) {
                        x.grow(tb[order[i]]);
                        y.grow(&cent[3 * order[i]]);
                    }
                    return std::make_pair(x, y);
                }));
            for (auto &x : f) {
                auto r = x.get();
                bb.grow(r.first);
                cb.grow(r.second);
            }
        } else {
            for (uint32_t i = b; i < e; i++) {
                bb.grow(tb[order[i]]);
                cb.grow(&cent[3 * order[i]]);
            }
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
        // bins of all three axes in one pass over the range (in parallel chunks when large)
        Bins all;
        if (nchunks > 1) {
            std::vector<std::future<Bins>> f;
            for (uint32_t q = 0; q < nchunks; ++q)
                f.push_back(std::async(std::launch::async, [&, q] {
                    const uint32_t i0 = b + (uint64_t)(e - b) * q / nchunks, i1 = b + (uint64_t)(e - b) * (q + 1) / nchunks;
                    return bin_range(i0, i1, cb);
                }));
            for (auto &x : f) all.merge(x.get());
        } else {
            all = bin_range(b, e, cb);
        }
        for (int ax = 0; ax < 3; ax++) {
            float ext = cb.hi[ax] - cb.lo[ax];
            if (!(ext > 0.0f)) continue;
            const Box *bins = all.box[ax];
            const uint32_t *cnt = all.cnt[ax];
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

int32_t leaf_ref(uint32_t start, uint32_t count) {
    if (count >= 32) throw std::runtime_error("BVH leaf too large");
    if (start > kLeafStartMask) throw std::runtime_error("too many triangles for the BVH2 leaf encoding");
    uint32_t enc = start | (count << kLeafCountShift);
    return (int32_t)~enc;
}

struct Tree {
    std::vector<BNode> nodes;
    std::vector<uint32_t> order;   // builder order: leaves index [start, start + count)
    int32_t root = -1;
    uint32_t depth = 0;
};

Tree build_tree(const float *tris, uint32_t n, int max_leaf) {
    Tree T;
    std::vector<Box> tb(n);
    std::vector<float> cent(3 * (size_t)n);
    T.order.resize(n);
    for (uint32_t t = 0; t < n; t++) {
        tb[t].empty();
        for (int k = 0; k < 3; k++) tb[t].grow(tris + 9 * (size_t)t + 3 * k);
        for (int c = 0; c < 3; c++)
            cent[3 * (size_t)t + c] = (tris[9 * (size_t)t + c] + tris[9 * (size_t)t + 3 + c] + tris[9 * (size_t)t + 6 + c]) * (1.0f / 3.0f);
        T.order[t] = t;
    }
    Builder B{tb, cent, T.order, max_leaf};
    T.nodes.reserve(2 * (size_t)n / std::max(1, max_leaf / 2) + 16);
    T.root = B.build(T.nodes, 0, n, 0);
    T.depth = B.max_depth.load() + 1;
    return T;
}

// Packs the binary tree into 64-byte nodes; leaf_start(i) is the position of
// leaf i's first triangle in the final triangle order.
template <class F>
std::vector<float> pack_bvh2(const Tree &T, F leaf_start) {
    const std::vector<BNode> &nodes = T.nodes;
    std::vector<float> out;
    const int32_t root = T.root;
    if (nodes[root].left < 0) {
        // single leaf: a root node with the leaf and an empty leaf
        out.assign(16, 0.0f);
        Box far;
        for (int i = 0; i < 3; i++) { far.lo[i] = far.hi[i] = 1e30f; }
        put_box(out.data(), nodes[root].box, far);
        int32_t c0 = leaf_ref(leaf_start(root), nodes[root].count), c1 = (int32_t)~0u;
        std::memcpy(&out[12], &c0, 4);
        std::memcpy(&out[13], &c1, 4);
        return out;
    }
    // internal nodes depth-first (left child directly after its parent)
    std::vector<int32_t> packed(nodes.size(), -1);
    std::vector<int32_t> stack, seq;
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
    out.assign(seq.size() * 16, 0.0f);
    for (size_t k = 0; k < seq.size(); k++) {
        const BNode &nd = nodes[seq[k]];
        const BNode &l = nodes[nd.left], &r = nodes[nd.right];
        float *dst = &out[16 * k];
        put_box(dst, l.box, r.box);
        int32_t c0 = l.left >= 0 ? packed[nd.left] : leaf_ref(leaf_start(nd.left), l.count);
        int32_t c1 = r.left >= 0 ? packed[nd.right] : leaf_ref(leaf_start(nd.right), r.count);
        std::memcpy(&dst[12], &c0, 4);
        std::memcpy(&dst[13], &c1, 4);
    }
    return out;
}

// ---- 8-wide collapse and quantisation

// Triangle range [start, start + count) of every subtree in the builder order
// (the builder partitions in place, so a subtree's triangles are contiguous).
void subtree_ranges(const std::vector<BNode> &nodes, int32_t root, std::vector<uint32_t> &start,
                    std::vector<uint32_t> &count) {
    start.assign(nodes.size(), 0);
    count.assign(nodes.size(), 0);
    std::vector<std::pair<int32_t, bool>> st{{root, false}};
    while (!st.empty()) {
        auto [i, done] = st.back();
        st.pop_back();
        const BNode &n = nodes[i];
        if (n.left < 0) {
            start[i] = n.start;
            count[i] = n.count;
        } else if (done) {
            start[i] = std::min(start[n.left], start[n.right]);
            count[i] = count[n.left] + count[n.right];
        } else {
            st.push_back({i, true});
            st.push_back({n.left, false});
            st.push_back({n.right, false});
        }
    }
}

// Collapse by dynamic programming over the binary tree (Ylitie, Karras and
// Laine, HPG 2017, section 3.1): cost(n, i) is the least SAH cost of the
// subtree n when it may occupy at most i child slots of its parent -- as one
// leaf (at most 3 triangles, area * c_prim * count), as one 8-wide node (area
// * c_node + the best split of its two children over 8 slots), or, for i >= 2,
// split between its children.  The tree's nodes are numbered parents first,
// so a reverse sweep visits children before parents.
struct Collapse {
    static constexpr float kNode = 1.0f, kPrim = 0.3f;
    std::vector<float> cost;         // 8 per node: cost(n, 1..8)
    std::vector<int8_t> split;       // 8 per node: 0 = one child, k = k slots to the left subtree
    std::vector<uint8_t> as_leaf;    // cost(n, 1) is the leaf option
    std::vector<int8_t> node_split;  // slots to the left child when n is an 8-wide node

    Collapse(const std::vector<BNode> &nodes, const std::vector<uint32_t> &count) {
        const size_t N = nodes.size();
        cost.assign(8 * N, 0.0f);
        split.assign(8 * N, 0);
        as_leaf.assign(N, 0);
        node_split.assign(N, 0);
        for (size_t q = N; q-- > 0;) {
            const BNode &nd = nodes[q];
            const float area = std::max(nd.box.area(), 0.0f);
            const float leaf = count[q] <= 3 ? area * kPrim * (float)count[q] : INFINITY;
            float *C = &cost[8 * q];
            if (nd.left < 0) {
                for (int i = 0; i < 8; i++) C[i] = leaf;
                as_leaf[q] = 1;
                continue;
            }
            const float *L = &cost[8 * (size_t)nd.left], *R = &cost[8 * (size_t)nd.right];
            float dist[9];
            int arg[9];
            for (int j = 2; j <= 8; j++) {
                dist[j] = INFINITY;
                arg[j] = 1;
                for (int k = 1; k < j; k++) {
                    const float c = L[k - 1] + R[j - k - 1];
                    if (c < dist[j]) { dist[j] = c; arg[j] = k; }
                }
            }
            const float node = area * kNode + dist[8];
            node_split[q] = (int8_t)arg[8];
            C[0] = std::min(leaf, node);
            as_leaf[q] = leaf <= node ? 1 : 0;
            for (int i = 2; i <= 8; i++) {
                if (dist[i] < C[0]) { C[i - 1] = dist[i]; split[8 * q + i - 1] = (int8_t)arg[i]; }
                else C[i - 1] = C[0];
            }
        }
    }
    // Subtrees that fill at most i slots for subtree q.
    void collect(const std::vector<BNode> &nodes, int32_t q, int i, int32_t *out, int &n) const {
        const int k = split[8 * (size_t)q + i - 1];
        if (k == 0) { out[n++] = q; return; }
        collect(nodes, nodes[q].left, k, out, n);
        collect(nodes, nodes[q].right, i - k, out, n);
    }
    // Children of the 8-wide node made from binary node q.
    int children(const std::vector<BNode> &nodes, int32_t q, int32_t C[8]) const {
        int n = 0;
        const int k = node_split[q];
        collect(nodes, nodes[q].left, k, C, n);
        collect(nodes, nodes[q].right, 8 - k, C, n);
        return n;
    }
};

// Slot s means "negative side of axis k" for every set bit k; children are
// assigned greedily by the score of their centre offset along that diagonal.
void assign_slots(const std::vector<BNode> &nodes, const Box &nb, const int32_t *C, int n, int32_t slot_child[8]) {
    double cn[3];
    for (int k = 0; k < 3; k++) cn[k] = 0.5 * ((double)nb.lo[k] + (double)nb.hi[k]);
    struct Cand {
        double score;
        int c, s;
    };
    Cand cand[64];
    int nc = 0;
    for (int c = 0; c < n; c++) {
        const Box &b = nodes[C[c]].box;
        double d[3];
        for (int k = 0; k < 3; k++) d[k] = 0.5 * ((double)b.lo[k] + (double)b.hi[k]) - cn[k];
        for (int sl = 0; sl < 8; sl++) {
            double sc = 0.0;
            for (int k = 0; k < 3; k++) sc += (sl >> k & 1) ? -d[k] : d[k];
            cand[nc++] = {sc, c, sl};
        }
    }
    // repeatedly take the best remaining (child, slot) pair (the first one on ties)
    bool used_c[8] = {false}, used_s[8] = {false};
    for (int s2 = 0; s2 < 8; s2++) slot_child[s2] = -1;
    for (int done = 0; done < n; ++done) {
        int best = -1;
        for (int q = 0; q < nc; q++)
            if (!used_c[cand[q].c] && !used_s[cand[q].s] && (best < 0 || cand[q].score > cand[best].score)) best = q;
        const Cand &x = cand[best];
        used_c[x.c] = used_s[x.s] = true;
        slot_child[x.s] = C[x.c];
    }
}

// Quantised child boxes: conservative (floor/ceil in double) and padded by
// one step on every side, which absorbs the rounding of the traversal's
// folded slab arithmetic (at most half a step).  The step s = 2^e covers the
// node extent in 252 steps and the origin sits at least one step below the
// node box (float rounding of p is below a quarter step because s is at least
// 2^-20 of the coordinates' magnitude), so padded planes stay within 0..255.
void quantize(uint32_t *w, const Box &nb, const Box *cb[8]) {
    uint8_t qlo[3][8], qhi[3][8];
    int eb[3];
    float p[3];
    for (int k = 0; k < 3; k++) {
        const double lo_n = nb.lo[k], hi_n = nb.hi[k];
        const double ext = hi_n - lo_n;
        const double mag = std::max(std::max(std::fabs(lo_n), std::fabs(hi_n)), 1e-30);
        int e = (int)std::floor(std::log2(mag)) - 20;
        if (ext > 0.0) e = std::max(e, (int)std::ceil(std::log2(ext / 252.0)));
        while (std::ldexp(252.0, e) < ext) ++e;
        if (e > 38) throw std::runtime_error("scene extent too large for the 8-wide node quantisation");
        e = std::max(-126, e);
        eb[k] = e + 127;
        const double scale = std::ldexp(1.0, e);
        // origin at least one step below the node box (rounded toward -inf)
        p[k] = (float)(lo_n - scale);
        if ((double)p[k] > lo_n - scale) p[k] = std::nextafter(p[k], -INFINITY);
        for (int s = 0; s < 8; s++) {
            if (!cb[s]) {   // empty slot: an inverted box that no ray hits
                qlo[k][s] = 255;
                qhi[k][s] = 0;
                continue;
            }
            const double lo = std::floor(((double)cb[s]->lo[k] - (double)p[k]) / scale) - 1.0;
            const double hi = std::ceil(((double)cb[s]->hi[k] - (double)p[k]) / scale) + 1.0;
            if (lo < 0.0 || hi > 255.0) throw std::runtime_error("8-wide child box outside its node's range");
            qlo[k][s] = (uint8_t)lo;
            qhi[k][s] = (uint8_t)hi;
        }
    }
    for (int k = 0; k < 3; k++) std::memcpy(&w[k], &p[k], 4);
    w[3] = (uint32_t)eb[0] | (uint32_t)eb[1] << 8 | (uint32_t)eb[2] << 16 | (w[3] & 0xff000000u);
    auto pack = [](const uint8_t *q, uint32_t *dst) {
        dst[0] = q[0] | q[1] << 8 | q[2] << 16 | (uint32_t)q[3] << 24;
        dst[1] = q[4] | q[5] << 8 | q[6] << 16 | (uint32_t)q[7] << 24;
    };
    pack(qlo[0], &w[8]);
    pack(qlo[1], &w[10]);
    pack(qlo[2], &w[12]);
    pack(qhi[0], &w[14]);
    pack(qhi[1], &w[16]);
    pack(qhi[2], &w[18]);
}

}  // namespace

Bvh2 build_bvh2(const float *tris, uint32_t n, int max_leaf) {
    Bvh2 out;
    if (n == 0) return out;
    Tree T = build_tree(tris, n, max_leaf);
    out.depth = T.depth;
    out.nodes = pack_bvh2(T, [&](int32_t i) { return T.nodes[i].start; });
    out.tri_order = std::move(T.order);
    return out;
}

BvhPair build_bvh_pair(const float *tris, uint32_t n) {
    BvhPair P;
    if (n == 0) return P;
    Tree T = build_tree(tris, n, 3);
    const std::vector<BNode> &nodes = T.nodes;
    std::vector<uint32_t> sub_start, sub_count;
    subtree_ranges(nodes, T.root, sub_start, sub_count);
    const Collapse dp(nodes, sub_count);
    auto is_leaf8 = [&](int32_t c) { return dp.as_leaf[c] != 0; };
    // new position of every binary leaf's first triangle
    std::vector<uint32_t> leaf_start(nodes.size(), 0);
    auto place_subtree = [&](int32_t c, uint32_t base) {   // c holds at most 3 triangles: at most 5 nodes
        int32_t st[8];
        int sp = 0;
        st[sp++] = c;
        while (sp > 0) {
            const int32_t i = st[--sp];
            if (nodes[i].left < 0) leaf_start[i] = base + (nodes[i].start - sub_start[c]);
            else { st[sp++] = nodes[i].left; st[sp++] = nodes[i].right; }
        }
    };
    std::vector<uint32_t> &order = P.bvh2.tri_order;
    order.reserve(n);
    std::vector<uint32_t> &W = P.bvh8.nodes;
    W.assign(20, 0u);
    struct Todo {
        uint32_t w;
        int32_t b;
        uint32_t depth;
    };
    std::vector<Todo> todo;
    todo.push_back({0, T.root, 1});
    uint32_t depth8 = 0;
    while (!todo.empty()) {
        Todo t = todo.back();
        todo.pop_back();
        depth8 = std::max(depth8, t.depth);
        int32_t C[8];
        int nc;
        if (is_leaf8(t.b)) {   // the whole tree is one leaf
            C[0] = t.b;
            nc = 1;
        } else {
            nc = dp.children(nodes, t.b, C);
        }
        int32_t slot_child[8];
        assign_slots(nodes, nodes[t.b].box, C, nc, slot_child);
        uint32_t ninternal = 0;
        for (int s = 0; s < 8; s++)
            if (slot_child[s] >= 0 && !is_leaf8(slot_child[s])) ++ninternal;
        const uint32_t child_base = (uint32_t)(W.size() / 20);
        W.resize(W.size() + 20 * (size_t)ninternal, 0u);
        const uint32_t tri_base = (uint32_t)order.size();
        uint32_t imask = 0, meta[8] = {0};
        Todo kids[8];
        int nkids = 0;
        uint32_t j = 0;
        const Box *cb[8];
        for (int s = 0; s < 8; s++) {
            const int32_t c = slot_child[s];
            cb[s] = c >= 0 ? &nodes[c].box : nullptr;
            if (c < 0) continue;
            if (!is_leaf8(c)) {
                imask |= 1u << s;
                meta[s] = 1u << 5 | (24u + (uint32_t)s);   // one hit bit at 24 + slot
                kids[nkids++] = {child_base + j++, c, t.depth + 1};
            } else {
                const uint32_t off = (uint32_t)order.size() - tri_base, cnt = sub_count[c];
                if (cnt < 1 || cnt > 3 || off > 21) throw std::runtime_error("BVH8 leaf layout");
                meta[s] = ((1u << cnt) - 1u) << 5 | off;   // cnt hit bits from off
                place_subtree(c, (uint32_t)order.size());
                for (uint32_t k = 0; k < cnt; k++) order.push_back(T.order[sub_start[c] + k]);
            }
        }
        uint32_t *w = &W[20 * (size_t)t.w];
        w[3] = imask << 24;
        w[4] = child_base;
        w[5] = tri_base;
        w[6] = meta[0] | meta[1] << 8 | meta[2] << 16 | meta[3] << 24;
        w[7] = meta[4] | meta[5] << 8 | meta[6] << 16 | meta[7] << 24;
        quantize(w, nodes[t.b].box, cb);
        for (int q = nkids - 1; q >= 0; --q) todo.push_back(kids[q]);
    }
    if (order.size() != n) throw std::runtime_error("BVH8 collapse lost triangles");
    P.bvh8.depth = depth8;
    P.bvh2.depth = T.depth;
    P.bvh2.nodes = pack_bvh2(T, [&](int32_t i) { return leaf_start[i]; });
    return P;
}

std::string check_bvh8(const std::vector<uint32_t> &W, const std::vector<uint32_t> &order, const float *tris,
                       uint32_t n) {
    if (order.size() != n) return "triangle order has the wrong size";
    std::vector<uint8_t> seen(n, 0);
    for (uint32_t o : order) {
        if (o >= n || seen[o]) return "triangle order is not a permutation";
        seen[o] = 1;
    }
    const uint32_t nw = (uint32_t)(W.size() / 20);
    if (nw == 0) return "8-wide tree is empty";
    std::vector<uint8_t> tri_ref(n, 0), node_ref(nw, 0);
    struct Item {
        uint32_t node;
        double lo[3], hi[3];   // the box the parent stores for this node
    };
    std::vector<Item> todo;
    Item root{0, {-1e300, -1e300, -1e300}, {1e300, 1e300, 1e300}};
    todo.push_back(root);
    node_ref[0] = 1;
    auto inside = [&](uint32_t pos, const double *lo, const double *hi) {
        const uint32_t t = order[pos];
        for (int v = 0; v < 3; v++)
            for (int k = 0; k < 3; k++) {
                double x = tris[9 * (size_t)t + 3 * v + k];
                if (x < lo[k] || x > hi[k]) return false;
            }
        return true;
    };
    while (!todo.empty()) {
        Item it = todo.back();
        todo.pop_back();
        const uint32_t *w = &W[20 * (size_t)it.node];
        float p[3];
        std::memcpy(p, w, 12);
        const uint32_t imask = w[3] >> 24;
        double scale[3];
        for (int k = 0; k < 3; k++) scale[k] = std::ldexp(1.0, (int)((w[3] >> (8 * k)) & 0xffu) - 127);
        auto q = [&](int plane, int k, int s) { return (double)((w[8 + 2 * (plane * 3 + k) + s / 4] >> (8 * (s % 4))) & 0xffu); };
        uint32_t j = 0;
        for (int s = 0; s < 8; s++) {
            const uint32_t m = (s < 4 ? w[6] : w[7]) >> (8 * (s & 3)) & 0xffu;
            double lo[3], hi[3];
            for (int k = 0; k < 3; k++) {
                lo[k] = (double)p[k] + q(0, k, s) * scale[k];
                hi[k] = (double)p[k] + q(1, k, s) * scale[k];
            }
            if (imask >> s & 1u) {
                if (m != (0x38u | (uint32_t)s)) return "8-wide internal child meta";
                const uint32_t c = w[4] + j++;
                if (c >= nw || node_ref[c]) return "8-wide child index out of range or shared";
                node_ref[c] = 1;
                Item ci{c, {lo[0], lo[1], lo[2]}, {hi[0], hi[1], hi[2]}};
                todo.push_back(ci);
            } else if (m) {
                const uint32_t cnt = (uint32_t)__builtin_popcount(m >> 5), off = m & 31u;
                if ((m >> 5) != (1u << cnt) - 1u) return "8-wide leaf meta is not a unary count";
                for (uint32_t k = 0; k < cnt; k++) {
                    const uint32_t pos = w[5] + off + k;
                    if (pos >= n || tri_ref[pos]) return "8-wide leaf triangle out of range or shared";
                    tri_ref[pos] = 1;
                    if (!inside(pos, lo, hi)) return "8-wide child box does not contain its triangle";
                    // and every ancestor box along the way
                    if (!inside(pos, it.lo, it.hi)) return "8-wide node box does not contain its triangle";
                }
            }
        }
        // child boxes of internal children must lie within this node's stored box
        (void)it;
    }
    for (uint32_t i = 0; i < n; i++)
        if (!tri_ref[i]) return "8-wide tree misses a triangle";
    for (uint32_t i = 0; i < nw; i++)
        if (!node_ref[i]) return "8-wide tree has an unreachable node";
    return std::string();
}

std::string check_bvh_pair(const BvhPair &P, const float *tris, uint32_t n) {
    const std::string e8 = check_bvh8(P.bvh8.nodes, P.bvh2.tri_order, tris, n);
    if (!e8.empty()) return e8;
    // ---- binary tree: leaves cover the order once
    std::vector<uint8_t> tri2(n, 0);
    const std::vector<float> &B = P.bvh2.nodes;
    const uint32_t nb = (uint32_t)(B.size() / 16);
    for (uint32_t i = 0; i < nb; i++)
        for (int c = 0; c < 2; c++) {
            int32_t ref;
            std::memcpy(&ref, &B[16 * (size_t)i + 12 + c], 4);
            if (ref >= 0) {
                if ((uint32_t)ref >= nb) return "binary child index out of range";
                continue;
            }
            const uint32_t enc = ~(uint32_t)ref, start = enc & kLeafStartMask, cnt = enc >> kLeafCountShift;
            for (uint32_t k = 0; k < cnt; k++) {
                if (start + k >= n || tri2[start + k]) return "binary leaf triangle out of range or shared";
                tri2[start + k] = 1;
            }
        }
    for (uint32_t i = 0; i < n; i++)
        if (!tri2[i]) return "binary tree misses a triangle";
    return std::string();
}

}  // namespace hk
