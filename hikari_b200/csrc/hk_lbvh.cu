// Tree build on the device, for scenes that must become renderable fast (the
// serving loop switching scenes, a scene edited between renders).  The host
// build (hk_bvh.cpp: binned SAH, SAH-optimal 8-wide collapse) gives the
// better trees; this one gives the same compressed 8-wide node format in a
// few milliseconds:
//
//   1. scene box of the triangle centroids (block reductions, atomics on
//      order-preserving integer images of the floats);
//   2. 64-bit keys: 30-bit Morton code of the centroid above the triangle
//      index (unique keys), sorted by radix sort (CUB);
//   3. binary hierarchy over the sorted keys by the longest common prefix
//      (Karras, "Maximizing Parallelism in the Construction of BVHs, Octrees,
//      and k-d Trees", HPG 2012): every node covers a contiguous key range;
//   4. node boxes bottom up: each leaf climbs and the second child to arrive
//      at a node merges the two boxes;
//   5. top-down collapse into 8-wide nodes, one frontier level per launch:
//      a node takes its binary node's two children and opens the child of
//      largest surface area until it has eight or none can open (a child of
//      at most three triangles stays a leaf), assigns children to the octant
//      slots like the host collapse, reserves its internal children and its
//      leaf triangles with atomics, and quantises its child boxes.
//
// Quantisation follows the host's rule (hk_bvh.cpp quantize): per axis a
// power-of-two step covering the node in 252 steps, the origin one step below
// the node box, child planes rounded outward and padded by one step.
#include <cub/device/device_radix_sort.cuh>

#include <cstdint>
#include <string>
#include <vector>

#include "hk_hostutil.h"
#include "hk_lbvh.h"

namespace hk {
namespace {

constexpr int kLbvhThreads = 256;

// float <-> unsigned key whose integer order is the float order
__device__ __forceinline__ uint32_t f2key(float f) {
    const uint32_t u = __float_as_uint(f);
    return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
__device__ __forceinline__ float key2f(uint32_t k) {
    return __uint_as_float((k & 0x80000000u) ? (k & 0x7fffffffu) : ~k);
}

struct Box3 {
    float lo[3], hi[3];
};
__device__ __forceinline__ Box3 tri_box(const float *t) {
    Box3 b;
    for (int k = 0; k < 3; k++) {
        b.lo[k] = fminf(fminf(t[k], t[3 + k]), t[6 + k]);
        b.hi[k] = fmaxf(fmaxf(t[k], t[3 + k]), t[6 + k]);
    }
    return b;
}
__device__ __forceinline__ Box3 merge(const Box3 &a, const Box3 &b) {
    Box3 r;
    for (int k = 0; k < 3; k++) {
        r.lo[k] = fminf(a.lo[k], b.lo[k]);
        r.hi[k] = fmaxf(a.hi[k], b.hi[k]);
    }
    return r;
}
__device__ __forceinline__ float half_area(const Box3 &b) {
    const float x = b.hi[0] - b.lo[0], y = b.hi[1] - b.lo[1], z = b.hi[2] - b.lo[2];
    return x * y + y * z + z * x;
}

// 1. centroid box: gkeys[0..2] min keys, [3..5] max keys
__global__ void centroid_box_kernel(const float *tris, uint32_t n, uint32_t *gkeys) {
    __shared__ uint32_t sk[6];
    if (threadIdx.x < 6) sk[threadIdx.x] = threadIdx.x < 3 ? 0xffffffffu : 0u;
    __syncthreads();
    uint32_t lo[3] = {0xffffffffu, 0xffffffffu, 0xffffffffu}, hi[3] = {0u, 0u, 0u};
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const float *t = tris + 9 * (size_t)i;
        for (int k = 0; k < 3; k++) {
            const uint32_t c = f2key((t[k] + t[3 + k] + t[6 + k]) * (1.0f / 3.0f));
            lo[k] = min(lo[k], c);
            hi[k] = max(hi[k], c);
        }
    }
    for (int k = 0; k < 3; k++) {
        atomicMin(&sk[k], lo[k]);
        atomicMax(&sk[3 + k], hi[k]);
    }
    __syncthreads();
    if (threadIdx.x < 3) atomicMin(&gkeys[threadIdx.x], sk[threadIdx.x]);
    else if (threadIdx.x < 6) atomicMax(&gkeys[threadIdx.x], sk[threadIdx.x]);
}

__device__ __forceinline__ uint32_t spread10(uint32_t v) {   // 10 bits -> every third bit
    v &= 0x3ffu;
    v = (v | (v << 16)) & 0x030000ffu;
    v = (v | (v << 8)) & 0x0300f00fu;
    v = (v | (v << 4)) & 0x030c30c3u;
    v = (v | (v << 2)) & 0x09249249u;
    return v;
}

// 2. keys: Morton code << 32 | triangle index
__global__ void morton_kernel(const float *tris, uint32_t n, const uint32_t *gkeys, unsigned long long *keys) {
    float lo[3], inv[3];
    for (int k = 0; k < 3; k++) {
        lo[k] = key2f(gkeys[k]);
        const float ext = key2f(gkeys[3 + k]) - lo[k];
        inv[k] = ext > 0.0f ? 1023.0f / ext : 0.0f;
    }
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const float *t = tris + 9 * (size_t)i;
        uint32_t q[3];
        for (int k = 0; k < 3; k++) {
            const float c = (t[k] + t[3 + k] + t[6 + k]) * (1.0f / 3.0f);
            q[k] = (uint32_t)fminf(fmaxf((c - lo[k]) * inv[k], 0.0f), 1023.0f);
        }
        const uint32_t m = spread10(q[0]) << 2 | spread10(q[1]) << 1 | spread10(q[2]);
        keys[i] = (unsigned long long)m << 32 | i;
    }
}

// Node numbering: internal nodes 0 .. n-2, leaf i (sorted position i) is n-1+i.
__device__ __forceinline__ int prefix(const unsigned long long *k, int n, int i, int j) {
    if (j < 0 || j >= n) return -1;
    return __clzll(k[i] ^ k[j]);
}

// 3. hierarchy: children and ranges of internal node i, parents of everything
__global__ void hierarchy_kernel(const unsigned long long *keys, int n, int2 *child, int2 *range, int *parent) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n - 1; i += gridDim.x * blockDim.x) {
        const int d = prefix(keys, n, i, i + 1) > prefix(keys, n, i, i - 1) ? 1 : -1;
        const int dmin = prefix(keys, n, i, i - d);
        int lmax = 2;
        while (prefix(keys, n, i, i + lmax * d) > dmin) lmax <<= 1;
        int l = 0;
        for (int t = lmax >> 1; t >= 1; t >>= 1)
            if (prefix(keys, n, i, i + (l + t) * d) > dmin) l += t;
        const int j = i + l * d;
        const int dnode = prefix(keys, n, i, j);
        int s = 0;
        for (int t = (l + 1) >> 1;; t = (t + 1) >> 1) {
            if (prefix(keys, n, i, i + (s + t) * d) > dnode) s += t;
            if (t == 1) break;
        }
        const int gamma = i + s * d + min(d, 0);
        const int first = min(i, j), last = max(i, j);
        const int left = first == gamma ? (n - 1) + gamma : gamma;
        const int right = last == gamma + 1 ? (n - 1) + gamma + 1 : gamma + 1;
        if (gamma < 0 || gamma > n - 2 || left >= 2 * n - 1 || right >= 2 * n - 1) continue;   // never: see the split search
        child[i] = make_int2(left, right);
        range[i] = make_int2(first, last);
        parent[left] = i;
        parent[right] = i;
    }
}

// a box another block wrote: read around the (incoherent) L1
__device__ __forceinline__ Box3 load_box(const Box3 *b) {
    Box3 r;
    const float *f = reinterpret_cast<const float *>(b);
    for (int k = 0; k < 3; k++) {
        r.lo[k] = __ldcg(f + k);
        r.hi[k] = __ldcg(f + 3 + k);
    }
    return r;
}

// 4. boxes bottom up
__global__ void boxes_kernel(const float *tris, const unsigned long long *keys, int n, const int2 *child,
                             const int *parent, unsigned *visits, Box3 *box) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const uint32_t t = (uint32_t)(keys[i] & 0xffffffffull);
        int node = (n - 1) + i;
        box[node] = tri_box(tris + 9 * (size_t)t);
        __threadfence();
        int p = n > 1 ? parent[node] : -1;
        while (p >= 0 && p < n - 1) {
            if (atomicAdd(&visits[p], 1u) == 0u) break;   // the first child to arrive stops
            __threadfence();
            const int2 c = child[p];
            box[p] = merge(load_box(box + c.x), load_box(box + c.y));
            __threadfence();
            node = p;
            p = p == 0 ? -1 : parent[p];
        }
    }
}

struct Frontier {
    uint32_t wide;   // 8-wide node index
    int32_t bin;     // binary node it is made from
};

__device__ __forceinline__ uint32_t node_count(const int2 *range, int n, int node) {
    if (node >= n - 1) return 1u;
    const int2 r = range[node];
    return (uint32_t)(r.y - r.x + 1);
}
__device__ __forceinline__ uint32_t node_first(const int2 *range, int n, int node) {
    return node >= n - 1 ? (uint32_t)(node - (n - 1)) : (uint32_t)range[node].x;
}

// Quantised child boxes of one 8-wide node (hk_bvh.cpp quantize, in double on
// the device).  Returns false where the extent does not fit the format.
__device__ bool quantize_dev(uint32_t *w, const Box3 &nb, const Box3 *cb, const bool *used) {
    uint8_t qlo[3][8], qhi[3][8];
    uint32_t eb[3];
    float p[3];
    for (int k = 0; k < 3; k++) {
        const double lo_n = nb.lo[k], hi_n = nb.hi[k];
        const double ext = hi_n - lo_n;
        const double mag = fmax(fmax(fabs(lo_n), fabs(hi_n)), 1e-30);
        int e = (int)floor(log2(mag)) - 20;
        if (ext > 0.0) e = max(e, (int)ceil(log2(ext / 252.0)));
        while (ldexp(252.0, e) < ext) ++e;
        if (e > 38) return false;
        e = max(-126, e);
        eb[k] = (uint32_t)(e + 127);
        const double scale = ldexp(1.0, e);
        p[k] = (float)(lo_n - scale);
        if ((double)p[k] > lo_n - scale) p[k] = nextafterf(p[k], -INFINITY);
        for (int s = 0; s < 8; s++) {
            if (!used[s]) {
                qlo[k][s] = 255;
                qhi[k][s] = 0;
                continue;
            }
            const double lo = floor(((double)cb[s].lo[k] - (double)p[k]) / scale) - 1.0;
            const double hi = ceil(((double)cb[s].hi[k] - (double)p[k]) / scale) + 1.0;
            if (lo < 0.0 || hi > 255.0) return false;
            qlo[k][s] = (uint8_t)lo;
            qhi[k][s] = (uint8_t)hi;
        }
    }
    for (int k = 0; k < 3; k++) w[k] = __float_as_uint(p[k]);
    w[3] = eb[0] | eb[1] << 8 | eb[2] << 16 | (w[3] & 0xff000000u);
    for (int a = 0; a < 6; a++) {
        const uint8_t *q = a < 3 ? qlo[a] : qhi[a - 3];
        w[8 + 2 * a] = q[0] | q[1] << 8 | q[2] << 16 | (uint32_t)q[3] << 24;
        w[9 + 2 * a] = q[4] | q[5] << 8 | q[6] << 16 | (uint32_t)q[7] << 24;
    }
    return true;
}

// 5. one level of the collapse.  ctr: [0] wide nodes allocated, [1]
// triangles placed, [2] next frontier size, [3] error flag (1: a node's
// extent does not fit the quantisation, 2: a reservation passed its buffer --
// the write is skipped)
__global__ void collapse_kernel(const unsigned long long *keys, int n, const int2 *child, const int2 *range,
                                const Box3 *box, const Frontier *in, uint32_t nin, Frontier *out, uint32_t *wnodes,
                                uint32_t *order, uint32_t *ctr, uint32_t max_wide) {
    for (uint32_t f = blockIdx.x * blockDim.x + threadIdx.x; f < nin; f += gridDim.x * blockDim.x) {
        const Frontier fr = in[f];
        int C[8];
        int nc = 0;
        const bool small = node_count(range, n, fr.bin) <= 3u;
        if (small) {   // the whole tree is one leaf
            C[nc++] = fr.bin;
        } else {
            const int2 c = child[fr.bin];
            if (c.x < 0 || c.y < 0 || c.x >= 2 * n - 1 || c.y >= 2 * n - 1) {
                atomicExch(&ctr[3], 2u);
                continue;
            }
            C[nc++] = c.x;
            C[nc++] = c.y;
            while (nc < 8) {   // open the child of largest area that can open
                int best = -1;
                float ba = -1.0f;
                for (int q = 0; q < nc; q++)
                    if (node_count(range, n, C[q]) > 3u) {
                        const float a = half_area(box[C[q]]);
                        if (a > ba) { ba = a; best = q; }
                    }
                if (best < 0) break;
                const int2 cc = child[C[best]];
                if (cc.x < 0 || cc.y < 0 || cc.x >= 2 * n - 1 || cc.y >= 2 * n - 1) {
                    atomicExch(&ctr[3], 2u);
                    break;
                }
                C[best] = cc.x;
                C[nc++] = cc.y;
            }
        }
        // octant slots (hk_bvh.cpp assign_slots): best remaining (child, slot) pair first
        const Box3 nb = box[fr.bin];
        double cn[3];
        for (int k = 0; k < 3; k++) cn[k] = 0.5 * ((double)nb.lo[k] + (double)nb.hi[k]);
        double score[8][8];
        for (int c = 0; c < nc; c++) {
            double d[3];
            for (int k = 0; k < 3; k++) d[k] = 0.5 * ((double)box[C[c]].lo[k] + (double)box[C[c]].hi[k]) - cn[k];
            for (int sl = 0; sl < 8; sl++) {
                double sc = 0.0;
                for (int k = 0; k < 3; k++) sc += (sl >> k & 1) ? -d[k] : d[k];
                score[c][sl] = sc;
            }
        }
        int slot_child[8];
        for (int s = 0; s < 8; s++) slot_child[s] = -1;
        bool used_c[8] = {false, false, false, false, false, false, false, false};
        bool used_s[8] = {false, false, false, false, false, false, false, false};
        for (int done = 0; done < nc; ++done) {
            int bc = -1, bs = -1;
            for (int c = 0; c < nc; c++)
                for (int s = 0; s < 8; s++)
                    if (!used_c[c] && !used_s[s] && (bc < 0 || score[c][s] > score[bc][bs])) { bc = c; bs = s; }
            used_c[bc] = used_s[bs] = true;
            slot_child[bs] = C[bc];
        }
        // reserve internal children and leaf triangles
        uint32_t ninternal = 0, nleaf_tris = 0;
        for (int s = 0; s < 8; s++) {
            if (slot_child[s] < 0) continue;
            const uint32_t cnt = node_count(range, n, slot_child[s]);
            if (cnt > 3u) ++ninternal;
            else nleaf_tris += cnt;
        }
        const uint32_t child_base = ninternal ? atomicAdd(&ctr[0], ninternal) : 0u;
        const uint32_t tri_base = nleaf_tris ? atomicAdd(&ctr[1], nleaf_tris) : atomicAdd(&ctr[1], 0u);
        if (fr.wide >= max_wide) { atomicExch(&ctr[3], 2u); continue; }
        uint32_t *w = wnodes + 20 * (size_t)fr.wide;
        uint32_t imask = 0, meta[8] = {0, 0, 0, 0, 0, 0, 0, 0}, j = 0, off = 0;
        Box3 cb[8];
        bool used[8];
        for (int s = 0; s < 8; s++) {
            const int c = slot_child[s];
            used[s] = c >= 0;
            if (c < 0) continue;
            cb[s] = box[c];
            const uint32_t cnt = node_count(range, n, c);
            if (cnt > 3u) {
                imask |= 1u << s;
                meta[s] = 1u << 5 | (24u + (uint32_t)s);
                const uint32_t o = atomicAdd(&ctr[2], 1u);
                if (o < max_wide) out[o] = Frontier{child_base + j, c};
                else atomicExch(&ctr[3], 2u);
                ++j;
            } else {
                meta[s] = ((1u << cnt) - 1u) << 5 | off;
                const uint32_t first = node_first(range, n, c);
                for (uint32_t k = 0; k < cnt; k++) {
                    if (tri_base + off + k < (uint32_t)n && first + k < (uint32_t)n)
                        order[tri_base + off + k] = (uint32_t)(keys[first + k] & 0xffffffffull);
                    else
                        atomicExch(&ctr[3], 2u);
                }
                off += cnt;
            }
        }
        w[3] = imask << 24;
        w[4] = child_base;
        w[5] = tri_base;
        w[6] = meta[0] | meta[1] << 8 | meta[2] << 16 | meta[3] << 24;
        w[7] = meta[4] | meta[5] << 8 | meta[6] << 16 | meta[7] << 24;
        if (!quantize_dev(w, nb, cb, used)) atomicExch(&ctr[3], 1u);
    }
}

int grid_for(uint64_t n) {
    const uint64_t g = (n + kLbvhThreads - 1) / kLbvhThreads;
    return (int)(g < 1 ? 1 : (g > 148ull * 16 ? 148ull * 16 : g));
}

}  // namespace

void build_bvh8_gpu(const float *tris_dev, uint32_t n, cudaStream_t st, GpuBvh8 &out) {
    if (n == 0) throw HkError{HK_ERR_INVALID, "empty scene"};
    DevBuf gkeys, keys, keys_sorted, child, range, parent, visits, box, fr[2], ctr, temp;
    gkeys.alloc(6 * sizeof(uint32_t));
    const uint32_t init[6] = {0xffffffffu, 0xffffffffu, 0xffffffffu, 0u, 0u, 0u};
    HK_CUDA(cudaMemcpyAsync(gkeys.p, init, sizeof init, cudaMemcpyHostToDevice, st));
    centroid_box_kernel<<<grid_for(n), kLbvhThreads, 0, st>>>(tris_dev, n, gkeys.as<uint32_t>());
    keys.alloc((size_t)n * 8);
    keys_sorted.alloc((size_t)n * 8);
    morton_kernel<<<grid_for(n), kLbvhThreads, 0, st>>>(tris_dev, n, gkeys.as<uint32_t>(),
                                                         keys.as<unsigned long long>());
    HK_CUDA(cudaGetLastError());
    // sort the 62 significant key bits (30-bit code above a 32-bit index)
    size_t temp_bytes = 0;
    HK_CUDA(cub::DeviceRadixSort::SortKeys(nullptr, temp_bytes, keys.as<unsigned long long>(),
                                           keys_sorted.as<unsigned long long>(), (int)n, 0, 62, st));
    temp.alloc(std::max<size_t>(temp_bytes, 16));
    HK_CUDA(cub::DeviceRadixSort::SortKeys(temp.p, temp_bytes, keys.as<unsigned long long>(),
                                           keys_sorted.as<unsigned long long>(), (int)n, 0, 62, st));
    const int nn = 2 * (int)n - 1;
    child.alloc((size_t)std::max(1, (int)n - 1) * sizeof(int2));
    range.alloc((size_t)std::max(1, (int)n - 1) * sizeof(int2));
    parent.alloc((size_t)nn * sizeof(int));
    visits.alloc((size_t)std::max(1, (int)n - 1) * sizeof(unsigned));
    box.alloc((size_t)nn * sizeof(Box3));
    HK_CUDA(cudaMemsetAsync(visits.p, 0, visits.bytes, st));
    HK_CUDA(cudaMemsetAsync(parent.p, 0xff, parent.bytes, st));   // -1: no parent yet
    HK_CUDA(cudaMemsetAsync(child.p, 0xff, child.bytes, st));     // -1: unset
    if (n > 1)
        hierarchy_kernel<<<grid_for(n), kLbvhThreads, 0, st>>>(keys_sorted.as<unsigned long long>(), (int)n,
                                                               child.as<int2>(), range.as<int2>(), parent.as<int>());
    boxes_kernel<<<grid_for(n), kLbvhThreads, 0, st>>>(tris_dev, keys_sorted.as<unsigned long long>(), (int)n,
                                                       child.as<int2>(), parent.as<int>(), visits.as<unsigned>(),
                                                       box.as<Box3>());
    HK_CUDA(cudaGetLastError());
    // collapse: at most n 8-wide nodes (every one has an internal child or is the root)
    const uint32_t max_wide = std::max(1u, n);
    out.nodes.alloc((size_t)max_wide * 20 * sizeof(uint32_t));
    out.order.alloc((size_t)n * sizeof(uint32_t));
    fr[0].alloc((size_t)max_wide * sizeof(Frontier));
    fr[1].alloc((size_t)max_wide * sizeof(Frontier));
    ctr.alloc(4 * sizeof(uint32_t));
    const Frontier f0{0u, 0};   // the root: internal node 0, or with one triangle its leaf (node n - 1 = 0)
    HK_CUDA(cudaMemcpyAsync(fr[0].p, &f0, sizeof f0, cudaMemcpyHostToDevice, st));
    uint32_t h_ctr[4] = {1u, 0u, 0u, 0u};   // the root is wide node 0
    HK_CUDA(cudaMemcpyAsync(ctr.p, h_ctr, sizeof h_ctr, cudaMemcpyHostToDevice, st));
    uint32_t nin = 1, depth = 0, cur = 0;
    while (nin > 0) {
        ++depth;
        if (depth > 1000) throw HkError{HK_ERR_CUDA, "device tree collapse did not end"};
        HK_CUDA(cudaMemsetAsync(ctr.as<uint32_t>() + 2, 0, sizeof(uint32_t), st));
        collapse_kernel<<<grid_for(nin), kLbvhThreads, 0, st>>>(
            keys_sorted.as<unsigned long long>(), (int)n, child.as<int2>(), range.as<int2>(), box.as<Box3>(),
            fr[cur].as<Frontier>(), nin, fr[cur ^ 1].as<Frontier>(), out.nodes.as<uint32_t>(),
            out.order.as<uint32_t>(), ctr.as<uint32_t>(), max_wide);
        HK_CUDA(cudaGetLastError());
        HK_CUDA(cudaMemcpyAsync(h_ctr, ctr.p, sizeof h_ctr, cudaMemcpyDeviceToHost, st));
        HK_CUDA(cudaStreamSynchronize(st));
        if (h_ctr[3] == 1u) throw HkError{HK_ERR_INVALID, "scene extent too large for the 8-wide node quantisation"};
        if (h_ctr[3] != 0u) throw HkError{HK_ERR_CUDA, "device tree collapse overran its buffers"};
        if (h_ctr[0] > max_wide || h_ctr[2] > max_wide) throw HkError{HK_ERR_CUDA, "device tree collapse overran its buffers"};
        nin = h_ctr[2];
        cur ^= 1;
    }
    if (h_ctr[1] != n) throw HkError{HK_ERR_CUDA, "device tree collapse placed " + std::to_string(h_ctr[1]) +
                                                      " of " + std::to_string(n) + " triangles"};
    out.nnodes = h_ctr[0];
    out.depth = depth;
}

}  // namespace hk

namespace hk {
namespace {
// 48-byte triangle records in leaf order: v0.xyz + original index, v1.xyz +
// mesh id, v2.xyz + 0 (the layout hk_host.cpp uploads for the host build)
__global__ void gather_records_kernel(const float *tris, const int32_t *tmesh, const uint32_t *order, uint32_t n,
                                      float4 *recs) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const uint32_t o = order[i];
        const float *t = tris + 9 * (size_t)o;
        recs[3 * (size_t)i] = make_float4(t[0], t[1], t[2], __int_as_float((int)o));
        recs[3 * (size_t)i + 1] = make_float4(t[3], t[4], t[5], __int_as_float(tmesh[o]));
        recs[3 * (size_t)i + 2] = make_float4(t[6], t[7], t[8], 0.0f);
    }
}
}  // namespace

void gather_tri_records(const float *tris_dev, const int32_t *tmesh_dev, const uint32_t *order_dev, uint32_t n,
                        float *recs_dev, cudaStream_t st) {
    gather_records_kernel<<<grid_for(n), kLbvhThreads, 0, st>>>(tris_dev, tmesh_dev, order_dev, n, (float4 *)recs_dev);
    HK_CUDA(cudaGetLastError());
}

}  // namespace hk
