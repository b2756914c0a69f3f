// Wavefront pathMIS kernels shared by the wavefront translation units: the
// queue helpers, the extend and shadow (traversal) kernels and the shade
// kernel template.  hk_wavefront.cu holds regen and the launch sequence;
// hk_wf_trace_*.cu instantiate the traversal kernels per tree kind and
// hk_wf_shade_*.cu the shade kernels per queue, so they compile in parallel.
#pragma once
#include "hk_shading.cuh"
#include "hk_wavefront.h"

namespace hk {

// ------------------------------------------------------------ helpers
__device__ __forceinline__ unsigned lane_id() { return threadIdx.x & 31u; }

// Warp-aggregated append to a queue counter: one atomic per warp.
__device__ __forceinline__ unsigned warp_append(unsigned *counter) {
    unsigned mask = __activemask();
    int leader = __ffs(mask) - 1;
    unsigned rank = __popc(mask & ((1u << lane_id()) - 1u));
    unsigned base = 0;
    if ((int)lane_id() == leader) base = atomicAdd(counter, (unsigned)__popc(mask));
    base = __shfl_sync(mask, base, leader);
    return base + rank;
}
// Append grouped by key (lanes with equal keys share one atomic).
__device__ __forceinline__ unsigned warp_append_keyed(unsigned *counters, int key) {
    unsigned mask = __activemask();
    unsigned peers = __match_any_sync(mask, key);
    int leader = __ffs(peers) - 1;
    unsigned rank = __popc(peers & ((1u << lane_id()) - 1u));
    unsigned base = 0;
    if ((int)lane_id() == leader) base = atomicAdd(counters + key, (unsigned)__popc(peers));
    base = __shfl_sync(peers, base, leader);
    return base + rank;
}
__device__ __forceinline__ void red_add_v4(float4 *addr, float a, float b, float c, float d) {
    asm volatile("red.global.add.v4.f32 [%0], {%1, %2, %3, %4};" ::"l"(addr), "f"(a), "f"(b), "f"(c), "f"(d)
                 : "memory");
}
__device__ __forceinline__ float4 f4(V3 v, float w) { return make_float4(v.x, v.y, v.z, w); }

// PerspectiveCamera::SampleRay (src/camera/PerspectiveCamera.cpp:71) at the
// job's resolution and pose; field of view and clip planes are the scene's.
__device__ __forceinline__ Ray camera_ray_job(const DevScene &S, const WfJob &J, float px, float py) {
    const float *M = J.cam;
    float u = px * (1.0f / (float)J.width), v = py * (1.0f / (float)J.height);
    V3 np = v3(S.cam_near * (1.0f - 2.0f * u) / S.cam_cot, S.cam_near * (1.0f - 2.0f * v) / (J.cam_aspect * S.cam_cot),
               S.cam_near);
    V3 dir = normalize(np);
    float invz = 1.0f / dir.z;
    Ray r;
    r.o = v3(M[3], M[7], M[11]);
    r.d = v3(M[0] * dir.x + M[1] * dir.y + M[2] * dir.z, M[4] * dir.x + M[5] * dir.y + M[6] * dir.z,
             M[8] * dir.x + M[9] * dir.y + M[10] * dir.z);
    r.tmin = S.cam_near * invz;
    r.tmax = S.cam_far * invz;
    return r;
}

__device__ __forceinline__ uint64_t wf_mix_seed(uint64_t seed, uint64_t s) {
    uint64_t z = seed + 0x9E3779B97F4A7C15ULL * (s + 1);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    return z ^ (z >> 31);
}

// Piece of the current plan that holds plan item w (pieces are sorted by plan_begin).
__device__ __forceinline__ int find_seg(const WfState &W, uint64_t w, int nseg) {
    int lo = 0, hi = nseg - 1;
    while (lo < hi) {
        int mid = (lo + hi + 1) >> 1;
        if (W.segs[mid].plan_begin <= w) lo = mid; else hi = mid - 1;
    }
    return lo;
}

// ImageBlock::Put into the job's global film with vector reductions.
__device__ __forceinline__ void splat_global(const DevScene &S, const WfJob &J, float px, float py, V3 val) {
    const int B = S.border, FW = (int)J.width + 2 * B, FH = (int)J.height + 2 * B;
    float *film = J.film;
    float cx = px - 0.5f - (0 - B), cy = py - 0.5f - (0 - B);
    int x0 = max((int)ceilf(cx - S.filt_radius), 0), y0 = max((int)ceilf(cy - S.filt_radius), 0);
    int x1 = min((int)floorf(cx + S.filt_radius), FW - 1), y1 = min((int)floorf(cy + S.filt_radius), FH - 1);
    float4 *F = reinterpret_cast<float4 *>(film);
    for (int y = y0; y <= y1; ++y) {
        float wy = __ldg(S.ftab + (int)(fabsf((float)y - cy) * S.filt_lookup));
        for (int x = x0; x <= x1; ++x) {
            float wx = __ldg(S.ftab + (int)(fabsf((float)x - cx) * S.filt_lookup));
            float w = wx * wy;
            if (w == 0.0f) continue;
            red_add_v4(F + (size_t)y * FW + x, (val.x * wx) * wy, (val.y * wx) * wy, (val.z * wx) * wy, w);
        }
    }
}
// ------------------------------------------------------------ extend
// Shared memory of the traversal short stacks: kShStack entries per thread.
__device__ __forceinline__ SharedStack make_stack() {
    extern __shared__ uint2 wf_stack_smem[];
    SharedStack s;
    s.sh = wf_stack_smem + threadIdx.x;
    s.stride = (int)blockDim.x;
    s.spill = nullptr;
    return s;
}

// The traversal kernels come in two register budgets: kMinBlocks = 0 leaves
// the budget to the compiler; kLeanBlocks asks for five resident blocks of
// 256 threads (at most 48 registers), more warps to hide the latency of the
// node and triangle fetches at the price of some spilling.  The autotuner
// picks per kernel (hk_wavefront_config.reg_lean).
constexpr int kLeanBlocks = 5;

// kShared: the warp's triangle tests shared out over its lanes (8-wide tree;
// the block's ray records in dynamic shared memory after the stacks).
template <int kAccel, int kMinBlocks, bool kShared>
__global__ void __launch_bounds__(256, kMinBlocks) wf_extend_kernel(DevScene S, WfState W, int cur, int steps, int min_idle) {
    const unsigned n = W.ctr->eq_count[cur];
    TravStats ts;
    WalkerOf<kAccel, SharedStack> wk;
    std::conditional_t<kAccel == kAccelBvh8, uint2, int> stack_mem[kAccel == kAccelBvh8 ? kStackSize - kShStack : kStackSize];
    if constexpr (kAccel == kAccelBvh8) {
        wk.stk = make_stack();
        wk.stk.spill = stack_mem;
    } else {
        wk.stack = stack_mem;
    }
    int slot = -1;
    auto load = [&](int i) {
        slot = W.eq[cur][i];
        const float4 o = W.ray_o[slot], d = W.ray_d[slot];
        Ray r;
        r.o = v3(o.x, o.y, o.z);
        r.d = v3(d.x, d.y, d.z);
        r.tmin = o.w;
        r.tmax = d.w;
        return r;
    };
    auto store = [&](int, const auto &w) {
        int type = 0;
        if (w.found) {
            const int mesh = __float_as_int(__ldg(S.tris + 3 * w.hit.tri + 1).w);
            const DevBsdf &B = S.bsdfs[S.meshes[mesh].bsdf];
            const bool map = B.type == kBumpMap || B.type == kNormalMap;
            type = B.deep ? kWfGenericQueue : wf_queue_of(B.type, B.textured != 0, map ? S.bsdfs[B.nested].type : -1);
            if (map && S.bsdfs[B.nested].deep) type = kWfGenericQueue;   // a map over a deep stack of layers
        }
        W.hit[slot] = make_float4(w.hit.t, w.hit.u, w.hit.v, __int_as_float(w.found ? w.hit.tri : -1));
        W.sq[type][warp_append_keyed(W.ctr->sq_count, type)] = slot;
    };
    if constexpr (kShared && kAccel == kAccelBvh8) {
        extern __shared__ uint2 wf_stack_smem[];
        float4 *rays = reinterpret_cast<float4 *>(wf_stack_smem + (size_t)blockDim.x * kShStack);
        trace_queue_shared<false>(S, wk, &W.ctr->ext_fetch, n, steps, min_idle, rays, load, store, ts);
    } else {
        trace_queue<false>(S, wk, &W.ctr->ext_fetch, n, steps, min_idle, load, store, ts);
    }
    unsigned long long nv = ts.nodes, nt = ts.tris;
    for (int o = 16; o > 0; o >>= 1) {
        nv += __shfl_down_sync(0xffffffffu, nv, o);
        nt += __shfl_down_sync(0xffffffffu, nt, o);
    }
    if (lane_id() == 0 && (nv || nt)) {
        atomicAdd(&W.ctr->node_visits, nv);
        atomicAdd(&W.ctr->tri_tests, nt);
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        atomicAdd(&W.ctr->rays, (unsigned long long)n);
        const unsigned k = W.ctr->log_n[0];   // one thread per launch; launches are stream-ordered
        if (k < (unsigned)kWfLaunchLog) W.ctr->log_rays[0][k] = n;
        W.ctr->log_n[0] = k + 1;
    }
}

// ------------------------------------------------------------ shade
__device__ __forceinline__ void finish(const WfState &W, int slot) { W.fq[warp_append(&W.ctr->fq_count)] = slot; }

// kMinBlocks = 0 leaves the register budget to the compiler; kLeanShade asks
// for four resident blocks of 256 threads (at most 64 registers): more warps
// to hide the latency of the path-state and scene gathers, at the price of
// some spilling.  Only the untextured queues (0-5) come in both budgets.
constexpr int kLeanShade = 4;
template <int kType, int kMinBlocks = 0>
__global__ void __launch_bounds__(256, kMinBlocks) wf_shade_kernel(DevScene S, WfState W, int nxt) {
    const int n = (int)W.ctr->sq_count[kType];
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const int slot = W.sq[kType][i];
        const float4 o4 = W.ray_o[slot], d4 = W.ray_d[slot];
        const V3 ro = v3(o4.x, o4.y, o4.z), rd = v3(d4.x, d4.y, d4.z);
        float4 b4 = W.beta[slot];
        V3 beta = v3(b4.x, b4.y, b4.z);
        float w_mats = b4.w;
        float4 p4 = W.pix[slot];
        const uint32_t dflags = (uint32_t)__float_as_int(p4.w);
        int depth = (int)(dflags & 0xffffu);
        uint32_t flags = dflags >> 16;
        const WfJob &J = W.jobs[__float_as_int(p4.z)];
        // radiance terms go to the path's accumulator with vector reductions
        // (as the unoccluded next-event terms do): shade neither reads nor
        // rewrites it
        if constexpr (kType == 0) {
            // miss (PathMISIntegrator.cpp:35-66); a new path's accumulator is zero
            V3 Le = v3(0, 0, 0);
            if (S.env_index >= 0 && (depth > 0 || !S.force_background)) Le = beta * env_eval(S, rd);
            else if (depth == 0) Le = ld3(S.background);
            if (!all_zero(Le)) red_add_v4(W.lacc + slot, Le.x, Le.y, Le.z, 0.0f);
            finish(W, slot);
            continue;
        } else {
            // queue -> top-level BSDF type (run-time dispatch for the generic
            // queue) and whether texture lookups are compiled in
            // kBumpQ: a bumpMap / normalMap over the rough type BT (the
            // records move through the perturbed frame, the nested BSDF is
            // evaluated with its type compiled in)
            constexpr bool kBumpQ = kType >= kWfBumpQueue0;
            constexpr int BT = kType == kWfGenericQueue
                                   ? -1
                                   : (kBumpQ ? kType - kWfBumpQueue0
                                             : (kType >= kWfTexturedQueue0 ? kType - kWfTexturedQueue0 : kType - 1));
            constexpr bool kTexQ = kType >= kWfGenericQueue;
            uint4 rs = W.rng[slot];
            Pcg32 rng;
            rng.state = (uint64_t)rs.x | ((uint64_t)rs.y << 32);
            rng.inc = (uint64_t)rs.z | ((uint64_t)rs.w << 32);
            float4 h4 = W.hit[slot];
            Hit h;
            h.t = h4.x; h.u = h4.y; h.v = h4.z; h.tri = __float_as_int(h4.w);
            Isect it;
            post_intersect(S, h, it);
            const DevMesh &m = S.meshes[it.mesh];
            const int bsdf = m.bsdf;
            if (m.emitter >= 0) {
                const DevAreaLight &AL = S.area_lights[__ldg(S.emitter_area + m.emitter)];
                ERec er;
                er.ref = ro; er.p = it.p; er.n = it.sh.n;
                V3 wi = er.p - er.ref; er.dist = norm(wi); er.wi = wi / er.dist;
                if (depth > 0) {
                    // MIS weight of the BSDF-sampled hit (PathMISIntegrator.cpp:122-140)
                    if (flags & kWfFlagForceMats) {
                        w_mats = 1.0f;
                    } else {
                        float4 pwi = W.prev_wi[slot], pwo = W.prev_wo[slot];
                        BRec pb;
                        pb.wi = v3(pwi.x, pwi.y, pwi.z);
                        pb.wo = v3(pwo.x, pwo.y, pwo.z);
                        pb.measure = __float_as_int(pwo.w);
                        pb.eta = 0.0f;
                        pb.tex = false;
                        pb.tu = pb.tv = 0.0f;
                        float plm = area_pdf(AL, er);
                        // a textured BSDF's pdf was taken when it sampled (its
                        // parameters depend on that vertex's texture lookups)
                        float pbm = S.bsdfs[__float_as_int(pwi.w)].textured ? W.prev_pdf[slot]
                                                                            : bsdf_pdf(S.bsdfs, __float_as_int(pwi.w), pb);
                        if (pbm + plm != 0.0f) w_mats = pbm / (pbm + plm);
                    }
                }
                const V3 Le = (beta * w_mats) * area_eval(AL, er);
                if (!all_zero(Le)) red_add_v4(W.lacc + slot, Le.x, Le.y, Le.z, 0.0f);
            }
            // screen-space partials of a camera ray's first hit (textured
            // materials only: Intersection::ComputeScreenSpacePartial)
            float4 duv = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
            BumpFrames bf;   // a bumpMap / normalMap vertex's frames (the generic queue only)
            if constexpr (BT < 0) {
                if (is_bump(S.bsdfs[bsdf])) bf = perturbed_frames(S, h, it, S.bsdfs[bsdf]);
            } else if constexpr (kBumpQ) {
                bf = perturbed_frames(S, h, it, S.bsdfs[bsdf]);
            }
            // what wireframe / curvature textures read at this vertex
            float3 geo = make_float3(INFINITY, 0.0f, 0.0f);
            if constexpr (kTexQ) {
                if (depth == 0 && S.ray_diff) {
                    V3 rx, ry;
                    camera_diff(S, J.cam, J.width, J.height, J.cam_aspect, p4.x, p4.y, rx, ry);
                    duv = screen_partials(S, h, it, ro, rx, ry);
                }
                if (S.bsdfs[bsdf].geo_tex) geo = tex_geometry(S, h, it);
            }
            // next-event estimation over every emitter (PathMISIntegrator.cpp:83-109)
            const V3 wi_local = to_local(it.sh, rd * -1.0f);
            for (int e = 0; e < S.nemitters; ++e) {
                ERec er;
                er.ref = it.p;
                er.dist = 0.0f;
                er.pdf = 0.0f;
                float u1 = rng.nextf();
                float ux = rng.nextf(), uy = rng.nextf();
                V3 ld = emitter_sample(S, e, er, ux, uy, u1);
                if (is_zero(ld)) continue;
                BRec br;
                br.wi = wi_local;
                br.wo = to_local(it.sh, er.wi);
                br.measure = kMeasureSolidAngle;
                br.eta = 0.0f;
                br.tex = kTexQ;   // lookups only in the kernels of textured materials
                br.tu = it.u;
                br.tv = it.v;
                if constexpr (kTexQ) {   // unread where lookups are compiled out
                    br.duv = duv;
                    br.geo = geo;
                }
                float pl = er.pdf;
                float pb;
                V3 f;
                if constexpr (BT < 0) {
                    pb = bsdf_pdf_b(S.bsdfs, bsdf, br, bf);
                    f = bsdf_eval_b(S.bsdfs, bsdf, br, bf);
                } else if constexpr (kBumpQ) {
                    pb = bump_pdf_t<BT>(S.bsdfs, bsdf, br, bf);
                    f = bump_eval_t<BT>(S.bsdfs, bsdf, br, bf);
                } else {
                    pb = bsdf_pdf_t<BT>(S.bsdfs, bsdf, br);
                    f = bsdf_eval_t<BT>(S.bsdfs, bsdf, br);
                }
                float w = (pl + pb != 0.0f) ? pl / (pl + pb) : 1.0f;
                float c = fabsf(br.wo.z);
                V3 contrib = v3((((beta.x * f.x) * c) * ld.x) * w, (((beta.y * f.y) * c) * ld.y) * w,
                                (((beta.z * f.z) * c) * ld.z) * w);
                if (all_zero(contrib)) continue;   // adds nothing whether occluded or not
                unsigned q = warp_append(&W.ctr->shadow_count);
                if (q < (unsigned)W.max_shadow) {
                    W.sh_o[q] = f4(it.p, __int_as_float(slot));
                    W.sh_d[q] = f4(er.p - it.p, 0.0f);
                    W.sh_c[q] = f4(contrib, 0.0f);
                }
            }
            // BSDF sampling (PathMISIntegrator.cpp:111-120)
            BRec br;
            br.wi = wi_local;
            br.wo = v3(0, 0, 0);
            br.measure = kMeasureUnknown;
            br.eta = 0.0f;
            br.tex = kTexQ;
            br.tu = it.u;
            br.tv = it.v;
            if constexpr (kTexQ) {
                br.duv = duv;
                br.geo = geo;
            }
            float sx = rng.nextf(), sy = rng.nextf();
            float u1 = needs_u1(S.bsdfs, bsdf) ? rng.nextf() : 0.0f;
            V3 F;
            if constexpr (BT < 0) F = bsdf_sample_b(S.bsdfs, bsdf, br, sx, sy, u1, bf);
            else if constexpr (kBumpQ) F = bump_sample_t<BT>(S.bsdfs, bsdf, br, sx, sy, u1, bf);
            else F = bsdf_sample_t<BT>(S.bsdfs, bsdf, br, sx, sy, u1);
            beta = beta * F;
            bool alive = !is_zero(beta);
            if (alive) {
                flags = (br.measure == kMeasureDiscrete) ? kWfFlagForceMats : 0u;
                if (flags) w_mats = 1.0f;
                // Russian roulette (PathMISIntegrator.cpp:142-151)
                if (depth >= J.rr_start) {
                    if (rng.nextf() < 0.95f) beta = beta * (1.0f / 0.95f);
                    else alive = false;
                }
                ++depth;
                if (depth >= J.depth) alive = false;   // the next hit would not be shaded
            }
            if (!alive) {
                finish(W, slot);
                continue;
            }
            W.ray_o[slot] = f4(it.p, kRayEps);
            W.ray_d[slot] = f4(to_world(it.sh, br.wo), __int_as_float(0x7f800000));
            W.beta[slot] = f4(beta, w_mats);
            W.pix[slot] = make_float4(p4.x, p4.y, p4.z, __int_as_float((int)((flags << 16) | (uint32_t)depth)));
            W.prev_wi[slot] = f4(br.wi, __int_as_float(bsdf));
            W.prev_wo[slot] = f4(br.wo, __int_as_float(br.measure));
            if constexpr (kTexQ) {
                // the MIS weight at an emitter hit next needs this BSDF's pdf of
                // the sampled direction (PathMISIntegrator.cpp:128)
                if (S.bsdfs[bsdf].textured && !(flags & kWfFlagForceMats)) {
                    BRec pr = br;
                    pr.eta = 0.0f;
                    if constexpr (BT < 0) W.prev_pdf[slot] = bsdf_pdf_b(S.bsdfs, bsdf, pr, bf);
                    else if constexpr (kBumpQ) W.prev_pdf[slot] = bump_pdf_t<BT>(S.bsdfs, bsdf, pr, bf);
                    else W.prev_pdf[slot] = bsdf_pdf_t<BT>(S.bsdfs, bsdf, pr);
                }
            }
            W.rng[slot] = make_uint4((uint32_t)rng.state, (uint32_t)(rng.state >> 32), (uint32_t)rng.inc,
                                     (uint32_t)(rng.inc >> 32));
            W.eq[nxt][warp_append(&W.ctr->eq_count[nxt])] = slot;
        }
    }
}

// ------------------------------------------------------------ shadow
// kShared: the warp's triangle tests shared out over its lanes (8-wide tree;
// the block's rays in dynamic shared memory after the stacks).
template <int kAccel, int kMinBlocks, bool kShared>
__global__ void __launch_bounds__(256, kMinBlocks) wf_shadow_kernel(DevScene S, WfState W, int steps, int min_idle) {
    const unsigned n = min(W.ctr->shadow_count, (unsigned)W.max_shadow);
    TravStats ts;
    WalkerOf<kAccel, SharedStack> wk;
    std::conditional_t<kAccel == kAccelBvh8, uint2, int> stack_mem[kAccel == kAccelBvh8 ? kStackSize - kShStack : kStackSize];
    if constexpr (kAccel == kAccelBvh8) {
        wk.stk = make_stack();
        wk.stk.spill = stack_mem;
    } else {
        wk.stack = stack_mem;
    }
    int slot = -1;
    auto load = [&](int i) {
        const float4 o = W.sh_o[i], d = W.sh_d[i];
        slot = __float_as_int(o.w);
        Ray r;
        r.o = v3(o.x, o.y, o.z);
        r.d = v3(d.x, d.y, d.z);
        r.tmin = kRayEps;
        r.tmax = 1.0f - kRayEps;
        return r;
    };
    auto store = [&](int i, const auto &w) {
        if (!w.found) {
            const float4 c = W.sh_c[i];
            red_add_v4(W.lacc + slot, c.x, c.y, c.z, 0.0f);
        }
    };
    if constexpr (kShared && kAccel == kAccelBvh8) {
        extern __shared__ uint2 wf_stack_smem[];
        float4 *rays = reinterpret_cast<float4 *>(wf_stack_smem + (size_t)blockDim.x * kShStack);
        trace_queue_shared<true>(S, wk, &W.ctr->sh_fetch, n, steps, min_idle, rays, load, store, ts);
    } else {
        trace_queue<true>(S, wk, &W.ctr->sh_fetch, n, steps, min_idle, load, store, ts);
    }
    unsigned long long nv = ts.nodes, nt = ts.tris;
    for (int o = 16; o > 0; o >>= 1) {
        nv += __shfl_down_sync(0xffffffffu, nv, o);
        nt += __shfl_down_sync(0xffffffffu, nt, o);
    }
    if (lane_id() == 0 && (nv || nt)) {
        atomicAdd(&W.ctr->node_visits_shadow, nv);
        atomicAdd(&W.ctr->tri_tests_shadow, nt);
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        atomicAdd(&W.ctr->shadow_rays, (unsigned long long)n);
        const unsigned k = W.ctr->log_n[1];
        if (k < (unsigned)kWfLaunchLog) W.ctr->log_rays[1][k] = n;
        W.ctr->log_n[1] = k + 1;
    }
}

// ------------------------------------------------------------ launchers
__host__ inline size_t wf_stack_bytes(int threads) { return (size_t)threads * kShStack * sizeof(uint2); }

// dynamic shared memory of a traversal launch: the short stacks, and the ray
// records where the triangle tests are shared out
__host__ inline size_t wf_shadow_smem(int threads, bool shared) {
    return wf_stack_bytes(threads) + (shared ? (size_t)threads * 2 * sizeof(float4) : 0);
}
template <int kAccel>
cudaError_t wf_launch_extend_t(const DevScene &S, const WfState &W, const WfLaunchConfig &C, int cur, cudaStream_t st) {
    const bool shared = kAccel == kAccelBvh8 && C.closest_tests == 2;
    const size_t smem = kAccel == kAccelBvh8 ? wf_shadow_smem(C.threads_extend, shared) : 0;
    const int a = C.fetch_steps, b = C.fetch_min_idle;
    if (shared) {
        if (C.lean_extend)
            wf_extend_kernel<kAccel, kLeanBlocks, true><<<C.blocks_extend, C.threads_extend, smem, st>>>(S, W, cur, a, b);
        else
            wf_extend_kernel<kAccel, 0, true><<<C.blocks_extend, C.threads_extend, smem, st>>>(S, W, cur, a, b);
    } else {
        if (C.lean_extend)
            wf_extend_kernel<kAccel, kLeanBlocks, false><<<C.blocks_extend, C.threads_extend, smem, st>>>(S, W, cur, a, b);
        else
            wf_extend_kernel<kAccel, 0, false><<<C.blocks_extend, C.threads_extend, smem, st>>>(S, W, cur, a, b);
    }
    return cudaGetLastError();
}
template <int kAccel>
cudaError_t wf_launch_shadow_t(const DevScene &S, const WfState &W, const WfLaunchConfig &C, cudaStream_t st) {
    const bool shared = kAccel == kAccelBvh8 && C.shadow_tests == 2;
    const size_t smem = kAccel == kAccelBvh8 ? wf_shadow_smem(C.threads_shadow, shared) : 0;
    DevScene SS = S;
    SS.postpone_any = S.postpone && C.shadow_tests == 1 ? 1 : 0;
    const int a = C.fetch_steps_shadow, b = C.fetch_min_idle_shadow;
    if (shared) {
        if (C.lean_shadow)
            wf_shadow_kernel<kAccel, kLeanBlocks, true><<<C.blocks_shadow, C.threads_shadow, smem, st>>>(SS, W, a, b);
        else
            wf_shadow_kernel<kAccel, 0, true><<<C.blocks_shadow, C.threads_shadow, smem, st>>>(SS, W, a, b);
    } else {
        if (C.lean_shadow)
            wf_shadow_kernel<kAccel, kLeanBlocks, false><<<C.blocks_shadow, C.threads_shadow, smem, st>>>(SS, W, a, b);
        else
            wf_shadow_kernel<kAccel, 0, false><<<C.blocks_shadow, C.threads_shadow, smem, st>>>(SS, W, a, b);
    }
    return cudaGetLastError();
}
// which: 0 extend, 2 shadow; lean: the kLeanBlocks register budget; shared:
// the kernel with shared triangle tests
template <int kAccel>
int wf_trace_occupancy_t(int which, int threads, bool lean, bool shared) {
    int n = 0;
    shared = shared && kAccel == kAccelBvh8;
    if (which == 0) {
        const size_t smem = kAccel == kAccelBvh8 ? wf_shadow_smem(threads, shared) : 0;
        if (shared) {
            if (lean)
                cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, wf_extend_kernel<kAccel, kLeanBlocks, true>, threads,
                                                              smem);
            else cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, wf_extend_kernel<kAccel, 0, true>, threads, smem);
        } else {
            if (lean)
                cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, wf_extend_kernel<kAccel, kLeanBlocks, false>, threads,
                                                              smem);
            else cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, wf_extend_kernel<kAccel, 0, false>, threads, smem);
        }
    } else {
        const size_t smem = kAccel == kAccelBvh8 ? wf_shadow_smem(threads, shared) : 0;
        if (shared) {
            if (lean)
                cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, wf_shadow_kernel<kAccel, kLeanBlocks, true>, threads,
                                                              smem);
            else cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, wf_shadow_kernel<kAccel, 0, true>, threads, smem);
        } else {
            if (lean)
                cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, wf_shadow_kernel<kAccel, kLeanBlocks, false>, threads,
                                                              smem);
            else cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, wf_shadow_kernel<kAccel, 0, false>, threads, smem);
        }
    }
    return n;
}
template <int kType>
cudaError_t wf_launch_shade_t(const DevScene &S, const WfState &W, const WfLaunchConfig &C, int nxt, cudaStream_t st) {
    if constexpr (kType <= 5) {
        if (C.lean_shade) {
            wf_shade_kernel<kType, kLeanShade><<<C.blocks_shade, C.threads_shade, 0, st>>>(S, W, nxt);
            return cudaGetLastError();
        }
    }
    wf_shade_kernel<kType><<<C.blocks_shade, C.threads_shade, 0, st>>>(S, W, nxt);
    return cudaGetLastError();
}
template <int kType>
int wf_shade_occupancy_t(int threads, bool lean) {
    int n = 0;
    if constexpr (kType <= 5) {
        if (lean) {
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, wf_shade_kernel<kType, kLeanShade>, threads, 0);
            return n;
        }
    }
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, wf_shade_kernel<kType>, threads, 0);
    return n;
}

}  // namespace hk
