// Wavefront pathMIS on sm_100a: the integrator of
// src/integrator/PathMISIntegrator.cpp:16-157 split at its ray casts so that
// every kernel runs one kind of work over a compacted queue.
//
//   regen   finished paths are splatted (ImageBlock::Put, src/core/Block.cpp:95)
//           into their job's film with 128-bit vector reductions; slots claim
//           new (job, tile, sample, pixel) work and start camera rays
//   extend  closest hit of every queued ray; the hit's material type picks
//           the shade queue
//   shade<T> one kernel per top-level BSDF type (and one for misses): emitter
//           hit with its MIS weight, next-event estimation over every emitter
//           (shadow rays queued with their contribution), BSDF sampling,
//           Russian roulette
//   shadow  any-hit of every queued shadow ray; unoccluded contributions are
//           added to their path's radiance
//
// This file holds regen and the launch sequence; the queue helpers and the
// extend / shade / shadow kernels are in hk_wf_kernels.cuh.
//
// The estimator is the reference's: the next-event MIS weight of an
// unoccluded emitter is its own pl / (pl + pb) (the reference updates its
// carried weight exactly when the shadow ray is unoccluded, and uses it right
// away); the emitter-hit weight is computed from the previous vertex's BSDF
// record and forced to 1 after an EDiscrete sample; Russian roulette runs
// before the continuation ray is traced (the reference traces first and
// discards the hit of a terminated path, which changes nothing).
#include "hk_wf_kernels.cuh"

namespace hk {

// The traversal and shade kernels are instantiated in hk_wf_trace_*.cu and
// hk_wf_shade_*.cu; this file only calls their launchers.
extern template cudaError_t wf_launch_extend_t<kAccelBvh8>(const DevScene &, const WfState &, const WfLaunchConfig &, int, cudaStream_t);
extern template cudaError_t wf_launch_extend_t<kAccelBvh2>(const DevScene &, const WfState &, const WfLaunchConfig &, int, cudaStream_t);
extern template cudaError_t wf_launch_shadow_t<kAccelBvh8>(const DevScene &, const WfState &, const WfLaunchConfig &, cudaStream_t);
extern template cudaError_t wf_launch_shadow_t<kAccelBvh2>(const DevScene &, const WfState &, const WfLaunchConfig &, cudaStream_t);
extern template int wf_trace_occupancy_t<kAccelBvh8>(int, int, bool, bool);
extern template int wf_trace_occupancy_t<kAccelBvh2>(int, int, bool, bool);
#define HK_WF_SHADE_EXTERN(K)                                                                                           \
    extern template cudaError_t wf_launch_shade_t<K>(const DevScene &, const WfState &, const WfLaunchConfig &, int, \
                                                     cudaStream_t);                                                 \
    extern template int wf_shade_occupancy_t<K>(int, bool)
HK_WF_SHADE_EXTERN(0);
HK_WF_SHADE_EXTERN(1);
HK_WF_SHADE_EXTERN(2);
HK_WF_SHADE_EXTERN(3);
HK_WF_SHADE_EXTERN(4);
HK_WF_SHADE_EXTERN(5);
HK_WF_SHADE_EXTERN(6);
HK_WF_SHADE_EXTERN(7);
HK_WF_SHADE_EXTERN(8);
HK_WF_SHADE_EXTERN(9);
HK_WF_SHADE_EXTERN(10);
HK_WF_SHADE_EXTERN(11);
HK_WF_SHADE_EXTERN(12);
HK_WF_SHADE_EXTERN(13);
HK_WF_SHADE_EXTERN(14);
HK_WF_SHADE_EXTERN(15);
HK_WF_SHADE_EXTERN(16);
#undef HK_WF_SHADE_EXTERN
static_assert(kWfTypes == 17, "launch_shade_all launches one kernel per shade queue");

// ------------------------------------------------------------ regen
// Splat and retire the finished paths, then give every finished or idle slot
// new work from the dispatch plan; slots that find none wait in the next idle
// list.  Queues read here: fq, idle[cur]; written: eq[cur], idle[cur ^ 1].
// Slot i of the n slots that want work (finished paths first, then idle
// slots) takes plan item next_work + i: the items are dealt without an
// atomic, and wf_reset_kernel advances next_work by n afterwards.  An item
// whose pixel lies outside its image (the partial tiles at the right and
// bottom edges) counts as work done and leaves its slot idle until the next
// iteration.  Appends to the extend and idle lists, the per-job finished
// counts and the change of the in-flight count are gathered per block in
// shared memory and added once per block and round: a global atomic per warp
// on a handful of addresses serialises at the L2.
__global__ void __launch_bounds__(256) wf_regen_kernel(DevScene S, WfState W, int cur) {
    __shared__ unsigned s_finished[kWfMaxJobs];
    __shared__ int s_active;
    __shared__ unsigned s_warp[2][8];   // per-warp counts, then offsets, of the extend / idle appends
    __shared__ unsigned s_base[2];
    for (int k = threadIdx.x; k < kWfMaxJobs; k += blockDim.x) s_finished[k] = 0u;
    if (threadIdx.x == 0) s_active = 0;
    __syncthreads();
    const int nf = (int)W.ctr->fq_count;
    const int n = nf + (int)W.ctr->idle_count[cur];
    const uint64_t total = W.ctr->total_work;
    const uint64_t first = W.ctr->next_work;
    const int nseg = (int)W.ctr->seg_count;
    const unsigned lane = lane_id(), warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
    unsigned long long dropped = 0;
    int active_delta = 0;
    for (int i0 = blockIdx.x * blockDim.x; i0 < n; i0 += gridDim.x * blockDim.x) {   // block-uniform rounds
        const int i = i0 + (int)threadIdx.x;
        int slot = -1;
        bool started = false;
        if (i < n) {
            if (i < nf) {
                slot = W.fq[i];
                float4 p = W.pix[slot];
                float4 L = W.lacc[slot];
                const int pj = __float_as_int(p.z);
                const WfJob &J = W.jobs[pj];
                V3 val = v3(L.x, L.y, L.z);
                if (is_valid(val)) splat_global(S, J, p.x, p.y, val);
                else ++dropped;
                atomicAdd(&s_finished[pj], 1u);
                --active_delta;
            } else {
                slot = W.idle[cur][i - nf];
            }
            const uint64_t w = first + (uint64_t)i;
            if (w < total) {
                const WfSeg &G = W.segs[find_seg(W, w, nseg)];
                const int j = G.job;
                const WfJob &J = W.jobs[j];
                const uint64_t l = G.job_begin + (w - G.plan_begin);
                const uint32_t p = (uint32_t)(l % kWfTilePixels);
                const uint64_t ts = l / kWfTilePixels;
                uint32_t s, t;
                if (J.sample_major) {
                    const uint64_t ntiles = J.work_count / ((uint64_t)J.spp * kWfTilePixels);
                    t = (uint32_t)(ts % ntiles);
                    s = (uint32_t)(ts / ntiles);
                } else {
                    s = (uint32_t)(ts % J.spp);
                    t = (uint32_t)(ts / J.spp);
                }
                const uint32_t x = (t % J.tiles_x) * kWfTileSide + p % kWfTileSide;
                const uint32_t y = (t / J.tiles_x) * kWfTileSide + p / kWfTileSide;
                if (x >= J.width || y >= J.height) {
                    atomicAdd(&s_finished[j], 1u);   // counted as work done: no path
                } else {
                    Pcg32 rng;
                    rng.seed(wf_mix_seed(J.seed, (uint64_t)J.sample_offset + s),
                             (uint64_t)y * J.width + x + (uint64_t)J.image_index * J.width * J.height);
                    float px = (float)x + rng.nextf(), py = (float)y + rng.nextf();
                    Ray r = camera_ray_job(S, J, px, py);
                    W.ray_o[slot] = f4(r.o, r.tmin);
                    W.ray_d[slot] = f4(r.d, r.tmax);
                    W.beta[slot] = make_float4(1.0f, 1.0f, 1.0f, 1.0f);
                    W.lacc[slot] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
                    W.pix[slot] = make_float4(px, py, __int_as_float(j), __int_as_float(0));
                    W.rng[slot] = make_uint4((uint32_t)rng.state, (uint32_t)(rng.state >> 32), (uint32_t)rng.inc,
                                             (uint32_t)(rng.inc >> 32));
                    ++active_delta;
                    started = true;
                }
            }
        }
        // block-aggregated appends: one atomic per list per block and round
        const bool to_idle = i < n && !started;
        const unsigned be = __ballot_sync(0xffffffffu, started), bi = __ballot_sync(0xffffffffu, to_idle);
        if (lane == 0) {
            s_warp[0][warp] = __popc(be);
            s_warp[1][warp] = __popc(bi);
        }
        __syncthreads();
        if (threadIdx.x < 2) {
            unsigned sum = 0;
            for (unsigned k = 0; k < nwarps; ++k) {
                const unsigned c = s_warp[threadIdx.x][k];
                s_warp[threadIdx.x][k] = sum;
                sum += c;
            }
            unsigned *ctr = threadIdx.x == 0 ? &W.ctr->eq_count[cur] : &W.ctr->idle_count[cur ^ 1];
            s_base[threadIdx.x] = sum ? atomicAdd(ctr, sum) : 0u;
        }
        __syncthreads();
        const unsigned below = (1u << lane) - 1u;
        if (started) W.eq[cur][s_base[0] + s_warp[0][warp] + __popc(be & below)] = slot;
        if (to_idle) W.idle[cur ^ 1][s_base[1] + s_warp[1][warp] + __popc(bi & below)] = slot;
        __syncthreads();   // s_warp and s_base are rewritten by the next round
    }
    if (dropped) atomicAdd(&W.ctr->dropped, dropped);
    // one atomic per warp into the block, one per block and job into HBM
    for (int o = 16; o > 0; o >>= 1) active_delta += __shfl_down_sync(0xffffffffu, active_delta, o);
    if (lane == 0 && active_delta) atomicAdd(&s_active, active_delta);
    __syncthreads();
    for (int k = threadIdx.x; k < kWfMaxJobs; k += blockDim.x)
        if (s_finished[k]) atomicAdd(W.jobs[k].finished, (unsigned long long)s_finished[k]);
    if (threadIdx.x == 0 && s_active) atomicAdd(&W.ctr->active, (unsigned)s_active);
}

// Reset the counters of the queues consumed by regen and of those the next
// phases fill.
__global__ void wf_reset_kernel(WfState W, int cur) {
    if (threadIdx.x == 0) {
        // regen dealt plan items next_work .. next_work + n - 1 to its n slots
        const unsigned long long dealt = W.ctr->next_work + W.ctr->fq_count + W.ctr->idle_count[cur];
        W.ctr->next_work = dealt < W.ctr->total_work ? dealt : W.ctr->total_work;
        W.ctr->fq_count = 0;
        W.ctr->idle_count[cur] = 0;
        W.ctr->eq_count[cur ^ 1] = 0;
        W.ctr->shadow_count = 0;
        W.ctr->ext_fetch = 0;
        W.ctr->sh_fetch = 0;
    }
    if (threadIdx.x < kWfTypes) W.ctr->sq_count[threadIdx.x] = 0;
}

// Empty pool: every slot in idle list 0, all queues and statistics zero.
__global__ void wf_init_kernel(WfState W) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < W.capacity; i += gridDim.x * blockDim.x) W.idle[0][i] = i;
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        WfCounters *c = W.ctr;
        c->eq_count[0] = c->eq_count[1] = 0;
        c->idle_count[0] = (unsigned)W.capacity;
        c->idle_count[1] = 0;
        for (int t = 0; t < kWfTypes; ++t) c->sq_count[t] = 0;
        c->fq_count = c->shadow_count = c->active = 0;
        c->ext_fetch = c->sh_fetch = 0;
        c->rays = c->shadow_rays = c->dropped = 0;
        c->node_visits = c->tri_tests = c->node_visits_shadow = c->tri_tests_shadow = 0;
        c->log_n[0] = c->log_n[1] = 0;
    }
}

// Add the engine's statistics to a caller's 7-slot u64 array.
__global__ void wf_counters_add_kernel(const WfCounters *c, unsigned long long *out) {
    if (threadIdx.x != 0) return;
    out[0] += c->rays;
    out[1] += c->shadow_rays;
    out[2] += c->dropped;
    out[3] += c->node_visits;
    out[4] += c->tri_tests;
    out[5] += c->node_visits_shadow;
    out[6] += c->tri_tests_shadow;
}

// ------------------------------------------------------------ launchers
static cudaError_t launch_extend(const DevScene &S, const WfState &W, const WfLaunchConfig &C, int cur, cudaStream_t st) {
    return S.accel == kAccelBvh8 ? wf_launch_extend_t<kAccelBvh8>(S, W, C, cur, st) : wf_launch_extend_t<kAccelBvh2>(S, W, C, cur, st);
}
static cudaError_t launch_shadow(const DevScene &S, const WfState &W, const WfLaunchConfig &C, cudaStream_t st) {
    return S.accel == kAccelBvh8 ? wf_launch_shadow_t<kAccelBvh8>(S, W, C, st) : wf_launch_shadow_t<kAccelBvh2>(S, W, C, st);
}
static cudaError_t launch_shade_all(const DevScene &S, const WfState &W, const WfLaunchConfig &C, int nxt, cudaStream_t st) {
    wf_launch_shade_t<0>(S, W, C, nxt, st);
    wf_launch_shade_t<1>(S, W, C, nxt, st);
    wf_launch_shade_t<2>(S, W, C, nxt, st);
    wf_launch_shade_t<3>(S, W, C, nxt, st);
    wf_launch_shade_t<4>(S, W, C, nxt, st);
    wf_launch_shade_t<5>(S, W, C, nxt, st);
    wf_launch_shade_t<6>(S, W, C, nxt, st);
    wf_launch_shade_t<7>(S, W, C, nxt, st);
    wf_launch_shade_t<8>(S, W, C, nxt, st);
    wf_launch_shade_t<9>(S, W, C, nxt, st);
    wf_launch_shade_t<10>(S, W, C, nxt, st);
    wf_launch_shade_t<11>(S, W, C, nxt, st);
    wf_launch_shade_t<12>(S, W, C, nxt, st);
    wf_launch_shade_t<13>(S, W, C, nxt, st);
    wf_launch_shade_t<14>(S, W, C, nxt, st);
    wf_launch_shade_t<15>(S, W, C, nxt, st);
    return wf_launch_shade_t<16>(S, W, C, nxt, st);
}

cudaError_t wf_launch_counters_add(const WfState &W, unsigned long long *out, cudaStream_t st) {
    wf_counters_add_kernel<<<1, 32, 0, st>>>(W.ctr, out);
    return cudaGetLastError();
}

cudaError_t wf_launch_init(const WfState &W, cudaStream_t st) {
    wf_init_kernel<<<(W.capacity + 255) / 256, 256, 0, st>>>(W);
    return cudaGetLastError();
}

cudaError_t wf_launch_iteration(const DevScene &S, const WfState &W, const WfLaunchConfig &C, int cur, cudaStream_t st) {
    const int nxt = cur ^ 1;
    wf_regen_kernel<<<C.blocks_regen, C.threads_regen, 0, st>>>(S, W, cur);
    wf_reset_kernel<<<1, 32, 0, st>>>(W, cur);
    launch_extend(S, W, C, cur, st);
    launch_shade_all(S, W, C, nxt, st);
    launch_shadow(S, W, C, st);
    return cudaGetLastError();
}

cudaError_t wf_launch_phase(const DevScene &S, const WfState &W, const WfLaunchConfig &C, int cur, int phase,
                            cudaStream_t st) {
    const int nxt = cur ^ 1;
    switch (phase) {
    case 0:
        wf_regen_kernel<<<C.blocks_regen, C.threads_regen, 0, st>>>(S, W, cur);
        wf_reset_kernel<<<1, 32, 0, st>>>(W, cur);
        break;
    case 1: launch_extend(S, W, C, cur, st); break;
    case 2: launch_shade_all(S, W, C, nxt, st); break;
    default: launch_shadow(S, W, C, st); break;
    }
    return cudaGetLastError();
}

int wf_occupancy(int which, int threads, int accel, bool lean, bool shared) {
    int n = 0;
    const bool w8 = accel == kAccelBvh8;
    switch (which) {
    case 0:
    case 2:
        return w8 ? wf_trace_occupancy_t<kAccelBvh8>(which, threads, lean, shared)
                  : wf_trace_occupancy_t<kAccelBvh2>(which, threads, lean, shared);
    case 1: return wf_shade_occupancy_t<5>(threads, lean);
    default: cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, wf_regen_kernel, threads, 0); break;
    }
    return n;
}

}  // namespace hk
