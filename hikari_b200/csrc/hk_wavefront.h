// Wavefront pathMIS: device-side structures shared by hk_wavefront.cu and the
// host driver in hk_host.cpp.
//
// A pool of `capacity` path slots lives in HBM as structure-of-arrays.  One
// iteration runs: regen (splat finished paths, claim new work for finished and
// idle slots, generate camera rays) -> extend (closest hit of every queued ray,
// classify by material) -> shade<material> (emission, MIS, next-event shadow
// rays, BSDF sampling, Russian roulette) -> shadow (any-hit, add unoccluded
// next-event terms).  Kernels use fixed persistent grids and read queue sizes
// and the dispatch plan from HBM, so iterations are captured once in a CUDA
// graph and replayed; jobs and plans change between replays.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>

#include "hk_device.h"

namespace hk {

// Shade queues: 0 miss; 1..5 the rough BSDF types without textures (type +
// 1), each shaded by a kernel compiled for that type with texture lookups
// compiled out; 6 the smooth, twoSided, bump- and normal-mapped BSDFs, shaded
// by one kernel that dispatches at run time; 7..11 the rough BSDF types with
// textured parameters (type + 7), each shaded by a kernel compiled for that
// type with texture lookups.
constexpr int kWfGenericQueue = 6;
constexpr int kWfTexturedQueue0 = 7;
constexpr int kWfBumpQueue0 = kWfTexturedQueue0 + kRoughCoating + 1;   // bumpMap / normalMap over a rough type
constexpr int kWfTypes = kWfBumpQueue0 + kRoughCoating + 1;
// Shade queue of a hit's top-level BSDF: 0 the miss queue; 1-5 the rough types
// without textures; 7-11 the same with textures; 12-16 bumpMap / normalMap
// wrapping a rough type (nested_type); 6 everything else (smooth BSDFs,
// twoSided, maps over them), dispatched at run time.
__host__ __device__ constexpr int wf_queue_of(int bsdf_type, bool textured = false, int nested_type = -1) {
    return bsdf_type <= kRoughCoating
               ? (textured ? kWfTexturedQueue0 + bsdf_type : bsdf_type + 1)
               : ((bsdf_type == kBumpMap || bsdf_type == kNormalMap) && nested_type >= 0 && nested_type <= kRoughCoating
                      ? kWfBumpQueue0 + nested_type
                      : kWfGenericQueue);
}
constexpr int kWfMaxJobs = 1024;   // job table entries of one engine
constexpr int kWfMaxSegs = 4096;   // pieces of one dispatch plan
constexpr int kWfTileSide = 16;
constexpr int kWfTilePixels = kWfTileSide * kWfTileSide;

// One image being rendered (a job): a view of the scene with its own film and
// resolution.  Jobs live in a table of kWfMaxJobs entries; a path records the
// index of its job.
struct WfJob {
    float *film;                    // (height+2B) x (width+2B) x 4, 16-byte aligned
    float cam[12];                  // camera-to-world rows (translation divided by w)
    unsigned long long *finished;   // work items of this job finished (device counter)
    uint64_t seed;
    uint64_t work_count;            // tiles * spp * 256 work items
    uint32_t spp, sample_offset, image_index, tiles_x;
    uint32_t width, height;
    float cam_aspect;               // width / height (PerspectiveCamera::Activate)
    int32_t depth, rr_start;
    // order of the job's work items: 0 tile by tile (all samples of a tile,
    // then the next tile: partial images show finished tiles); 1 sample by
    // sample (every tile's sample s, then s + 1: the paths in flight splat
    // over the whole image rather than over a few tiles)
    int32_t sample_major;
};

// One piece of the dispatch plan: work items [plan_begin, next piece's
// plan_begin) of the plan are the job's items starting at job_begin.  The host
// writes a plan between chunks of iterations; slots claim plan items in order.
struct WfSeg {
    uint64_t plan_begin;
    uint64_t job_begin;
    int32_t job;
    int32_t pad;
};

// Device-wide counters of the engine (one struct in HBM).  The first three
// fields are the dispatch head, rewritten by the host with each plan.
constexpr int kWfLaunchLog = 1024;   // launches whose ray counts the counters keep

struct WfCounters {
    unsigned long long next_work;      // next plan item to hand out
    unsigned long long total_work;     // plan items in the current plan
    unsigned int seg_count;            // pieces in the current plan
    unsigned int pad0;
    unsigned int eq_count[2];          // extend queues (ping-pong)
    unsigned int idle_count[2];        // slots without a path (ping-pong)
    unsigned int sq_count[kWfTypes];   // shade queues per material type
    unsigned int fq_count;             // finished paths awaiting splat + regeneration
    unsigned int shadow_count;         // next-event shadow rays
    unsigned int active;               // paths in flight
    unsigned int ext_fetch, sh_fetch;  // rays claimed by the extend / shadow kernels (dynamic fetch)
    unsigned int pad1;
    unsigned long long rays, shadow_rays, dropped;
    unsigned long long node_visits, tri_tests;                 // closest-hit traversal (extend)
    unsigned long long node_visits_shadow, tri_tests_shadow;   // any-hit traversal (shadow)
    // rays of each extend (0) / shadow (1) launch since the last reset, in
    // launch order (profiling; the host's status copies stop before it)
    unsigned int log_n[2];
    unsigned int log_rays[2][kWfLaunchLog];
};

// Path state: one 160-byte record per slot, five 32-byte sectors, the fields
// a kernel reads together in one sector: (ray o, ray d) extend and shade;
// (throughput, pixel) shade and regen; (rng, hit) shade; (previous BSDF record
// wi, wo) shade at emitter hits; (radiance, previous pdf) regen and the
// next-event reductions.  Slots are visited in queue order, i.e. scattered, so
// a separate array per field would fetch a whole sector for each 16-byte field.
constexpr size_t kSlotBytes = 160;
// One field of every slot's record: f[slot] is the field of that slot.
template <class T>
struct SlotField {
    T *p;   // the field in slot 0's record
    __host__ __device__ __forceinline__ T &operator[](size_t slot) const {
        return *reinterpret_cast<T *>(reinterpret_cast<char *>(p) + slot * kSlotBytes);
    }
    __host__ __device__ __forceinline__ T *operator+(size_t slot) const { return &(*this)[slot]; }
};

struct WfState {
    int capacity;
    int max_shadow;                    // shadow queue capacity
    // per-slot path state (byte offset in the slot's record)
    SlotField<float4> ray_o;      //   0: o.xyz, tmin
    SlotField<float4> ray_d;      //  16: d.xyz, tmax
    SlotField<float4> beta;       //  32: throughput.xyz, w_mats
    SlotField<float4> pix;        //  48: film x, film y, bits(job), bits(depth | flags << 16)
    SlotField<uint4> rng;         //  64: pcg32 state, increment
    SlotField<float4> hit;        //  80: t, u, v, bits(tri in leaf order or -1)
    SlotField<float4> prev_wi;    //  96: previous vertex: BSDF record wi.xyz, bits(bsdf id)
    SlotField<float4> prev_wo;    // 112: previous vertex: BSDF record wo.xyz, bits(measure)
    SlotField<float4> lacc;       // 128: radiance.xyz (next-event terms added atomically), -
    SlotField<float> prev_pdf;    // 144: previous vertex: its BSDF's pdf of the sampled direction (textured
                                  //      materials only)
    // queues
    int *eq[2];
    int *idle[2];
    int *sq[kWfTypes];
    int *fq;
    float4 *sh_o;       // shadow origin.xyz, bits(slot)
    float4 *sh_d;       // shadow direction.xyz (unnormalised), -
    float4 *sh_c;       // contribution.xyz, -
    WfCounters *ctr;
    const WfJob *jobs;
    const WfSeg *segs;
};

// flags in the high half of pix.w
constexpr uint32_t kWfFlagForceMats = 1u;   // previous BSDF sample was EDiscrete

struct WfLaunchConfig {
    int blocks_extend, threads_extend;
    int blocks_shade, threads_shade;
    int blocks_shadow, threads_shadow;
    int blocks_regen, threads_regen;
    int fetch_steps, fetch_min_idle;                 // dynamic ray fetch of the extend kernel
    int fetch_steps_shadow, fetch_min_idle_shadow;   // and of the shadow kernel
    int lean_extend, lean_shadow;                    // traversal kernels with the smaller register budget
    int lean_shade;                                  // untextured shade kernels with the smaller register budget
    int shadow_tests;   // shadow rays' triangle tests: 0 per lane, 1 postponed, 2 shared over the warp
    int closest_tests;  // closest-hit rays' triangle tests: 0 per lane (postponed where the tree allows), 2 shared
};

// empty pool: every slot idle, queues and statistics zero (the dispatch head is the host's)
cudaError_t wf_launch_init(const WfState &W, cudaStream_t st);
// one iteration with extend queue `cur` (0/1)
cudaError_t wf_launch_iteration(const DevScene &S, const WfState &W, const WfLaunchConfig &C, int cur, cudaStream_t st);
// one phase of an iteration: 0 regen + reset, 1 extend, 2 shade (all materials), 3 shadow
cudaError_t wf_launch_phase(const DevScene &S, const WfState &W, const WfLaunchConfig &C, int cur, int phase,
                            cudaStream_t st);
// out[0..6] += rays, shadow rays, dropped, node visits, triangle tests, shadow node visits, shadow tests
cudaError_t wf_launch_counters_add(const WfState &W, unsigned long long *out, cudaStream_t st);
// resident blocks per SM of a kernel (which: 0 extend, 1 shade, 2 shadow, 3
// regen); lean: the traversal kernels' smaller register budget
int wf_occupancy(int which, int threads, int accel, bool lean = false, bool shared = false);

}  // namespace hk
