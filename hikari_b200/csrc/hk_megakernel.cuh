// The plain megakernel (the drop-in): PathMISIntegrator::Li per thread,
// persistent CTAs pulling (tile, sample-chunk) work items, film splatted
// through the reconstruction filter into a shared-memory tile and flushed
// once per item.  Each instantiation (tree kind x texture lookups) is compiled
// in its own translation unit (hk_render_*.cu).
#pragma once
#include "hk_kernels.h"
#include "hk_shading.cuh"

namespace hk {

// ------------------------------------------------------------ integrator
struct PathCounters {
    uint32_t rays, shadow;
    TravStats trav;
};

__device__ __forceinline__ uint32_t mesh_emitter(const DevScene &S, int mesh) { return (uint32_t)S.meshes[mesh].emitter; }

// PathMISIntegrator::Li (src/integrator/PathMISIntegrator.cpp:16-157), with
// every reference quirk: Russian roulette p = 0.95 from depth rr_start
// (reference: every bounce), NEE over all emitters, MIS state carried across
// bounces, unweighted environment on BSDF-sampled misses, the EDiscrete
// override and Eigen's |c| <= 1e-5 zero test on throughput and NEE values.
// kTex: the scene has textured materials (texture lookups compiled in); the
// first hit's texture lookups filter with the camera ray's differentials
// through film position (px, py), later hits have none (src/core/
// Intersection.cpp:35).
template <int kAccel, bool kTex>
__device__ V3 li_pathmis(const DevScene &S, Pcg32 &rng, Ray ray, float px, float py, int depth_max, int rr_start,
                         PathCounters &pc) {
    Hit hn, hc;   // the next hit; the current vertex's hit
    bool found_next = false;
    Isect it, itn;
    float4 duv = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    BumpFrames bf;   // a bumpMap / normalMap vertex's frames (kTex only)
    V3 L = v3(0, 0, 0), beta = v3(1, 1, 1);
    int depth = 0;
    float w_ems = 1.0f, w_mats = 1.0f;
    const bool has_env = S.env_index >= 0;
    while (depth < depth_max) {
        if (depth == 0) {
            Hit h;
            pc.rays++;
            if (!trace<kAccel, false>(S, ray, h, pc.trav)) {
                if (has_env && !S.force_background) { L = L + beta * env_eval(S, ray.d); break; }
                return ld3(S.background);
            }
            post_intersect(S, h, it);
            hc = h;
            if (kTex && S.ray_diff) {
                V3 rx, ry;
                camera_diff(S, S.cam, S.width, S.height, S.cam_aspect, px, py, rx, ry);
                duv = screen_partials(S, h, it, ray.o, rx, ry);
            }
        } else {
            if (kTex) duv = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
            if (found_next) {
                it = itn;
                hc = hn;
            } else {
                if (has_env) L = L + beta * env_eval(S, ray.d);
                break;
            }
        }
        const DevMesh &m = S.meshes[it.mesh];
        const int bsdf = m.bsdf;
        float3 geo = make_float3(INFINITY, 0.0f, 0.0f);
        if constexpr (kTex) {
            if (is_bump(S.bsdfs[bsdf])) bf = perturbed_frames(S, hc, it, S.bsdfs[bsdf]);
            if (S.bsdfs[bsdf].geo_tex) geo = tex_geometry(S, hc, it);
        }
        if (m.emitter >= 0) {
            const DevAreaLight &AL = S.area_lights[__ldg(S.emitter_area + m.emitter)];
            ERec er;
            er.ref = ray.o; er.p = it.p; er.n = it.sh.n;
            V3 wi = er.p - er.ref; er.dist = norm(wi); er.wi = wi / er.dist;
            L = L + (beta * w_mats) * area_eval(AL, er);
        }
        for (int e = 0; e < S.nemitters; ++e) {
            ERec er;
            er.ref = it.p;
            er.dist = 0.0f;
            er.pdf = 0.0f;
            float u1 = rng.nextf();
            float ux = rng.nextf(), uy = rng.nextf();
            V3 ld = emitter_sample(S, e, er, ux, uy, u1);
            float pl = er.pdf;
            if (!is_zero(ld)) {
                // the BSDF term first, the shadow ray only for a non-zero
                // contribution (an occluded ray adds nothing either way; the
                // reference updates WeightEMS only for an unoccluded ray, and
                // every use recomputes it, as the emitter pdf of a non-zero
                // sample is positive)
                BRec br;
                br.wi = to_local(it.sh, ray.d * -1.0f);
                br.wo = to_local(it.sh, er.wi);
                br.measure = kMeasureSolidAngle;
                br.eta = 0.0f;
                br.tu = it.u; br.tv = it.v; br.tex = kTex; br.duv = duv; br.geo = geo;
                float pb;
                V3 f;
                if constexpr (kTex) {
                    pb = bsdf_pdf_b(S.bsdfs, bsdf, br, bf);
                    f = bsdf_eval_b(S.bsdfs, bsdf, br, bf);
                } else {
                    pb = bsdf_pdf(S.bsdfs, bsdf, br);
                    f = bsdf_eval(S.bsdfs, bsdf, br);
                }
                const float w = (pl + pb != 0.0f) ? pl / (pl + pb) : w_ems;
                const float c = fabsf(br.wo.z);
                const V3 contrib = v3((((beta.x * f.x) * c) * ld.x) * w, (((beta.y * f.y) * c) * ld.y) * w,
                                      (((beta.z * f.z) * c) * ld.z) * w);
                if (!all_zero(contrib)) {
                    Ray sr;
                    sr.o = it.p; sr.d = er.p - it.p; sr.tmin = kRayEps; sr.tmax = 1.0f - kRayEps;
                    Hit sh;
                    pc.shadow++;
                    if (!trace<kAccel, true>(S, sr, sh, pc.trav)) {
                        w_ems = w;
                        L = L + contrib;
                    }
                }
            }
        }
        BRec br;
        br.wi = to_local(it.sh, ray.d * -1.0f);
        br.wo = v3(0, 0, 0);
        br.measure = kMeasureUnknown;
        br.eta = 0.0f;
        br.tu = it.u; br.tv = it.v; br.tex = kTex; br.duv = duv; br.geo = geo;
        float sx = rng.nextf(), sy = rng.nextf();
        float u1 = needs_u1(S.bsdfs, bsdf) ? rng.nextf() : 0.0f;
        V3 F;
        if constexpr (kTex) F = bsdf_sample_b(S.bsdfs, bsdf, br, sx, sy, u1, bf);
        else F = bsdf_sample(S.bsdfs, bsdf, br, sx, sy, u1);
        ray.o = it.p;
        ray.d = to_world(it.sh, br.wo);
        ray.tmin = kRayEps;
        ray.tmax = __int_as_float(0x7f800000);
        beta = beta * F;
        if (is_zero(beta)) break;
        // Russian roulette (PathMISIntegrator.cpp:142-151) and the depth bound
        // before the continuation ray is traced: the reference traces first and
        // ends the path afterwards, discarding the hit; the trace draws no
        // random numbers, so the stream is consumed in the same order
        if (depth >= rr_start) {
            if (rng.nextf() < 0.95f) beta = beta * (1.0f / 0.95f);
            else break;
        }
        ++depth;
        if (depth >= depth_max) break;   // the next hit would not be shaded
        pc.rays++;
        found_next = trace<kAccel, false>(S, ray, hn, pc.trav);
        if (found_next) {
            post_intersect(S, hn, itn);
            const DevMesh &mn = S.meshes[itn.mesh];
            if (mn.emitter >= 0) {
                const DevAreaLight &AL = S.area_lights[__ldg(S.emitter_area + mn.emitter)];
                ERec er;
                er.ref = it.p; er.p = itn.p; er.n = itn.sh.n;
                V3 wi = er.p - er.ref; er.dist = norm(wi); er.wi = wi / er.dist;
                float plm = area_pdf(AL, er);
                float pbm;
                if constexpr (kTex) pbm = bsdf_pdf_b(S.bsdfs, bsdf, br, bf);
                else pbm = bsdf_pdf(S.bsdfs, bsdf, br);
                if (pbm + plm != 0.0f) w_mats = pbm / (pbm + plm);
            }
        }
        if (br.measure == kMeasureDiscrete) { w_ems = 0.0f; w_mats = 1.0f; }
    }
    return L;
}

// ------------------------------------------------------------ megakernel
// ImageBlock::Put (src/core/Block.cpp:95) into a shared tile covering film
// columns [fx0, fx0 + tw) and rows [fy0, fy0 + th).
__device__ __forceinline__ void splat_shared(const DevScene &S, float *tile, int tw, int th, int fx0, int fy0, int FW,
                                             int FH, float px, float py, V3 val) {
    const int B = S.border;
    float cx = px - 0.5f - (0 - B), cy = py - 0.5f - (0 - B);
    int x0 = max((int)ceilf(cx - S.filt_radius), 0), y0 = max((int)ceilf(cy - S.filt_radius), 0);
    int x1 = min((int)floorf(cx + S.filt_radius), FW - 1), y1 = min((int)floorf(cy + S.filt_radius), FH - 1);
    for (int y = y0; y <= y1; ++y) {
        float wy = S.ftab[(int)(fabsf((float)y - cy) * S.filt_lookup)];
        int ty = y - fy0;
        for (int x = x0; x <= x1; ++x) {
            float wx = S.ftab[(int)(fabsf((float)x - cx) * S.filt_lookup)];
            int tx = x - fx0;
            float w = wx * wy;
            if (w == 0.0f || tx < 0 || ty < 0 || tx >= tw || ty >= th) continue;
            float *c = tile + 4 * (ty * tw + tx);
            atomicAdd(c + 0, (val.x * wx) * wy);
            atomicAdd(c + 1, (val.y * wx) * wy);
            atomicAdd(c + 2, (val.z * wx) * wy);
            atomicAdd(c + 3, w);
        }
    }
}

__device__ __forceinline__ uint64_t mix_seed(uint64_t seed, uint64_t s0) {
    uint64_t z = seed + 0x9E3779B97F4A7C15ULL * (s0 + 1);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    return z ^ (z >> 31);
}

template <int kAccel, bool kTex>
__global__ void __launch_bounds__(kTileThreads) render_pathmis_kernel(DevScene S, RenderLaunch P) {
    extern __shared__ float tile[];
    __shared__ int s_item;
    const int FW = (int)S.width + 2 * S.border, FH = (int)S.height + 2 * S.border;
    const int tw = kTile + P.margin_hi - P.margin_lo;
    const int th = tw;
    const int n_tile_cells = tw * th * 4;
    for (int i = threadIdx.x; i < n_tile_cells; i += blockDim.x) tile[i] = 0.0f;
    const int lx = threadIdx.x % kTile, ly = threadIdx.x / kTile;
    PathCounters pc{0, 0, TravStats()};
    uint32_t dropped = 0;
    for (;;) {
        __syncthreads();
        if (threadIdx.x == 0) s_item = (int)atomicAdd(P.work_counter, 1u);
        __syncthreads();
        const int item = s_item;
        if (item >= P.n_items) break;
        const int tile_id = item / P.n_chunks, chunk = item % P.n_chunks;
        const int tx0 = (tile_id % P.tiles_x) * kTile, ty0 = (tile_id / P.tiles_x) * kTile;
        const int x = tx0 + lx, y = ty0 + ly;
        // film coordinates of the shared tile's first cell
        const int fx0 = tx0 + P.margin_lo, fy0 = ty0 + P.margin_lo;
        if (x < (int)S.width && y < (int)S.height) {
            const int s0 = P.sample_offset + chunk * P.spp_per_item;
            const int s1 = min(s0 + P.spp_per_item, P.sample_offset + P.spp);
            const uint64_t stream = (uint64_t)y * S.width + x + (uint64_t)P.image_index * S.width * S.height;
            for (int s = s0; s < s1; ++s) {
                // one stream per (seed, sample, pixel, image), as the wavefront
                // draws it: the image does not depend on the work split or the form
                Pcg32 rng;
                rng.seed(mix_seed(P.seed, (uint64_t)s), stream);
                float px = (float)x + rng.nextf(), py = (float)y + rng.nextf();
                Ray r = camera_ray(S, px, py);
                V3 L = li_pathmis<kAccel, kTex>(S, rng, r, px, py, P.depth, P.rr_start, pc);
                if (!is_valid(L)) { ++dropped; continue; }
                splat_shared(S, tile, tw, th, fx0, fy0, FW, FH, px, py, L);
            }
        }
        __syncthreads();
        // flush the tile: one global atomic per touched film cell and channel
        for (int i = threadIdx.x; i < tw * th; i += blockDim.x) {
            float4 c = reinterpret_cast<float4 *>(tile)[i];
            if (c.w == 0.0f && c.x == 0.0f && c.y == 0.0f && c.z == 0.0f) continue;
            int fx = fx0 + i % tw, fy = fy0 + i / tw;
            if (fx >= 0 && fy >= 0 && fx < FW && fy < FH) {
                float *dst = P.film + 4 * ((size_t)fy * FW + fx);
                atomicAdd(dst + 0, c.x);
                atomicAdd(dst + 1, c.y);
                atomicAdd(dst + 2, c.z);
                atomicAdd(dst + 3, c.w);
            }
            reinterpret_cast<float4 *>(tile)[i] = make_float4(0, 0, 0, 0);
        }
    }
    // per-warp counter reduction (64-bit: node counts of one thread can pass 2^32)
    unsigned long long r = pc.rays, sh = pc.shadow, dr = dropped, nv = pc.trav.nodes, nt = pc.trav.tris;
    for (int o = 16; o > 0; o >>= 1) {
        r += __shfl_down_sync(0xffffffffu, r, o);
        sh += __shfl_down_sync(0xffffffffu, sh, o);
        dr += __shfl_down_sync(0xffffffffu, dr, o);
        nv += __shfl_down_sync(0xffffffffu, nv, o);
        nt += __shfl_down_sync(0xffffffffu, nt, o);
    }
    if ((threadIdx.x & 31) == 0 && P.counters) {
        atomicAdd(P.counters + 0, r);
        atomicAdd(P.counters + 1, sh);
        atomicAdd(P.counters + 2, dr);
        atomicAdd(P.counters + 3, nv);
        atomicAdd(P.counters + 4, nt);
    }
}

template <int kAccel, bool kTex>
cudaError_t launch_render_t(const DevScene &S, const RenderLaunch &P, int grid, cudaStream_t st) {
    const int tw = kTile + P.margin_hi - P.margin_lo;
    const size_t smem = (size_t)tw * tw * 4 * sizeof(float);
    render_pathmis_kernel<kAccel, kTex><<<grid, kTileThreads, smem, st>>>(S, P);
    return cudaGetLastError();
}
template <int kAccel, bool kTex>
int render_occupancy_t(int margin_lo, int margin_hi) {
    int n = 0;
    const size_t smem = (size_t)(kTile + margin_hi - margin_lo) * (kTile + margin_hi - margin_lo) * 16;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, render_pathmis_kernel<kAccel, kTex>, kTileThreads, smem);
    return n;
}

}  // namespace hk
