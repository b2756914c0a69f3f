// sm_100a kernels of the pathMIS core:
//   * render_pathmis: the plain megakernel (one thread per pixel sample
//     stream, persistent CTAs pulling (tile, sample-chunk) work items, film
//     splatted through the reconstruction filter into a shared-memory tile and
//     flushed once per item);
//   * film_resolve, trace_rays, bsdf_batch and record-query kernels used by
//     the C-ABI and its parity tests.
#include <cstdio>
#include <mutex>

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
        if constexpr (kTex) {
            if (is_bump(S.bsdfs[bsdf])) bf = perturbed_frames(S, hc, it, S.bsdfs[bsdf]);
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
                Ray sr;
                sr.o = it.p; sr.d = er.p - it.p; sr.tmin = kRayEps; sr.tmax = 1.0f - kRayEps;
                Hit sh;
                pc.shadow++;
                if (!trace<kAccel, true>(S, sr, sh, pc.trav)) {
                    BRec br;
                    br.wi = to_local(it.sh, ray.d * -1.0f);
                    br.wo = to_local(it.sh, er.wi);
                    br.measure = kMeasureSolidAngle;
                    br.eta = 0.0f;
                    br.tu = it.u; br.tv = it.v; br.tex = kTex; br.duv = duv;
                    float pb;
                    V3 f;
                    if constexpr (kTex) {
                        pb = bsdf_pdf_b(S.bsdfs, bsdf, br, bf);
                        f = bsdf_eval_b(S.bsdfs, bsdf, br, bf);
                    } else {
                        pb = bsdf_pdf(S.bsdfs, bsdf, br);
                        f = bsdf_eval(S.bsdfs, bsdf, br);
                    }
                    if (pl + pb != 0.0f) w_ems = pl / (pl + pb);
                    float c = fabsf(br.wo.z);
                    L = L + v3((((beta.x * f.x) * c) * ld.x) * w_ems, (((beta.y * f.y) * c) * ld.y) * w_ems,
                               (((beta.z * f.z) * c) * ld.z) * w_ems);
                }
            }
        }
        BRec br;
        br.wi = to_local(it.sh, ray.d * -1.0f);
        br.wo = v3(0, 0, 0);
        br.measure = kMeasureUnknown;
        br.eta = 0.0f;
        br.tu = it.u; br.tv = it.v; br.tex = kTex; br.duv = duv;
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
        if (depth >= rr_start) {
            if (rng.nextf() < 0.95f) beta = beta * (1.0f / 0.95f);
            else break;
        }
        ++depth;
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
            Pcg32 rng;
            rng.seed(mix_seed(P.seed, (uint64_t)s0), (uint64_t)y * S.width + x + (uint64_t)P.image_index * S.width * S.height);
            for (int s = s0; s < s1; ++s) {
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

// Block.cpp:61 ToBitmap: interior pixels divided by their filter weight.
__global__ void film_resolve_kernel(const float *film, float *rgb, int W, int H, int B) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= W * H) return;
    int x = i % W, y = i / W;
    float4 c = reinterpret_cast<const float4 *>(film)[(size_t)(y + B) * (W + 2 * B) + (x + B)];
    float r = 0.0f, g = 0.0f, b = 0.0f;
    if (c.w != 0.0f) { r = c.x / c.w; g = c.y / c.w; b = c.z / c.w; }
    rgb[3 * (size_t)i + 0] = r;
    rgb[3 * (size_t)i + 1] = g;
    rgb[3 * (size_t)i + 2] = b;
}

// Ray queries: rays are n x 8 floats (o, d, tmin, tmax).  Reported triangle
// ids are the ORIGINAL global triangle indices (mesh order).
template <int kAccel>
__global__ void trace_rays_kernel(DevScene S, uint64_t n, const float *rays, int32_t *tri, float *t, float *u, float *v,
                                  int any_hit, unsigned long long *visit_counter) {
    TravStats ts;
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        const float4 *rp = reinterpret_cast<const float4 *>(rays + 8 * i);
        float4 a = __ldg(rp), b = __ldg(rp + 1);
        Ray r;
        r.o = v3(a.x, a.y, a.z);
        r.d = v3(a.w, b.x, b.y);
        r.tmin = b.z;
        r.tmax = b.w;
        Hit h;
        bool f = any_hit ? trace<kAccel, true>(S, r, h, ts) : trace<kAccel, false>(S, r, h, ts);
        if (any_hit) { tri[i] = f ? 1 : 0; continue; }
        tri[i] = f ? __float_as_int(__ldg(S.tris + 3 * h.tri).w) : -1;
        if (t) t[i] = f ? h.t : 0.0f;
        if (u) u[i] = f ? h.u : 0.0f;
        if (v) v[i] = f ? h.v : 0.0f;
    }
    if (visit_counter) {
        unsigned long long nodes = ts.nodes, tris = ts.tris;
        for (int o = 16; o > 0; o >>= 1) {
            nodes += __shfl_down_sync(0xffffffffu, nodes, o);
            tris += __shfl_down_sync(0xffffffffu, tris, o);
        }
        if ((threadIdx.x & 31) == 0) {
            atomicAdd(visit_counter, nodes);
            atomicAdd(visit_counter + 1, tris);
        }
    }
}

// Config-2 BSDF batch: per record Sample (wo, weight, pdf of the sampled
// direction, measure), Eval and Pdf at the given wo with ESolidAngle.
// One instantiation per top-level BSDF type (the host picks the id's type),
// so a launch carries only that BSDF's code.
template <int BT, bool kTex>
__global__ void bsdf_batch_kernel(DevScene S, int bsdf, uint64_t n, const float *wi, const float *u2, const float *u1,
                                  const float *wo, const float *uv, const float *duv, float *s_wo, float *s_w,
                                  float *s_pdf, int32_t *s_m, float *e_rgb, float *p_pdf) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        BRec r;
        r.wi = v3(wi[3 * i], wi[3 * i + 1], wi[3 * i + 2]);
        r.wo = v3(0, 0, 0);
        r.measure = kMeasureUnknown;
        r.eta = 0.0f;
        r.tex = kTex;
        r.tu = kTex ? uv[2 * i] : 0.0f;
        r.tv = kTex ? uv[2 * i + 1] : 0.0f;
        r.duv = (kTex && duv) ? make_float4(duv[4 * i], duv[4 * i + 1], duv[4 * i + 2], duv[4 * i + 3])
                              : make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        V3 w = bsdf_sample_t<BT>(S.bsdfs, bsdf, r, u2[2 * i], u2[2 * i + 1], u1 ? u1[i] : 0.0f);
        if (s_wo) { s_wo[3 * i] = r.wo.x; s_wo[3 * i + 1] = r.wo.y; s_wo[3 * i + 2] = r.wo.z; }
        if (s_w) { s_w[3 * i] = w.x; s_w[3 * i + 1] = w.y; s_w[3 * i + 2] = w.z; }
        if (s_m) s_m[i] = r.measure;
        if (s_pdf) s_pdf[i] = all_zero(w) ? 0.0f : bsdf_pdf_t<BT>(S.bsdfs, bsdf, r);
        BRec q;
        q.wi = r.wi;
        q.wo = v3(wo[3 * i], wo[3 * i + 1], wo[3 * i + 2]);
        q.measure = kMeasureSolidAngle;
        q.eta = 0.0f;
        q.tex = kTex;
        q.tu = r.tu;
        q.tv = r.tv;
        q.duv = r.duv;
        if (e_rgb) {
            V3 e = bsdf_eval_t<BT>(S.bsdfs, bsdf, q);
            e_rgb[3 * i] = e.x; e_rgb[3 * i + 1] = e.y; e_rgb[3 * i + 2] = e.z;
        }
        if (p_pdf) p_pdf[i] = bsdf_pdf_t<BT>(S.bsdfs, bsdf, q);
    }
}

// Texture2D::Eval(Isect, filter = true) of texture `tex` at n texture
// coordinates uv (n x 2) with screen-space partials duv (n x 4, or null): out n x 3.
__global__ void texture_eval_kernel(DevScene S, const DevTexture *T, int tex, uint64_t n, const float *uv,
                                    const float *duv, float *out) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        const float4 d = duv ? make_float4(duv[4 * i], duv[4 * i + 1], duv[4 * i + 2], duv[4 * i + 3])
                             : make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        const V3 c = tex_eval(T, tex, uv[2 * i], uv[2 * i + 1], d);
        out[3 * i] = c.x; out[3 * i + 1] = c.y; out[3 * i + 2] = c.z;
    }
}
cudaError_t launch_texture_eval(const DevScene &S, const DevTexture *T, int tex, uint64_t n, const float *uv,
                                const float *duv, float *out, cudaStream_t st) {
    const int g = (int)(n / 128 + 1 < 148 * 64 ? n / 128 + 1 : 148 * 64);
    texture_eval_kernel<<<g, 128, 0, st>>>(S, T, tex, n, uv, duv, out);
    return cudaGetLastError();
}

// Emitter record queries (parity tests).  in: n x 8 (ref xyz, ux, uy, u1, -, -)
// out: n x 16 (p, n, wi, pdf, dist, value xyz, pad)
__global__ void emitter_sample_kernel(DevScene S, int e, uint64_t n, const float *in, float *out) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        const float *q = in + 8 * i;
        ERec r;
        r.ref = v3(q[0], q[1], q[2]);
        r.dist = 0.0f;
        r.pdf = 0.0f;
        r.p = r.n = r.wi = v3(0, 0, 0);
        V3 val = emitter_sample(S, e, r, q[3], q[4], q[5]);
        float *o = out + 16 * i;
        o[0] = r.p.x; o[1] = r.p.y; o[2] = r.p.z; o[3] = r.n.x; o[4] = r.n.y; o[5] = r.n.z;
        o[6] = r.wi.x; o[7] = r.wi.y; o[8] = r.wi.z; o[9] = r.pdf; o[10] = r.dist;
        o[11] = val.x; o[12] = val.y; o[13] = val.z; o[14] = 0.0f; o[15] = 0.0f;
    }
}

// Camera rays for film positions: in n x 2, out n x 8
__global__ void camera_rays_kernel(DevScene S, uint64_t n, const float *pos, float *out) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        Ray r = camera_ray(S, pos[2 * i], pos[2 * i + 1]);
        float *o = out + 8 * i;
        o[0] = r.o.x; o[1] = r.o.y; o[2] = r.o.z; o[3] = r.d.x; o[4] = r.d.y; o[5] = r.d.z; o[6] = r.tmin; o[7] = r.tmax;
    }
}

// Environment Eval for world directions: in n x 3, out n x 3 (+ env Pdf in pdf[])
__global__ void env_eval_kernel(DevScene S, uint64_t n, const float *wi, float *out, float *pdf) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        V3 d = v3(wi[3 * i], wi[3 * i + 1], wi[3 * i + 2]);
        V3 c = env_eval(S, d);
        out[3 * i] = c.x; out[3 * i + 1] = c.y; out[3 * i + 2] = c.z;
        if (pdf) pdf[i] = env_pdf(S, d);
    }
}

// ------------------------------------------------------------ static scratch
// Scratch for hk_render_image_static, the entry point for callers that cannot
// allocate device memory.  Every GPU that loads the library holds this array
// (about 4.3 MB) until the process exits; all calls share it.
static __device__ __align__(256) unsigned long long g_render_scratch[kStaticScratchWords];

cudaError_t static_render_scratch(void **out) {
    static std::mutex mu;
    static void *ptrs[kStaticMaxDevices] = {};
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= kStaticMaxDevices) return cudaErrorInvalidDevice;
    std::lock_guard<std::mutex> lock(mu);
    if (!ptrs[dev]) {
        // the host-side name of the array is not a device address: ask the runtime
        void *p = nullptr;
        e = cudaGetSymbolAddress(&p, g_render_scratch);
        if (e != cudaSuccess) return e;
        ptrs[dev] = p;
    }
    *out = ptrs[dev];
    return cudaSuccess;
}

// ------------------------------------------------------------ launchers
static int grid_for(uint64_t n, int threads) {
    uint64_t g = (n + threads - 1) / threads;
    if (g > 148ull * 32) g = 148ull * 32;
    return (int)(g < 1 ? 1 : g);
}

cudaError_t launch_render(const DevScene &S, const RenderLaunch &P, int grid, cudaStream_t st) {
    const int tw = kTile + P.margin_hi - P.margin_lo;
    size_t smem = (size_t)tw * tw * 4 * sizeof(float);
    if (S.accel == kAccelBvh8) {
        if (S.textured) render_pathmis_kernel<kAccelBvh8, true><<<grid, kTileThreads, smem, st>>>(S, P);
        else render_pathmis_kernel<kAccelBvh8, false><<<grid, kTileThreads, smem, st>>>(S, P);
    } else {
        if (S.textured) render_pathmis_kernel<kAccelBvh2, true><<<grid, kTileThreads, smem, st>>>(S, P);
        else render_pathmis_kernel<kAccelBvh2, false><<<grid, kTileThreads, smem, st>>>(S, P);
    }
    return cudaGetLastError();
}
cudaError_t launch_resolve(const float *film, float *rgb, int W, int H, int B, cudaStream_t st) {
    int n = W * H;
    film_resolve_kernel<<<(n + 255) / 256, 256, 0, st>>>(film, rgb, W, H, B);
    return cudaGetLastError();
}
cudaError_t launch_trace(const DevScene &S, uint64_t n, const float *rays, int32_t *tri, float *t, float *u, float *v,
                         int any_hit, unsigned long long *visits, cudaStream_t st) {
    if (S.accel == kAccelBvh8)
        trace_rays_kernel<kAccelBvh8><<<grid_for(n, 128), 128, 0, st>>>(S, n, rays, tri, t, u, v, any_hit, visits);
    else
        trace_rays_kernel<kAccelBvh2><<<grid_for(n, 128), 128, 0, st>>>(S, n, rays, tri, t, u, v, any_hit, visits);
    return cudaGetLastError();
}
cudaError_t launch_bsdf_batch(const DevScene &S, int bsdf, int type, uint64_t n, const float *wi, const float *u2, const float *u1,
                              const float *wo, const float *uv, const float *duv, float *s_wo, float *s_w, float *s_pdf,
                              int32_t *s_m, float *e_rgb, float *p_pdf, cudaStream_t st) {
    const int g = grid_for(n, 256);
#define HK_BSDF_BATCH(T)                                                                                          \
    case T:                                                                                                       \
        if (uv) bsdf_batch_kernel<T, true><<<g, 256, 0, st>>>(S, bsdf, n, wi, u2, u1, wo, uv, duv, s_wo, s_w, s_pdf, s_m, e_rgb, p_pdf); \
        else bsdf_batch_kernel<T, false><<<g, 256, 0, st>>>(S, bsdf, n, wi, u2, u1, wo, uv, duv, s_wo, s_w, s_pdf, s_m, e_rgb, p_pdf); \
        break
    switch (type) {
        HK_BSDF_BATCH(kDiffuse);
        HK_BSDF_BATCH(kRoughConductor);
        HK_BSDF_BATCH(kRoughDielectric);
        HK_BSDF_BATCH(kRoughPlastic);
        HK_BSDF_BATCH(kRoughCoating);
        HK_BSDF_BATCH(kMirror);
        HK_BSDF_BATCH(kConductor);
        HK_BSDF_BATCH(kDielectric);
        HK_BSDF_BATCH(kPlastic);
        HK_BSDF_BATCH(kTwoSided);
        HK_BSDF_BATCH(kCoating);
        HK_BSDF_BATCH(kRoughDiffuse);
    default: return cudaErrorInvalidValue;
    }
#undef HK_BSDF_BATCH
    return cudaGetLastError();
}
cudaError_t launch_emitter_sample(const DevScene &S, int e, uint64_t n, const float *in, float *out, cudaStream_t st) {
    emitter_sample_kernel<<<grid_for(n, 128), 128, 0, st>>>(S, e, n, in, out);
    return cudaGetLastError();
}
cudaError_t launch_camera_rays(const DevScene &S, uint64_t n, const float *pos, float *out, cudaStream_t st) {
    camera_rays_kernel<<<grid_for(n, 128), 128, 0, st>>>(S, n, pos, out);
    return cudaGetLastError();
}
cudaError_t launch_env_eval(const DevScene &S, uint64_t n, const float *wi, float *out, float *pdf, cudaStream_t st) {
    env_eval_kernel<<<grid_for(n, 128), 128, 0, st>>>(S, n, wi, out, pdf);
    return cudaGetLastError();
}
int render_occupancy(int margin_lo, int margin_hi, int accel, bool textured) {
    int n = 0;
    const size_t smem = (size_t)(kTile + margin_hi - margin_lo) * (kTile + margin_hi - margin_lo) * 16;
    if (accel == kAccelBvh8) {
        if (textured) cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, render_pathmis_kernel<kAccelBvh8, true>, kTileThreads, smem);
        else cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, render_pathmis_kernel<kAccelBvh8, false>, kTileThreads, smem);
    } else {
        if (textured) cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, render_pathmis_kernel<kAccelBvh2, true>, kTileThreads, smem);
        else cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, render_pathmis_kernel<kAccelBvh2, false>, kTileThreads, smem);
    }
    return n;
}

}  // namespace hk
