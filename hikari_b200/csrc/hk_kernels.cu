// sm_100a kernels of the pathMIS core:
//   * film_resolve, trace_rays and the record-query kernels used by the C-ABI
//     and its parity tests;
//   * the dispatch from the launch interface to the megakernel
//     (hk_megakernel.cuh, instantiated in hk_render_*.cu) and the BSDF batch
//     (hk_batch.cuh, instantiated in hk_batch_*.cu).
#include <cstdio>
#include <mutex>

#include "hk_kernels.h"
#include "hk_shading.cuh"

namespace hk {
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
    if (S.accel == kAccelBvh8)
        return S.textured ? launch_render_t<kAccelBvh8, true>(S, P, grid, st) : launch_render_t<kAccelBvh8, false>(S, P, grid, st);
    return S.textured ? launch_render_t<kAccelBvh2, true>(S, P, grid, st) : launch_render_t<kAccelBvh2, false>(S, P, grid, st);
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
#define HK_BSDF_BATCH(T) \
    case T: return launch_bsdf_batch_t<T>(S, bsdf, n, wi, u2, u1, wo, uv, duv, s_wo, s_w, s_pdf, s_m, e_rgb, p_pdf, g, st)
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
        HK_BSDF_BATCH(-1);   // layers nested deeper than one level: run-time dispatch
    default: return cudaErrorInvalidValue;
    }
#undef HK_BSDF_BATCH
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
    if (accel == kAccelBvh8)
        return textured ? render_occupancy_t<kAccelBvh8, true>(margin_lo, margin_hi) : render_occupancy_t<kAccelBvh8, false>(margin_lo, margin_hi);
    return textured ? render_occupancy_t<kAccelBvh2, true>(margin_lo, margin_hi) : render_occupancy_t<kAccelBvh2, false>(margin_lo, margin_hi);
}

}  // namespace hk
