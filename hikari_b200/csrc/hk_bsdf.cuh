// Device BSDFs of the pathMIS core: diffuse, roughConductor, roughDielectric,
// roughPlastic, roughCoating and coating, roughDiffuse, the smooth mirror,
// conductor, dielectric and plastic, and twoSided; layers (coatings, twoSided)
// stack up to kNestLevels deep (one level inline, deeper stacks through the
// deep_* functions),
// with the Beckmann/GGX microfacet distribution and the 1D rough-transmittance
// lookups.
//
// Each function follows the reference method cited beside it, in the same
// float evaluation order, so results agree with the reference to the ulp
// differences of CUDA's expf/logf/sinf/cosf/powf against the host libm.
#pragma once
#include "hk_device.h"
#include "hk_math.cuh"

namespace hk {

struct BRec {
    V3 wi, wo;
    float eta;
    int measure;
    float tu, tv;   // texture coordinates of the intersection (Record.Isect.UV)
    float4 duv;     // their screen-space partials (dUdX, dVdX, dUdY, dVdY): a camera ray's first hit, else 0
    bool tex;       // textures are looked up (false in kernels that shade untextured materials only)
    // what the wireframe and curvature textures read at the intersection: the
    // distance from P to the nearest edge line of the hit triangle, the mean
    // and the Gaussian curvature (tex_geometry); without an intersection the
    // wireframe reads its interior colour and the curvature black
    float3 geo = make_float3(INFINITY, 0.0f, 0.0f);
};

// ------------------------------------------------------------ microfacet
// src/core/MicrofacetDistribution.cpp
struct Mfd {
    int type;
    float au, av;
};
__device__ __forceinline__ Mfd mfd_make(int type, float au, float av) {   // ctor :10-26
    return Mfd{type, clampf(au, 5e-4f, 1.0f), clampf(av, 5e-4f, 1.0f)};
}
__device__ __forceinline__ float mfd_eval(const Mfd &d, V3 m) {   // Eval :34
    if (m.z <= 0.0f) return 0.0f;
    float c2 = m.z * m.z;
    float be = ((m.x * m.x) / (d.au * d.au) + (m.y * m.y) / (d.av * d.av)) / c2;
    float r;
    if (d.type == kBeckmann) {
        r = expf(-be) / (kPi * d.au * d.av * c2 * c2);
    } else {
        float root = (1.0f + be) * c2;
        r = 1.0f / (kPi * d.au * d.av * root * root);
    }
    if (r * m.z < 1e-20f) r = 0.0f;
    return r;
}
__device__ __forceinline__ float mfd_project_roughness(const Mfd &d, V3 v) {   // :238
    float inv = 1.0f / sin_theta2(v);
    if (d.au == d.av || inv <= 0.0f) return d.au;
    float c2 = v.x * v.x * inv, s2 = v.y * v.y * inv;
    return sqrtf(c2 * d.au * d.au + s2 * d.av * d.av);
}
__device__ __forceinline__ float mfd_g1(const Mfd &d, V3 v, V3 m) {   // SmithG1 :82
    if (dot(v, m) * v.z <= 0.0f) return 0.0f;
    float tt = fabsf(tan_theta(v));
    if (tt == 0.0f) return 1.0f;
    float a = mfd_project_roughness(d, v);
    if (d.type == kBeckmann) {
        float x = 1.0f / (a * tt);
        if (x >= 1.6f) return 1.0f;
        float x2 = x * x;
        return (3.535f * x + 2.181f * x2) / (1.0f + 2.276f * x + 2.577f * x2);
    }
    float root = a * tt;
    return 2.0f / (1.0f + hypot2(1.0f, root));
}
__device__ __forceinline__ float mfd_g(const Mfd &d, V3 wi, V3 wo, V3 m) { return mfd_g1(d, wi, m) * mfd_g1(d, wo, m); }
__device__ __forceinline__ V3 mfd_sample(const Mfd &d, float ux, float uy, float &pdf) {   // SampleAll :148
    float sp, cp, a2;
    if (d.au == d.av) {
        float ph = (2.0f * kPi) * uy;
        sincosf(ph, &sp, &cp);
        a2 = d.au * d.au;
    } else {
        float ph = atanf(d.av / d.au * tanf(kPi + 2.0f * kPi * uy)) + kPi * floorf(2.0f * uy + 0.5f);
        sincosf(ph, &sp, &cp);
        float cs = cp / d.au, ss = sp / d.av;
        a2 = 1.0f / (cs * cs + ss * ss);
    }
    float cm;
    if (d.type == kBeckmann) {
        float t2 = a2 * -logf(1.0f - ux);
        cm = 1.0f / sqrtf(1.0f + t2);
        pdf = (1.0f - ux) / (kPi * d.au * d.av * cm * cm * cm);
    } else {
        float t2 = a2 * ux / (1.0f - ux);
        cm = 1.0f / sqrtf(1.0f + t2);
        float tmp = 1.0f + t2 / a2;
        pdf = (float)kInvPiD / (d.au * d.av * cm * cm * cm * tmp * tmp);
    }
    if (pdf < 1e-20f) pdf = 0.0f;
    float sm = sqrtf(fmaxf(0.0f, 1.0f - cm * cm));
    return v3(sm * cp, sm * sp, cm);
}
__device__ __forceinline__ float mfd_pdf(const Mfd &d, V3 m) { return mfd_eval(d, m) * m.z; }   // PdfAll :231

// ------------------------------------------------------------ fresnel
// FresnelDielectric (src/core/Common.cpp:494)
__device__ __forceinline__ float fresnel_dielectric(float ci, float eta, float inv_eta, float &ct) {
    if (eta == 1.0f) { ct = -ci; return 0.0f; }
    float sc = (ci > 0.0f) ? inv_eta : eta;
    float ct2 = 1.0f - (1.0f - ci * ci) * (sc * sc);
    if (ct2 <= 0.0f) { ct = 0.0f; return 1.0f; }
    float cii = fabsf(ci), ctt = sqrtf(ct2);
    float rs = (cii - eta * ctt) / (cii + eta * ctt);
    float rp = (eta * cii - ctt) / (eta * cii + ctt);
    ct = (ci > 0.0f) ? -ctt : ctt;
    return 0.5f * (rs * rs + rp * rp);
}
// FresnelConductor (src/core/Common.cpp:529), one channel
__device__ __forceinline__ float fresnel_conductor1(float ci, float eta, float k) {
    float ci2 = ci * ci, si2 = 1.0f - ci2;
    float e2 = eta * eta, k2 = k * k;
    float t0 = e2 - k2 - si2;
    float a2b2 = sqrtf(t0 * t0 + 4.0f * e2 * k2);
    float t1 = a2b2 + ci2;
    float a = sqrtf(0.5f * (a2b2 + t0));
    float t2 = 2.0f * ci * a;
    float rs = (t1 - t2) / (t1 + t2);
    float t3 = ci2 * a2b2 + si2 * si2;
    float t4 = t2 * si2;
    float rp = rs * ((t3 - t4) / (t3 + t4));
    return 0.5f * (rp + rs);
}
__device__ __forceinline__ V3 reflect_m(V3 wi, V3 m) { return m * (2.0f * dot(wi, m)) - wi; }   // :616
__device__ __forceinline__ V3 refract_m(V3 wi, V3 m, float ct, float eta, float inv_eta) {   // :622
    float e = (ct < 0.0f ? inv_eta : eta);
    return m * (dot(wi, m) * e + ct) - wi * e;
}

// ------------------------------------------------------------ RFT
// EvalCubicInterpolate1D over [0,1] (src/core/Common.cpp:230) on the activated table
__device__ __forceinline__ float cubic1d01(float x, const float *val, int size) {
    if (!(x >= 0.0f && x <= 1.0f)) return 0.0f;
    float t = ((x - 0.0f) * (size - 1)) / (1.0f - 0.0f);
    int k = (int)t;
    k = k > size - 2 ? size - 2 : k;
    k = k < 0 ? 0 : k;
    float f0 = __ldg(val + k), f1 = __ldg(val + k + 1), d0, d1;
    d0 = (k > 0) ? 0.5f * (f1 - __ldg(val + k - 1)) : f1 - f0;
    d1 = (k + 2 < size) ? 0.5f * (__ldg(val + k + 2) - f0) : f1 - f0;
    t = t - (float)k;
    float t2 = t * t, t3 = t2 * t;
    return (2.0f * t3 - 3.0f * t2 + 1) * f0 + (-2.0f * t3 + 3.0f * t2) * f1 + (t3 - 2.0f * t2 + t) * d0 +
           (t3 - t2) * d1;
}
// EvalCubicInterpolate2D over [0,1]^2 (src/core/Common.cpp:285) of a
// [y][x] table with sx x samples and sy y samples
__device__ __forceinline__ bool cubic_knot_weights(float p, int size, float *w, int &knot) {
    if (!(p >= 0.0f && p <= 1.0f)) return false;
    float t = ((p - 0.0f) * (float)(size - 1)) / (1.0f - 0.0f);
    knot = min((int)t, size - 2);
    t = t - (float)knot;
    const float t2 = t * t, t3 = t2 * t;
    w[0] = 0.0f;
    w[1] = 2.0f * t3 - 3.0f * t2 + 1;
    w[2] = -2.0f * t3 + 3.0f * t2;
    w[3] = 0.0f;
    const float d0 = t3 - 2.0f * t2 + t, d1 = t3 - t2;
    if (knot > 0) { w[2] += 0.5f * d0; w[0] -= 0.5f * d0; }
    else { w[2] += d0; w[1] -= d0; }
    if (knot + 2 < size) { w[3] += 0.5f * d1; w[1] -= 0.5f * d1; }
    else { w[2] += d1; w[1] -= d1; }
    return true;
}
__device__ __forceinline__ float cubic2d01(float px, float py, const float *val, int sx, int sy) {
    float wx[4], wy[4];
    int kx, ky;
    if (!cubic_knot_weights(px, sx, wx, kx) || !cubic_knot_weights(py, sy, wy, ky)) return 0.0f;
    float r = 0.0f;
#pragma unroll
    for (int y = -1; y <= 2; y++) {
        const float w_y = wy[y + 1];
#pragma unroll
        for (int x = -1; x <= 2; x++) {
            const float wxy = wx[x + 1] * w_y;
            if (wxy == 0) continue;
            r += __ldg(val + (ky + y) * sx + kx + x) * wxy;
        }
    }
    return r;
}
// RoughTransmittance::Eval (src/core/RoughTransmitance.cpp:48-87): eta fixed,
// alpha fixed (the activated 1D table) or, under a textured alpha, per query
// (the 2D table over warped cos and warped alpha)
__device__ __forceinline__ float rft_eval(const DevBsdf &b, float c, float alpha) {
    float wc = powf(fabsf(c), 0.25f);
    if (c < 0.0f) return 0.0f;
    if (b.alpha_tex) {
        const float wa = powf((alpha - b.rft_amin) / (b.rft_amax - b.rft_amin), 0.25f);
        return clampf(cubic2d01(wc, wa, b.rft2d, b.rft_n, b.rft_an), 0.0f, 1.0f);
    }
    return clampf(cubic1d01(wc, b.rft, b.rft_n), 0.0f, 1.0f);
}
// roughPlastic's 1 - IntData.EvalDiffuse(alpha) (:119-132): activated, or per query
__device__ __forceinline__ float plastic_fdr(const DevBsdf &b, float alpha) {
    if (!b.alpha_tex) return b.fdr_int;
    const float wa = powf((alpha - b.rft_amin) / (b.rft_amax - b.rft_amin), 0.25f);
    return 1.0f - clampf(cubic1d01(wa, b.rft_diff, b.rft_an), 0.0f, 1.0f);
}

__device__ __forceinline__ V3 ld_rgb(const float *p) { return v3(p[0], p[1], p[2]); }

// ------------------------------------------------------------ textures
// Texture2D::Eval(Isect) (src/core/Texture.cpp:211): UV scaled and offset, then
// CheckerboardTexture::Eval (src/texture/CheckerboardTexture.cpp:24) or
// GridTexture::Eval (src/texture/GridTexture.cpp:26); ScaleTexture::Eval
// (src/texture/ScaleTexture.cpp:17) scales its nested texture, innermost first.
__device__ __forceinline__ int mod_positive(int a, int b) {
    int q = a % b;
    return q < 0 ? q + b : q;
}
// ---- bitmaps: MipMap<T> (include/core/MipMap.hpp) over the pyramid built on
// the host.  All arithmetic follows the reference's float order; the level of
// detail uses the device log2f (the host's log2f may differ in the last place,
// which moves the lerp between two levels by as much).
// MipMap::Texel :244 -- outside the level, or everywhere with a "black" wrap mode, black.
__device__ __forceinline__ V3 mip_texel(const DevTexture &t, int l, int x, int y) {
    const int w = 1 << max(0, t.lw - l), h = 1 << max(0, t.lh - l);
    if (t.black || x < 0 || x >= w || y < 0 || y >= h) return v3(0, 0, 0);
    const uint32_t i = t.lvl_off[l] + (uint32_t)y * (uint32_t)w + (uint32_t)x;
    if (t.channels == 1) {
        const float r = __ldg(t.texels + i);
        return v3(r, r, r);
    }
    const float4 c = __ldg(reinterpret_cast<const float4 *>(t.texels) + i);
    return v3(c.x, c.y, c.z);
}
// MipMap::Triangle :412
__device__ __forceinline__ V3 mip_triangle(const DevTexture &t, int l, float u, float v) {
    l = clampi(l, 0, t.levels - 1);
    const float U = u * (float)(1 << max(0, t.lw - l)) - 0.5f, Vv = v * (float)(1 << max(0, t.lh - l)) - 0.5f;
    const int u0 = (int)floorf(U), v0 = (int)floorf(Vv);
    const float du = U - (float)u0, dv = Vv - (float)v0;
    const float a = (1.0f - du) * (1.0f - dv), b = (1.0f - du) * dv, c = du * (1.0f - dv), d = du * dv;
    V3 r = mip_texel(t, l, u0, v0) * a;
    r = r + mip_texel(t, l, u0, v0 + 1) * b;
    r = r + mip_texel(t, l, u0 + 1, v0) * c;
    return r + mip_texel(t, l, u0 + 1, v0 + 1) * d;
}
__device__ __forceinline__ V3 lerp3(float x, V3 a, V3 b) { return a * (1.0f - x) + b * x; }
// MipMap::Lookup(UV, Width) :287 (bilinear with width 0, trilinear)
__device__ __forceinline__ V3 mip_lookup_width(const DevTexture &t, float u, float v, float width) {
    const float level = (float)t.levels - 1.0f + log2f(fmaxf(width, 1e-8f));
    if (level < 0.0f) return mip_triangle(t, 0, u, v);
    if (level >= (float)(t.levels - 1)) return mip_texel(t, t.levels - 1, 0, 0);
    const int il = (int)floorf(level);
    return lerp3(level - (float)il, mip_triangle(t, il, u, v), mip_triangle(t, il + 1, u, v));
}
// MipMap::EWA :427.  The scan is bounded to 4096 x 4096 texels (reached only
// with a maxAnisotropy of the order of a thousand or more).
static __device__ __noinline__ V3 mip_ewa(const DevTexture &t, int l, float u, float v, float d0x, float d0y, float d1x,
                                   float d1y) {
    if (l >= t.levels) return mip_texel(t, t.levels - 1, 0, 0);
    const float W = (float)(1 << max(0, t.lw - l)), H = (float)(1 << max(0, t.lh - l));
    u = u * W - 0.5f;
    v = v * H - 0.5f;
    d0x *= W; d0y *= H; d1x *= W; d1y *= H;
    float A = (d0y * d0y + d1y * d1y) + 1.0f;
    float B = -2.0f * (d0x * d0y + d1x * d1y);
    float C = (d0x * d0x + d1x * d1x) + 1.0f;
    const float invf = 1.0f / (A * C - (B * B) * 0.25f);
    A *= invf; B *= invf; C *= invf;
    const float det = (-B) * B + (4.0f * A) * C;
    const float invdet = 1.0f / det;
    const float usq = sqrtf(det * C), vsq = sqrtf(A * det);
    const int u0 = (int)ceilf(u - (2.0f * invdet) * usq), v0 = (int)ceilf(v - (2.0f * invdet) * vsq);
    const int u1 = min((int)floorf(u + (2.0f * invdet) * usq), u0 + 4095);
    const int v1 = min((int)floorf(v + (2.0f * invdet) * vsq), v0 + 4095);
    V3 sum = v3(0, 0, 0);
    float sw = 0.0f;
    for (int iv = v0; iv <= v1; ++iv) {
        const float dv = (float)iv - v;
        for (int iu = u0; iu <= u1; ++iu) {
            const float du = (float)iu - u;
            const float r2 = ((A * du) * du + (B * du) * dv) + (C * dv) * dv;
            if (r2 < 1.0f) {
                const float wt = __ldg(t.lut + min((int)(r2 * (float)kEwaLutSize), kEwaLutSize - 1));
                sum = sum + mip_texel(t, l, iu, iv) * wt;
                sw += wt;
            }
        }
    }
    return v3(sum.x / sw, sum.y / sw, sum.z / sw);
}
// MipMap::Lookup(UV, D0, D1) :309
__device__ __forceinline__ V3 mip_lookup_diff(const DevTexture &t, float u, float v, float d0x, float d0y, float d1x,
                                              float d1y) {
    if (t.filter == kFilterTrilinear) {
        const float w = fmaxf(fmaxf(fabsf(d0x), fabsf(d0y)), fmaxf(fabsf(d1x), fabsf(d1y)));
        return mip_lookup_width(t, u, v, 2.0f * w);
    }
    if (d0x * d0x + d0y * d0y < d1x * d1x + d1y * d1y) {
        float a = d0x, b = d0y;
        d0x = d1x; d0y = d1y; d1x = a; d1y = b;
    }
    const float major = sqrtf(d0x * d0x + d0y * d0y);
    float minor = sqrtf(d1x * d1x + d1y * d1y);
    if (minor * t.max_aniso < major && minor > 0.0f) {
        const float sc = major / (minor * t.max_aniso);
        d1x *= sc; d1y *= sc;
        minor *= sc;
    }
    if (minor == 0.0f) return mip_triangle(t, 0, u, v);
    const float lod = fmaxf(0.0f, (float)t.levels - 1.0f + log2f(minor));
    const float ilod = floorf(lod);
    return lerp3(lod - ilod, mip_ewa(t, (int)ilod, u, v, d0x, d0y, d1x, d1y),
                 mip_ewa(t, (int)(ilod + 1.0f), u, v, d0x, d0y, d1x, d1y));
}
// BitmapTexture::Eval(UV, D0, D1) (src/texture/BitmapTexture.cpp:101) after
// Texture2D::Eval (src/core/Texture.cpp:211) scaled UV and the partials
static __device__ __noinline__ V3 bitmap_eval(const DevTexture &t, float u, float v, float4 d) {
    if (t.filter == kFilterNearest)
        return mip_texel(t, 0, (int)floorf(u * (float)(1 << t.lw)), (int)floorf(v * (float)(1 << t.lh)));
    if (t.filter == kFilterBilinear) return mip_lookup_width(t, u, v, 0.0f);
    return mip_lookup_diff(t, u, v, d.x * t.uv_scale[0], d.y * t.uv_scale[1], d.z * t.uv_scale[0],
                           d.w * t.uv_scale[1]);
}

// MipMap::EvalGradient (include/core/MipMap.hpp:363) at level l, unscaled UV
__device__ __forceinline__ void mip_gradient(const DevTexture &t, int l, float u, float v, V3 &gu, V3 &gv) {
    const float W = (float)(1 << max(0, t.lw - l)), H = (float)(1 << max(0, t.lh - l));
    const float U = u * W - 0.5f, Vv = v * H - 0.5f;
    const int x = (int)floorf(U), y = (int)floorf(Vv);
    const float dx = U - (float)x, dy = Vv - (float)y;
    const V3 p00 = mip_texel(t, l, x, y), p10 = mip_texel(t, l, x + 1, y);
    const V3 p01 = mip_texel(t, l, x, y + 1), p11 = mip_texel(t, l, x + 1, y + 1);
    const V3 tmp = (p01 + p10) - p11;
    gu = ((p10 + p00 * (dy - 1.0f)) - tmp * dy) * W;
    gv = ((p01 + p00 * (dx - 1.0f)) - tmp * dx) * H;
}
__device__ __forceinline__ V3 pattern_eval(const DevTexture &t, float u, float v);
// SmoothStep (include/core/Common.hpp:994) with Clamp (:752)
__device__ __forceinline__ float smooth_step(float lo, float hi, float x) {
    float v = (x - lo) / (hi - lo);
    v = v < 0.0f ? 0.0f : (v > 1.0f ? 1.0f : v);
    return v * v * (-2.0f * v + 3.0f);
}
// WireframeTexture::Eval (src/texture/WireframeTexture.cpp:22) and
// CurvatureTexture::Eval (src/texture/CurvatureTexture.cpp:34) from the hit's
// edge distance and curvatures (geo, see BRec)
__device__ __forceinline__ V3 geo_tex_eval(const DevTexture &t, float3 geo) {
    if (t.kind == kTexWireframe) {
        const float w = t.width;
        const float al = smooth_step(w * (1.0f - t.scale), w, geo.x);
        return ld_rgb(t.b) * (1.0f - al) + ld_rgb(t.a) * al;
    }
    const float val = t.count ? geo.z : geo.y;
    if (val < 0.0f) {
        const float x = -val * t.scale;
        return ld_rgb(t.b) * (1.0f < x ? 1.0f : x);   // std::min(x, 1)
    }
    if (val > 0.0f) {
        const float x = val * t.scale;
        return ld_rgb(t.a) * (1.0f < x ? 1.0f : x);
    }
    return v3(0, 0, 0);
}
// filter: Texture::Eval(Isect, bFilter) -- unfiltered bitmaps read the nearest texel (BitmapTexture::Eval(UV) :134)
__device__ __forceinline__ V3 tex_eval(const DevTexture *T, int id, float tu, float tv, float4 duv, bool filter = true,
                                       float3 geo = make_float3(INFINITY, 0.0f, 0.0f)) {
    float sc[4];
    int ns = 0;
    while (T[id].kind == kTexScale && ns < 4) {
        sc[ns++] = T[id].scale;
        id = T[id].nested;
    }
    const DevTexture &t = T[id];
    const float u = tu * t.uv_scale[0] + t.uv_offset[0], v = tv * t.uv_scale[1] + t.uv_offset[1];
    V3 c;
    if (t.kind == kTexBitmap) {
        c = filter ? bitmap_eval(t, u, v, duv)
                   : mip_texel(t, 0, (int)floorf(u * (float)(1 << t.lw)), (int)floorf(v * (float)(1 << t.lh)));
    } else if (t.kind == kTexWireframe || t.kind == kTexCurvature) {
        c = geo_tex_eval(t, geo);
    } else {
        c = pattern_eval(t, u, v);
    }
    while (ns > 0) c = c * sc[--ns];
    return c;
}
// Texture::EvalGradient(Isect) (src/core/Texture.cpp:227): gradient at the
// UNSCALED coordinates times the UV scale; bitmaps: MipMap::EvalGradient at
// level 0 (zero with nearest filtering, BitmapTexture.cpp:145); procedural:
// forward differences with step 1e-4 (:235); ScaleTexture scales (:24).
__device__ __forceinline__ void tex_gradient(const DevTexture *T, int id, float tu, float tv, V3 &gu, V3 &gv) {
    float sc[4];
    int ns = 0;
    while (T[id].kind == kTexScale && ns < 4) {
        sc[ns++] = T[id].scale;
        id = T[id].nested;
    }
    const DevTexture &t = T[id];
    if (t.kind == kTexBitmap) {
        if (t.filter == kFilterNearest) gu = gv = v3(0, 0, 0);
        else mip_gradient(t, 0, tu, tv, gu, gv);
    } else {
        const float eps = 1e-4f;
        const V3 c = pattern_eval(t, tu, tv), cu = pattern_eval(t, tu + eps, tv), cv = pattern_eval(t, tu, tv + eps);
        gu = v3((cu.x - c.x) / eps, (cu.y - c.y) / eps, (cu.z - c.z) / eps);
        gv = v3((cv.x - c.x) / eps, (cv.y - c.y) / eps, (cv.z - c.z) / eps);
    }
    gu = gu * t.uv_scale[0];
    gv = gv * t.uv_scale[1];
    while (ns > 0) {
        --ns;
        gu = gu * sc[ns];
        gv = gv * sc[ns];
    }
}
// CheckerboardTexture / GridTexture::Eval(UV) at scaled coordinates
__device__ __forceinline__ V3 pattern_eval(const DevTexture &t, float u, float v) {
    V3 c;
    if (t.kind == kTexCheckerboard) {
        bool ex = mod_positive(mod_positive((int)(u * t.count), t.count), 2) == 0;
        bool ey = mod_positive(mod_positive((int)(v * t.count), t.count), 2) == 0;
        c = (ex ^ ey) ? ld_rgb(t.a) : ld_rgb(t.b);
    } else {
        float su = u * (float)(t.count - 1), sv = v * (float)(t.count - 1);
        float dx = su - floorf(su), dy = sv - floorf(sv);
        if (dx > 0.5f) dx -= 1.0f;
        if (dy > 0.5f) dy -= 1.0f;
        c = (fabsf(dx) < t.width || fabsf(dy) < t.width) ? ld_rgb(t.a) : ld_rgb(t.b);
    }
    return c;
}
// A BSDF parameter at the query's intersection: its texture or its constant.
// slot: 0 kd, 1 ks, 2 ks_refract, 3 sigma_a, 4 alpha(U), 5 alphaV
__device__ __forceinline__ V3 par_rgb(const DevBsdf &b, int slot, const float *c, const BRec &r) {
    if (r.tex) {
        const int t = b.tex[slot];
        if (t) return tex_eval(b.textures, t - 1, r.tu, r.tv, r.duv, true, r.geo);
    }
    return ld_rgb(c);
}
__device__ __forceinline__ float par_alpha(const DevBsdf &b, int slot, float c, const BRec &r) {
    if (r.tex) {
        const int t = b.tex[slot];
        if (t) return tex_eval(b.textures, t - 1, r.tu, r.tv, r.duv, true, r.geo).x;
    }
    return c;
}

// ------------------------------------------------------------ diffuse
// src/bsdf/DiffuseBSDF.cpp:20-67
__device__ __forceinline__ V3 diffuse_sample(const DevBsdf &b, BRec &r, float ux, float uy) {
    if (r.wi.z <= 0) return v3(0, 0, 0);
    r.measure = kMeasureSolidAngle;
    r.wo = square_to_cos_hemi(ux, uy);
    r.eta = 1.0f;
    return par_rgb(b, 0, b.kd, r);
}
__device__ __forceinline__ V3 diffuse_eval(const DevBsdf &b, const BRec &r) {
    if (r.measure != kMeasureSolidAngle || r.wi.z <= 0 || r.wo.z <= 0) return v3(0, 0, 0);
    return par_rgb(b, 0, b.kd, r) * (float)kInvPiD;
}
__device__ __forceinline__ float diffuse_pdf(const BRec &r) {
    if (r.measure != kMeasureSolidAngle || r.wi.z <= 0 || r.wo.z <= 0) return 0.0f;
    return (float)kInvPiD * r.wo.z;
}

// ------------------------------------------------------------ roughConductor
// src/bsdf/RoughConductorBSDF.cpp:54-154
__device__ __forceinline__ Mfd bsdf_mfd(const DevBsdf &b, const BRec &r) {
    const float au = par_alpha(b, 4, b.alpha_u, r);
    return mfd_make(b.distribution, au, b.anisotropic ? par_alpha(b, 5, b.alpha_v, r) : au);
}
__device__ __forceinline__ V3 conductor_fresnel(const DevBsdf &b, float c) {
    return v3(fresnel_conductor1(c, b.eta_c[0], b.k_c[0]), fresnel_conductor1(c, b.eta_c[1], b.k_c[1]),
              fresnel_conductor1(c, b.eta_c[2], b.k_c[2]));
}
__device__ __forceinline__ V3 conductor_sample(const DevBsdf &b, BRec &r, float ux, float uy) {
    r.measure = kMeasureSolidAngle;
    float ci = r.wi.z;
    if (ci <= 0.0f) return v3(0, 0, 0);
    Mfd d = bsdf_mfd(b, r);
    float pdf;
    V3 m = mfd_sample(d, ux, uy, pdf);
    if (pdf == 0.0f) return v3(0, 0, 0);
    r.wo = reflect_m(r.wi, m);
    r.eta = 1.0f;
    if (r.wo.z < 0.0f) return v3(0, 0, 0);
    float mdw = dot(m, r.wi);
    V3 F = conductor_fresnel(b, mdw);
    float G = mfd_g(d, r.wi, r.wo, m);
    float D = mfd_eval(d, m);
    float den = pdf * r.wi.z;
    const V3 ks = par_rgb(b, 1, b.ks, r);
    return v3((((ks.x * F.x) * D) * G) * mdw / den, (((ks.y * F.y) * D) * G) * mdw / den,
              (((ks.z * F.z) * D) * G) * mdw / den);
}
__device__ __forceinline__ V3 conductor_eval(const DevBsdf &b, const BRec &r) {
    float ci = r.wi.z, co = r.wo.z;
    if (r.measure != kMeasureSolidAngle || ci <= 0.0f || co <= 0.0f) return v3(0, 0, 0);
    V3 h = normalize(r.wi + r.wo);
    Mfd d = bsdf_mfd(b, r);
    float D = mfd_eval(d, h);
    if (D == 0.0f) return v3(0, 0, 0);
    V3 F = conductor_fresnel(b, dot(h, r.wi)) * par_rgb(b, 1, b.ks, r);
    float G = mfd_g(d, r.wi, r.wo, h);
    float dg = D * G, den = 4.0f * ci;
    return v3(dg * F.x / den, dg * F.y / den, dg * F.z / den);
}
__device__ __forceinline__ float conductor_pdf(const DevBsdf &b, const BRec &r) {
    float ci = r.wi.z, co = r.wo.z;
    if (r.measure != kMeasureSolidAngle || ci <= 0.0f || co <= 0.0f) return 0.0f;
    V3 h = normalize(r.wi + r.wo);
    Mfd d = bsdf_mfd(b, r);
    return mfd_pdf(d, h) / (4.0f * fabsf(dot(h, r.wo)));
}

// ------------------------------------------------------------ roughDielectric
// src/bsdf/RoughDielectricBSDF.cpp:57-281.  u1 is the Next1D draw the
// reference takes from the record's sampler inside Sample (:92).
__device__ __forceinline__ V3 dielectric_sample(const DevBsdf &b, BRec &r, float ux, float uy, float u1) {
    r.measure = kMeasureSolidAngle;
    float ci = r.wi.z;
    if (ci == 0.0f) return v3(0, 0, 0);
    Mfd d = bsdf_mfd(b, r);
    Mfd sd = d;
    float s = 1.2f - 0.2f * sqrtf(fabsf(ci));
    sd.au *= s;
    sd.av *= s;
    float pdf;
    V3 m = mfd_sample(sd, ux, uy, pdf);
    if (pdf == 0.0f) return v3(0, 0, 0);
    float ct;
    float F = fresnel_dielectric(dot(r.wi, m), b.eta, b.inv_eta, ct);
    bool refl = !(u1 > F);
    V3 W;
    if (refl) {
        r.wo = reflect_m(r.wi, m);
        r.eta = 1.0f;
        if (r.wo.z * ci <= 0.0f) return v3(0, 0, 0);
        W = par_rgb(b, 1, b.ks, r);
    } else {
        if (ct == 0.0f) return v3(0, 0, 0);
        r.wo = refract_m(r.wi, m, ct, b.eta, b.inv_eta);
        r.eta = (ct < 0.0f ? b.eta : b.inv_eta);
        if (r.wo.z * ci >= 0.0f) return v3(0, 0, 0);
        float fac = (ct < 0.0f ? b.inv_eta : b.eta);
        W = par_rgb(b, 2, b.ks_refract, r) * (fac * fac);
    }
    float v = fabsf(mfd_eval(d, m) * mfd_g(d, r.wi, r.wo, m) * dot(r.wi, m) / (pdf * ci));
    return W * v;
}
__device__ __forceinline__ V3 dielectric_eval(const DevBsdf &b, const BRec &r) {
    float ci = r.wi.z, co = r.wo.z;
    if (r.measure != kMeasureSolidAngle || ci == 0.0f) return v3(0, 0, 0);
    bool refl = ci * co > 0.0f;
    float e = ci > 0.0f ? b.eta : b.inv_eta;
    V3 h = refl ? normalize(r.wi + r.wo) : normalize(r.wi + r.wo * e);
    h = h * signum(h.z);
    Mfd d = bsdf_mfd(b, r);
    float D = mfd_eval(d, h);
    if (D == 0.0f) return v3(0, 0, 0);
    float ct;
    float F = fresnel_dielectric(dot(r.wi, h), b.eta, b.inv_eta, ct);
    float G = mfd_g(d, r.wi, r.wo, h);
    if (refl) return par_rgb(b, 1, b.ks, r) * (F * D * G / (4.0f * fabsf(ci)));
    float sd = dot(r.wi, h) + e * dot(r.wo, h);
    float val = ((1.0f - F) * D * G * e * e * dot(r.wi, h) * dot(r.wo, h)) / (ci * sd * sd);
    float fac = (ci < 0.0f ? b.inv_eta : b.eta);
    return par_rgb(b, 2, b.ks_refract, r) * fabsf(val * fac * fac);
}
__device__ __forceinline__ float dielectric_pdf(const DevBsdf &b, const BRec &r) {
    if (r.measure != kMeasureSolidAngle) return 0.0f;
    float ci = r.wi.z, co = r.wo.z;
    if (ci == 0.0f || co == 0.0f) return 0.0f;
    bool refl = ci * co > 0.0f;
    V3 h;
    float J;
    if (refl) {
        h = normalize(r.wi + r.wo);
        J = 1.0f / (4.0f * dot(r.wo, h));
    } else {
        float e = ci > 0.0f ? b.eta : b.inv_eta;
        h = normalize(r.wi + r.wo * e);
        float sd = dot(r.wi, h) + e * dot(r.wo, h);
        J = (e * e * dot(r.wo, h)) / (sd * sd);
    }
    h = h * signum(h.z);
    Mfd d = bsdf_mfd(b, r);
    float s = 1.2f - 0.2f * sqrtf(fabsf(ci));
    d.au *= s;
    d.av *= s;
    float ct;
    float F = fresnel_dielectric(dot(r.wi, h), b.eta, b.inv_eta, ct);
    float pdf = mfd_pdf(d, h) * (refl ? F : (1.0f - F));
    return fabsf(pdf * J);
}

// ------------------------------------------------------------ roughPlastic
// The roughness of roughPlastic / roughCoating: the activated constant, or the
// texture's first channel clamped to [5e-4, 1] (RoughPlasticBSDF.cpp:77)
__device__ __forceinline__ float coat_alpha(const DevBsdf &b, const BRec &r) {
    return b.alpha_tex ? clampf(par_alpha(b, 4, b.alpha_u, r), 5e-4f, 1.0f) : b.alpha_u;
}
// src/bsdf/RoughPlasticBSDF.cpp:66-192
__device__ __forceinline__ V3 plastic_eval(const DevBsdf &b, const BRec &r) {
    float ci = r.wi.z, co = r.wo.z;
    if (r.measure == kMeasureUnknown || ci <= 0.0f || co <= 0.0f) return v3(0, 0, 0);
    const float a = coat_alpha(b, r);
    Mfd d = mfd_make(b.distribution, a, a);
    float ct;
    V3 h = normalize(r.wi + r.wo);
    float D = mfd_eval(d, h);
    float F = fresnel_dielectric(dot(r.wi, h), b.eta, b.inv_eta, ct);
    float G = mfd_g(d, r.wi, r.wi, h);   // G(Wi, Wi, H) as the reference does (:146)
    float val = F * D * G / (4.0f * ci);
    V3 res = par_rgb(b, 1, b.ks, r) * val;
    V3 dif = par_rgb(b, 0, b.kd, r);
    float t12 = rft_eval(b, ci, d.au), t21 = rft_eval(b, co, d.au);
    float fdr = plastic_fdr(b, d.au);
    if (b.nonlinear) dif = v3(dif.x / (1.0f - dif.x * fdr), dif.y / (1.0f - dif.y * fdr), dif.z / (1.0f - dif.z * fdr));
    else dif = dif / (1.0f - fdr);
    // INV_PI is a double literal in the reference: the scalar is formed in double
    float k = (float)(kInvPiD * co * t12 * t21 * b.inv_eta2);
    return res + dif * k;
}
__device__ __forceinline__ float plastic_spec_pdf(const DevBsdf &b, float ci, float alpha) {
    float sp = 1.0f - rft_eval(b, ci, alpha);
    return (sp * b.spec_w) / (sp * b.spec_w + (1.0f - sp) * (1.0f - b.spec_w));
}
__device__ __forceinline__ float plastic_pdf(const DevBsdf &b, const BRec &r) {
    float ci = r.wi.z, co = r.wo.z;
    if (r.measure == kMeasureUnknown || ci <= 0.0f || co <= 0.0f) return 0.0f;
    const float a = coat_alpha(b, r);
    Mfd d = mfd_make(b.distribution, a, a);
    V3 h = normalize(r.wi + r.wo);
    float sp = plastic_spec_pdf(b, ci, d.au), dp = 1.0f - sp;
    float J = 1.0f / (4.0f * dot(r.wo, h));
    float res = mfd_pdf(d, h) * J * sp;
    res += dp * cos_hemi_pdf(r.wo);
    return res;
}
__device__ __forceinline__ V3 plastic_sample(const DevBsdf &b, BRec &r, float ux, float uy) {
    float ci = r.wi.z;
    if (ci <= 0.0f) return v3(0, 0, 0);
    const float a = coat_alpha(b, r);
    Mfd d = mfd_make(b.distribution, a, a);
    float sp = plastic_spec_pdf(b, ci, d.au), dp = 1.0f - sp;
    bool spec;
    if (uy < sp) { uy /= sp; spec = true; }
    else { uy = (uy - sp) / (1.0f - sp); spec = false; }
    if (spec) {
        float pdf;
        V3 m = mfd_sample(d, ux, uy, pdf);
        r.wo = reflect_m(r.wi, m);
        r.measure = kMeasureDiscrete;
    } else {
        r.wo = square_to_cos_hemi(ux, uy);
        r.measure = kMeasureSolidAngle;
    }
    r.eta = 1.0f;
    V3 h = normalize(r.wi + r.wo);
    float J = 1.0f / (4.0f * dot(r.wo, h));
    float P = mfd_pdf(d, h) * J * sp + dp * cos_hemi_pdf(r.wo);
    if (P == 0.0f) return v3(0, 0, 0);
    return plastic_eval(b, r) / P;
}

// ------------------------------------------------------------ smooth BSDFs
// Delta-direction match |d . wo - 1| <= DeltaEpsilon (include/core/Common.hpp:46);
// DeltaEpsilon is the double literal 1e-3, so the comparison is made in double.
__device__ __forceinline__ bool delta_match(V3 d, V3 wo) { return (double)fabsf(dot(d, wo) - 1.0f) <= 1e-3; }
// Reflect / Refract about the local normal (src/core/Common.cpp:606-615)
__device__ __forceinline__ V3 reflect_n(V3 wi) { return v3(-wi.x, -wi.y, wi.z); }
__device__ __forceinline__ V3 refract_n(V3 wi, float ct, float eta, float inv_eta) {
    float sc = -(ct < 0.0f ? inv_eta : eta);
    return v3(sc * wi.x, sc * wi.y, ct);
}

// src/bsdf/MirrorBSDF.cpp:15-55 (the measure is set only past the cosine test);
// ConductorBSDF's Eval / Pdf use the same match (src/bsdf/ConductorBSDF.cpp:46-70)
__device__ __forceinline__ bool mirror_match(const BRec &r) {
    return r.wi.z > 0.0f && r.wo.z > 0.0f && r.measure == kMeasureDiscrete && delta_match(reflect_n(r.wi), r.wo);
}
__device__ __forceinline__ V3 mirror_sample(BRec &r) {
    if (r.wi.z <= 0) return v3(0, 0, 0);
    r.wo = reflect_n(r.wi);
    r.measure = kMeasureDiscrete;
    r.eta = 1.0f;
    return v3(1, 1, 1);
}
__device__ __forceinline__ V3 mirror_eval(const BRec &r) { return mirror_match(r) ? v3(1, 1, 1) : v3(0, 0, 0); }
__device__ __forceinline__ float mirror_pdf(const BRec &r) { return mirror_match(r) ? 1.0f : 0.0f; }

// src/bsdf/ConductorBSDF.cpp:32-70 (eta_c = intIOR / extIOR on every channel)
__device__ __forceinline__ V3 sconductor_sample(const DevBsdf &b, BRec &r) {
    r.measure = kMeasureDiscrete;
    float ci = r.wi.z;
    if (ci <= 0.0f) return v3(0, 0, 0);
    V3 F = conductor_fresnel(b, ci);
    r.wo = reflect_n(r.wi);
    r.eta = 1.0f;
    return par_rgb(b, 1, b.ks, r) * F;
}
__device__ __forceinline__ V3 sconductor_eval(const DevBsdf &b, const BRec &r) {
    if (!mirror_match(r)) return v3(0, 0, 0);
    return par_rgb(b, 1, b.ks, r) * conductor_fresnel(b, r.wi.z);
}

// src/bsdf/DielectricBSDF.cpp:33-110 (Eval and Pdf test no measure)
__device__ __forceinline__ V3 sdielectric_sample(const DevBsdf &b, BRec &r, float ux) {
    r.measure = kMeasureDiscrete;
    float ct;
    float F = fresnel_dielectric(r.wi.z, b.eta, b.inv_eta, ct);
    if (ux < F) {
        r.wo = reflect_n(r.wi);
        r.eta = 1.0f;
        return par_rgb(b, 1, b.ks, r);
    }
    r.wo = refract_n(r.wi, ct, b.eta, b.inv_eta);
    r.eta = ct < 0.0f ? b.eta : b.inv_eta;
    float f = ct < 0.0f ? b.inv_eta : b.eta;   // radiance transport
    return par_rgb(b, 2, b.ks_refract, r) * (f * f);
}
// Eval and Pdf share the lobe test: 0 none, 1 reflection, 2 refraction with
// cos(theta_t) < 0 (entering), 3 refraction leaving
__device__ __forceinline__ float sdielectric_lobe(const DevBsdf &b, const BRec &r, int &lobe) {
    float ci = r.wi.z, co = r.wo.z, ct;
    float F = fresnel_dielectric(ci, b.eta, b.inv_eta, ct);
    lobe = 0;
    if (ci * co >= 0.0f) {
        if (delta_match(reflect_n(r.wi), r.wo)) lobe = 1;
    } else if (delta_match(refract_n(r.wi, ct, b.eta, b.inv_eta), r.wo)) {
        lobe = ct < 0.0f ? 2 : 3;
    }
    return F;
}
__device__ __forceinline__ V3 sdielectric_eval(const DevBsdf &b, const BRec &r) {
    int lobe;
    float F = sdielectric_lobe(b, r, lobe);
    if (lobe == 1) return par_rgb(b, 1, b.ks, r) * F;
    if (lobe == 0) return v3(0, 0, 0);
    float f = lobe == 2 ? b.inv_eta : b.eta;
    return (par_rgb(b, 2, b.ks_refract, r) * (f * f)) * (1.0f - F);
}
__device__ __forceinline__ float sdielectric_pdf(const DevBsdf &b, const BRec &r) {
    int lobe;
    float F = sdielectric_lobe(b, r, lobe);
    return lobe == 0 ? 0.0f : (lobe == 1 ? F : 1.0f - F);
}

// src/bsdf/PlasticBSDF.cpp:33-142 (fdr_int = ApproxFresnelDiffuseReflectance(1 / eta))
__device__ __forceinline__ float splastic_spec_pdf(const DevBsdf &b, float Fi) {
    return (Fi * b.spec_w) / (Fi * b.spec_w + (1.0f - Fi) * (1.0f - b.spec_w));
}
__device__ __forceinline__ V3 splastic_diffuse(const DevBsdf &b, const BRec &r) {
    V3 dif = par_rgb(b, 0, b.kd, r);
    float fdr = b.fdr_int;
    if (b.nonlinear) return v3(dif.x / (1.0f - dif.x * fdr), dif.y / (1.0f - dif.y * fdr), dif.z / (1.0f - dif.z * fdr));
    return dif / (1.0f - fdr);
}
__device__ __forceinline__ V3 splastic_sample(const DevBsdf &b, BRec &r, float ux, float uy) {
    float ci = r.wi.z;
    if (ci <= 0.0f) return v3(0, 0, 0);
    float ct;
    float Fi = fresnel_dielectric(ci, b.eta, b.inv_eta, ct);
    float sp = splastic_spec_pdf(b, Fi);
    r.eta = 1.0f;
    if (ux < sp) {
        r.measure = kMeasureDiscrete;
        r.wo = reflect_n(r.wi);
        return (par_rgb(b, 1, b.ks, r) * Fi) / sp;
    }
    r.measure = kMeasureSolidAngle;
    r.wo = square_to_cos_hemi((ux - sp) / (1.0f - sp), uy);
    float Fo = fresnel_dielectric(r.wo.z, b.eta, b.inv_eta, ct);
    return splastic_diffuse(b, r) * (b.inv_eta2 * (1.0f - Fi) * (1.0f - Fo) / (1.0f - sp));
}
__device__ __forceinline__ V3 splastic_eval(const DevBsdf &b, const BRec &r) {
    float ci = r.wi.z, co = r.wo.z;
    if (r.measure == kMeasureUnknown || ci <= 0.0f || co <= 0.0f) return v3(0, 0, 0);
    float ct;
    float Fi = fresnel_dielectric(ci, b.eta, b.inv_eta, ct);
    if (r.measure == kMeasureDiscrete) return delta_match(reflect_n(r.wi), r.wo) ? par_rgb(b, 1, b.ks, r) * Fi : v3(0, 0, 0);
    float Fo = fresnel_dielectric(co, b.eta, b.inv_eta, ct);
    return splastic_diffuse(b, r) * (cos_hemi_pdf(r.wo) * b.inv_eta2 * (1.0f - Fi) * (1.0f - Fo));
}
__device__ __forceinline__ float splastic_pdf(const DevBsdf &b, const BRec &r) {
    float ci = r.wi.z, co = r.wo.z;
    if (r.measure == kMeasureUnknown || ci <= 0.0f || co <= 0.0f) return 0.0f;
    float ct;
    float Fi = fresnel_dielectric(ci, b.eta, b.inv_eta, ct);
    float sp = splastic_spec_pdf(b, Fi);
    if (r.measure == kMeasureDiscrete) return delta_match(reflect_n(r.wi), r.wo) ? 1.0f - sp : 0.0f;   // as :118
    return cos_hemi_pdf(r.wo) * (1.0f - sp);
}

// ------------------------------------------------------------ roughDiffuse
// src/bsdf/RoughDiffuseBSDF.cpp:19-140 (Oren-Nayar: the full model or the fast
// approximation); std::max / std::min / SafeAcos / SafeSqrt as the reference
// spells them (include/core/Common.hpp:818-839)
__device__ __forceinline__ float max_f(float a, float b) { return (a < b) ? b : a; }
__device__ __forceinline__ float min_f(float a, float b) { return (b < a) ? b : a; }
__device__ __forceinline__ float safe_acos(float v) { return acosf(min_f(1.0f, max_f(-1.0f, v))); }
__device__ __forceinline__ float safe_sqrt(float v) { return sqrtf(max_f(0.0f, v)); }
__device__ __forceinline__ float frame_sin_theta(V3 v) {   // Frame::SinTheta (src/core/Frame.cpp:38)
    float t = sin_theta2(v);
    return t <= 0.0f ? 0.0f : sqrtf(t);
}
__device__ __forceinline__ float frame_sin_phi(V3 v) {   // :68
    float t = frame_sin_theta(v);
    return t == 0.0f ? 1.0f : clampf(v.y / t, -1.0f, 1.0f);
}
__device__ __forceinline__ float frame_cos_phi(V3 v) {   // :78
    float t = frame_sin_theta(v);
    return t == 0.0f ? 1.0f : clampf(v.x / t, -1.0f, 1.0f);
}
__device__ __forceinline__ V3 roughdiffuse_eval(const DevBsdf &b, const BRec &r) {
    float ci = r.wi.z, co = r.wo.z;
    if (ci <= 0.0f || co <= 0.0f || r.measure != kMeasureSolidAngle) return v3(0, 0, 0);
    float sigma = clampf(par_alpha(b, 4, b.alpha_u, r), 5e-4f, 1.0f) * 0.70710678118655f;
    float s2 = sigma * sigma;
    float sti = frame_sin_theta(r.wi), sto = frame_sin_theta(r.wo);
    float cpd = 0.0f;
    if (sti > 1e-4f && sto > 1e-4f) {
        float spi = frame_sin_phi(r.wi), cpi = frame_cos_phi(r.wi);
        float spo = frame_sin_phi(r.wo), cpo = frame_cos_phi(r.wo);
        cpd = cpi * cpo + spi * spo;
    }
    const float inv_pi = (float)kInvPiD;
    if (b.fast_approx) {
        float A = 1.0f - 0.5f * s2 / (s2 + 0.33f);
        float B = 0.45f * s2 / (s2 + 0.09f);
        float sa, tb;
        if (ci > co) { sa = sto; tb = sti / ci; }
        else { sa = sti; tb = sto / co; }
        return par_rgb(b, 0, b.kd, r) * (inv_pi * co * (A + B * max_f(cpd, 0.0f) * sa * tb));
    }
    float thi = safe_acos(ci), tho = safe_acos(co);
    float al = max_f(thi, tho), be = min_f(thi, tho);
    float sa, sb, tb;
    if (ci > co) { sa = sto; sb = sti; tb = sti / ci; }
    else { sa = sti; sb = sto; tb = sto / co; }
    float t1 = s2 / (s2 + 0.09f);
    float t2 = (4.0f * (float)(kInvPiD * kInvPiD)) * al * be;
    float t3 = 2.0f * be * inv_pi;
    float C1 = 1.0f - 0.5f * s2 / (s2 + 0.33f);
    float C2 = 0.45f * t1;
    float C3 = 0.125f * t1 * t2 * t2;
    float C4 = 0.17f * s2 / (s2 + 0.13f);
    if (cpd > 0.0f) C2 *= sa;
    else C2 *= sa - t3 * t3 * t3;
    float th = (sa + sb) / (safe_sqrt(1.0f - sa * sa) + safe_sqrt(1.0f - sb * sb));
    if (isinf(th) || isnan(th)) return v3(0, 0, 0);
    V3 rho = par_rgb(b, 0, b.kd, r);
    V3 lr1 = rho * (C1 + cpd * C2 * tb + (1.0f - fabsf(cpd)) * C3 * th);
    V3 lr2 = (rho * rho) * (C4 * (1.0f - cpd * t3 * t3));
    return (lr1 + lr2) * (inv_pi * co);
}
__device__ __forceinline__ float roughdiffuse_pdf(const BRec &r) {
    if (r.wi.z <= 0.0f || r.wo.z <= 0.0f || r.measure != kMeasureSolidAngle) return 0.0f;
    return cos_hemi_pdf(r.wo);
}
__device__ __forceinline__ V3 roughdiffuse_sample(const DevBsdf &b, BRec &r, float ux, float uy) {
    r.measure = kMeasureSolidAngle;
    if (r.wi.z <= 0.0f) return v3(0, 0, 0);
    r.wo = square_to_cos_hemi(ux, uy);
    r.eta = 1.0f;
    float pdf = cos_hemi_pdf(r.wo);
    if (pdf == 0.0f) return v3(0, 0, 0);
    return roughdiffuse_eval(b, r) / pdf;
}

// ------------------------------------------------------------ dispatch (leaf BSDFs)
__device__ __forceinline__ V3 leaf_eval(const DevBsdf &b, const BRec &r) {
    switch (b.type) {
    case kDiffuse: return diffuse_eval(b, r);
    case kRoughConductor: return conductor_eval(b, r);
    case kRoughDielectric: return dielectric_eval(b, r);
    case kRoughPlastic: return plastic_eval(b, r);
    case kMirror: return mirror_eval(r);
    case kConductor: return sconductor_eval(b, r);
    case kDielectric: return sdielectric_eval(b, r);
    case kRoughDiffuse: return roughdiffuse_eval(b, r);
    default: return splastic_eval(b, r);
    }
}
__device__ __forceinline__ float leaf_pdf(const DevBsdf &b, const BRec &r) {
    switch (b.type) {
    case kDiffuse: return diffuse_pdf(r);
    case kRoughConductor: return conductor_pdf(b, r);
    case kRoughDielectric: return dielectric_pdf(b, r);
    case kRoughPlastic: return plastic_pdf(b, r);
    case kMirror:
    case kConductor: return mirror_pdf(r);
    case kDielectric: return sdielectric_pdf(b, r);
    case kRoughDiffuse: return roughdiffuse_pdf(r);
    default: return splastic_pdf(b, r);
    }
}
__device__ __forceinline__ V3 leaf_sample(const DevBsdf &b, BRec &r, float ux, float uy, float u1) {
    switch (b.type) {
    case kDiffuse: return diffuse_sample(b, r, ux, uy);
    case kRoughConductor: return conductor_sample(b, r, ux, uy);
    case kRoughDielectric: return dielectric_sample(b, r, ux, uy, u1);
    case kRoughPlastic: return plastic_sample(b, r, ux, uy);
    case kMirror: return mirror_sample(r);
    case kConductor: return sconductor_sample(b, r);
    case kDielectric: return sdielectric_sample(b, r, ux);
    case kRoughDiffuse: return roughdiffuse_sample(b, r, ux, uy);
    default: return splastic_sample(b, r, ux, uy);
    }
}

// ------------------------------------------------------------ roughCoating
// src/bsdf/RoughCoatingBSDF.cpp:62-385 over one nested leaf BSDF
__device__ __forceinline__ V3 coat_refract(V3 wi, float inv_eta) {   // RefractIn :347 / RefractOut :367
    bool entering = wi.z > 0.0f;
    float st2 = inv_eta * inv_eta * sin_theta2(wi);
    if (st2 >= 1.0f) return v3(0, 0, 0);
    float ct = sqrtf(1.0f - st2);
    return v3(inv_eta * wi.x, inv_eta * wi.y, entering ? ct : -ct);
}
__device__ __forceinline__ V3 coating_eval(const DevBsdf &b, const DevBsdf &nb, const BRec &r) {
    float ci = r.wi.z, co = r.wo.z;
    if (ci * co <= 0.0f) return v3(0, 0, 0);
    const float a = coat_alpha(b, r);
    Mfd d = mfd_make(b.distribution, a, a);
    V3 h = normalize(r.wi + r.wo) * signum(r.wo.z);
    float ct;
    float D = mfd_eval(d, h);
    float F = fresnel_dielectric(fabsf(dot(r.wi, h)), b.eta, b.inv_eta, ct);
    float G = mfd_g(d, r.wi, r.wo, h);
    float den = 4.0f * fabsf(ci);
    const V3 ks = par_rgb(b, 1, b.ks, r);
    V3 res = v3((((ks.x * F) * D) * G) / den, (((ks.y * F) * D) * G) / den, (((ks.z * F) * D) * G) / den);
    BRec ri = r;
    ri.wi = coat_refract(r.wi, b.inv_eta);
    ri.wo = coat_refract(r.wo, b.inv_eta);
    V3 nv = leaf_eval(nb, ri);
    float ti = rft_eval(b, fabsf(ci), d.au), to = rft_eval(b, fabsf(co), d.au);
    nv = v3(nv.x * ti * to, nv.y * ti * to, nv.z * ti * to);
    V3 sa = par_rgb(b, 3, b.sigma_a, r) * b.thickness;
    if (!is_zero(sa)) {
        float q = 1.0f / fabsf(ri.wi.z) + 1.0f / fabsf(ri.wo.z);
        nv = nv * v3(expf(-sa.x * q), expf(-sa.y * q), expf(-sa.z * q));
    }
    if (r.measure == kMeasureSolidAngle) nv = nv * (b.inv_eta * b.inv_eta * r.wo.z / ri.wo.z);
    return res + nv;
}
__device__ __forceinline__ float coating_pdf(const DevBsdf &b, const DevBsdf &nb, const BRec &r) {
    V3 h = normalize(r.wi + r.wo) * signum(r.wo.z);
    const float a = coat_alpha(b, r);
    Mfd d = mfd_make(b.distribution, a, a);
    float ci = r.wi.z, co = r.wo.z;
    float r12 = 1.0f - rft_eval(b, fabsf(ci), d.au);
    float sp = (r12 * b.spec_w) / (r12 * b.spec_w + (1.0f - r12) * (1.0f - b.spec_w));
    float np = 1.0f - sp;
    float res = 0.0f;
    if (ci * co > 0.0f) {
        float J = 1.0f / (4.0f * fabsf(dot(r.wo, h)));
        res = mfd_pdf(d, h) * J * sp;
    }
    BRec ri = r;
    ri.wi = coat_refract(r.wi, b.inv_eta);
    ri.wo = coat_refract(r.wo, b.inv_eta);
    float p = leaf_pdf(nb, ri);
    if (ri.measure == kMeasureSolidAngle) p *= b.inv_eta * b.inv_eta * co / ri.wo.z;
    return res + p * np;
}
__device__ __forceinline__ V3 coating_sample(const DevBsdf &b, const DevBsdf &nb, BRec &r, float ux, float uy, float u1) {
    const float a = coat_alpha(b, r);
    Mfd d = mfd_make(b.distribution, a, a);
    float aci = fabsf(r.wi.z);
    float r12 = 1.0f - rft_eval(b, aci, d.au);
    float sp = (r12 * b.spec_w) / (r12 * b.spec_w + (1.0f - r12) * (1.0f - b.spec_w));
    bool spec;
    if (ux < sp) { spec = true; ux /= sp; }
    else { spec = false; ux = (ux - sp) / (1.0f - sp); }
    if (spec) {
        float pdf;
        V3 m = mfd_sample(d, ux, uy, pdf);
        r.wo = reflect_m(r.wi, m);
        r.measure = kMeasureDiscrete;
        r.eta = 1.0f;
        if (r.wo.z * r.wo.z <= 0.0f) return v3(0, 0, 0);
    } else {
        V3 wib = r.wi;
        r.wi = coat_refract(r.wi, b.inv_eta);
        V3 res = leaf_sample(nb, r, ux, uy, u1);
        r.wi = wib;
        if (is_zero(res)) return v3(0, 0, 0);
        r.wo = coat_refract(r.wo, b.eta);
        if (is_zero(r.wo)) return v3(0, 0, 0);
    }
    float P = coating_pdf(b, nb, r);
    if (P == 0.0f) return v3(0, 0, 0);
    return coating_eval(b, nb, r) / P;
}

// ------------------------------------------------------------ coating
// src/bsdf/CoatingBSDF.cpp:28-302: a smooth dielectric layer over one leaf BSDF
__device__ __forceinline__ V3 scoat_refract_in(const DevBsdf &b, V3 wi, float &R) {   // RefractIn :290
    float ct;
    R = fresnel_dielectric(fabsf(wi.z), b.eta, b.inv_eta, ct);
    return v3(b.inv_eta * wi.x, b.inv_eta * wi.y, -signum(wi.z) * ct);
}
__device__ __forceinline__ V3 scoat_refract_out(const DevBsdf &b, V3 wi, float &R) {   // RefractOut :297
    float ct;
    R = fresnel_dielectric(fabsf(wi.z), b.inv_eta, b.eta, ct);
    return v3(b.eta * wi.x, b.eta * wi.y, -signum(wi.z) * ct);
}
__device__ __forceinline__ V3 scoat_absorb(const DevBsdf &b, const BRec &r, V3 res, V3 wi_int, V3 wo_int) {
    V3 sa = par_rgb(b, 3, b.sigma_a, r) * b.thickness;
    if (is_zero(sa)) return res;
    float q = 1.0f / fabsf(wi_int.z) + 1.0f / fabsf(wo_int.z);
    return res * v3(expf(-sa.x * q), expf(-sa.y * q), expf(-sa.z * q));
}
__device__ __forceinline__ float scoat_spec_pdf(const DevBsdf &b, float R12) {
    return (R12 * b.spec_w) / (R12 * b.spec_w + (1.0f - R12) * (1.0f - b.spec_w));
}
__device__ __forceinline__ V3 scoating_sample(const DevBsdf &b, const DevBsdf &nb, BRec &r, float ux, float uy, float u1) {
    float R12;
    V3 wip = scoat_refract_in(b, r.wi, R12);
    float sp = scoat_spec_pdf(b, R12);
    if (ux < sp) {
        r.wo = reflect_n(r.wi);
        r.eta = 1.0f;
        r.measure = kMeasureDiscrete;
        return par_rgb(b, 1, b.ks, r) * (R12 / sp);
    }
    ux = (ux - sp) / (1.0f - sp);
    if (R12 == 1.0f) return v3(0, 0, 0);
    V3 wib = r.wi;
    r.wi = wip;
    V3 res = leaf_sample(nb, r, ux, uy, u1);
    r.wi = wib;
    if (is_zero(res)) return v3(0, 0, 0);
    V3 wop = r.wo;
    res = scoat_absorb(b, r, res, wip, wop);
    float R21;
    r.wo = scoat_refract_out(b, wop, R21);
    if (R21 == 1.0f) return v3(0, 0, 0);
    res = res / (1.0f - sp);
    return res * ((1.0f - R12) * (1.0f - R21));
}
__device__ __forceinline__ V3 scoating_eval(const DevBsdf &b, const DevBsdf &nb, const BRec &r) {
    if (r.measure == kMeasureDiscrete) {
        if (!delta_match(reflect_n(r.wi), r.wo)) return v3(0, 0, 0);
        float ct;
        return par_rgb(b, 1, b.ks, r) * fresnel_dielectric(fabsf(r.wi.z), b.eta, b.inv_eta, ct);
    }
    float R12, R21;
    BRec ri = r;
    ri.wi = scoat_refract_in(b, r.wi, R12);
    ri.wo = scoat_refract_in(b, r.wo, R21);
    if (R12 == 1.0f || R21 == 1.0f) return v3(0, 0, 0);
    V3 res = (leaf_eval(nb, ri) * (1.0f - R12)) * (1.0f - R21);
    res = scoat_absorb(b, r, res, ri.wi, ri.wo);
    if (r.measure == kMeasureSolidAngle) res = res * (b.inv_eta * b.inv_eta * r.wo.z / ri.wo.z);
    return res;
}
__device__ __forceinline__ float scoating_pdf(const DevBsdf &b, const DevBsdf &nb, const BRec &r) {
    float R12;
    V3 wip = scoat_refract_in(b, r.wi, R12);
    float sp = scoat_spec_pdf(b, R12);
    if (r.measure == kMeasureDiscrete) return delta_match(reflect_n(r.wi), r.wo) ? sp : 0.0f;
    float R21;
    BRec ri = r;
    ri.wi = wip;
    ri.wo = scoat_refract_in(b, r.wo, R21);
    if (R12 == 1.0f || R21 == 1.0f) return 0.0f;
    float p = leaf_pdf(nb, ri);
    if (r.measure == kMeasureSolidAngle) p *= b.inv_eta * b.inv_eta * r.wo.z / ri.wo.z;
    return p * (1.0f - sp);
}

// ------------------------------------------------------------ full dispatch
// A layer is a leaf BSDF or a (rough) coating over a leaf; a twoSided BSDF picks
// one layer per side (src/bsdf/TwoSidedBSDF.cpp:19-67), mirroring z for the
// back side.  Deeper stacks go through deep_* below.
__device__ __forceinline__ V3 layer_eval(const DevBsdf *bs, const DevBsdf &b, const BRec &r) {
    if (b.type == kRoughCoating) return coating_eval(b, bs[b.nested], r);
    if (b.type == kCoating) return scoating_eval(b, bs[b.nested], r);
    return leaf_eval(b, r);
}
__device__ __forceinline__ float layer_pdf(const DevBsdf *bs, const DevBsdf &b, const BRec &r) {
    if (b.type == kRoughCoating) return coating_pdf(b, bs[b.nested], r);
    if (b.type == kCoating) return scoating_pdf(b, bs[b.nested], r);
    return leaf_pdf(b, r);
}
__device__ __forceinline__ V3 layer_sample(const DevBsdf *bs, const DevBsdf &b, BRec &r, float ux, float uy, float u1) {
    if (b.type == kRoughCoating) return coating_sample(b, bs[b.nested], r, ux, uy, u1);
    if (b.type == kCoating) return scoating_sample(b, bs[b.nested], r, ux, uy, u1);
    return leaf_sample(b, r, ux, uy, u1);
}
__device__ __forceinline__ V3 twosided_eval(const DevBsdf *bs, const DevBsdf &b, const BRec &r) {
    BRec c = r;
    if (c.wi.z > 0.0f) return layer_eval(bs, bs[b.nested], c);
    c.wi.z *= -1.0f;
    c.wo.z *= -1.0f;
    return layer_eval(bs, bs[b.nested2], c);
}
__device__ __forceinline__ float twosided_pdf(const DevBsdf *bs, const DevBsdf &b, const BRec &r) {
    BRec c = r;
    if (c.wi.z > 0.0f) return layer_pdf(bs, bs[b.nested], c);
    c.wi.z *= -1.0f;
    c.wo.z *= -1.0f;
    return layer_pdf(bs, bs[b.nested2], c);
}
__device__ __forceinline__ V3 twosided_sample(const DevBsdf *bs, const DevBsdf &b, BRec &r, float ux, float uy, float u1) {
    const bool flip = r.wi.z < 0.0f;
    if (flip) r.wi.z *= -1.0f;
    V3 res = layer_sample(bs, bs[flip ? b.nested2 : b.nested], r, ux, uy, u1);
    if (flip) {
        r.wi.z *= -1.0f;
        if (!is_zero(res)) r.wo.z *= -1.0f;
    }
    return res;
}
// ---- stacks deeper than one layer (a coating over a coating or a twoSided, a
// twoSided over a twoSided or over a coated coating; the host flags them `deep`
// and bounds them to kNestLevels layers).  The reference evaluates a stack by
// recursion (each coating calls its nested BSDF, src/bsdf/RoughCoatingBSDF.cpp,
// src/bsdf/CoatingBSDF.cpp, src/bsdf/TwoSidedBSDF.cpp); here one loop walks
// down the stack, recording what each layer adds and multiplies, evaluates the
// leaf once, and applies the layers on the way back up in the reference's
// operation order -- the same arithmetic as coating_* / scoating_* above, in
// three compact out-of-line functions.
static __device__ __noinline__ V3 deep_leaf_eval(const DevBsdf &b, const BRec &r) { return leaf_eval(b, r); }
static __device__ __noinline__ float deep_leaf_pdf(const DevBsdf &b, const BRec &r) { return leaf_pdf(b, r); }
static __device__ __noinline__ V3 deep_leaf_sample(const DevBsdf &b, BRec &r, float ux, float uy, float u1) {
    return leaf_sample(b, r, ux, uy, u1);
}
struct DeepLayer {
    int kind;        // 0 roughCoating, 1 coating, 2 twoSided (no arithmetic on the way up)
    bool has_e, has_s;
    V3 add, e;       // eval: the layer's own lobe; its absorption factor
    float m1, m2;    // eval: rft in and out (roughCoating), 1 - R12 and 1 - R21 (coating); pdf: the nested weight
    float s;         // the solid-angle factor of the refraction
};
static __device__ __noinline__ V3 deep_eval(const DevBsdf *bs, int id, const BRec &r0) {
    DeepLayer L[kNestLevels];
    int n = 0;
    BRec c = r0;
    V3 v = v3(0, 0, 0);
    bool stop = false;
    for (;;) {
        const DevBsdf &b = bs[id];
        if (n == kNestLevels || !(b.type == kRoughCoating || b.type == kCoating || b.type == kTwoSided)) {
            v = deep_leaf_eval(b, c);
            break;
        }
        DeepLayer &l = L[n++];
        l.kind = b.type == kRoughCoating ? 0 : b.type == kCoating ? 1 : 2;
        l.has_e = l.has_s = false;
        if (l.kind == 2) {   // TwoSidedBSDF::Eval (:46)
            if (c.wi.z > 0.0f) {
                id = b.nested;
            } else {
                c.wi.z *= -1.0f;
                c.wo.z *= -1.0f;
                id = b.nested2;
            }
            continue;
        }
        BRec ri = c;
        if (l.kind == 0) {   // RoughCoatingBSDF::Eval (coating_eval)
            const float ci = c.wi.z, co = c.wo.z;
            if (ci * co <= 0.0f) { stop = true; break; }
            const float a = coat_alpha(b, c);
            Mfd d = mfd_make(b.distribution, a, a);
            V3 h = normalize(c.wi + c.wo) * signum(c.wo.z);
            float ct;
            float D = mfd_eval(d, h);
            float F = fresnel_dielectric(fabsf(dot(c.wi, h)), b.eta, b.inv_eta, ct);
            float G = mfd_g(d, c.wi, c.wo, h);
            float den = 4.0f * fabsf(ci);
            const V3 ks = par_rgb(b, 1, b.ks, c);
            l.add = v3((((ks.x * F) * D) * G) / den, (((ks.y * F) * D) * G) / den, (((ks.z * F) * D) * G) / den);
            ri.wi = coat_refract(c.wi, b.inv_eta);
            ri.wo = coat_refract(c.wo, b.inv_eta);
            l.m1 = rft_eval(b, fabsf(ci), d.au);
            l.m2 = rft_eval(b, fabsf(co), d.au);
            V3 sa = par_rgb(b, 3, b.sigma_a, c) * b.thickness;
            if (!is_zero(sa)) {
                float q = 1.0f / fabsf(ri.wi.z) + 1.0f / fabsf(ri.wo.z);
                l.e = v3(expf(-sa.x * q), expf(-sa.y * q), expf(-sa.z * q));
                l.has_e = true;
            }
        } else {             // CoatingBSDF::Eval (scoating_eval)
            if (c.measure == kMeasureDiscrete) {
                float ct;
                v = delta_match(reflect_n(c.wi), c.wo)
                        ? par_rgb(b, 1, b.ks, c) * fresnel_dielectric(fabsf(c.wi.z), b.eta, b.inv_eta, ct)
                        : v3(0, 0, 0);
                --n;
                break;
            }
            float R12, R21;
            ri.wi = scoat_refract_in(b, c.wi, R12);
            ri.wo = scoat_refract_in(b, c.wo, R21);
            if (R12 == 1.0f || R21 == 1.0f) { stop = true; break; }
            l.m1 = 1.0f - R12;
            l.m2 = 1.0f - R21;
            V3 sa = par_rgb(b, 3, b.sigma_a, c) * b.thickness;
            if (!is_zero(sa)) {
                float q = 1.0f / fabsf(ri.wi.z) + 1.0f / fabsf(ri.wo.z);
                l.e = v3(expf(-sa.x * q), expf(-sa.y * q), expf(-sa.z * q));
                l.has_e = true;
            }
        }
        if (c.measure == kMeasureSolidAngle) { l.s = b.inv_eta * b.inv_eta * c.wo.z / ri.wo.z; l.has_s = true; }
        c = ri;
        id = b.nested;
    }
    if (stop) { v = v3(0, 0, 0); --n; }   // the layer that stopped contributes zero
    for (int k = n - 1; k >= 0; --k) {
        const DeepLayer &l = L[k];
        if (l.kind == 2) continue;
        if (l.kind == 0) {
            V3 nv = v3(v.x * l.m1 * l.m2, v.y * l.m1 * l.m2, v.z * l.m1 * l.m2);
            if (l.has_e) nv = nv * l.e;
            if (l.has_s) nv = nv * l.s;
            v = l.add + nv;
        } else {
            V3 res = (v * l.m1) * l.m2;
            if (l.has_e) res = res * l.e;
            if (l.has_s) res = res * l.s;
            v = res;
        }
    }
    return v;
}
static __device__ __noinline__ float deep_pdf(const DevBsdf *bs, int id, const BRec &r0) {
    DeepLayer L[kNestLevels];
    int n = 0;
    BRec c = r0;
    float p = 0.0f;
    for (;;) {
        const DevBsdf &b = bs[id];
        if (n == kNestLevels || !(b.type == kRoughCoating || b.type == kCoating || b.type == kTwoSided)) {
            p = deep_leaf_pdf(b, c);
            break;
        }
        DeepLayer &l = L[n++];
        l.kind = b.type == kRoughCoating ? 0 : b.type == kCoating ? 1 : 2;
        l.has_s = false;
        if (l.kind == 2) {   // TwoSidedBSDF::Pdf (:61)
            if (c.wi.z > 0.0f) {
                id = b.nested;
            } else {
                c.wi.z *= -1.0f;
                c.wo.z *= -1.0f;
                id = b.nested2;
            }
            continue;
        }
        BRec ri = c;
        if (l.kind == 0) {   // RoughCoatingBSDF::Pdf (coating_pdf)
            V3 h = normalize(c.wi + c.wo) * signum(c.wo.z);
            const float a = coat_alpha(b, c);
            Mfd d = mfd_make(b.distribution, a, a);
            const float ci = c.wi.z, co = c.wo.z;
            float r12 = 1.0f - rft_eval(b, fabsf(ci), d.au);
            float sp = (r12 * b.spec_w) / (r12 * b.spec_w + (1.0f - r12) * (1.0f - b.spec_w));
            l.m1 = 1.0f - sp;
            l.add.x = 0.0f;
            if (ci * co > 0.0f) {
                float J = 1.0f / (4.0f * fabsf(dot(c.wo, h)));
                l.add.x = mfd_pdf(d, h) * J * sp;
            }
            ri.wi = coat_refract(c.wi, b.inv_eta);
            ri.wo = coat_refract(c.wo, b.inv_eta);
            if (ri.measure == kMeasureSolidAngle) { l.s = b.inv_eta * b.inv_eta * co / ri.wo.z; l.has_s = true; }
        } else {             // CoatingBSDF::Pdf (scoating_pdf)
            float R12, R21;
            V3 wip = scoat_refract_in(b, c.wi, R12);
            float sp = scoat_spec_pdf(b, R12);
            if (c.measure == kMeasureDiscrete) {
                p = delta_match(reflect_n(c.wi), c.wo) ? sp : 0.0f;
                --n;
                break;
            }
            ri.wi = wip;
            ri.wo = scoat_refract_in(b, c.wo, R21);
            if (R12 == 1.0f || R21 == 1.0f) { p = 0.0f; --n; break; }
            l.m1 = 1.0f - sp;
            if (c.measure == kMeasureSolidAngle) { l.s = b.inv_eta * b.inv_eta * c.wo.z / ri.wo.z; l.has_s = true; }
        }
        c = ri;
        id = b.nested;
    }
    for (int k = n - 1; k >= 0; --k) {
        const DeepLayer &l = L[k];
        if (l.kind == 2) continue;
        if (l.has_s) p *= l.s;
        p = l.kind == 0 ? l.add.x + p * l.m1 : p * l.m1;
    }
    return p;
}
static __device__ __noinline__ V3 deep_sample(const DevBsdf *bs, int id0, BRec &r, float ux, float uy, float u1) {
    struct Down {
        int id, kind;   // kind: 0 roughCoating, 1 coating, 2 twoSided
        bool spec;      // roughCoating: the layer's own lobe was sampled (the walk ended here)
        V3 wi, wip;     // wi on entering the layer; coating: wi refracted into it
        float r12, sp;  // coating: the entering Fresnel reflectance and the specular probability
    } L[kNestLevels];
    int n = 0, id = id0;
    V3 res = v3(0, 0, 0);
    for (;;) {   // down: each layer picks its lobe and passes the refracted wi on
        const DevBsdf &b = bs[id];
        if (n == kNestLevels || !(b.type == kRoughCoating || b.type == kCoating || b.type == kTwoSided)) {
            res = deep_leaf_sample(b, r, ux, uy, u1);
            break;
        }
        Down &l = L[n++];
        l.id = id;
        l.kind = b.type == kRoughCoating ? 0 : b.type == kCoating ? 1 : 2;
        l.spec = false;
        l.wi = r.wi;
        if (l.kind == 2) {   // TwoSidedBSDF::Sample (:21)
            const bool flip = r.wi.z < 0.0f;
            if (flip) r.wi.z *= -1.0f;
            l.spec = flip;   // twoSided: whether the back side was taken
            id = flip ? b.nested2 : b.nested;
            continue;
        }
        if (l.kind == 0) {   // RoughCoatingBSDF::Sample (coating_sample)
            const float a = coat_alpha(b, r);
            Mfd d = mfd_make(b.distribution, a, a);
            float aci = fabsf(r.wi.z);
            float r12 = 1.0f - rft_eval(b, aci, d.au);
            float sp = (r12 * b.spec_w) / (r12 * b.spec_w + (1.0f - r12) * (1.0f - b.spec_w));
            if (ux < sp) {
                ux /= sp;
                l.spec = true;
                float pdf;
                V3 m = mfd_sample(d, ux, uy, pdf);
                r.wo = reflect_m(r.wi, m);
                r.measure = kMeasureDiscrete;
                r.eta = 1.0f;
                res = r.wo.z * r.wo.z <= 0.0f ? v3(0, 0, 0) : v3(1, 1, 1);
                break;
            }
            ux = (ux - sp) / (1.0f - sp);
            r.wi = coat_refract(r.wi, b.inv_eta);
        } else {             // CoatingBSDF::Sample (scoating_sample)
            float R12;
            l.wip = scoat_refract_in(b, r.wi, R12);
            l.r12 = R12;
            l.sp = scoat_spec_pdf(b, R12);
            if (ux < l.sp) {
                r.wo = reflect_n(r.wi);
                r.eta = 1.0f;
                r.measure = kMeasureDiscrete;
                res = par_rgb(b, 1, b.ks, r) * (R12 / l.sp);
                --n;
                break;
            }
            ux = (ux - l.sp) / (1.0f - l.sp);
            if (R12 == 1.0f) { res = v3(0, 0, 0); --n; break; }
            r.wi = l.wip;
        }
        id = b.nested;
    }
    for (int k = n - 1; k >= 0; --k) {   // up: each layer refracts wo out and weighs the sample
        const Down &l = L[k];
        const DevBsdf &b = bs[l.id];
        if (l.kind == 2) {
            if (l.spec) {
                r.wi.z *= -1.0f;
                if (!is_zero(res)) r.wo.z *= -1.0f;
            }
            continue;
        }
        if (l.kind == 0) {
            if (!l.spec) {
                r.wi = l.wi;
                if (is_zero(res)) continue;
                r.wo = coat_refract(r.wo, b.eta);
                if (is_zero(r.wo)) { res = v3(0, 0, 0); continue; }
            } else if (is_zero(res)) {
                continue;
            }
            float P = deep_pdf(bs, l.id, r);
            res = P == 0.0f ? v3(0, 0, 0) : deep_eval(bs, l.id, r) / P;
            continue;
        }
        r.wi = l.wi;
        if (is_zero(res)) continue;
        V3 wop = r.wo;
        res = scoat_absorb(b, r, res, l.wip, wop);
        float R21;
        r.wo = scoat_refract_out(b, wop, R21);
        if (R21 == 1.0f) { res = v3(0, 0, 0); continue; }
        res = res / (1.0f - l.sp);
        res = res * ((1.0f - l.r12) * (1.0f - R21));
    }
    return res;
}

__device__ __forceinline__ V3 bsdf_eval(const DevBsdf *bs, int id, const BRec &r) {
    const DevBsdf &b = bs[id];
    if (b.deep) return deep_eval(bs, id, r);
    if (b.type == kTwoSided) return twosided_eval(bs, b, r);
    return layer_eval(bs, b, r);
}
__device__ __forceinline__ float bsdf_pdf(const DevBsdf *bs, int id, const BRec &r) {
    const DevBsdf &b = bs[id];
    if (b.deep) return deep_pdf(bs, id, r);
    if (b.type == kTwoSided) return twosided_pdf(bs, b, r);
    return layer_pdf(bs, b, r);
}
// u1 is consumed only by a roughDielectric (top-level or under a coating); the
// caller draws it lazily through needs_u1().  A twoSided BSDF nests no
// transmission, so it never draws one.
__device__ __forceinline__ bool needs_u1(const DevBsdf *bs, int id) {
    if (bs[id].type == kBumpMap || bs[id].type == kNormalMap) id = bs[id].nested;
    const DevBsdf &b = bs[id];
    if (b.type == kRoughDielectric) return true;
    if (b.deep) {   // a stack of coatings over a rough dielectric
        if (b.type == kTwoSided) return false;
        int k = b.nested;
        for (int l = 1; l < kNestLevels && (bs[k].type == kRoughCoating || bs[k].type == kCoating); ++l) k = bs[k].nested;
        return bs[k].type == kRoughDielectric;
    }
    return (b.type == kRoughCoating || b.type == kCoating) && bs[b.nested].type == kRoughDielectric;
}
__device__ __forceinline__ V3 bsdf_sample(const DevBsdf *bs, int id, BRec &r, float ux, float uy, float u1) {
    const DevBsdf &b = bs[id];
    if (b.deep) return deep_sample(bs, id, r, ux, uy, u1);
    if (b.type == kTwoSided) return twosided_sample(bs, b, r, ux, uy, u1);
    return layer_sample(bs, b, r, ux, uy, u1);
}

// ---- bumpMap / normalMap (src/bsdf/BumpMapBSDF.cpp, src/bsdf/NormalMapBSDF.cpp).
// The perturbed frame depends on the intersection only, so the shading code
// computes it once per vertex (perturbed_frames, hk_shading.cuh) and these
// wrappers move each record between the shading frame and the perturbed one
// through world space, as the reference does; other BSDFs pass through.
struct BumpFrames {
    Frame sh, pf;   // the intersection's shading frame and its perturbed frame
};
__device__ __forceinline__ bool is_bump(const DevBsdf &b) { return b.type == kBumpMap || b.type == kNormalMap; }
// BumpMapBSDF::Eval / Pdf (:56, :80): zero where a direction changes side
__device__ __forceinline__ bool bump_record(const BumpFrames &f, const BRec &r, BRec &q) {
    q = r;
    q.wi = to_local(f.pf, to_world(f.sh, r.wi));
    q.wo = to_local(f.pf, to_world(f.sh, r.wo));
    return !(r.wo.z * q.wo.z <= 0.0f || r.wi.z * q.wi.z <= 0.0f);
}
static __device__ __noinline__ V3 bump_eval(const DevBsdf *bs, int id, const BRec &r, const BumpFrames &f) {
    BRec q;
    if (!bump_record(f, r, q)) return v3(0, 0, 0);
    return bsdf_eval(bs, bs[id].nested, q);
}
static __device__ __noinline__ float bump_pdf(const DevBsdf *bs, int id, const BRec &r, const BumpFrames &f) {
    BRec q;
    if (!bump_record(f, r, q)) return 0.0f;
    return bsdf_pdf(bs, bs[id].nested, q);
}
// BumpMapBSDF::Sample (:22)
static __device__ __noinline__ V3 bump_sample(const DevBsdf *bs, int id, BRec &r, float ux, float uy, float u1,
                                       const BumpFrames &f) {
    BRec q = r;
    q.wi = to_local(f.pf, to_world(f.sh, r.wi));
    q.wo = v3(0, 0, 0);
    q.measure = kMeasureUnknown;
    if (r.wi.z * q.wi.z <= 0.0f) return v3(0, 0, 0);
    const V3 res = bsdf_sample(bs, bs[id].nested, q, ux, uy, u1);
    if (!is_zero(res)) {
        r.wo = to_local(f.sh, to_world(f.pf, q.wo));
        r.eta = q.eta;
        r.measure = q.measure;
        if (r.wo.z * q.wo.z <= 0.0f) return v3(0, 0, 0);
    }
    return res;
}
// run-time dispatch including the wrappers (f is read only for them)
__device__ __forceinline__ V3 bsdf_eval_b(const DevBsdf *bs, int id, const BRec &r, const BumpFrames &f) {
    return is_bump(bs[id]) ? bump_eval(bs, id, r, f) : bsdf_eval(bs, id, r);
}
__device__ __forceinline__ float bsdf_pdf_b(const DevBsdf *bs, int id, const BRec &r, const BumpFrames &f) {
    return is_bump(bs[id]) ? bump_pdf(bs, id, r, f) : bsdf_pdf(bs, id, r);
}
__device__ __forceinline__ V3 bsdf_sample_b(const DevBsdf *bs, int id, BRec &r, float ux, float uy, float u1,
                                            const BumpFrames &f) {
    return is_bump(bs[id]) ? bump_sample(bs, id, r, ux, uy, u1, f) : bsdf_sample(bs, id, r, ux, uy, u1);
}

}  // namespace hk

namespace hk {
// Dispatch with the top-level BSDF type known at compile time (the wavefront
// shades one material type per kernel, so each kernel carries one BSDF);
// BT < 0 dispatches at run time.
template <int BT>
__device__ __forceinline__ V3 bsdf_eval_t(const DevBsdf *bs, int id, const BRec &r) {
    const DevBsdf &b = bs[id];
    if constexpr (BT < 0) return bsdf_eval(bs, id, r);
    else if constexpr (BT == kDiffuse) return diffuse_eval(b, r);
    else if constexpr (BT == kRoughConductor) return conductor_eval(b, r);
    else if constexpr (BT == kRoughDielectric) return dielectric_eval(b, r);
    else if constexpr (BT == kRoughPlastic) return plastic_eval(b, r);
    else if constexpr (BT == kRoughCoating) return coating_eval(b, bs[b.nested], r);
    else if constexpr (BT == kMirror) return mirror_eval(r);
    else if constexpr (BT == kConductor) return sconductor_eval(b, r);
    else if constexpr (BT == kDielectric) return sdielectric_eval(b, r);
    else if constexpr (BT == kPlastic) return splastic_eval(b, r);
    else if constexpr (BT == kCoating) return scoating_eval(b, bs[b.nested], r);
    else if constexpr (BT == kRoughDiffuse) return roughdiffuse_eval(b, r);
    else return twosided_eval(bs, b, r);
}
template <int BT>
__device__ __forceinline__ float bsdf_pdf_t(const DevBsdf *bs, int id, const BRec &r) {
    const DevBsdf &b = bs[id];
    if constexpr (BT < 0) return bsdf_pdf(bs, id, r);
    else if constexpr (BT == kDiffuse) return diffuse_pdf(r);
    else if constexpr (BT == kRoughConductor) return conductor_pdf(b, r);
    else if constexpr (BT == kRoughDielectric) return dielectric_pdf(b, r);
    else if constexpr (BT == kRoughPlastic) return plastic_pdf(b, r);
    else if constexpr (BT == kRoughCoating) return coating_pdf(b, bs[b.nested], r);
    else if constexpr (BT == kMirror || BT == kConductor) return mirror_pdf(r);
    else if constexpr (BT == kDielectric) return sdielectric_pdf(b, r);
    else if constexpr (BT == kPlastic) return splastic_pdf(b, r);
    else if constexpr (BT == kCoating) return scoating_pdf(b, bs[b.nested], r);
    else if constexpr (BT == kRoughDiffuse) return roughdiffuse_pdf(r);
    else return twosided_pdf(bs, b, r);
}
template <int BT>
__device__ __forceinline__ V3 bsdf_sample_t(const DevBsdf *bs, int id, BRec &r, float ux, float uy, float u1) {
    const DevBsdf &b = bs[id];
    if constexpr (BT < 0) return bsdf_sample(bs, id, r, ux, uy, u1);
    else if constexpr (BT == kDiffuse) return diffuse_sample(b, r, ux, uy);
    else if constexpr (BT == kRoughConductor) return conductor_sample(b, r, ux, uy);
    else if constexpr (BT == kRoughDielectric) return dielectric_sample(b, r, ux, uy, u1);
    else if constexpr (BT == kRoughPlastic) return plastic_sample(b, r, ux, uy);
    else if constexpr (BT == kRoughCoating) return coating_sample(b, bs[b.nested], r, ux, uy, u1);
    else if constexpr (BT == kMirror) return mirror_sample(r);
    else if constexpr (BT == kConductor) return sconductor_sample(b, r);
    else if constexpr (BT == kDielectric) return sdielectric_sample(b, r, ux);
    else if constexpr (BT == kPlastic) return splastic_sample(b, r, ux, uy);
    else if constexpr (BT == kCoating) return scoating_sample(b, bs[b.nested], r, ux, uy, u1);
    else if constexpr (BT == kRoughDiffuse) return roughdiffuse_sample(b, r, ux, uy);
    else return twosided_sample(bs, b, r, ux, uy, u1);
}

// bumpMap / normalMap id wrapping a BSDF of type BT known at compile time:
// the wrappers above with the nested call dispatched statically
template <int BT>
__device__ __forceinline__ V3 bump_eval_t(const DevBsdf *bs, int id, const BRec &r, const BumpFrames &f) {
    BRec q;
    if (!bump_record(f, r, q)) return v3(0, 0, 0);
    return bsdf_eval_t<BT>(bs, bs[id].nested, q);
}
template <int BT>
__device__ __forceinline__ float bump_pdf_t(const DevBsdf *bs, int id, const BRec &r, const BumpFrames &f) {
    BRec q;
    if (!bump_record(f, r, q)) return 0.0f;
    return bsdf_pdf_t<BT>(bs, bs[id].nested, q);
}
template <int BT>
__device__ __forceinline__ V3 bump_sample_t(const DevBsdf *bs, int id, BRec &r, float ux, float uy, float u1,
                                            const BumpFrames &f) {
    BRec q = r;
    q.wi = to_local(f.pf, to_world(f.sh, r.wi));
    q.wo = v3(0, 0, 0);
    q.measure = kMeasureUnknown;
    if (r.wi.z * q.wi.z <= 0.0f) return v3(0, 0, 0);
    const V3 res = bsdf_sample_t<BT>(bs, bs[id].nested, q, ux, uy, u1);
    if (!is_zero(res)) {
        r.wo = to_local(f.sh, to_world(f.pf, q.wo));
        r.eta = q.eta;
        r.measure = q.measure;
        if (r.wo.z * q.wo.z <= 0.0f) return v3(0, 0, 0);
    }
    return res;
}
}  // namespace hk
