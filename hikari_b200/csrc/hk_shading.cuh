// Emitters, camera, intersection post-processing and film splatting of the
// pathMIS core (device side).
#pragma once
#include "hk_bsdf.cuh"
#include "hk_device.h"
#include "hk_math.cuh"
#include "hk_traverse.cuh"

namespace hk {

// ------------------------------------------------------------ intersection
struct Isect {
    V3 p;
    Frame sh;
    int mesh;
    float u, v;   // texture coordinates (0 without them)
};

// normalized() of an expression over MatrixXf columns (dynamic size): Eigen
// reduces the squared norm left to right, ((x*x + y*y) + z*z), where a
// fixed-size vector reduces x*x + (y*y + z*z)
__device__ __forceinline__ V3 normalize_dyn(V3 a) {
    float z = (a.x * a.x + a.y * a.y) + a.z * a.z;
    return z > 0.0f ? a / sqrtf(z) : a;
}
// Frame(N, dPdU) (src/core/Frame.cpp:7): tangent by Gram-Schmidt against N
__device__ __forceinline__ Frame frame_from_n_dpdu(V3 n, V3 dpdu) {
    Frame f;
    f.n = n;
    f.s = normalize(dpdu - n * dot(n, dpdu));
    f.t = cross(n, f.s);
    return f;
}

// Triangle::PostIntersect (src/core/Mesh.cpp:67-172): position and texture
// coordinates from barycentrics; the shading frame from the face normal, from
// interpolated vertex normals, or -- with normals and texture coordinates --
// from the interpolated normal and dP/du.
__device__ __forceinline__ void post_intersect(const DevScene &S, const Hit &h, Isect &it) {
    const float4 *tp = S.tris + 3 * h.tri;
    float4 q0 = __ldg(tp), q1 = __ldg(tp + 1), q2 = __ldg(tp + 2);
    V3 p0 = xyz(q0), p1 = xyz(q1), p2 = xyz(q2);
    float b0 = 1 - (h.u + h.v), b1 = h.u, b2 = h.v;
    it.p = (p0 * b0 + p1 * b1) + p2 * b2;
    it.mesh = __float_as_int(q1.w);
    it.u = it.v = 0.0f;
    const DevMesh &m = S.meshes[it.mesh];
    const uint32_t orig = (uint32_t)__float_as_int(q0.w);
    float2 t0, t1, t2;
    if (m.has_uv) {
        t0 = __ldg(S.tri_uv + 3 * orig);
        t1 = __ldg(S.tri_uv + 3 * orig + 1);
        t2 = __ldg(S.tri_uv + 3 * orig + 2);
        it.u = (b0 * t0.x + b1 * t1.x) + b2 * t2.x;
        it.v = (b0 * t0.y + b1 * t1.y) + b2 * t2.y;
    }
    if (m.has_normals) {
        const float4 *np = S.tri_normals + 3 * orig;
        V3 n0 = xyz(__ldg(np)), n1 = xyz(__ldg(np + 1)), n2 = xyz(__ldg(np + 2));
        if (m.has_uv) {
            V3 dp1 = p1 - p0, dp2 = p2 - p0;
            float du1 = t1.x - t0.x, dv1 = t1.y - t0.y, du2 = t2.x - t0.x, dv2 = t2.y - t0.y;
            if (norm(cross(dp1, dp2)) == 0.0f) {
                it.sh = frame_from_n(normalize(cross(dp1, dp2)));   // the geometric frame
                return;
            }
            float det = du1 * dv2 - dv1 * du2;
            if (det != 0.0f) {
                float inv = 1.0f / det;
                V3 dpdu = (dp1 * dv2 - dp2 * dv1) * inv;
                V3 ns = (n0 * b0 + n1 * b1) + n2 * b2;
                ns = ns * (1.0f / norm(ns));
                it.sh = frame_from_n_dpdu(ns, dpdu);
                return;
            }
        }
        it.sh = frame_from_n(normalize_dyn((n0 * b0 + n1 * b1) + n2 * b2));
    } else {
        it.sh = frame_from_n(normalize(cross(p1 - p0, p2 - p0)));
    }
}

// dP/du, dP/dv and the geometric normal of a hit as Triangle::PostIntersect
// leaves them (src/core/Mesh.cpp:106-156): false without UV partials (a mesh
// without normals or texture coordinates, a zero-area triangle).
__device__ __forceinline__ bool uv_tangents(const DevScene &S, const Hit &h, const Isect &it, V3 &dpdu, V3 &dpdv,
                                            V3 &ng) {
    const DevMesh &m = S.meshes[it.mesh];
    if (!m.has_uv || !m.has_normals) return false;
    const float4 *tp = S.tris + 3 * h.tri;
    const float4 q0 = __ldg(tp), q1 = __ldg(tp + 1), q2 = __ldg(tp + 2);
    const V3 p0 = xyz(q0), dp1 = xyz(q1) - p0, dp2 = xyz(q2) - p0;
    const V3 c = cross(dp1, dp2);
    if (norm(c) == 0.0f) return false;
    const uint32_t orig = (uint32_t)__float_as_int(q0.w);
    const float2 t0 = __ldg(S.tri_uv + 3 * orig), t1 = __ldg(S.tri_uv + 3 * orig + 1), t2 = __ldg(S.tri_uv + 3 * orig + 2);
    const float du1 = t1.x - t0.x, dv1 = t1.y - t0.y, du2 = t2.x - t0.x, dv2 = t2.y - t0.y;
    const float det = du1 * dv2 - dv1 * du2;
    if (det == 0.0f) {
        dpdu = it.sh.s;
        dpdv = it.sh.t;
    } else {
        const float inv = 1.0f / det;
        dpdu = (dp1 * dv2 - dp2 * dv1) * inv;
        dpdv = (dp1 * (-du2) + dp2 * du1) * inv;
    }
    ng = normalize(c);
    return true;
}

// What the wireframe and curvature textures read at a hit (BRec::geo): the
// distance from P to the nearest of the hit triangle's edge lines
// (WireframeTexture::Eval, src/texture/WireframeTexture.cpp:60-72), and the
// mean and Gaussian curvature from the first and second fundamental forms
// (Shape::ComputeCurvature, src/core/Shape.cpp:30-51) with dN/du, dN/dv as
// Triangle::PostIntersect forms them (src/core/Mesh.cpp:137-156); 0 without
// UV partials.
__device__ __forceinline__ float3 tex_geometry(const DevScene &S, const Hit &h, const Isect &it) {
    const float4 *tp = S.tris + 3 * h.tri;
    const float4 q0 = __ldg(tp), q1 = __ldg(tp + 1), q2 = __ldg(tp + 2);
    const V3 ps[3] = {xyz(q0), xyz(q1), xyz(q2)};
    float min_d2 = 3.402823466e38f;   // std::numeric_limits<float>::max()
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        const V3 cur = ps[i], nxt = ps[(i + 1) % 3];
        const V3 d1 = normalize(nxt - cur), d2 = it.p - cur;
        const V3 e = (cur + d1 * dot(d1, d2)) - it.p;
        const float d2e = dot(e, e);
        min_d2 = d2e < min_d2 ? d2e : min_d2;   // std::min
    }
    float3 g = make_float3(sqrtf(min_d2), 0.0f, 0.0f);
    const DevMesh &m = S.meshes[it.mesh];
    if (!m.has_uv || !m.has_normals) return g;
    const V3 p0 = ps[0], dp1 = ps[1] - p0, dp2 = ps[2] - p0;
    if (norm(cross(dp1, dp2)) == 0.0f) return g;   // no UV partials
    const uint32_t orig = (uint32_t)__float_as_int(q0.w);
    const float2 t0 = __ldg(S.tri_uv + 3 * orig), t1 = __ldg(S.tri_uv + 3 * orig + 1), t2 = __ldg(S.tri_uv + 3 * orig + 2);
    const float du1 = t1.x - t0.x, dv1 = t1.y - t0.y, du2 = t2.x - t0.x, dv2 = t2.y - t0.y;
    const float det = du1 * dv2 - dv1 * du2;
    V3 dpdu, dpdv, dndu = v3(0, 0, 0), dndv = v3(0, 0, 0);
    if (det == 0.0f) {
        dpdu = it.sh.s;
        dpdv = it.sh.t;
    } else {
        const float inv = 1.0f / det;
        dpdu = (dp1 * dv2 - dp2 * dv1) * inv;
        dpdv = (dp1 * (-du2) + dp2 * du1) * inv;
        const float4 *np = S.tri_normals + 3 * orig;
        const V3 n0 = xyz(__ldg(np)), n1 = xyz(__ldg(np + 1)), n2 = xyz(__ldg(np + 2));
        const float b0 = 1 - (h.u + h.v), b1 = h.u, b2 = h.v;
        V3 ns = (n0 * b0 + n1 * b1) + n2 * b2;
        const float inv_ln = 1.0f / norm(ns);
        ns = ns * inv_ln;
        V3 dnu = (n1 - n0) * inv_ln;
        dnu = dnu - ns * dot(ns, dnu);
        V3 dnv = (n2 - n0) * inv_ln;
        dnv = dnv - ns * dot(ns, dnv);
        dndu = (dnu * dv2 - dnv * dv1) * inv;
        dndv = (dnu * (-du2) + dnv * du1) * inv;
    }
    const float E = dot(dpdu, dpdu), F = dot(dpdu, dpdv), G = dot(dpdv, dpdv);
    const float L = -dot(dpdu, dndu), M = -dot(dpdv, dndu), N = -dot(dpdv, dndv);
    const float inv_denom = 1.0f / (E * G - F * F);
    g.z = (L * N - M * M) * inv_denom;
    g.y = 0.5f * ((L * G - 2.0f * M * F) + N * E) * inv_denom;
    return g;
}

// Intersection::ComputeScreenSpacePartial (src/core/Intersection.cpp:30) of
// the first hit of a camera ray from o with differential directions rx, ry:
// (dUdX, dVdX, dUdY, dVdY), zero where the hit has no UV partials.
__device__ __forceinline__ float4 screen_partials(const DevScene &S, const Hit &h, const Isect &it, V3 o, V3 rx, V3 ry) {
    const float4 zero = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    V3 dpdu, dpdv, n;
    if (!uv_tangents(S, h, it, dpdu, dpdv, n)) return zero;
    if (is_zero(dpdu) && is_zero(dpdv)) return zero;
    const float pp = dot(n, it.p), po = dot(n, o);
    const float prx = dot(n, rx), pry = dot(n, ry);
    if (prx == 0.0f || pry == 0.0f) return zero;
    const float tx = (pp - po) / prx, ty = (pp - po) / pry;
    const float ax = fabsf(n.x), ay = fabsf(n.y), az = fabsf(n.z);
    int a0, a1;
    if (ax > ay && ax > az) { a0 = 1; a1 = 2; }
    else if (ay > az) { a0 = 0; a1 = 2; }
    else { a0 = 0; a1 = 1; }
    auto c_of = [](V3 a, int k) { return k == 0 ? a.x : (k == 1 ? a.y : a.z); };
    const float A00 = c_of(dpdu, a0), A01 = c_of(dpdv, a0), A10 = c_of(dpdu, a1), A11 = c_of(dpdv, a1);
    const V3 px = o + rx * tx, py = o + ry * ty;
    float4 r;
    // SolveLinearSystem2x2 (include/core/Common.hpp:881), its failure defaults
    const float d = A00 * A11 - A01 * A10;
    const bool ok = fabsf(d) > 1.0f / 3.40282347e+38f;
    const float id = ok ? 1.0f / d : 0.0f;
    const float bx0 = c_of(px, a0) - c_of(it.p, a0), bx1 = c_of(px, a1) - c_of(it.p, a1);
    const float by0 = c_of(py, a0) - c_of(it.p, a0), by1 = c_of(py, a1) - c_of(it.p, a1);
    r.x = ok ? (A11 * bx0 - A01 * bx1) * id : 1.0f;
    r.y = ok ? (A00 * bx1 - A10 * bx0) * id : 0.0f;
    r.z = ok ? (A11 * by0 - A01 * by1) * id : 0.0f;
    r.w = ok ? (A00 * by1 - A10 * by0) * id : 1.0f;
    return r;
}

// BumpMapBSDF::GetPerturbebFrame (src/bsdf/BumpMapBSDF.cpp:172) and
// NormalMapBSDF::GetPerturbebFrame (src/bsdf/NormalMapBSDF.cpp:169) for the
// hit's BSDF b (a bumpMap or normalMap); the host admits these BSDFs only on
// meshes with normals and texture coordinates.
__device__ __forceinline__ BumpFrames perturbed_frames(const DevScene &S, const Hit &h, const Isect &it,
                                                       const DevBsdf &b) {
    BumpFrames f;
    f.sh = it.sh;
    V3 dpdu = v3(0, 0, 0), dpdv = v3(0, 0, 0), ng = it.sh.n;
    uv_tangents(S, h, it, dpdu, dpdv, ng);
    Frame &p = f.pf;
    if (b.type == kBumpMap) {
        V3 gu, gv;
        tex_gradient(b.textures, b.tex[0] - 1, it.u, it.v, gu, gv);
        const float ddu = luminance(gu), ddv = luminance(gv);
        const V3 n = it.sh.n;
        const V3 pu = dpdu + n * (ddu - dot(n, dpdu)), pv = dpdv + n * (ddv - dot(n, dpdv));
        p.n = normalize(cross(pu, pv));
        p.s = normalize(pu - p.n * dot(p.n, pu));
        p.t = cross(p.n, p.s);
        if (dot(p.n, ng) < 0.0f) p.n = p.n * -1.0f;
    } else {
        const V3 c = tex_eval(b.textures, b.tex[0] - 1, it.u, it.v, make_float4(0.0f, 0.0f, 0.0f, 0.0f), false);
        p.n = normalize(to_world(it.sh, v3(2.0f * c.x - 1.0f, 2.0f * c.y - 1.0f, 2.0f * c.z - 1.0f)));
        p.s = normalize(dpdu - p.n * dot(p.n, dpdu));
        p.t = cross(p.n, p.s);
    }
    return f;
}

// ------------------------------------------------------------ emitters
struct ERec {
    V3 ref, p, n, wi;
    float pdf, dist;
};

// std::lower_bound over cdf[0..n] then clamp to [0, n-1] (src/core/DiscretePDF.cpp:41-46)
__device__ __forceinline__ int cdf_find(const float *cdf, int n, float u) {
    int lo = 0, hi = n + 1;
    while (lo < hi) {
        int mid = (lo + hi) >> 1;
        if (__ldg(cdf + mid) < u) lo = mid + 1; else hi = mid;
    }
    return clampi(lo - 1, 0, n - 1);
}

// cdf_find through a guide table (cutpoint method): g[k] is the first index
// with cdf >= k / kEnvGuide, so the lower bound of u lies in [g[k], g[k+1]]
// for k = floor(u * kEnvGuide) and the search there returns cdf_find's index.
__device__ __forceinline__ int cdf_find_guided(const float *cdf, int n, float u, const int32_t *g) {
    const int k = min((int)(u * (float)kEnvGuide), kEnvGuide - 1);
    int lo = __ldg(g + k), hi = __ldg(g + k + 1);
    while (lo < hi) {
        int mid = (lo + hi) >> 1;
        if (__ldg(cdf + mid) < u) lo = mid + 1; else hi = mid;
    }
    return clampi(lo - 1, 0, n - 1);
}

// AreaLight::Pdf / Eval (src/emitter/AreaLight.cpp:38,59)
__device__ __forceinline__ float area_pdf(const DevAreaLight &L, const ERec &r) {
    float gd = fabsf(dot(r.wi * -1.0f, r.n));
    if (gd == 0.0f) return 0.0f;
    float gn = r.dist * r.dist;
    return L.inv_area * (gn / gd);
}
__device__ __forceinline__ V3 area_eval(const DevAreaLight &L, const ERec &r) {
    return dot(r.n, r.wi) < 0.0f ? ld3(L.radiance) : v3(0, 0, 0);
}
// AreaLight::Sample (src/emitter/AreaLight.cpp:14) with Mesh::SamplePosition (src/core/Mesh.cpp:273)
__device__ __forceinline__ V3 area_sample(const DevScene &S, const DevAreaLight &L, ERec &r, float ux, float uy, float u1) {
    int ti = cdf_find(S.light_cdf + L.cdf0, (int)L.ntri, u1);
    float sq = sqrtf(1.0f - ux);
    float al = 1.0f - sq, be = uy * sq, ga = 1.0f - al - be;
    const float4 *tp = S.light_tris + 3 * (L.tri0 + ti);
    V3 p0 = xyz(__ldg(tp)), p1 = xyz(__ldg(tp + 1)), p2 = xyz(__ldg(tp + 2));
    r.p = (p0 * ga + p1 * al) + p2 * be;
    const float4 *np = S.light_normals + 3 * (L.tri0 + ti);
    float4 n0 = __ldg(np);
    if (n0.w != 0.0f) {
        V3 n1 = xyz(__ldg(np + 1)), n2 = xyz(__ldg(np + 2));
        r.n = (xyz(n0) * ga + n1 * al) + n2 * be;
    } else {
        r.n = normalize(cross(p1 - p0, p2 - p0));
    }
    V3 wi = r.p - r.ref;
    r.dist = norm(wi);
    r.wi = normalize(wi);
    r.pdf = area_pdf(L, r);
    if (r.pdf == 0.0f || isinf(r.pdf)) return v3(0, 0, 0);
    return area_eval(L, r) / r.pdf;
}

__device__ __forceinline__ V3 mat3(const float *m, V3 v) {
    return v3(m[0] * v.x + m[1] * v.y + m[2] * v.z, m[3] * v.x + m[4] * v.y + m[5] * v.z,
              m[6] * v.x + m[7] * v.y + m[8] * v.z);
}
// SphericalCoordinates (src/core/Common.cpp:481)
__device__ __forceinline__ void spherical_coords(V3 d, float &th, float &ph) {
    th = acosf(d.z);
    ph = atan2f(d.y, d.x);
    if (ph < 0) ph += 2.0f * kPi;
}
__device__ __forceinline__ V3 env_texel(const DevScene &S, int y, int x) {
    return xyz(__ldg(S.env_rgb + (uint64_t)y * S.env_w + x));
}
// DiscretePDF1D::SampleContinuous (src/core/DiscretePDF.cpp:39), the index
// found through the CDF's guide table
__device__ __forceinline__ float sample_cont(const float *cdf, const float *func, float integral, int n, float u,
                                             float &pdf, int &idx, const int32_t *guide) {
    idx = cdf_find_guided(cdf, n, u, guide);
    float c0 = __ldg(cdf + idx), c1 = __ldg(cdf + idx + 1);
    float du = u - c0;
    if (c1 - c0 > 0.0f) du /= (c1 - c0);
    pdf = __ldg(func + idx) / integral;
    return ((float)idx + du) / (float)n;
}
// ConstantLight::Sample (src/emitter/ConstantLight.cpp:15)
__device__ __forceinline__ V3 const_sample(const DevScene &S, ERec &r, float ux, float uy) {
    float th = uy * kPi;
    float st = sinf(th);
    if (st != 0.0f) r.pdf = 1.0f / (2.0f * (float)(3.14159265358979323846 * 3.14159265358979323846) * st);
    else return v3(0, 0, 0);
    float ph = ux * (float)(2.0 * 3.14159265358979323846);
    float ct = cosf(th), sp = sinf(ph), cp = cosf(ph);
    r.wi = v3(st * cp, st * sp, ct);   // SphericalDirection (src/core/Common.cpp:467)
    r.n = r.wi * -1.0f;
    r.p = r.ref + (r.wi * r.dist) * 2.0f;
    return ld3(S.env_const) / r.pdf;
}
// PointLight::Sample (src/emitter/PointLight.cpp:15), DirectionalLight::Sample
// (src/emitter/DirectionalLight.cpp:18); both report pdf 1
__device__ __forceinline__ V3 delta_sample(const DevScene &S, int k, ERec &r) {
    const float4 a = __ldg(S.delta_lights + 2 * k), c = __ldg(S.delta_lights + 2 * k + 1);
    r.pdf = 1.0f;
    if (a.w == 0.0f) {
        r.p = v3(a.x, a.y, a.z);
        V3 wi = r.p - r.ref;
        r.dist = norm(wi);
        r.wi = normalize(wi);
        r.n = r.wi * -1.0f;
        return v3(c.x, c.y, c.z) * (1.0f / ((4.0f * kPi) * (r.dist * r.dist)));
    }
    r.wi = normalize(v3(a.x, a.y, a.z)) * -1.0f;
    r.p = r.ref + r.wi * (2.0f * r.dist);
    r.n = r.wi * -1.0f;
    return v3(c.x, c.y, c.z);
}
// EnvironmentLight::Sample (src/emitter/EnvironmentLight.cpp:41)
__device__ __forceinline__ V3 env_sample(const DevScene &S, ERec &r, float ux, float uy) {
    if (S.env_kind == kEnvConstant) return const_sample(S, r, ux, uy);
    float py, px;
    int iy, ix;
    float dy = sample_cont(S.env_marg_cdf, S.env_marg_func, S.env_marg_int, (int)S.env_h, uy, py, iy, S.env_marg_guide);
    float dx = sample_cont(S.env_cond_cdf + (uint64_t)iy * (S.env_w + 1), S.env_cond_func + (uint64_t)iy * S.env_w,
                           __ldg(S.env_cond_int + iy), (int)S.env_w, ux, px, ix,
                           S.env_cond_guide + (uint64_t)iy * (kEnvGuide + 1));
    float mp = px * py;
    float th = dy * kPi, st = sinf(th);
    if (mp == 0.0f) return v3(0, 0, 0);
    if (st != 0.0f) r.pdf = mp / (2.0f * (float)(3.14159265358979323846 * 3.14159265358979323846) * st);
    else return v3(0, 0, 0);
    float ph = dx * (float)(2.0 * 3.14159265358979323846);
    float sp = sinf(ph), cp = cosf(ph), ct = cosf(th);
    V3 dir = v3(st * cp, st * sp, ct);   // SphericalDirection (src/core/Common.cpp:467)
    r.wi = mat3(S.env_to_world, dir);
    r.n = r.wi * -1.0f;
    r.p = r.ref + (r.wi * r.dist) * 2.0f;
    V3 rad = env_texel(S, iy, ix);
    if (!is_valid(rad)) return v3(0, 0, 0);
    return (rad * S.env_scale) / r.pdf;
}
// EnvironmentLight::Pdf (:78) with DiscretePDF2D::Pdf (src/core/DiscretePDF.cpp:127)
__device__ __forceinline__ float env_pdf(const DevScene &S, V3 wi) {
    float th, ph;
    if (S.env_kind == kEnvConstant) {   // ConstantLight::Pdf (src/emitter/ConstantLight.cpp:36)
        spherical_coords(wi, th, ph);
        float st = sinf(th);
        if (st == 0.0f) return 0.0f;
        return 1.0f / (2.0f * (float)(3.14159265358979323846 * 3.14159265358979323846) * st);
    }
    spherical_coords(mat3(S.env_to_local, wi), th, ph);
    float st = sinf(th);
    if (st == 0.0f) return 0.0f;
    float u = ph / (float)(2.0 * 3.14159265358979323846), v = th / (float)3.14159265358979323846;
    int X = clampi((int)(u * S.env_w), 0, (int)S.env_w - 1), Y = clampi((int)(v * S.env_h), 0, (int)S.env_h - 1);
    float p = __ldg(S.env_cond_func + (uint64_t)Y * S.env_w + X) / S.env_marg_int;
    return p / (2.0f * (float)(3.14159265358979323846 * 3.14159265358979323846) * st);
}
// EnvironmentLight::Eval (:92): nearest texel
__device__ __forceinline__ V3 env_eval(const DevScene &S, V3 wi) {
    if (S.env_kind == kEnvConstant) return ld3(S.env_const);   // ConstantLight::Eval (:47)
    float th, ph;
    spherical_coords(mat3(S.env_to_local, wi), th, ph);
    if (isnan(th) || isnan(ph)) return v3(0, 0, 0);
    float X = clampf(ph / (float)(2.0 * 3.14159265358979323846) * (float)S.env_w, 0.0f, (float)(S.env_w - 1.0f));
    float Y = clampf(th / (float)3.14159265358979323846 * (float)S.env_h, 0.0f, (float)(S.env_h - 1.0f));
    V3 rad = env_texel(S, (int)Y, (int)X);
    if (!is_valid(rad)) return v3(0, 0, 0);
    return rad * S.env_scale;
}

// Emitter::Sample of emitter e (Scene order) for next-event estimation: the
// integrator gives environment and directional emitters the scene's
// bounding-sphere radius as Distance (PathMISIntegrator.cpp:87-90)
__device__ __forceinline__ V3 emitter_sample(const DevScene &S, int e, ERec &er, float ux, float uy, float u1) {
    const int ai = __ldg(S.emitter_area + e);
    if (ai >= 0) return area_sample(S, S.area_lights[ai], er, ux, uy, u1);
    er.dist = S.scene_radius;
    if (ai == -1) return env_sample(S, er, ux, uy);
    return delta_sample(S, -2 - ai, er);
}

// ------------------------------------------------------------ camera
// PerspectiveCamera::SampleRay (src/camera/PerspectiveCamera.cpp:77) with the
// sample->camera projective map inverted in closed form.
__device__ __forceinline__ Ray camera_ray(const DevScene &S, float px, float py) {
    float u = px * (1.0f / (float)S.width), v = py * (1.0f / (float)S.height);
    V3 np = v3(S.cam_near * (1.0f - 2.0f * u) / S.cam_cot, S.cam_near * (1.0f - 2.0f * v) / (S.cam_aspect * S.cam_cot),
               S.cam_near);
    V3 dir = normalize(np);
    float invz = 1.0f / dir.z;
    const float *M = S.cam;
    Ray r;
    r.o = v3(M[3], M[7], M[11]);
    r.d = v3(M[0] * dir.x + M[1] * dir.y + M[2] * dir.z, M[4] * dir.x + M[5] * dir.y + M[6] * dir.z,
             M[8] * dir.x + M[9] * dir.y + M[10] * dir.z);
    r.tmin = S.cam_near * invz;
    r.tmax = S.cam_far * invz;
    return r;
}

// The differential ray directions of PerspectiveCamera::SampleRay (:94-98):
// through the near-plane point moved by m_dX / m_dY (:64), one pixel along x
// / y, in the closed form of the near-plane map.  M: row-major 3x4
// camera-to-world; width, height, aspect: the image's.
__device__ __forceinline__ void camera_diff(const DevScene &S, const float *M, uint32_t width, uint32_t height,
                                            float aspect, float px, float py, V3 &rx, V3 &ry) {
    const float iw = 1.0f / (float)width, ih = 1.0f / (float)height;
    const float u = px * iw, v = py * ih;
    const V3 np = v3(S.cam_near * (1.0f - 2.0f * u) / S.cam_cot, S.cam_near * (1.0f - 2.0f * v) / (aspect * S.cam_cot),
                     S.cam_near);
    const float dx = S.cam_near * (1.0f - 2.0f * iw) / S.cam_cot - S.cam_near / S.cam_cot;
    const float dy = S.cam_near * (1.0f - 2.0f * ih) / (aspect * S.cam_cot) - S.cam_near / (aspect * S.cam_cot);
    const V3 a = normalize(v3(np.x + dx, np.y, np.z)), b = normalize(v3(np.x, np.y + dy, np.z));
    rx = v3(M[0] * a.x + M[1] * a.y + M[2] * a.z, M[4] * a.x + M[5] * a.y + M[6] * a.z,
            M[8] * a.x + M[9] * a.y + M[10] * a.z);
    ry = v3(M[0] * b.x + M[1] * b.y + M[2] * b.z, M[4] * b.x + M[5] * b.y + M[6] * b.z,
            M[8] * b.x + M[9] * b.y + M[10] * b.z);
}

}  // namespace hk
