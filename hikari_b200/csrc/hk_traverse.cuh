// Software BVH traversal for sm_100a (B200 has no RT cores).
//
// Nodes are 64-byte BVH2 records (both child boxes in one node, fetched with
// four 128-bit read-only loads); triangles are pre-gathered 48-byte records
// in leaf order.  Closest-hit rays test triangles with the watertight test
// of Woop, Benthin and Wald (JCGT 2013), accepting both windings like the
// reference's Moller-Trumbore (src/core/Mesh.cpp:340) and the reference's
// closest-hit rule: a hit with t in [tmin, tmax] replaces the current one,
// tmax shrinks to its t (src/acceleration/HLBVHAcceleration.cpp:229-240).
// Any-hit (shadow) rays test with the reference's Moller-Trumbore itself, the
// test its shadow query applies, and stop at the first triangle it accepts.
#pragma once
#include "hk_device.h"
#include "hk_math.cuh"

#include <type_traits>

namespace hk {

struct Ray {
    V3 o, d;
    float tmin, tmax;
};

struct Hit {
    float t, u, v;    // u, v: weights of the 2nd and 3rd vertex (reference UV)
    int tri;          // index in leaf order, -1 = miss
};

// Per-ray constants of the watertight test.
struct WatertightRay {
    int kx, ky, kz;
    float sx, sy, sz;
};
__device__ __forceinline__ float comp(V3 v, int k) { return k == 0 ? v.x : (k == 1 ? v.y : v.z); }
__device__ __forceinline__ WatertightRay watertight_setup(V3 d) {
    WatertightRay w;
    float ax = fabsf(d.x), ay = fabsf(d.y), az = fabsf(d.z);
    w.kz = (ax > ay) ? (ax > az ? 0 : 2) : (ay > az ? 1 : 2);
    w.kx = w.kz + 1 == 3 ? 0 : w.kz + 1;
    w.ky = w.kx + 1 == 3 ? 0 : w.kx + 1;
    float dz = comp(d, w.kz);
    if (dz < 0.0f) { int t = w.kx; w.kx = w.ky; w.ky = t; }   // keep winding
    w.sx = comp(d, w.kx) / dz;
    w.sy = comp(d, w.ky) / dz;
    w.sz = 1.0f / dz;
    return w;
}

// Returns true and t, u, v when the ray hits triangle (a, b, c) with t in [tmin, tmax].
__device__ __forceinline__ bool intersect_watertight(const WatertightRay &w, V3 o, V3 a, V3 b, V3 c, float tmin,
                                                     float tmax, float &t, float &u, float &v) {
    V3 A = a - o, B = b - o, C = c - o;
    float Az = comp(A, w.kz), Bz = comp(B, w.kz), Cz = comp(C, w.kz);
    float Ax = comp(A, w.kx) - w.sx * Az, Ay = comp(A, w.ky) - w.sy * Az;
    float Bx = comp(B, w.kx) - w.sx * Bz, By = comp(B, w.ky) - w.sy * Bz;
    float Cx = comp(C, w.kx) - w.sx * Cz, Cy = comp(C, w.ky) - w.sy * Cz;
    float U = Cx * By - Cy * Bx;
    float Vv = Ax * Cy - Ay * Cx;
    float W = Bx * Ay - By * Ax;
    if (U == 0.0f || Vv == 0.0f || W == 0.0f) {   // edge: redo in double (watertight fallback)
        double CxBy = (double)Cx * (double)By, CyBx = (double)Cy * (double)Bx;
        U = (float)(CxBy - CyBx);
        double AxCy = (double)Ax * (double)Cy, AyCx = (double)Ay * (double)Cx;
        Vv = (float)(AxCy - AyCx);
        double BxAy = (double)Bx * (double)Ay, ByAx = (double)By * (double)Ax;
        W = (float)(BxAy - ByAx);
    }
    if ((U < 0.0f || Vv < 0.0f || W < 0.0f) && (U > 0.0f || Vv > 0.0f || W > 0.0f)) return false;
    float det = U + Vv + W;
    if (det == 0.0f) return false;
    Az *= w.sz; Bz *= w.sz; Cz *= w.sz;
    float T = U * Az + Vv * Bz + W * Cz;
    float rcp = 1.0f / det;
    float tt = T * rcp;
    if (!(tt >= tmin && tt <= tmax)) return false;
    t = tt;
    u = Vv * rcp;
    v = W * rcp;
    return true;
}

__device__ __forceinline__ float4 ldg4(const float4 *p) { return __ldg(p); }

// The reference's Moller-Trumbore arithmetic (Mesh::RayIntersect,
// src/core/Mesh.cpp:340-384), used to re-evaluate the winning triangle so that
// the reported t and barycentrics -- and so the shading point -- are the
// reference's own numbers.  Returns false where the reference's test rejects
// (|det| < 1e-8 or a barycentric outside [0,1] by rounding): the watertight
// values are kept there.
__device__ __forceinline__ bool refine_mt(V3 o, V3 d, V3 p0, V3 p1, V3 p2, float tmin, float tmax, float &t, float &u,
                                          float &v) {
    V3 e1 = p1 - p0, e2 = p2 - p0;
    V3 pv = cross(d, e2);
    float det = dot(e1, pv);
    if (det > -1e-8f && det < 1e-8f) return false;
    float inv = 1.0f / det;
    V3 tv = o - p0;
    float uu = dot(tv, pv) * inv;
    if (uu < 0.0f || uu > 1.0f) return false;
    V3 qv = cross(tv, e1);
    float vv = dot(d, qv) * inv;
    if (vv < 0.0f || uu + vv > 1.0f) return false;
    float tt = dot(e2, qv) * inv;
    if (!(tt >= tmin && tt <= tmax)) return false;
    t = tt;
    u = uu;
    v = vv;
    return true;
}

// Any-hit test of a shadow ray: Mesh::RayIntersect (src/core/Mesh.cpp:340-384)
// as the reference's shadow query runs it (HLBVHAcceleration::RayIntersect
// returns on the first triangle it accepts), so the occlusion decision is the
// reference's own.  No barycentrics or t leave the function.
__device__ __forceinline__ bool occludes_mt(V3 o, V3 d, V3 p0, V3 p1, V3 p2, float tmin, float tmax) {
    const V3 e1 = p1 - p0, e2 = p2 - p0;
    const V3 pv = cross(d, e2);
    const float det = dot(e1, pv);
    if (det > -1e-8f && det < 1e-8f) return false;
    const float inv = 1.0f / det;
    const V3 tv = o - p0;
    const float uu = dot(tv, pv) * inv;
    if (uu < 0.0f || uu > 1.0f) return false;
    const V3 qv = cross(tv, e1);
    const float vv = dot(d, qv) * inv;
    if (vv < 0.0f || uu + vv > 1.0f) return false;
    const float tt = dot(e2, qv) * inv;
    return tt >= tmin && tt <= tmax;
}

// Three-input min / max (PTX min.f32 / max.f32 with three sources, sm_100a).
__device__ __forceinline__ float fmax3f(float a, float b, float c) {
    float r;
    asm("max.f32 %0, %1, %2, %3;" : "=f"(r) : "f"(a), "f"(b), "f"(c));
    return r;
}
__device__ __forceinline__ float fmin3f(float a, float b, float c) {
    float r;
    asm("min.f32 %0, %1, %2, %3;" : "=f"(r) : "f"(a), "f"(b), "f"(c));
    return r;
}

// Slab test of two child boxes against the ray interval; explicit FMAs (the
// result only prunes, it never changes which triangle is reported).
__device__ __forceinline__ void box2(const float4 a, const float4 b, const float4 c, V3 idir, V3 ood, float tmin,
                                     float tmax, bool &hit0, bool &hit1, float &t0, float &t1) {
    float c0lox = __fmaf_rn(a.x, idir.x, -ood.x), c0hix = __fmaf_rn(a.y, idir.x, -ood.x);
    float c0loy = __fmaf_rn(a.z, idir.y, -ood.y), c0hiy = __fmaf_rn(a.w, idir.y, -ood.y);
    float c1lox = __fmaf_rn(b.x, idir.x, -ood.x), c1hix = __fmaf_rn(b.y, idir.x, -ood.x);
    float c1loy = __fmaf_rn(b.z, idir.y, -ood.y), c1hiy = __fmaf_rn(b.w, idir.y, -ood.y);
    float c0loz = __fmaf_rn(c.x, idir.z, -ood.z), c0hiz = __fmaf_rn(c.y, idir.z, -ood.z);
    float c1loz = __fmaf_rn(c.z, idir.z, -ood.z), c1hiz = __fmaf_rn(c.w, idir.z, -ood.z);
    float n0 = fmax3f(fminf(c0lox, c0hix), fminf(c0loy, c0hiy), fmaxf(fminf(c0loz, c0hiz), tmin));
    float f0 = fmin3f(fmaxf(c0lox, c0hix), fmaxf(c0loy, c0hiy), fminf(fmaxf(c0loz, c0hiz), tmax));
    float n1 = fmax3f(fminf(c1lox, c1hix), fminf(c1loy, c1hiy), fmaxf(fminf(c1loz, c1hiz), tmin));
    float f1 = fmin3f(fmaxf(c1lox, c1hix), fmaxf(c1loy, c1hiy), fminf(fmaxf(c1loz, c1hiz), tmax));
    // slack of a few ulps keeps boxes of axis-aligned, zero-thickness geometry
    hit0 = n0 <= f0 * 1.00000024f + 1e-30f;
    hit1 = n1 <= f1 * 1.00000024f + 1e-30f;
    t0 = n0;
    t1 = n1;
}

// Per-thread traversal statistics (node fetches and triangle tests), the
// basis of the algorithmic-bytes roofline.
struct TravStats {
    uint32_t nodes = 0, tris = 0;
};

// Binary-tree traversal as a resumable walker: begin() sets a ray up, each
// step() visits one node (box test of both children, leaf triangles tested
// at once, near child next, far child pushed) and returns true when the ray
// is done; end() adds the statistics and re-evaluates the closest hit with the
// reference's arithmetic.  A single-leaf tree is stored as a root whose child0
// is the leaf and child1 an empty box.
struct Bvh2Walker {
    V3 o, d, idir, ood;
    float tmin, tmax, tmax0;
    WatertightRay w;
    int node, sp;
    bool found;
    Hit hit;
    uint32_t nvis, ntri;
    int *stack;   // kStackSize entries owned by the caller (kept out of the walker so it stays in registers)

    __device__ __forceinline__ void begin(const DevScene &S, const Ray &ray) {
        o = ray.o;
        d = ray.d;
        // zero components -> tiny signed values: inverse stays finite, no 0*inf NaN
        const float tiny = 1e-30f;
        const V3 dd = v3(fabsf(d.x) < tiny ? copysignf(tiny, d.x) : d.x, fabsf(d.y) < tiny ? copysignf(tiny, d.y) : d.y,
                         fabsf(d.z) < tiny ? copysignf(tiny, d.z) : d.z);
        idir = v3(1.0f / dd.x, 1.0f / dd.y, 1.0f / dd.z);
        ood = v3(o.x * idir.x, o.y * idir.y, o.z * idir.z);
        w = watertight_setup(d);
        tmin = ray.tmin;
        tmax = tmax0 = ray.tmax;
        node = S.nnodes == 0 ? -1 : 0;
        sp = 0;
        found = false;
        hit.tri = -1;
        nvis = ntri = 0;
    }

    template <bool kAnyHit>
    __device__ __forceinline__ bool step(const DevScene &S) {
        if (node < 0) return true;
        const float4 *np = S.nodes + 4 * node;
        const float4 a = ldg4(np), b = ldg4(np + 1), c = ldg4(np + 2), e = ldg4(np + 3);
        const int c0 = __float_as_int(e.x), c1 = __float_as_int(e.y);
        ++nvis;
        bool h0, h1;
        float t0, t1;
        box2(a, b, c, idir, ood, tmin, tmax, h0, h1, t0, t1);
        int next = -0x7fffffff;   // sentinel: pop
        int leafs[2];
        int nleaf = 0;
        int inner[2];
        float tin[2];
        int ninner = 0;
        if (h0) { if (c0 < 0) leafs[nleaf++] = c0; else { inner[ninner] = c0; tin[ninner++] = t0; } }
        if (h1) { if (c1 < 0) leafs[nleaf++] = c1; else { inner[ninner] = c1; tin[ninner++] = t1; } }
        for (int l = 0; l < nleaf; ++l) {
            const uint32_t enc = ~(uint32_t)leafs[l];
            const uint32_t start = enc & kLeafStartMask, cnt = enc >> kLeafCountShift;
            ntri += cnt;
            for (uint32_t i = 0; i < cnt; ++i) {
                const float4 *tp = S.tris + 3 * (start + i);
                const float4 p0 = ldg4(tp), p1 = ldg4(tp + 1), p2 = ldg4(tp + 2);
                if constexpr (kAnyHit) {
                    if (occludes_mt(o, d, xyz(p0), xyz(p1), xyz(p2), tmin, tmax)) {
                        found = true;
                        hit.tri = (int)(start + i);
                        return true;
                    }
                } else {
                    float tt, uu, vv;
                    if (intersect_watertight(w, o, xyz(p0), xyz(p1), xyz(p2), tmin, tmax, tt, uu, vv)) {
                        found = true;
                        hit.t = tt; hit.u = uu; hit.v = vv; hit.tri = (int)(start + i);
                        tmax = tt;
                    }
                }
            }
        }
        if (ninner == 2) {
            const bool swap = tin[1] < tin[0];
            const int nearc = swap ? inner[1] : inner[0], farc = swap ? inner[0] : inner[1];
            if (sp < kStackSize) stack[sp++] = farc;
            next = nearc;
        } else if (ninner == 1) {
            next = inner[0];
        }
        if (next == -0x7fffffff) {
            if (sp == 0) return true;
            next = stack[--sp];
        }
        node = next;
        return false;
    }

    template <bool kAnyHit>
    __device__ __forceinline__ void end(const DevScene &S, TravStats &st) {
        st.nodes += nvis;
        st.tris += ntri;
        if (found && !kAnyHit) {
            const float4 *tp = S.tris + 3 * hit.tri;
            refine_mt(o, d, xyz(ldg4(tp)), xyz(ldg4(tp + 1)), xyz(ldg4(tp + 2)), tmin, tmax0, hit.t, hit.u, hit.v);
        }
    }
};

// Closest hit (any_hit = false) or first hit (any_hit = true).
template <bool kAnyHit>
__device__ __forceinline__ bool trace_bvh2(const DevScene &S, const Ray &ray, Hit &hit, TravStats &st) {
    int stack[kStackSize];
    Bvh2Walker wk;
    wk.stack = stack;
    wk.begin(S, ray);
    while (!wk.template step<kAnyHit>(S)) {}
    wk.template end<kAnyHit>(S, st);
    hit = wk.hit;
    return wk.found;
}

// ------------------------------------------------------------ 8-wide tree
// Traversal of the compressed 8-wide BVH (hk_bvh.h), following Ylitie, Karras
// and Laine (HPG 2017): a node group is (first child index, hit bits of the
// internal children << 24 | imask), a triangle group is (first triangle,
// hit bits 0..23).  Hit bits of internal children sit at slot ^ (7 ^ octant),
// so the lowest set bit is the nearest child.  A warp vote postpones the
// triangle tests of lanes that are few among the active ones while they still
// have nodes to visit, so that lanes intersect triangles together.

constexpr int kShStack = 8;   // entries per thread kept in shared memory

// Traversal stack in local memory (e: kStackSize entries owned by the caller).
struct LocalStack {
    uint2 *e;
    int sp = 0;
    // The tree depth bound keeps sp below kStackSize; past it an entry would be dropped, never written out of bounds.
    __device__ __forceinline__ void push(uint2 v) {
        if (sp < kStackSize) e[sp++] = v;
    }
    __device__ __forceinline__ uint2 pop() { return e[--sp]; }
};

// Short stack: the top kShStack entries of each thread in shared memory
// (sh[k * stride], one column per thread), deeper entries in local memory.
struct SharedStack {
    uint2 *sh;
    int stride;
    int sp = 0;
    uint2 *spill;   // kStackSize - kShStack entries in local memory, owned by the caller
    __device__ __forceinline__ void push(uint2 v) {
        if (sp < kShStack) sh[sp++ * stride] = v;
        else if (sp < kStackSize) { spill[sp - kShStack] = v; ++sp; }
    }
    __device__ __forceinline__ uint2 pop() {
        --sp;
        return sp < kShStack ? sh[sp * stride] : spill[sp - kShStack];
    }
};

__device__ __forceinline__ uint4 ldg4u(const uint4 *p) { return __ldg(p); }

// Byte k of x as a float in [0, 255]: a byte permute builds the float
// 2^23 + q (exponent byte 0x4B, q in the low mantissa byte), and subtracting
// 2^23 is exact -- two full-rate instructions instead of an integer-to-float
// conversion.
template <int k>
__device__ __forceinline__ float qbyte(uint32_t x) {
    return __uint_as_float(__byte_perm(x, 0x4B000000u, 0x7440u | k)) - 8388608.0f;
}
// Two FMAs in one instruction (PTX fma.rn.f32x2, sm_100a): each lane is an
// IEEE round-to-nearest FMA, the same result as two __fmaf_rn.
__device__ __forceinline__ float2 fma2(float2 a, float2 b, float2 c) {
    float2 r;
    asm("{\n\t.reg .b64 pa, pb, pc, pr;\n\t"
        "mov.b64 pa, {%2, %3};\n\tmov.b64 pb, {%4, %5};\n\tmov.b64 pc, {%6, %7};\n\t"
        "fma.rn.f32x2 pr, pa, pb, pc;\n\tmov.b64 {%0, %1}, pr;\n\t}"
        : "=f"(r.x), "=f"(r.y)
        : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y), "f"(c.x), "f"(c.y));
    return r;
}

// The float 2^23 + q without the subtraction: the slab offsets of a node are
// shifted by -2^23 steps instead (one rounding of at most half a step, which
// the one-step padding of the quantised boxes absorbs).
template <int k>
__device__ __forceinline__ float qbyte_biased(uint32_t x) {
    return __uint_as_float(__byte_perm(x, 0x4B000000u, 0x7440u | k));
}

template <class Stack>
struct Bvh8Walker {
    V3 o, d, idir;
    float tmin, tmax, tmax0;
    WatertightRay w;
    uint32_t oct, ko;
    uint2 ng, tg;
    bool found;
    Hit hit;
    uint32_t nvis, ntri;
    Stack stk;

    __device__ __forceinline__ void begin(const DevScene &S, const Ray &ray) {
        o = ray.o;
        d = ray.d;
        // |1/d| <= 1e20 keeps 2^23 steps of up to 2^38 (the largest step the build emits) finite
        const float tiny = 1e-20f;
        const V3 dd = v3(fabsf(d.x) < tiny ? copysignf(tiny, d.x) : d.x, fabsf(d.y) < tiny ? copysignf(tiny, d.y) : d.y,
                         fabsf(d.z) < tiny ? copysignf(tiny, d.z) : d.z);
        idir = v3(1.0f / dd.x, 1.0f / dd.y, 1.0f / dd.z);
        oct = (idir.x < 0.0f ? 1u : 0u) | (idir.y < 0.0f ? 2u : 0u) | (idir.z < 0.0f ? 4u : 0u);
        ko = 7u ^ oct;
        w = watertight_setup(d);
        tmin = ray.tmin;
        tmax = tmax0 = ray.tmax;
        // the root as slot 0 of a virtual parent (nothing for an empty tree)
        ng = make_uint2(0u, S.nwnodes == 0 ? 0u : ((1u << (24 + ko)) | 1u));
        tg = make_uint2(0u, 0u);
        stk.sp = 0;
        found = false;
        hit.tri = -1;
        nvis = ntri = 0;
    }

    // One node visit (or one popped triangle group) and its triangle tests.
    template <bool kAnyHit>
    __device__ __forceinline__ bool step(const DevScene &S) {
        if (ng.y > 0x00ffffffu) {
            const uint32_t b = __ffs(ng.y >> 24) - 1;
            ng.y &= ~(1u << (24 + b));
            const uint32_t slot = b ^ ko;
            const uint32_t child = ng.x + __popc(ng.y & 0xffu & ((1u << slot) - 1u));
            if (ng.y > 0x00ffffffu) stk.push(ng);
            visit(S, child);
        } else {
            tg = ng;   // a postponed triangle group from the stack (or nothing)
            ng = make_uint2(0u, 0u);
        }
        if (kAnyHit ? S.postpone_any : S.postpone) {   // any-hit rays only where the launch asks
            const unsigned act = __activemask();
            const unsigned want = __ballot_sync(act, tg.y != 0u);
            if (tg.y != 0u && ng.y > 0x00ffffffu && __popc(want) * 5 < __popc(act)) {
                stk.push(tg);
                tg.y = 0u;
            }
        }
        while (tg.y != 0u) {
            const uint32_t tri = tg.x + (__ffs(tg.y) - 1);
            tg.y &= tg.y - 1u;
            ++ntri;
            const float4 *tp = S.tris + 3 * (size_t)tri;
            const float4 p0 = ldg4(tp), p1 = ldg4(tp + 1), p2 = ldg4(tp + 2);
            if constexpr (kAnyHit) {
                if (occludes_mt(o, d, xyz(p0), xyz(p1), xyz(p2), tmin, tmax)) {
                    found = true;
                    hit.tri = (int)tri;
                    return true;
                }
            } else {
                float tt, uu, vv;
                if (intersect_watertight(w, o, xyz(p0), xyz(p1), xyz(p2), tmin, tmax, tt, uu, vv)) {
                    found = true;
                    hit.t = tt; hit.u = uu; hit.v = vv; hit.tri = (int)tri;
                    tmax = tt;
                }
            }
        }
        if (ng.y <= 0x00ffffffu) {
            if (stk.sp == 0) return true;
            ng = stk.pop();
        }
        return false;
    }

    // One step of an any-hit ray with the warp's triangle tests shared out:
    // every lane of the warp calls it (alive: the lane holds a ray).  Alive
    // lanes visit a node (or pop a triangle group); the triangles of all
    // lanes' groups are then numbered in lane order and tested 32 at a time,
    // lane j taking triangle r + j of the numbering against its owner's ray
    // (rays: the warp's rays in shared memory, origin + tmin then direction +
    // tmax per lane), and a lane is occluded when any of its triangles is.
    // The serial loop of step() runs as many rounds as the warp's largest
    // group, with the other lanes idle; this runs ceil(sum / 32).
    __device__ __forceinline__ bool step_any_shared(const DevScene &S, bool alive, const float4 *rays) {
        const unsigned lane = threadIdx.x & 31u;
        uint2 grp = make_uint2(0u, 0u);
        if (alive) {
            if (ng.y > 0x00ffffffu) {
                const uint32_t b = __ffs(ng.y >> 24) - 1;
                ng.y &= ~(1u << (24 + b));
                const uint32_t slot = b ^ ko;
                const uint32_t child = ng.x + __popc(ng.y & 0xffu & ((1u << slot) - 1u));
                if (ng.y > 0x00ffffffu) stk.push(ng);
                visit(S, child);
                grp = tg;
            } else {
                grp = ng;   // a postponed triangle group from the stack (or nothing)
                ng = make_uint2(0u, 0u);
            }
            tg = make_uint2(0u, 0u);
        }
        const uint32_t cnt = __popc(grp.y);
        uint32_t incl = cnt;   // inclusive prefix of the counts in lane order
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t v = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= (unsigned)o) incl += v;
        }
        const uint32_t total = __shfl_sync(0xffffffffu, incl, 31);
        const uint32_t excl = incl - cnt;
        ntri += cnt;
        bool occluded = false;
        for (uint32_t r = 0; r < total; r += 32) {   // warp-uniform
            const uint32_t w = r + lane;
            // owner: the number of lanes whose inclusive prefix is <= w
            // (binary lifting; every index read stays within 0..31)
            uint32_t own = 0;
#pragma unroll
            for (uint32_t b = 16; b > 0; b >>= 1) {
                const uint32_t v = __shfl_sync(0xffffffffu, incl, own + b - 1);
                if (v <= w) own += b;
            }
            const uint32_t obase = __shfl_sync(0xffffffffu, grp.x, own);
            const uint32_t omask = __shfl_sync(0xffffffffu, grp.y, own);
            const uint32_t oexcl = __shfl_sync(0xffffffffu, excl, own);
            bool hit = false;
            if (w < total) {
                const uint32_t tri = obase + __fns(omask, 0u, (int)(w - oexcl) + 1);
                const float4 *tp = S.tris + 3 * (size_t)tri;
                const float4 p0 = ldg4(tp), p1 = ldg4(tp + 1), p2 = ldg4(tp + 2);
                const float4 ro = rays[2 * own], rd = rays[2 * own + 1];
                hit = occludes_mt(xyz(ro), xyz(rd), xyz(p0), xyz(p1), xyz(p2), ro.w, rd.w);
            }
            const uint32_t hb = __ballot_sync(0xffffffffu, hit);
            // the lanes that tested this lane's triangles in round r
            const int lo = max((int)excl - (int)r, 0), hi = min((int)incl - (int)r, 32);
            if (lo < hi) {
                const uint32_t upto = hi >= 32 ? 0xffffffffu : ((1u << hi) - 1u);
                if (hb & upto & ~((1u << lo) - 1u)) occluded = true;
            }
        }
        if (!alive) return false;
        if (occluded) {
            found = true;
            return true;
        }
        if (ng.y <= 0x00ffffffu) {
            if (stk.sp == 0) return true;
            ng = stk.pop();
        }
        return false;
    }

    // One step of a closest-hit ray with the warp's triangle tests shared out,
    // numbered and dealt as in step_any_shared: lane j of round r tests
    // triangle r + j with the watertight test against its owner's ray (rays:
    // origin + tmin and the packed watertight constants per lane; the owner's
    // current tmax by shuffle).  Per owner the hit of least t wins and, on
    // equal t, the one later in the owner's test order: the hit that the
    // serial loop of step() keeps, since it accepts t <= tmax and then shrinks
    // tmax to t.  A group that spans two rounds sees the first round's tmax in
    // the second, as the serial loop would.
    __device__ __forceinline__ bool step_closest_shared(const DevScene &S, bool alive, const float4 *rays) {
        const unsigned lane = threadIdx.x & 31u;
        uint2 grp = make_uint2(0u, 0u);
        if (alive) {
            if (ng.y > 0x00ffffffu) {
                const uint32_t b = __ffs(ng.y >> 24) - 1;
                ng.y &= ~(1u << (24 + b));
                const uint32_t slot = b ^ ko;
                const uint32_t child = ng.x + __popc(ng.y & 0xffu & ((1u << slot) - 1u));
                if (ng.y > 0x00ffffffu) stk.push(ng);
                visit(S, child);
                grp = tg;
            } else {
                grp = ng;
                ng = make_uint2(0u, 0u);
            }
            tg = make_uint2(0u, 0u);
        }
        const uint32_t cnt = __popc(grp.y);
        uint32_t incl = cnt;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t v = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= (unsigned)o) incl += v;
        }
        const uint32_t total = __shfl_sync(0xffffffffu, incl, 31);
        const uint32_t excl = incl - cnt;
        ntri += cnt;
        for (uint32_t r = 0; r < total; r += 32) {   // warp-uniform
            const uint32_t w = r + lane;
            uint32_t own = 0;
#pragma unroll
            for (uint32_t b = 16; b > 0; b >>= 1) {
                const uint32_t v = __shfl_sync(0xffffffffu, incl, own + b - 1);
                if (v <= w) own += b;
            }
            const uint32_t obase = __shfl_sync(0xffffffffu, grp.x, own);
            const uint32_t omask = __shfl_sync(0xffffffffu, grp.y, own);
            const uint32_t oexcl = __shfl_sync(0xffffffffu, excl, own);
            const float otmax = __shfl_sync(0xffffffffu, tmax, own);
            // (t, 31 - lane): the least key is the least t, then the latest lane
            unsigned long long key = ~0ull;
            float tt = 0.0f, uu = 0.0f, vv = 0.0f;
            uint32_t tri = 0u;
            if (w < total) {
                tri = obase + __fns(omask, 0u, (int)(w - oexcl) + 1);
                const float4 *tp = S.tris + 3 * (size_t)tri;
                const float4 p0 = ldg4(tp), p1 = ldg4(tp + 1), p2 = ldg4(tp + 2);
                const float4 ro = rays[2 * own], rw = rays[2 * own + 1];
                const uint32_t kp = __float_as_uint(rw.w);
                WatertightRay wr;
                wr.kx = (int)(kp & 3u);
                wr.ky = (int)((kp >> 2) & 3u);
                wr.kz = (int)((kp >> 4) & 3u);
                wr.sx = rw.x;
                wr.sy = rw.y;
                wr.sz = rw.z;
                if (intersect_watertight(wr, xyz(ro), xyz(p0), xyz(p1), xyz(p2), ro.w, otmax, tt, uu, vv)) {
                    const uint32_t tb = __float_as_uint(tt);
                    const uint32_t ord = (tb & 0x80000000u) ? ~tb : (tb | 0x80000000u);   // order of the floats
                    key = ((unsigned long long)ord << 32) | (31u - lane);
                }
            }
            // least key within each owner's run of lanes (runs are contiguous)
#pragma unroll
            for (int s = 1; s < 32; s <<= 1) {
                const unsigned long long k2 = __shfl_down_sync(0xffffffffu, key, s);
                const uint32_t o2 = __shfl_down_sync(0xffffffffu, own, s);
                if (lane + (unsigned)s < 32u && o2 == own && k2 < key) key = k2;
            }
            // this lane's run in round r starts at lane lo
            const int lo = max((int)excl - (int)r, 0), hi = min((int)incl - (int)r, 32);
            const unsigned long long mk = __shfl_sync(0xffffffffu, key, lo < hi ? lo : 0);
            const uint32_t wl = 31u - (uint32_t)(mk & 31u);
            const float wt = __shfl_sync(0xffffffffu, tt, wl), wu = __shfl_sync(0xffffffffu, uu, wl),
                        wv = __shfl_sync(0xffffffffu, vv, wl);
            const uint32_t wtri = __shfl_sync(0xffffffffu, tri, wl);
            if (lo < hi && mk != ~0ull) {
                found = true;
                hit.t = wt; hit.u = wu; hit.v = wv; hit.tri = (int)wtri;
                tmax = wt;
            }
        }
        if (!alive) return false;
        if (ng.y <= 0x00ffffffu) {
            if (stk.sp == 0) return true;
            ng = stk.pop();
        }
        return false;
    }

    // The per-lane record step_closest_shared reads: origin + tmin, and the
    // watertight constants with kx | ky << 2 | kz << 4 in the last word.
    __device__ __forceinline__ void closest_record(float4 *dst) const {
        dst[0] = make_float4(o.x, o.y, o.z, tmin);
        dst[1] = make_float4(w.sx, w.sy, w.sz, __uint_as_float((uint32_t)w.kx | ((uint32_t)w.ky << 2) | ((uint32_t)w.kz << 4)));
    }

    // Intersect the 8 children of node `child`: ng / tg become its groups.
    __device__ __forceinline__ void visit(const DevScene &S, uint32_t child) {
        const uint4 *np = S.wnodes + 5 * (size_t)child;
        const uint4 n0 = ldg4u(np), n1 = ldg4u(np + 1), n2 = ldg4u(np + 2), n3 = ldg4u(np + 3), n4 = ldg4u(np + 4);
        ++nvis;
        const float adx = __uint_as_float((n0.w & 0xffu) << 23) * idir.x;
        const float ady = __uint_as_float(((n0.w >> 8) & 0xffu) << 23) * idir.y;
        const float adz = __uint_as_float(((n0.w >> 16) & 0xffu) << 23) * idir.z;
        const float ox = __fmaf_rn(-8388608.0f, adx, (__uint_as_float(n0.x) - o.x) * idir.x);
        const float oy = __fmaf_rn(-8388608.0f, ady, (__uint_as_float(n0.y) - o.y) * idir.y);
        const float oz = __fmaf_rn(-8388608.0f, adz, (__uint_as_float(n0.z) - o.z) * idir.z);
        const uint32_t imask = n0.w >> 24;
        // meta of internal children: slot ^ (7 ^ octant) in the position bits
        const uint32_t in0 = ((imask & 0xfu) * 0x00204081u) & 0x01010101u;
        const uint32_t in1 = ((imask >> 4) * 0x00204081u) & 0x01010101u;
        const uint32_t meta0 = n1.z ^ (in0 * ko), meta1 = n1.w ^ (in1 * ko);
        // near / far planes per axis (lo planes first for a positive direction)
        const uint32_t nx0 = oct & 1u ? n3.z : n2.x, nx1 = oct & 1u ? n3.w : n2.y;
        const uint32_t fx0 = oct & 1u ? n2.x : n3.z, fx1 = oct & 1u ? n2.y : n3.w;
        const uint32_t ny0 = oct & 2u ? n4.x : n2.z, ny1 = oct & 2u ? n4.y : n2.w;
        const uint32_t fy0 = oct & 2u ? n2.z : n4.x, fy1 = oct & 2u ? n2.w : n4.y;
        const uint32_t nz0 = oct & 4u ? n4.z : n3.x, nz1 = oct & 4u ? n4.w : n3.y;
        const uint32_t fz0 = oct & 4u ? n3.x : n4.z, fz1 = oct & 4u ? n3.y : n4.w;
        uint32_t hits = 0;
        const float t0 = tmin, t1 = tmax;
        const float2 adx2 = make_float2(adx, adx), ady2 = make_float2(ady, ady), adz2 = make_float2(adz, adz);
        const float2 ox2 = make_float2(ox, ox), oy2 = make_float2(oy, oy), oz2 = make_float2(oz, oz);
        auto test_child = [&](auto kk, uint32_t xn, uint32_t xf, uint32_t yn, uint32_t yf, uint32_t zn, uint32_t zf,
                              uint32_t meta) {
            constexpr int k = decltype(kk)::value;
            // near and far plane of an axis in one packed FMA
            const float2 tx = fma2(make_float2(qbyte_biased<k>(xn), qbyte_biased<k>(xf)), adx2, ox2);
            const float2 ty = fma2(make_float2(qbyte_biased<k>(yn), qbyte_biased<k>(yf)), ady2, oy2);
            const float2 tz = fma2(make_float2(qbyte_biased<k>(zn), qbyte_biased<k>(zf)), adz2, oz2);
            const float tn = fmax3f(tx.x, ty.x, fmaxf(tz.x, t0));
            const float tf = fmin3f(tx.y, ty.y, fminf(tz.y, t1));
            const uint32_t m = __byte_perm(meta, 0u, 0x4440u | k);
            if (tn <= tf * 1.00000024f + 1e-30f) hits |= (m >> 5) << (m & 31u);
        };
        test_child(std::integral_constant<int, 0>{}, nx0, fx0, ny0, fy0, nz0, fz0, meta0);
        test_child(std::integral_constant<int, 1>{}, nx0, fx0, ny0, fy0, nz0, fz0, meta0);
        test_child(std::integral_constant<int, 2>{}, nx0, fx0, ny0, fy0, nz0, fz0, meta0);
        test_child(std::integral_constant<int, 3>{}, nx0, fx0, ny0, fy0, nz0, fz0, meta0);
        test_child(std::integral_constant<int, 0>{}, nx1, fx1, ny1, fy1, nz1, fz1, meta1);
        test_child(std::integral_constant<int, 1>{}, nx1, fx1, ny1, fy1, nz1, fz1, meta1);
        test_child(std::integral_constant<int, 2>{}, nx1, fx1, ny1, fy1, nz1, fz1, meta1);
        test_child(std::integral_constant<int, 3>{}, nx1, fx1, ny1, fy1, nz1, fz1, meta1);
        ng = make_uint2(n1.x, (hits & 0xff000000u) | imask);
        tg = make_uint2(n1.y, hits & 0x00ffffffu);
    }

    template <bool kAnyHit>
    __device__ __forceinline__ void end(const DevScene &S, TravStats &st) {
        st.nodes += nvis;
        st.tris += ntri;
        if (found && !kAnyHit) {
            const float4 *tp = S.tris + 3 * hit.tri;
            refine_mt(o, d, xyz(ldg4(tp)), xyz(ldg4(tp + 1)), xyz(ldg4(tp + 2)), tmin, tmax0, hit.t, hit.u, hit.v);
        }
    }
};

template <bool kAnyHit>
__device__ __forceinline__ bool trace_bvh8(const DevScene &S, const Ray &ray, Hit &hit, TravStats &st) {
    uint2 stack[kStackSize];
    Bvh8Walker<LocalStack> wk;
    wk.stk.e = stack;
    wk.begin(S, ray);
    while (!wk.template step<kAnyHit>(S)) {}
    wk.template end<kAnyHit>(S, st);
    hit = wk.hit;
    return wk.found;
}

// Closest hit (kAnyHit = false) or first hit in the tree kAccel; kernels are
// instantiated per tree and the host launches the scene's one.
template <int kAccel, bool kAnyHit>
__device__ __forceinline__ bool trace(const DevScene &S, const Ray &ray, Hit &hit, TravStats &st) {
    if constexpr (kAccel == kAccelBvh8) return trace_bvh8<kAnyHit>(S, ray, hit, st);
    else return trace_bvh2<kAnyHit>(S, ray, hit, st);
}

// Walker type of a tree.
template <int kAccel, class Stack>
using WalkerOf = std::conditional_t<kAccel == kAccelBvh8, Bvh8Walker<Stack>, Bvh2Walker>;

// Traverses n rays of a queue with dynamic fetching: a lane whose ray is done
// takes the next unclaimed ray, so lanes do not idle until the warp's longest
// ray ends (persistent while-while traversal with ray replacement, Aila and
// Laine, "Understanding the Efficiency of Ray Traversal on GPUs", HPG 2009).
// A warp claims kFetchChunk consecutive queue entries with one atomic on
// *fetch and hands them to its lanes itself (one atomic per refill would
// serialise at the L2 on that one address).  Lanes check for a refill every
// `steps` node visits; while other lanes still traverse, a warp refills only
// once at least `min_idle` lanes are idle.  load(i) returns ray i;
// store(i, walker) consumes the result.  Every lane of the warp must call
// this (full-warp votes).
constexpr unsigned kFetchChunk = 128;

template <bool kAnyHit, class Walker, class Load, class Store>
__device__ __forceinline__ void trace_queue(const DevScene &S, Walker &wk, unsigned *fetch, unsigned n, int steps,
                                            int min_idle, Load load, Store store, TravStats &st) {
    const unsigned lane = threadIdx.x & 31u;
    int item = -1;
    bool exhausted = false;
    unsigned chunk_next = 0, chunk_end = 0;   // warp-uniform: unhanded entries of the claimed chunk
    for (;;) {
        const unsigned want = __ballot_sync(0xffffffffu, item < 0 && !exhausted);
        const unsigned busy = __ballot_sync(0xffffffffu, item >= 0);
        if (want && (busy == 0u || __popc(want) >= min_idle)) {
            const unsigned k = __popc(want), rank = __popc(want & ((1u << lane) - 1u));
            const unsigned avail = chunk_end - chunk_next;
            unsigned idx = chunk_next + rank;
            if (k > avail) {   // warp-uniform: claim the next chunk for the lanes past the old one
                unsigned base = 0;
                if ((int)lane == __ffs(want) - 1) base = atomicAdd(fetch, kFetchChunk);
                base = __shfl_sync(0xffffffffu, base, __ffs(want) - 1);
                if (rank >= avail) idx = base + (rank - avail);
                chunk_next = base + (k - avail);
                chunk_end = base + kFetchChunk;
            } else {
                chunk_next += k;
            }
            if (want >> lane & 1u) {
                if (idx < n) {
                    item = (int)idx;
                    wk.begin(S, load(item));
                } else {
                    exhausted = true;
                }
            }
        }
        if (!__any_sync(0xffffffffu, item >= 0)) break;
        if (item >= 0) {
            for (int k = 0; k < steps; ++k) {
                if (wk.template step<kAnyHit>(S)) {
                    wk.template end<kAnyHit>(S, st);
                    store(item, wk);
                    item = -1;
                    break;
                }
            }
        }
    }
}

// trace_queue with the warp's triangle tests shared out
// (Bvh8Walker::step_any_shared for any-hit rays, step_closest_shared for
// closest-hit rays): the same refills, but every lane takes every step, lanes
// without a ray as idle partners.  rays: 2 float4 per thread of the block
// (shared memory), written here when a lane takes a ray.
template <bool kAnyHit, class Walker, class Load, class Store>
__device__ __forceinline__ void trace_queue_shared(const DevScene &S, Walker &wk, unsigned *fetch, unsigned n,
                                                   int steps, int min_idle, float4 *rays, Load load, Store store,
                                                   TravStats &st) {
    const unsigned lane = threadIdx.x & 31u;
    float4 *mine = rays + 2 * threadIdx.x;
    const float4 *warp_rays = rays + 2 * (threadIdx.x & ~31u);
    int item = -1;
    bool exhausted = false;
    unsigned chunk_next = 0, chunk_end = 0;
    for (;;) {
        const unsigned want = __ballot_sync(0xffffffffu, item < 0 && !exhausted);
        const unsigned busy = __ballot_sync(0xffffffffu, item >= 0);
        if (want && (busy == 0u || __popc(want) >= min_idle)) {
            const unsigned k = __popc(want), rank = __popc(want & ((1u << lane) - 1u));
            const unsigned avail = chunk_end - chunk_next;
            unsigned idx = chunk_next + rank;
            if (k > avail) {
                unsigned base = 0;
                if ((int)lane == __ffs(want) - 1) base = atomicAdd(fetch, kFetchChunk);
                base = __shfl_sync(0xffffffffu, base, __ffs(want) - 1);
                if (rank >= avail) idx = base + (rank - avail);
                chunk_next = base + (k - avail);
                chunk_end = base + kFetchChunk;
            } else {
                chunk_next += k;
            }
            if (want >> lane & 1u) {
                if (idx < n) {
                    item = (int)idx;
                    const Ray r = load(item);
                    wk.begin(S, r);
                    if constexpr (kAnyHit) {
                        mine[0] = make_float4(r.o.x, r.o.y, r.o.z, r.tmin);
                        mine[1] = make_float4(r.d.x, r.d.y, r.d.z, r.tmax);
                    } else {
                        wk.closest_record(mine);
                    }
                } else {
                    exhausted = true;
                }
            }
        }
        if (!__any_sync(0xffffffffu, item >= 0)) break;
        __syncwarp();   // the new rays are visible to the warp's other lanes
        for (int k = 0; k < steps; ++k) {
            bool done;
            if constexpr (kAnyHit) done = wk.step_any_shared(S, item >= 0, warp_rays);
            else done = wk.step_closest_shared(S, item >= 0, warp_rays);
            if (item >= 0 && done) {
                wk.template end<kAnyHit>(S, st);
                store(item, wk);
                item = -1;
            }
            if (!__any_sync(0xffffffffu, item >= 0)) break;
        }
        __syncwarp();   // every read of a lane's ray precedes its replacement
    }
}

}  // namespace hk
