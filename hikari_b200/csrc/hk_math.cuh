// Device math for the pathMIS core: 3-vectors in the reference's float
// evaluation order, pcg32, shading frames and the sampling warps.
//
// The library is compiled with -fmad=false so that products and sums round
// like the reference's x86 build (no FMA contraction); 3-vector dot products
// reduce as x + (y + z), which is how Eigen 3.3 unrolls a fixed-size redux
// (ext/eigen/Eigen/src/Core/Redux.h:91).  Where rounding cannot change a
// result (box tests) the code uses explicit __fmaf_rn.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace hk {

constexpr float kPi = 3.14159265358979323846f;
constexpr double kInvPiD = 0.31830988618379067154;
constexpr float kRayEps = 1e-4f;     // Epsilon, include/core/Common.hpp:43

struct V3 { float x, y, z; };
__device__ __forceinline__ V3 v3(float x, float y, float z) { return V3{x, y, z}; }
__device__ __forceinline__ V3 operator+(V3 a, V3 b) { return v3(a.x + b.x, a.y + b.y, a.z + b.z); }
__device__ __forceinline__ V3 operator-(V3 a, V3 b) { return v3(a.x - b.x, a.y - b.y, a.z - b.z); }
__device__ __forceinline__ V3 operator*(V3 a, V3 b) { return v3(a.x * b.x, a.y * b.y, a.z * b.z); }
__device__ __forceinline__ V3 operator*(V3 a, float s) { return v3(a.x * s, a.y * s, a.z * s); }
__device__ __forceinline__ V3 operator/(V3 a, float s) { return v3(a.x / s, a.y / s, a.z / s); }
__device__ __forceinline__ float dot(V3 a, V3 b) { return a.x * b.x + (a.y * b.y + a.z * b.z); }
__device__ __forceinline__ V3 cross(V3 a, V3 b) {
    return v3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
__device__ __forceinline__ float norm(V3 a) { return sqrtf(dot(a, a)); }
// MatrixBase::normalized(): a / sqrt(squaredNorm) when squaredNorm > 0
__device__ __forceinline__ V3 normalize(V3 a) {
    float z = dot(a, a);
    return z > 0.0f ? a / sqrtf(z) : a;
}
__device__ __forceinline__ V3 xyz(float4 f) { return v3(f.x, f.y, f.z); }
__device__ __forceinline__ V3 ld3(const float *p) { return v3(p[0], p[1], p[2]); }
// DenseBase::isZero() with Eigen's float dummy_precision: every |c| <= 1e-5
__device__ __forceinline__ bool is_zero(V3 a) {
    return fabsf(a.x) <= 1e-5f && fabsf(a.y) <= 1e-5f && fabsf(a.z) <= 1e-5f;
}
__device__ __forceinline__ bool all_zero(V3 a) { return a.x == 0.0f && a.y == 0.0f && a.z == 0.0f; }
// Color3f::IsValid (src/core/Color.cpp:44)
__device__ __forceinline__ bool is_valid(V3 a) {
    return !(a.x < 0.0f || !isfinite(a.x) || a.y < 0.0f || !isfinite(a.y) || a.z < 0.0f || !isfinite(a.z));
}
// Color3f::GetLuminance (src/core/Color.cpp:95)
__device__ __forceinline__ float luminance(V3 c) { return c.x * 0.212671f + c.y * 0.715160f + c.z * 0.072169f; }
__device__ __forceinline__ float clampf(float v, float lo, float hi) { return v < lo ? lo : (v > hi ? hi : v); }
__device__ __forceinline__ int clampi(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }
__device__ __forceinline__ float signum(float v) { return copysignf(1.0f, v); }
// Hypot2 (include/core/Common.hpp:829)
__device__ __forceinline__ float hypot2(float a, float b) {
    float r;
    if (fabsf(a) > fabsf(b)) { r = b / a; r = fabsf(a) * sqrtf(1.0f + r * r); }
    else if (b != 0.0f) { r = a / b; r = fabsf(b) * sqrtf(1.0f + r * r); }
    else r = 0.0f;
    return r;
}

// ---------------------------------------------------------------- pcg32
// PCG-XSH-RR 64/32 (O'Neill 2014), the generator of ext/pcg32/pcg32.h.
struct Pcg32 {
    uint64_t state, inc;
    __device__ __forceinline__ uint32_t next() {
        uint64_t old = state;
        state = old * 0x5851f42d4c957f2dULL + inc;
        uint32_t xs = (uint32_t)(((old >> 18u) ^ old) >> 27u);
        uint32_t rot = (uint32_t)(old >> 59u);
        return __funnelshift_r(xs, xs, rot);
    }
    __device__ __forceinline__ void seed(uint64_t initstate, uint64_t initseq) {
        state = 0u;
        inc = (initseq << 1u) | 1u;
        next();
        state += initstate;
        next();
    }
    // nextFloat: 23 random mantissa bits in [1,2) minus 1
    __device__ __forceinline__ float nextf() { return __uint_as_float((next() >> 9) | 0x3f800000u) - 1.0f; }
};

// ---------------------------------------------------------------- frames
struct Frame { V3 s, t, n; };
// CoordinateSystem (src/core/Common.cpp:591) / Frame(N) (src/core/Frame.cpp:18)
__device__ __forceinline__ Frame frame_from_n(V3 n) {
    Frame f;
    f.n = n;
    if (fabsf(n.x) > fabsf(n.y)) {
        float inv = 1.0f / sqrtf(n.x * n.x + n.z * n.z);
        f.t = v3(n.z * inv, 0.0f, -n.x * inv);
    } else {
        float inv = 1.0f / sqrtf(n.y * n.y + n.z * n.z);
        f.t = v3(0.0f, n.z * inv, -n.y * inv);
    }
    f.s = cross(f.t, f.n);
    return f;
}
__device__ __forceinline__ V3 to_local(const Frame &f, V3 v) { return v3(dot(v, f.s), dot(v, f.t), dot(v, f.n)); }
__device__ __forceinline__ V3 to_world(const Frame &f, V3 v) { return (f.s * v.x + f.t * v.y) + f.n * v.z; }
__device__ __forceinline__ float tan_theta(V3 v) {
    float t = 1.0f - v.z * v.z;
    if (t <= 0.0f) return 0.0f;
    return sqrtf(t) / v.z;
}
__device__ __forceinline__ float sin_theta2(V3 v) { return 1.0f - v.z * v.z; }

// ---------------------------------------------------------------- warps
// Concentric square->disk map (Sampling::SquareToUniformDisk, src/core/Sampling.cpp:29)
__device__ __forceinline__ void square_to_disk(float ux, float uy, float &dx, float &dy) {
    float ox = 2.0f * ux - 1.0f, oy = 2.0f * uy - 1.0f;
    if (ox == 0.0f && oy == 0.0f) { dx = 0.0f; dy = 0.0f; return; }
    float th, r;
    if (fabsf(ox) > fabsf(oy)) { r = ox; th = kPi * 0.25f * (oy / ox); }
    else { r = oy; th = kPi * 0.5f - kPi * 0.25f * (ox / oy); }
    dx = r * cosf(th);
    dy = r * sinf(th);
}
// Sampling::SquareToCosineHemisphere (src/core/Sampling.cpp:97)
__device__ __forceinline__ V3 square_to_cos_hemi(float ux, float uy) {
    float dx, dy;
    square_to_disk(ux, uy, dx, dy);
    float z = sqrtf(1.0f - dx * dx - dy * dy);
    if (isnan(z)) z = 0.0f;
    return v3(dx, dy, z);
}
// Sampling::SquareToCosineHemispherePdf (src/core/Sampling.cpp:110)
__device__ __forceinline__ float cos_hemi_pdf(V3 v) {
    return (norm(v) - 1.0f <= 1e-6f && v.z >= 0.0f) ? v.z / kPi : 0.0f;
}

}  // namespace hk
