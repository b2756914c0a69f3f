/*
 * hk_oracle.c -- CPU restatement of Hikari's pathMIS hot path (checker only).
 *
 * TEST INFRASTRUCTURE: loaded by tests/, __graft_entry__.smoke() and the
 * cpu_baseline leg of bench.py, never by the product.  Citations are
 * reference-project paths (file:line).  Arithmetic is float in the
 * reference's evaluation order; film accumulation is double.
 *
 * Build: oracle/build.py (gcc -O2 -fopenmp -ffp-contract=off).
 */
#define _GNU_SOURCE
#include "hk_oracle.h"

#include <float.h>
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define PI_F 3.14159265358979323846f
#define INV_PI_D 0.31830988618379067154
#define EPS_RAY 1e-4f

static __thread char g_err[512];
const char *ho_last_error(void) { return g_err; }
static int fail(const char *m) { snprintf(g_err, sizeof g_err, "%s", m); return -1; }

/* ------------------------------------------------------------------ vec */
typedef struct { float x, y, z; } v3;
static inline v3 V(float x, float y, float z) { v3 r = {x, y, z}; return r; }
static inline v3 add(v3 a, v3 b) { return V(a.x + b.x, a.y + b.y, a.z + b.z); }
static inline v3 sub(v3 a, v3 b) { return V(a.x - b.x, a.y - b.y, a.z - b.z); }
static inline v3 mul(v3 a, v3 b) { return V(a.x * b.x, a.y * b.y, a.z * b.z); }
static inline v3 scl(v3 a, float s) { return V(a.x * s, a.y * s, a.z * s); }
static inline v3 divs(v3 a, float s) { return V(a.x / s, a.y / s, a.z / s); }
/* Eigen 3.3 fixed-size dot/squaredNorm reduce as a binary tree: x + (y + z)
 * (redux_novec_unroller, ext/eigen/Eigen/src/Core/Redux.h:91) */
static inline float dot(v3 a, v3 b) { return a.x * b.x + (a.y * b.y + a.z * b.z); }
static inline v3 cross(v3 a, v3 b) {
    return V(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
static inline float norm(v3 a) { return sqrtf(dot(a, a)); }
/* Eigen MatrixBase::normalized(): divide by sqrt(squaredNorm) if > 0 */
static inline v3 normalize(v3 a) {
    float z = dot(a, a);
    return z > 0.0f ? divs(a, sqrtf(z)) : a;
}
static inline v3 vload(const float *p) { return V(p[0], p[1], p[2]); }
static inline void vstore(float *p, v3 a) { p[0] = a.x; p[1] = a.y; p[2] = a.z; }
/* Eigen DenseBase::isZero(): every |c| <= 1e-5f (dummy_precision<float>) */
static inline int is_zero(v3 a) {
    return fabsf(a.x) <= 1e-5f && fabsf(a.y) <= 1e-5f && fabsf(a.z) <= 1e-5f;
}
/* Color3f::IsValid  src/core/Color.cpp:44 */
static inline int is_valid(v3 a) {
    return !(a.x < 0.0f || !isfinite(a.x) || a.y < 0.0f || !isfinite(a.y) || a.z < 0.0f ||
             !isfinite(a.z));
}
/* Color3f::GetLuminance  src/core/Color.cpp:95 */
static inline float lum(v3 c) { return c.x * 0.212671f + c.y * 0.715160f + c.z * 0.072169f; }
static inline float clampf(float v, float lo, float hi) { return v < lo ? lo : (v > hi ? hi : v); }
static inline int clampi(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }
/* Signum  include/core/Common.hpp:901 */
static inline float signum(float v) { return copysignf(1.0f, v); }
/* Hypot2  include/core/Common.hpp:829 */
static float hypot2(float a, float b) {
    float r;
    if (fabsf(a) > fabsf(b)) { r = b / a; r = fabsf(a) * sqrtf(1.0f + r * r); }
    else if (b != 0.0f) { r = a / b; r = fabsf(b) * sqrtf(1.0f + r * r); }
    else r = 0.0f;
    return r;
}

/* ------------------------------------------------------------------ pcg32 */
/* O'Neill's PCG-XSH-RR 64/32 as packaged in ext/pcg32/pcg32.h:29-110 */
#define PCG_MULT 0x5851f42d4c957f2dULL
uint32_t ho_pcg32_next(ho_pcg32 *r) {
    uint64_t old = r->state;
    r->state = old * PCG_MULT + r->inc;
    uint32_t xs = (uint32_t)(((old >> 18u) ^ old) >> 27u);
    uint32_t rot = (uint32_t)(old >> 59u);
    return (xs >> rot) | (xs << ((~rot + 1u) & 31));
}
void ho_pcg32_seed(ho_pcg32 *r, uint64_t initstate, uint64_t initseq) {
    r->state = 0u;
    r->inc = (initseq << 1u) | 1u;
    ho_pcg32_next(r);
    r->state += initstate;
    ho_pcg32_next(r);
}
float ho_pcg32_nextf(ho_pcg32 *r) {
    union { uint32_t u; float f; } x;
    x.u = (ho_pcg32_next(r) >> 9) | 0x3f800000u;
    return x.f - 1.0f;
}
static void pcg_default(ho_pcg32 *r) { r->state = 0x853c49e6748fea9bULL; r->inc = 0xda3e39cb94b95bdbULL; }

/* ------------------------------------------------------------------ frame */
typedef struct { v3 s, t, n; } frame;
/* CoordinateSystem  src/core/Common.cpp:591 ; Frame(N)  src/core/Frame.cpp:18 */
static frame frame_from_n(v3 n) {
    frame f; f.n = n;
    if (fabsf(n.x) > fabsf(n.y)) {
        float inv = 1.0f / sqrtf(n.x * n.x + n.z * n.z);
        f.t = V(n.z * inv, 0.0f, -n.x * inv);
    } else {
        float inv = 1.0f / sqrtf(n.y * n.y + n.z * n.z);
        f.t = V(0.0f, n.z * inv, -n.y * inv);
    }
    f.s = cross(f.t, f.n);
    return f;
}
static inline v3 to_local(const frame *f, v3 v) { return V(dot(v, f->s), dot(v, f->t), dot(v, f->n)); }
static inline v3 to_world(const frame *f, v3 v) {
    return add(add(scl(f->s, v.x), scl(f->t, v.y)), scl(f->n, v.z));
}
/* Frame::TanTheta / SinTheta2  src/core/Frame.cpp:47,57 */
static inline float tan_theta(v3 v) {
    float t = 1.0f - v.z * v.z;
    if (t <= 0.0f) return 0.0f;
    return sqrtf(t) / v.z;
}
static inline float sin_theta2(v3 v) { return 1.0f - v.z * v.z; }

/* --------------------------------------------------------------- sampling */
/* Sampling::SquareToUniformDisk  src/core/Sampling.cpp:29 (concentric map) */
static void square_to_disk(float ux, float uy, float *dx, float *dy) {
    float ox = 2.0f * ux - 1.0f, oy = 2.0f * uy - 1.0f;
    if (ox == 0.0f && oy == 0.0f) { *dx = 0.0f; *dy = 0.0f; return; }
    float th, r;
    if (fabsf(ox) > fabsf(oy)) { r = ox; th = PI_F * 0.25f * (oy / ox); }
    else { r = oy; th = PI_F * 0.5f - PI_F * 0.25f * (ox / oy); }
    *dx = r * cosf(th);
    *dy = r * sinf(th);
}
/* Sampling::SquareToCosineHemisphere  src/core/Sampling.cpp:97 */
static v3 square_to_cos_hemi(float ux, float uy) {
    float dx, dy;
    square_to_disk(ux, uy, &dx, &dy);
    float z = sqrtf(1.0f - dx * dx - dy * dy);
    if (isnan(z)) z = 0.0f;
    return V(dx, dy, z);
}
/* Sampling::SquareToCosineHemispherePdf  src/core/Sampling.cpp:110 */
static float cos_hemi_pdf(v3 v) {
    return (norm(v) - 1.0f <= 1e-6f && v.z >= 0.0f) ? v.z / PI_F : 0.0f;
}

/* ----------------------------------------------------------- microfacet */
/* src/core/MicrofacetDistribution.cpp */
typedef struct { int type; float au, av; } mfd;
static mfd mfd_make(int type, float au, float av) {   /* :10-26 */
    mfd d; d.type = type;
    d.au = clampf(au, 5e-4f, 1.0f);
    d.av = clampf(av, 5e-4f, 1.0f);
    return d;
}
static inline int mfd_iso(const mfd *d) { return d->au == d->av; }
static float mfd_eval(const mfd *d, v3 m) {   /* :34 */
    if (m.z <= 0.0f) return 0.0f;
    float c2 = m.z * m.z;
    float be = ((m.x * m.x) / (d->au * d->au) + (m.y * m.y) / (d->av * d->av)) / c2;
    float r;
    if (d->type == HO_BECKMANN) {
        r = expf(-be) / (PI_F * d->au * d->av * c2 * c2);
    } else {
        float root = (1.0f + be) * c2;
        r = 1.0f / (PI_F * d->au * d->av * root * root);
    }
    if (r * m.z < 1e-20f) r = 0.0f;
    return r;
}
static float mfd_project_roughness(const mfd *d, v3 v) {   /* :238 */
    float inv = 1.0f / sin_theta2(v);
    if (mfd_iso(d) || inv <= 0.0f) return d->au;
    float c2 = v.x * v.x * inv, s2 = v.y * v.y * inv;
    return sqrtf(c2 * d->au * d->au + s2 * d->av * d->av);
}
static float mfd_g1(const mfd *d, v3 v, v3 m) {   /* :82 */
    if (dot(v, m) * v.z <= 0.0f) return 0.0f;
    float tt = fabsf(tan_theta(v));
    if (tt == 0.0f) return 1.0f;
    float a = mfd_project_roughness(d, v);
    if (d->type == HO_BECKMANN) {
        float x = 1.0f / (a * tt);
        if (x >= 1.6f) return 1.0f;
        float x2 = x * x;
        return (3.535f * x + 2.181f * x2) / (1.0f + 2.276f * x + 2.577f * x2);
    }
    float root = a * tt;
    return 2.0f / (1.0f + hypot2(1.0f, root));
}
static inline float mfd_g(const mfd *d, v3 wi, v3 wo, v3 m) { return mfd_g1(d, wi, m) * mfd_g1(d, wo, m); }
static v3 mfd_sample(const mfd *d, float ux, float uy, float *pdf) {   /* SampleAll :148 */
    float cm = 0.0f, sp, cp, a2;
    if (mfd_iso(d)) {
        float ph = (2.0f * PI_F) * uy;
        sp = sinf(ph); cp = cosf(ph);
        a2 = d->au * d->au;
    } else {
        float ph = atanf(d->av / d->au * tanf(PI_F + 2.0f * PI_F * uy)) + PI_F * floorf(2.0f * uy + 0.5f);
        sp = sinf(ph); cp = cosf(ph);
        float cs = cp / d->au, ss = sp / d->av;
        a2 = 1.0f / (cs * cs + ss * ss);
    }
    if (d->type == HO_BECKMANN) {
        float t2 = a2 * -logf(1.0f - ux);
        cm = 1.0f / sqrtf(1.0f + t2);
        *pdf = (1.0f - ux) / (PI_F * d->au * d->av * cm * cm * cm);
    } else {
        float t2 = a2 * ux / (1.0f - ux);
        cm = 1.0f / sqrtf(1.0f + t2);
        float tmp = 1.0f + t2 / a2;
        *pdf = (float)INV_PI_D / (d->au * d->av * cm * cm * cm * tmp * tmp);
    }
    if (*pdf < 1e-20f) *pdf = 0.0f;
    float sm = sqrtf(fmaxf(0.0f, 1.0f - cm * cm));
    return V(sm * cp, sm * sp, cm);
}
static inline float mfd_pdf(const mfd *d, v3 m) { return mfd_eval(d, m) * m.z; }   /* PdfAll :231 */

/* ---------------------------------------------------------------- fresnel */
/* FresnelDielectric  src/core/Common.cpp:494 */
static float fresnel_dielectric(float ci, float eta, float inv_eta, float *ct) {
    if (eta == 1.0f) { *ct = -ci; return 0.0f; }
    float sc = (ci > 0.0f) ? inv_eta : eta;
    float ct2 = 1.0f - (1.0f - ci * ci) * (sc * sc);
    if (ct2 <= 0.0f) { *ct = 0.0f; return 1.0f; }
    float cii = fabsf(ci), ctt = sqrtf(ct2);
    float rs = (cii - eta * ctt) / (cii + eta * ctt);
    float rp = (eta * cii - ctt) / (eta * cii + ctt);
    *ct = (ci > 0.0f) ? -ctt : ctt;
    return 0.5f * (rs * rs + rp * rp);
}
/* FresnelConductor  src/core/Common.cpp:529 (per channel) */
static float fresnel_conductor1(float ci, float eta, float k) {
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
static v3 fresnel_conductor(float ci, const float *eta, const float *k) {
    return V(fresnel_conductor1(ci, eta[0], k[0]), fresnel_conductor1(ci, eta[1], k[1]),
             fresnel_conductor1(ci, eta[2], k[2]));
}
/* Reflect / Refract in global coordinates  src/core/Common.cpp:616-626 */
static inline v3 reflect_m(v3 wi, v3 m) { return sub(scl(m, 2.0f * dot(wi, m)), wi); }
static inline v3 refract_m(v3 wi, v3 m, float ct, float eta, float inv_eta) {
    float e = (ct < 0.0f ? inv_eta : eta);
    return sub(scl(m, dot(wi, m) * e + ct), scl(wi, e));
}

/* ------------------------------------------------------- cubic / RFT */
/* EvalCubicInterpolate1D  src/core/Common.cpp:230 */
static float cubic1d(float x, const float *val, int size, float mn, float mx) {
    if (!(x >= mn && x <= mx)) return 0.0f;
    float t = ((x - mn) * (size - 1)) / (mx - mn);
    int k = (int)t; if (k > size - 2) k = size - 2; if (k < 0) k = 0;
    float f0 = val[k], f1 = val[k + 1], d0, d1;
    d0 = (k > 0) ? 0.5f * (val[k + 1] - val[k - 1]) : val[k + 1] - val[k];
    d1 = (k + 2 < size) ? 0.5f * (val[k + 2] - val[k]) : val[k + 1] - val[k];
    t = t - (float)k;
    float t2 = t * t, t3 = t2 * t;
    return (2.0f * t3 - 3.0f * t2 + 1) * f0 + (-2.0f * t3 + 3.0f * t2) * f1 + (t3 - 2.0f * t2 + t) * d0 +
           (t3 - t2) * d1;
}
/* knot weights shared by EvalCubicInterpolate2D/3D  src/core/Common.cpp:299-336 */
static int cubic_weights(float p, int size, float *w, int *knot) {
    if (!(p >= 0.0f && p <= 1.0f)) return 0;
    float t = ((p - 0.0f) * (float)(size - 1)) / (1.0f - 0.0f);
    int k = (int)t; if (k > size - 2) k = size - 2;
    *knot = k;
    t = t - (float)k;
    float t2 = t * t, t3 = t2 * t;
    w[0] = 0.0f; w[1] = 2.0f * t3 - 3.0f * t2 + 1; w[2] = -2.0f * t3 + 3.0f * t2; w[3] = 0.0f;
    float d0 = t3 - 2.0f * t2 + t, d1 = t3 - t2;
    if (k > 0) { w[2] += 0.5f * d0; w[0] -= 0.5f * d0; }
    else { w[2] += d0; w[1] -= d0; }
    if (k + 2 < size) { w[3] += 0.5f * d1; w[1] -= 0.5f * d1; }
    else { w[2] += d1; w[1] -= d1; }
    return 1;
}
/* EvalCubicInterpolate2D on [0,1]^2  src/core/Common.cpp:285 */
static float cubic2d(float px, float py, const float *val, int sx, int sy) {
    float w[2][4]; int kn[2];
    if (!cubic_weights(px, sx, w[0], &kn[0])) return 0.0f;
    if (!cubic_weights(py, sy, w[1], &kn[1])) return 0.0f;
    float r = 0.0f;
    for (int y = -1; y <= 2; y++) {
        float wy = w[1][y + 1];
        for (int x = -1; x <= 2; x++) {
            float wxy = w[0][x + 1] * wy;
            if (wxy == 0) continue;
            r += val[(kn[1] + y) * sx + kn[0] + x] * wxy;
        }
    }
    return r;
}
/* EvalCubicInterpolate3D on [0,1]^3  src/core/Common.cpp:373 */
static float cubic3d(float px, float py, float pz, const float *val, int sx, int sy, int sz) {
    float w[3][4]; int kn[3];
    if (!cubic_weights(px, sx, w[0], &kn[0])) return 0.0f;
    if (!cubic_weights(py, sy, w[1], &kn[1])) return 0.0f;
    if (!cubic_weights(pz, sz, w[2], &kn[2])) return 0.0f;
    float r = 0.0f;
    for (int z = -1; z <= 2; z++) {
        float wz = w[2][z + 1];
        for (int y = -1; y <= 2; y++) {
            float wyz = w[1][y + 1] * wz;
            for (int x = -1; x <= 2; x++) {
                float wxyz = w[0][x + 1] * wyz;
                if (wxyz == 0) continue;
                r += val[((kn[2] + z) * sy + (kn[1] + y)) * sx + kn[0] + x] * wxyz;
            }
        }
    }
    return r;
}

typedef struct {
    uint64_t eta_n, alpha_n, theta_n, t_size, d_size;
    float eta_min, eta_max, alpha_min, alpha_max;
    const float *trans;   /* eta_n*alpha_n*theta_n*2 */
    const float *diff;    /* eta_n*alpha_n*2 */
    float *owned;
} rft_table;

/* RoughTransmittance ctor  src/core/RoughTransmitance.cpp:9 (file layout) */
static int rft_parse(rft_table *t, const void *bytes, uint64_t n) {
    const unsigned char *b = (const unsigned char *)bytes;
    if (n < 56) return fail("rft: short header");
    uint64_t h[5]; float f[4];
    memcpy(h, b, 40); memcpy(f, b + 40, 16);
    t->eta_n = h[0]; t->alpha_n = h[1]; t->theta_n = h[2]; t->t_size = h[3]; t->d_size = h[4];
    t->eta_min = f[0]; t->eta_max = f[1]; t->alpha_min = f[2]; t->alpha_max = f[3];
    if (56 + 4 * (t->t_size + t->d_size) > n) return fail("rft: short body");
    t->owned = (float *)malloc(4 * (t->t_size + t->d_size));
    memcpy(t->owned, b + 56, 4 * (t->t_size + t->d_size));
    t->trans = t->owned; t->diff = t->owned + t->t_size;
    return 0;
}
/* SetEta  src/core/RoughTransmitance.cpp:170 -> 2D [alpha][theta] + diffuse[alpha] */
static void rft_set_eta(const rft_table *t, float eta, float *t2d, float *d1d) {
    const float *pt = t->trans, *pd = t->diff;
    int E = (int)t->eta_n, A = (int)t->alpha_n, T = (int)t->theta_n;
    if (eta < 1.0f) { pt += (uint64_t)E * A * T; pd += (uint64_t)E * A; eta = 1.0f / eta; }
    if (eta < t->eta_min) eta = t->eta_min;
    float we = powf((eta - t->eta_min) / (t->eta_max - t->eta_min), 0.25f);
    float da = 1.0f / (A - 1.0f), dt = 1.0f / (T - 1.0f);
    for (int i = 0; i < A; i++) {
        for (int j = 0; j < T; j++)
            t2d[i * T + j] = cubic3d(j * dt, i * da, we, pt, T, A, E);
        d1d[i] = cubic2d(i * da, we, pd, A, E);
    }
}
/* SetAlpha  src/core/RoughTransmitance.cpp:237 -> 1D [theta] + diffuse scalar */
static void rft_set_alpha(const rft_table *t, const float *t2d, const float *d1d, float alpha,
                          float *t1d, float *dscalar) {
    int A = (int)t->alpha_n, T = (int)t->theta_n;
    float wa = powf((alpha - t->alpha_min) / (t->alpha_max - t->alpha_min), 0.25f);
    float dt = 1.0f / (T - 1.0f);
    for (int i = 0; i < T; i++) t1d[i] = cubic2d(i * dt, wa, t2d, T, A);
    *dscalar = cubic1d(wa, d1d, A, 0.0f, 1.0f);
}
/* Eval with eta and alpha fixed  src/core/RoughTransmitance.cpp:48-70 */
static float rft_eval1d(const float *t1d, int T, float c) {
    float wc = powf(fabsf(c), 0.25f);
    if (c < 0.0f) return 0.0f;
    return clampf(cubic1d(wc, t1d, T, 0.0f, 1.0f), 0.0f, 1.0f);
}
/* Eval with eta fixed, alpha per query (:71-87): the 2D cubic over warped cos, alpha */
static float rft_eval2d(const float *t2d, int T, int A, float amin, float amax, float c, float alpha) {
    float wc = powf(fabsf(c), 0.25f);
    if (c < 0.0f) return 0.0f;
    float wa = powf((alpha - amin) / (amax - amin), 0.25f);
    return clampf(cubic2d(wc, wa, t2d, T, A), 0.0f, 1.0f);
}

/* ------------------------------------------------------------------ BSDF */
#define RFT_MAX_THETA 128
typedef struct {
    ho_bsdf_desc d;
    float eta, inv_eta, inv_eta2;      /* dielectric-type relative IOR */
    float eta_c[3], k_c[3];            /* conductor eta and k/extIOR */
    float spec_w;                      /* m_SpecularSamplingWeight */
    float rft[RFT_MAX_THETA];          /* activated 1D transmittance table */
    int rft_n;
    float fdr_int;                     /* plastic: 1 - IntData.EvalDiffuse(alpha) */
    /* a textured alpha of roughPlastic / roughCoating: the transmittance left
     * 2D after SetEta ([alpha][theta]) and the plastic's diffuse one over alpha */
    int alpha_tex, rft_an;
    float rft_amin, rft_amax;
    float *rft2d, *rft_diff;
    const ho_texture_desc *textures;   /* the scene's textures (set when finalized) */
    struct mip_t *const *mips;         /* their MIP pyramids (bitmaps; NULL otherwise) */
} bsdf_t;

/* uv: Record.Isect.UV; duv: its screen-space partials (dUdX, dVdX, dUdY, dVdY);
 * it: the record's intersection (frames and dP/du, dP/dv for bumpMap /
 * normalMap), NULL in queries without one */
/* dpdu / dpdv with has_uvp: Isect.dPdU / dPdV and bHasUVPartial (set with normals and texture coordinates) */
/* edge_d, curv_h, curv_k: what the wireframe and curvature textures read (the
 * distance from p to the nearest edge line of the hit triangle, the mean and
 * Gaussian curvature from the UV partials), set only for meshes whose BSDF
 * uses one of them */
typedef struct isect_s {
    v3 p; frame sh, geo; int mesh; float t; float uv[2]; v3 dpdu, dpdv; int has_uvp;
    v3 dndu, dndv; float edge_d, curv_h, curv_k;
} isect_t;
typedef struct { v3 wi, wo; float eta; int measure; float uv[2]; float duv[4]; const isect_t *it; } brec;

/* ------------------------------------------------------------ bitmap textures */
/* LoadImageFromFileR / LoadImageFromFileRGB (src/core/Texture.cpp:12, :74):
 * 8-bit pixels -> gamma-corrected floats, rows flipped (row 0 = v 0 = the
 * image's bottom row), average over x-major order.  MipMap<T> (include/core/
 * MipMap.hpp:67): Lanczos resampling to power-of-two sizes, then a 2x2 box
 * pyramid; lookups Lookup(UV) :281 (nearest), Lookup(UV, width) :287
 * (bilinear / trilinear), Lookup(UV, D0, D1) :309 (trilinear or EWA). */
#define HO_MIP_MAX 32
typedef struct mip_t {
    int ch, levels, black, trilinear;
    float max_aniso;
    int w[HO_MIP_MAX], h[HO_MIP_MAX];
    float *lv[HO_MIP_MAX];     /* 3 floats per texel (one channel: all three equal) */
    float avg[3];
} mip_t;

static float ewa_lut[128];    /* MipMap::s_WeightLut: exp(-2 r^2) - exp(-2) at r^2 = i / 127 */
static void ewa_lut_init(void) {
    if (ewa_lut[0] != 0.0f) return;
    for (int i = 0; i < 128; i++) {
        float alpha = 2.0f, r2 = (float)i / (float)(128 - 1);
        ewa_lut[i] = expf(-alpha * r2) - expf(-alpha);
    }
}
static void mip_free(mip_t *m) {
    if (!m) return;
    for (int i = 0; i < m->levels; i++) free(m->lv[i]);
    free(m);
}
static int is_pow2(int v) { return v && !(v & (v - 1)); }
static int round_up_pow2(int v) {
    v--; v |= v >> 1; v |= v >> 2; v |= v >> 4; v |= v >> 8; v |= v >> 16;
    return v + 1;
}
static int log2_int(uint32_t v) { int r = 0; while (v >>= 1) r++; return r; }
static int mod_int(int a, int b) { int r = a % b; return r < 0 ? r + b : r; }
static int clamp_int(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }
/* Lanczos (src/core/MipMap.cpp:5), as written there: sin(x tau)/(x tau) * sin(x)/x */
static float lanczos(float x, float tau) {
    x = fabsf(x);
    float sa = sinf(x * tau) / (x * tau);
    float lz = sinf(x) / x;
    return sa * lz;
}
typedef struct { int first; float w[4]; } rs_weight;
/* MipMap::GetResampleWeights :386 */
static rs_weight *resample_weights(int old_n, int new_n) {
    rs_weight *W = malloc(sizeof *W * (size_t)new_n);
    const float fw = 2.0f;
    for (int i = 0; i < new_n; i++) {
        float center = ((float)i + 0.5f) * (float)old_n / (float)new_n;
        W[i].first = (int)floorf((center - fw) + 0.5f);
        for (int j = 0; j < 4; j++) {
            float pos = (float)(W[i].first + j) + 0.5f;
            W[i].w[j] = lanczos((pos - center) / fw, 2.0f);
        }
        float inv = 1.0f / (((W[i].w[0] + W[i].w[1]) + W[i].w[2]) + W[i].w[3]);
        for (int j = 0; j < 4; j++) W[i].w[j] *= inv;
    }
    return W;
}
static int wrap_index(int x, int n, int wrap) {
    if (wrap == HO_WRAP_REPEAT) return mod_int(x, n);
    if (wrap == HO_WRAP_CLAMP) return clamp_int(x, 0, n - 1);
    return x;
}
/* MipMap::Texel :244 -- any coordinate outside the level, and every texel
 * when a wrap mode is "black", reads black (the wrap switch that follows is
 * reached only for coordinates already inside). */
static inline v3 mip_texel(const mip_t *m, int l, int x, int y) {
    if (m->black || x < 0 || x >= m->w[l] || y < 0 || y >= m->h[l]) return V(0, 0, 0);
    return vload(m->lv[l] + 3 * ((size_t)y * m->w[l] + x));
}
static float clamp_max(float v) { return v < 0.0f ? 0.0f : (v > FLT_MAX ? FLT_MAX : v); }
/* texels: w * h * 3 floats (gamma-corrected, flipped); ch 1 stores x in all three. */
static mip_t *mip_build(const float *texels, int w, int h, int ch, int wrap_u, int wrap_v, int trilinear,
                        float max_aniso) {
    ewa_lut_init();
    mip_t *m = calloc(1, sizeof *m);
    m->ch = ch; m->trilinear = trilinear; m->max_aniso = max_aniso;
    m->black = wrap_u == HO_WRAP_BLACK || wrap_v == HO_WRAP_BLACK;
    int W = w, H = h;
    float *l0;
    if (!is_pow2(w) || !is_pow2(h)) {
        W = round_up_pow2(w); H = round_up_pow2(h);
        rs_weight *uw = resample_weights(w, W);
        l0 = malloc(sizeof(float) * 3 * (size_t)W * H);
        for (int v = 0; v < h; v++)
            for (int u = 0; u < W; u++) {
                float acc[3] = {0, 0, 0};
                for (int j = 0; j < 4; j++) {
                    int ou = wrap_index(uw[u].first + j, w, wrap_u);
                    if (ou >= 0 && ou < w)
                        for (int c = 0; c < 3; c++) acc[c] += uw[u].w[j] * texels[3 * ((size_t)v * w + ou) + c];
                }
                for (int c = 0; c < 3; c++) l0[3 * ((size_t)v * W + u) + c] = acc[c];
            }
        free(uw);
        rs_weight *vw = resample_weights(h, H);
        float *col = malloc(sizeof(float) * 3 * (size_t)H);
        for (int u = 0; u < W; u++) {
            for (int v = 0; v < H; v++) {
                float acc[3] = {0, 0, 0};
                for (int j = 0; j < 4; j++) {
                    int ov = wrap_index(vw[v].first + j, h, wrap_v);
                    if (ov >= 0 && ov < h)
                        for (int c = 0; c < 3; c++) acc[c] += vw[v].w[j] * l0[3 * ((size_t)ov * W + u) + c];
                }
                for (int c = 0; c < 3; c++) col[3 * v + c] = acc[c];
            }
            for (int v = 0; v < H; v++)
                for (int c = 0; c < 3; c++) l0[3 * ((size_t)v * W + u) + c] = clamp_max(col[3 * v + c]);
        }
        free(col); free(vw);
    } else {
        l0 = malloc(sizeof(float) * 3 * (size_t)W * H);
        memcpy(l0, texels, sizeof(float) * 3 * (size_t)W * H);
    }
    m->levels = 1 + log2_int((uint32_t)(W > H ? W : H));
    m->w[0] = W; m->h[0] = H; m->lv[0] = l0;
    for (int i = 1; i < m->levels; i++) {
        int ur = m->w[i - 1] / 2 > 1 ? m->w[i - 1] / 2 : 1, vr = m->h[i - 1] / 2 > 1 ? m->h[i - 1] / 2 : 1;
        m->w[i] = ur; m->h[i] = vr;
        m->lv[i] = malloc(sizeof(float) * 3 * (size_t)ur * vr);
        for (int v = 0; v < vr; v++)
            for (int u = 0; u < ur; u++) {
                v3 a = mip_texel(m, i - 1, 2 * u, 2 * v), b = mip_texel(m, i - 1, 2 * u + 1, 2 * v);
                v3 c = mip_texel(m, i - 1, 2 * u, 2 * v + 1), d = mip_texel(m, i - 1, 2 * u + 1, 2 * v + 1);
                vstore(m->lv[i] + 3 * ((size_t)v * ur + u), scl(add(add(add(a, b), c), d), 0.25f));
            }
    }
    return m;
}
/* MipMap::Triangle :412 (bilinear at one level) */
static v3 mip_triangle(const mip_t *m, int l, float u, float v) {
    l = clamp_int(l, 0, m->levels - 1);
    float U = u * (float)m->w[l] - 0.5f, Vv = v * (float)m->h[l] - 0.5f;
    int u0 = (int)floorf(U), v0 = (int)floorf(Vv);
    float du = U - (float)u0, dv = Vv - (float)v0;
    v3 t00 = mip_texel(m, l, u0, v0), t01 = mip_texel(m, l, u0, v0 + 1);
    v3 t10 = mip_texel(m, l, u0 + 1, v0), t11 = mip_texel(m, l, u0 + 1, v0 + 1);
    float a = (1.0f - du) * (1.0f - dv), b = (1.0f - du) * dv, c = du * (1.0f - dv), d = du * dv;
    return add(add(add(scl(t00, a), scl(t01, b)), scl(t10, c)), scl(t11, d));
}
static v3 lerp3(float t, v3 a, v3 b) { return add(scl(a, 1.0f - t), scl(b, t)); }
/* MipMap::EvalGradient :363 (bilinear slope at one level, unscaled UV) */
static void mip_gradient(const mip_t *m, int l, float u, float v, v3 *g) {
    float U = u * (float)m->w[l] - 0.5f, Vv = v * (float)m->h[l] - 0.5f;
    int x = (int)floorf(U), y = (int)floorf(Vv);
    float dx = U - (float)x, dy = Vv - (float)y;
    v3 p00 = mip_texel(m, l, x, y), p10 = mip_texel(m, l, x + 1, y);
    v3 p01 = mip_texel(m, l, x, y + 1), p11 = mip_texel(m, l, x + 1, y + 1);
    v3 tmp = sub(add(p01, p10), p11);
    g[0] = scl(sub(add(p10, scl(p00, dy - 1.0f)), scl(tmp, dy)), (float)m->w[l]);
    g[1] = scl(sub(add(p01, scl(p00, dx - 1.0f)), scl(tmp, dx)), (float)m->h[l]);
}
/* MipMap::Lookup(UV, Width) :287 */
static v3 mip_lookup_width(const mip_t *m, float u, float v, float width) {
    float level = (float)m->levels - 1.0f + log2f(fmaxf(width, 1e-8f));
    if (level < 0.0f) return mip_triangle(m, 0, u, v);
    if (level >= (float)(m->levels - 1)) return mip_texel(m, m->levels - 1, 0, 0);
    int il = (int)floorf(level);
    float delta = level - (float)il;
    return lerp3(delta, mip_triangle(m, il, u, v), mip_triangle(m, il + 1, u, v));
}
/* MipMap::EWA :427 */
static v3 mip_ewa(const mip_t *m, int l, float u, float v, float d0x, float d0y, float d1x, float d1y) {
    if (l >= m->levels) return mip_texel(m, m->levels - 1, 0, 0);
    float W = (float)m->w[l], H = (float)m->h[l];
    u = u * W - 0.5f; v = v * H - 0.5f;
    d0x *= W; d0y *= H; d1x *= W; d1y *= H;
    float A = (d0y * d0y + d1y * d1y) + 1.0f;
    float B = -2.0f * (d0x * d0y + d1x * d1y);
    float C = (d0x * d0x + d1x * d1x) + 1.0f;
    float invf = 1.0f / (A * C - (B * B) * 0.25f);
    A *= invf; B *= invf; C *= invf;
    float det = (-B) * B + (4.0f * A) * C;
    float invdet = 1.0f / det;
    float usq = sqrtf(det * C), vsq = sqrtf(A * det);
    int u0 = (int)ceilf(u - (2.0f * invdet) * usq), u1 = (int)floorf(u + (2.0f * invdet) * usq);
    int v0 = (int)ceilf(v - (2.0f * invdet) * vsq), v1 = (int)floorf(v + (2.0f * invdet) * vsq);
    v3 sum = V(0, 0, 0);
    float sw = 0.0f;
    for (int iv = v0; iv <= v1; ++iv) {
        float dv = (float)iv - v;
        for (int iu = u0; iu <= u1; ++iu) {
            float du = (float)iu - u;
            float r2 = ((A * du) * du + (B * du) * dv) + (C * dv) * dv;
            if (r2 < 1.0f) {
                int idx = (int)(r2 * 128.0f);
                if (idx > 127) idx = 127;
                float wt = ewa_lut[idx];
                sum = add(sum, scl(mip_texel(m, l, iu, iv), wt));
                sw += wt;
            }
        }
    }
    return divs(sum, sw);
}
/* MipMap::Lookup(UV, D0, D1) :309 */
static v3 mip_lookup_diff(const mip_t *m, float u, float v, float d0x, float d0y, float d1x, float d1y) {
    if (m->trilinear) {
        float w = fmaxf(fmaxf(fabsf(d0x), fabsf(d0y)), fmaxf(fabsf(d1x), fabsf(d1y)));
        return mip_lookup_width(m, u, v, 2.0f * w);
    }
    if (d0x * d0x + d0y * d0y < d1x * d1x + d1y * d1y) {
        float tx = d0x, ty = d0y; d0x = d1x; d0y = d1y; d1x = tx; d1y = ty;
    }
    float major = sqrtf(d0x * d0x + d0y * d0y), minor = sqrtf(d1x * d1x + d1y * d1y);
    if (minor * m->max_aniso < major && minor > 0.0f) {
        float sc = major / (minor * m->max_aniso);
        d1x *= sc; d1y *= sc;
        minor *= sc;
    }
    if (minor == 0.0f) return mip_triangle(m, 0, u, v);
    float lod = fmaxf(0.0f, (float)m->levels - 1.0f + log2f(minor));
    float ilod = floorf(lod);
    return lerp3(lod - ilod, mip_ewa(m, (int)ilod, u, v, d0x, d0y, d1x, d1y),
                 mip_ewa(m, (int)(ilod + 1.0f), u, v, d0x, d0y, d1x, d1y));
}
/* BitmapTexture::Eval(UV, D0, D1) (src/texture/BitmapTexture.cpp:101) after
 * Texture2D::Eval (src/core/Texture.cpp:211) scaled and offset UV and D. */
static v3 bitmap_eval(const ho_texture_desc *t, const mip_t *m, const float *uvi, const float *duv) {
    float u = uvi[0] * t->uv_scale[0] + t->uv_offset[0], v = uvi[1] * t->uv_scale[1] + t->uv_offset[1];
    if (t->filter == HO_FILTER_NEAREST || !duv)   /* Eval(UV): the unfiltered lookup (:134) */
        return mip_texel(m, 0, (int)floorf(u * (float)m->w[0]), (int)floorf(v * (float)m->h[0]));
    if (t->filter == HO_FILTER_BILINEAR) return mip_lookup_width(m, u, v, 0.0f);
    return mip_lookup_diff(m, u, v, duv[0] * t->uv_scale[0], duv[1] * t->uv_scale[1], duv[2] * t->uv_scale[0],
                           duv[3] * t->uv_scale[1]);
}

struct ho_scene;
static v3 bsdf_eval(const struct ho_scene *s, int id, const brec *r);
static float bsdf_pdf(const struct ho_scene *s, int id, const brec *r);
static v3 bsdf_sample(const struct ho_scene *s, int id, brec *r, float ux, float uy, ho_pcg32 *rng,
                      const float *u1fixed);

/* ------------------------------------------------------------------ scene */
typedef struct {
    uint32_t v0, nv, t0, nt;
    int32_t bsdf, emitter;
    int has_n;
    int has_uv;        /* texture coordinates present (ho_scene_set_mesh_uv) */
    float *cdf;        /* nt+1 area CDF (DiscretePDF1D) */
    float *func;       /* nt areas */
    float func_int;    /* m_FuncIntegral */
    float inv_area;    /* Mesh::m_InvMeshArea */
    v3 radiance;
    int geo_tex;       /* its BSDF uses a wireframe or curvature texture: hits compute their inputs */
} mesh_t;

typedef struct { int n; float *func; float *cdf; float integral; } pdf1d;

typedef struct { float bmin[3], bmax[3]; int32_t left_or_first, count, axis, right; } bnode;

struct ho_scene {
    /* 1: Sampler::Next2D returns (second draw, first draw), the order the
     * reference's Point2f(nextFloat(), nextFloat()) takes when its arguments
     * are evaluated right to left (GCC; the order is unspecified in C++).
     * 0 (default): (first, second), the order the CUDA kernels use. */
    int swap2d;
    int nb, cap_b; bsdf_t *bsdfs;
    int ntex, cap_tex; ho_texture_desc *tex; struct mip_t **mips;
    int ray_diff;                      /* a bitmap texture filters with the camera ray's differentials */
    int nm, cap_m; mesh_t *meshes;
    float *P; float *N; float *UV; uint32_t nv, cap_v;   /* global vertices (world space); UV 2 per vertex */
    uint32_t *F; int32_t *tri_mesh; uint32_t nt, cap_t;
    rft_table rft[2]; int has_rft[2];
    /* emitters in Scene::AddChild order: meshes (XML order), env appended */
    int n_emit; int32_t emit_mesh[64]; int env_index;
    /* env */
    int has_env; uint32_t ew, eh; float *env; float env_scale; float to_world[9], to_local[9];
    int env_const_on; v3 env_const;                   /* ConstantLight instead of the map */
    /* point / directional lights: emit_mesh codes -2 - k */
    int n_delta; struct { int directional; v3 vec, color; } delta[64];
    pdf1d *env_rows; pdf1d env_marg;
    /* camera */
    uint32_t W, H; float cam[16]; float fov, near_c, far_c;
    float cot, aspect;
    /* filter */
    int filt_kind; float filt_r, filt_p0, filt_p1; float ftab[33]; float lookup; int border;
    v3 background; int force_bg;
    /* bvh */
    bnode *nodes; int nnodes; uint32_t *order;
    float bbox[6];
    int finalized;
};

ho_scene *ho_scene_create(void) {
    ho_scene *s = (ho_scene *)calloc(1, sizeof(ho_scene));
    s->filt_kind = 2; s->filt_r = 2.0f; s->filt_p0 = 0.5f;    /* DEFAULT_CAMERA_RFILTER gaussian */
    s->env_index = -1;
    return s;
}
void ho_scene_destroy(ho_scene *s) {
    if (!s) return;
    for (int i = 0; i < s->nm; i++) { free(s->meshes[i].cdf); free(s->meshes[i].func); }
    for (int i = 0; i < s->ntex; i++) mip_free(s->mips[i]);
    free(s->mips);
    free(s->meshes); free(s->bsdfs); free(s->tex); free(s->P); free(s->N); free(s->UV); free(s->F); free(s->tri_mesh);
    for (int i = 0; i < 2; i++) free(s->rft[i].owned);
    free(s->env);
    if (s->env_rows) { for (uint32_t i = 0; i < s->eh; i++) { free(s->env_rows[i].func); free(s->env_rows[i].cdf); } }
    free(s->env_rows); free(s->env_marg.func); free(s->env_marg.cdf);
    free(s->nodes); free(s->order);
    free(s);
}
int ho_scene_set_rft(ho_scene *s, int dist, const void *bytes, uint64_t n) {
    if (dist < 0 || dist > 1) return fail("bad distribution");
    if (rft_parse(&s->rft[dist], bytes, n)) return -1;
    if (s->rft[dist].theta_n > RFT_MAX_THETA) return fail("rft theta too large");
    s->has_rft[dist] = 1;
    return 0;
}
static int push_texture(ho_scene *s, const ho_texture_desc *d, mip_t *m) {
    if (s->ntex == s->cap_tex) {
        s->cap_tex = s->cap_tex ? 2 * s->cap_tex : 8;
        s->tex = realloc(s->tex, s->cap_tex * sizeof *s->tex);
        s->mips = realloc(s->mips, s->cap_tex * sizeof *s->mips);
    }
    s->tex[s->ntex] = *d;
    s->mips[s->ntex] = m;
    return s->ntex++;
}
int ho_scene_add_texture(ho_scene *s, const ho_texture_desc *d) {
    const int geo = d->kind == HO_TEX_WIREFRAME || d->kind == HO_TEX_CURVATURE;
    if ((d->kind < HO_TEX_CHECKERBOARD || d->kind > HO_TEX_SCALE) && !geo) return fail("unknown texture kind");
    if (d->kind == HO_TEX_SCALE && (d->nested < 0 || d->nested >= s->ntex)) return fail("scale texture needs a nested texture");
    if (d->kind != HO_TEX_SCALE && !geo && d->count <= 0) return fail("texture block / line count must be positive");
    return push_texture(s, d, NULL);
}
/* BitmapTexture ctor (src/texture/BitmapTexture.cpp:7) over LoadImageFromFileR
 * / LoadImageFromFileRGB (src/core/Texture.cpp:12, :74) and MipMap. */
int ho_scene_add_bitmap(ho_scene *s, const ho_texture_desc *d, const uint8_t *pix, int w, int h) {
    if (d->kind != HO_TEX_BITMAP) return fail("bitmap texture expected");
    if (d->channels != 1 && d->channels != 3) return fail("bitmap channel must be r (1) or rgb (3)");
    if (w <= 0 || h <= 0 || w > (1 << 15) || h > (1 << 15) || !pix) return fail("invalid bitmap size");
    if (d->filter < HO_FILTER_NEAREST || d->filter > HO_FILTER_EWA) return fail("invalid filter type");
    if (d->wrap_u < 0 || d->wrap_u > 2 || d->wrap_v < 0 || d->wrap_v > 2) return fail("invalid wrap mode");
    const int ch = d->channels;
    const float inv255 = 1.0f / 255.0f, inv_gamma = 1.0f / d->gamma;
    float *t = malloc(sizeof(float) * 3 * (size_t)w * h);
    float avg[3] = {0, 0, 0};
    for (int x = 0; x < w; x++)
        for (int y = 0; y < h; y++) {
            size_t ld = (size_t)y * w + x, st = (size_t)(h - 1 - y) * w + x;
            for (int c = 0; c < 3; c++) {
                int cc = ch == 1 ? 0 : c;
                float val = (float)pix[ld * ch + cc] * inv255;
                val = inv_gamma == 1.0f ? val : powf(val, inv_gamma);   /* GammaCorrect (include/core/Common.hpp:982) */
                t[3 * st + c] = val;
                avg[c] += val;
            }
        }
    mip_t *m = mip_build(t, w, h, ch, d->wrap_u, d->wrap_v, d->filter == HO_FILTER_TRILINEAR, d->max_anisotropy);
    free(t);
    for (int c = 0; c < 3; c++) m->avg[c] = avg[c] / (float)(w * h);
    if (d->filter >= HO_FILTER_TRILINEAR) s->ray_diff = 1;
    return push_texture(s, d, m);
}
int ho_scene_add_bsdf(ho_scene *s, const ho_bsdf_desc *d) {
    if (s->nb == s->cap_b) { s->cap_b = s->cap_b ? 2 * s->cap_b : 8; s->bsdfs = realloc(s->bsdfs, s->cap_b * sizeof(bsdf_t)); }
    bsdf_t *b = &s->bsdfs[s->nb]; memset(b, 0, sizeof *b);
    b->d = *d;
    return s->nb++;
}
int ho_scene_add_mesh(ho_scene *s, const float *pos, uint32_t nv, const uint32_t *idx, uint32_t nt,
                      const float *nrm, int32_t bsdf, const float *rad) {
    if (s->nm == s->cap_m) { s->cap_m = s->cap_m ? 2 * s->cap_m : 8; s->meshes = realloc(s->meshes, s->cap_m * sizeof(mesh_t)); }
    if (s->nv + nv > s->cap_v) {
        while (s->nv + nv > s->cap_v) s->cap_v = s->cap_v ? 2 * s->cap_v : 1024;
        s->P = realloc(s->P, 3ull * s->cap_v * 4); s->N = realloc(s->N, 3ull * s->cap_v * 4);
        s->UV = realloc(s->UV, 2ull * s->cap_v * 4);
    }
    if (s->nt + nt > s->cap_t) {
        while (s->nt + nt > s->cap_t) s->cap_t = s->cap_t ? 2 * s->cap_t : 1024;
        s->F = realloc(s->F, 3ull * s->cap_t * 4); s->tri_mesh = realloc(s->tri_mesh, 4ull * s->cap_t);
    }
    mesh_t *m = &s->meshes[s->nm]; memset(m, 0, sizeof *m);
    m->v0 = s->nv; m->nv = nv; m->t0 = s->nt; m->nt = nt; m->bsdf = bsdf; m->emitter = -1;
    m->has_n = nrm != NULL;
    memcpy(s->P + 3ull * s->nv, pos, 12ull * nv);
    if (nrm) memcpy(s->N + 3ull * s->nv, nrm, 12ull * nv);
    for (uint64_t i = 0; i < 3ull * nt; i++) {
        if (idx[i] >= nv) return fail("mesh index out of range");
        s->F[3ull * s->nt + i] = idx[i] + s->nv;
    }
    for (uint32_t i = 0; i < nt; i++) s->tri_mesh[s->nt + i] = s->nm;
    if (rad) {
        if (s->n_emit >= 64) return fail("too many emitters");
        m->radiance = vload(rad);
        m->emitter = s->n_emit;
        s->emit_mesh[s->n_emit++] = s->nm;
    }
    memset(s->UV + 2ull * s->nv, 0, 8ull * nv);
    s->nv += nv; s->nt += nt;
    return s->nm++;
}
/* Texture coordinates of a mesh (2 per vertex, the OBJ "vt" of each vertex). */
int ho_scene_set_mesh_uv(ho_scene *s, int mesh, const float *uv) {
    if (mesh < 0 || mesh >= s->nm || !uv) return fail("bad mesh id");
    mesh_t *m = &s->meshes[mesh];
    memcpy(s->UV + 2ull * m->v0, uv, 8ull * m->nv);
    m->has_uv = 1;
    return 0;
}
static void mat3_inverse(const float *m, float *o) {
    double a = m[0], b = m[1], c = m[2], d = m[3], e = m[4], f = m[5], g = m[6], h = m[7], i = m[8];
    double det = a * (e * i - f * h) - b * (d * i - f * g) + c * (d * h - e * g);
    o[0] = (float)((e * i - f * h) / det); o[1] = (float)((c * h - b * i) / det); o[2] = (float)((b * f - c * e) / det);
    o[3] = (float)((f * g - d * i) / det); o[4] = (float)((a * i - c * g) / det); o[5] = (float)((c * d - a * f) / det);
    o[6] = (float)((d * h - e * g) / det); o[7] = (float)((b * g - a * h) / det); o[8] = (float)((a * e - b * d) / det);
}
static inline v3 mat3_mul(const float *m, v3 v) {
    return V(m[0] * v.x + m[1] * v.y + m[2] * v.z, m[3] * v.x + m[4] * v.y + m[5] * v.z,
             m[6] * v.x + m[7] * v.y + m[8] * v.z);
}
/* DiscretePDF1D ctor  src/core/DiscretePDF.cpp:5 */
static void pdf1d_build(pdf1d *p, const float *f, int n) {
    p->n = n; p->func = malloc(4ull * n); p->cdf = malloc(4ull * (n + 1));
    memcpy(p->func, f, 4ull * n);
    p->cdf[0] = 0.0f;
    for (int i = 1; i < n + 1; i++) p->cdf[i] = p->cdf[i - 1] + p->func[i - 1] / n;
    p->integral = p->cdf[n];
    if (p->integral == 0.0f) for (int i = 1; i < n + 1; i++) p->cdf[i] = (float)i / (float)n;
    else for (int i = 1; i < n + 1; i++) p->cdf[i] /= p->integral;
}
/* std::lower_bound then clamp to [0, n-1]  src/core/DiscretePDF.cpp:41-46 */
static int cdf_find(const float *cdf, int n, float u) {
    int lo = 0, hi = n + 1;            /* first index with cdf[i] >= u */
    while (lo < hi) { int mid = (lo + hi) >> 1; if (cdf[mid] < u) lo = mid + 1; else hi = mid; }
    int idx = lo - 1; if (idx < 0) idx = 0; if (idx > n - 1) idx = n - 1;
    return idx;
}
/* DiscretePDF1D::SampleContinuous  src/core/DiscretePDF.cpp:39 */
static float pdf1d_sample_cont(const pdf1d *p, float u, float *pdf, int *pidx) {
    int idx = cdf_find(p->cdf, p->n, u);
    *pidx = idx;
    float du = u - p->cdf[idx];
    if (p->cdf[idx + 1] - p->cdf[idx] > 0.0f) du /= (p->cdf[idx + 1] - p->cdf[idx]);
    *pdf = p->func[idx] / p->integral;
    return ((float)idx + du) / (float)p->n;
}
int ho_scene_set_envmap(ho_scene *s, const float *rgb, uint32_t w, uint32_t h, const float *tw16, float scale) {
    if (s->has_env) return fail("only one environment emitter");   /* Scene.cpp:198 */
    s->has_env = 1; s->ew = w; s->eh = h; s->env_scale = scale;
    s->env = malloc(12ull * w * h); memcpy(s->env, rgb, 12ull * w * h);
    for (int r = 0; r < 3; r++) for (int c = 0; c < 3; c++) s->to_world[3 * r + c] = tw16[4 * r + c];
    mat3_inverse(s->to_world, s->to_local);
    /* EnvironmentLight ctor  src/emitter/EnvironmentLight.cpp:8-31 */
    float *L = malloc(4ull * w * h);
    for (uint32_t y = 0; y < h; y++) {
        float th = (float)(y + 0.5f) / h * PI_F;
        float st = sinf(th);
        for (uint32_t x = 0; x < w; x++) L[(uint64_t)y * w + x] = lum(vload(rgb + 3ull * ((uint64_t)y * w + x))) * st;
    }
    s->env_rows = calloc(h, sizeof(pdf1d));
    float *marg = malloc(4ull * h);
    for (uint32_t y = 0; y < h; y++) { pdf1d_build(&s->env_rows[y], L + (uint64_t)y * w, (int)w); marg[y] = s->env_rows[y].integral; }
    pdf1d_build(&s->env_marg, marg, (int)h);
    free(marg); free(L);
    if (s->n_emit >= 64) return fail("too many emitters");
    s->env_index = s->n_emit;
    s->emit_mesh[s->n_emit++] = -1;
    return 0;
}
/* ConstantLight ctor  src/emitter/ConstantLight.cpp:8; Scene::AddChild :191 */
int ho_scene_set_constant_light(ho_scene *s, const float *rgb) {
    if (s->has_env) return fail("only one environment emitter");
    if (s->n_emit >= 64) return fail("too many emitters");
    s->has_env = 1; s->env_const_on = 1; s->env_const = vload(rgb);
    s->env_index = s->n_emit;
    s->emit_mesh[s->n_emit++] = -1;
    return 0;
}
/* PointLight / DirectionalLight ctors  src/emitter/PointLight.cpp:8, DirectionalLight.cpp:8 */
static int add_delta_light(ho_scene *s, int directional, const float *color, const float *vec) {
    if (s->n_emit >= 64 || s->n_delta >= 64) return fail("too many emitters");
    s->delta[s->n_delta].directional = directional;
    s->delta[s->n_delta].color = vload(color);
    s->delta[s->n_delta].vec = vload(vec);
    s->emit_mesh[s->n_emit++] = -2 - s->n_delta++;
    return 0;
}
int ho_scene_add_point_light(ho_scene *s, const float *power, const float *pos) { return add_delta_light(s, 0, power, pos); }
int ho_scene_add_directional_light(ho_scene *s, const float *irr, const float *dir) { return add_delta_light(s, 1, irr, dir); }
int ho_scene_set_camera(ho_scene *s, uint32_t w, uint32_t h, const float *tw16, float fov, float n, float f) {
    s->W = w; s->H = h; memcpy(s->cam, tw16, 64); s->fov = fov; s->near_c = n; s->far_c = f;
    return 0;
}
int ho_scene_set_filter(ho_scene *s, int kind, float r, float p0, float p1) {
    s->filt_kind = kind; s->filt_r = r; s->filt_p0 = p0; s->filt_p1 = p1; return 0;
}
int ho_scene_set_background(ho_scene *s, const float *rgb, int force) { s->background = vload(rgb); s->force_bg = force; return 0; }

/* filters  src/filter/{Box,Tent,Gaussian,MitchellNetraval}Filter.cpp */
static float filter_eval(const ho_scene *s, float x) {
    switch (s->filt_kind) {
    case 0: return 1.0f;
    case 1: return fmaxf(0.0f, 1.0f - fabsf(x));
    case 2: {
        float a = -1.0f / (2.0f * s->filt_p0 * s->filt_p0);
        return fmaxf(0.0f, expf(a * x * x) - expf(a * s->filt_r * s->filt_r));
    }
    default: {
        float B = s->filt_p0, C = s->filt_p1;
        x = fabsf(2.0f * x / s->filt_r);
        float x2 = x * x, x3 = x2 * x;
        if (x < 1.0f) return 1.0f / 6.0f * ((12.0f - 9.0f * B - 6.0f * C) * x3 + (-18.0f + 12.0f * B + 6.0f * C) * x2 + (6.0f - 2.0f * B));
        if (x < 2.0f) return 1.0f / 6.0f * ((-B - 6 * C) * x3 + (6.0f * B + 30.0f * C) * x2 + (-12.0f * B - 48.0f * C) * x + (8.0f * B + 24.0f * C));
        return 0.0f;
    }
    }
}

static int bvh_build(ho_scene *s);

static float approx_fresnel_diffuse(float e);
/* Whether a BSDF has a transmission lobe (EDeltaTransmission / EGlossyTransmission;
 * coatings inherit their nested BSDF's types, RoughCoatingBSDF.cpp:317). */
static int bsdf_transmits(const ho_scene *s, int id, int depth) {
    if (id < 0 || id >= s->nb || depth > 8) return 0;
    const ho_bsdf_desc *d = &s->bsdfs[id].d;
    switch (d->type) {
    case HO_BSDF_ROUGH_DIELECTRIC: case HO_BSDF_DIELECTRIC: return 1;
    case HO_BSDF_ROUGH_COATING:
    case HO_BSDF_COATING: return bsdf_transmits(s, d->nested, depth + 1);
    case HO_BSDF_TWO_SIDED:
        return bsdf_transmits(s, d->nested, depth + 1) || bsdf_transmits(s, d->nested2, depth + 1);
    case HO_BSDF_BUMP_MAP: case HO_BSDF_NORMAL_MAP: return bsdf_transmits(s, d->nested, depth + 1);
    default: return 0;
    }
}

/* BSDF activation: RoughPlasticBSDF::Activate :261, RoughCoatingBSDF::Activate :315 */
static v3 tex_average(const ho_texture_desc *T, mip_t *const *M, int id);
/* Texture::GetAverage of a parameter: the texture's average or the constant */
static v3 par_average(const ho_scene *s, const ho_bsdf_desc *d, int slot, const float *c) {
    return d->tex[slot] ? tex_average(s->tex, s->mips, d->tex[slot] - 1) : vload(c);
}
/* channel 0 of Texture::GetMinimum / GetMaximum, for the roughness range
 * check of a textured alpha (checkerboard / grid / wireframe: the smaller and
 * larger colour; scale: the nested range scaled; bitmap: the level-0 texels;
 * curvature: [0, 1]) */
static void tex_range0(const ho_scene *s, int id, float *lo, float *hi) {
    const ho_texture_desc *t = &s->tex[id];
    if (t->kind == HO_TEX_SCALE) {
        tex_range0(s, t->nested, lo, hi);
        *lo *= t->scale; *hi *= t->scale;
        return;
    }
    if (t->kind == HO_TEX_CURVATURE) { *lo = 0.0f; *hi = 1.0f; return; }
    if (t->kind == HO_TEX_BITMAP) {
        const mip_t *m = s->mips[id];
        float mn = FLT_MAX, mx = -FLT_MAX;
        for (int64_t i = 0; i < (int64_t)m->w[0] * m->h[0]; i++) {
            mn = fminf(mn, m->lv[0][3 * i]);
            mx = fmaxf(mx, m->lv[0][3 * i]);
        }
        *lo = mn; *hi = mx;
        return;
    }
    *lo = fminf(t->a[0], t->b[0]);
    *hi = fmaxf(t->a[0], t->b[0]);
}
static int activate_bsdf(ho_scene *s, bsdf_t *b) {
    const ho_bsdf_desc *d = &b->d;
    b->textures = s->tex;
    b->mips = s->mips;
    for (int k = 0; k < 6; k++)
        if (d->tex[k] < 0 || d->tex[k] > s->ntex) return fail("invalid texture id");
    b->eta = d->int_ior / d->ext_ior;
    b->inv_eta = 1.0f / b->eta;
    b->inv_eta2 = b->inv_eta * b->inv_eta;
    for (int c = 0; c < 3; c++) { b->eta_c[c] = d->eta[c]; b->k_c[c] = d->k[c] / d->ext_ior; }
    if (d->type == HO_BSDF_ROUGH_PLASTIC || d->type == HO_BSDF_ROUGH_COATING) {
        int dist = d->distribution;
        if (!s->has_rft[dist]) return fail("missing RFT table");
        const rft_table *t = &s->rft[dist];
        float alpha = clampf(d->alpha_u, 5e-4f, 1.0f);
        float e = b->eta < 1.0f ? 1.0f / b->eta : b->eta;        /* CheckEta :315 */
        if (e < t->eta_min || e > t->eta_max) return fail("eta outside RFT range");
        int A = (int)t->alpha_n, T = (int)t->theta_n;
        float *t2d = malloc(4ull * A * T), *d1d = malloc(4ull * A);
        float dsc;
        b->alpha_tex = d->tex[4] != 0;
        if (b->alpha_tex) {   /* CheckAlpha(GetMinimum / GetMaximum) (RoughPlasticBSDF.cpp:268) */
            float lo, hi;
            tex_range0(s, d->tex[4] - 1, &lo, &hi);
            if (lo < t->alpha_min || lo > t->alpha_max || hi < t->alpha_min || hi > t->alpha_max)
                return fail("alpha outside RFT range");
        } else if (alpha < t->alpha_min || alpha > t->alpha_max) {
            return fail("alpha outside RFT range");
        }
        rft_set_eta(t, b->eta, t2d, d1d);
        b->rft_n = T;
        b->rft_an = A;
        b->rft_amin = t->alpha_min;
        b->rft_amax = t->alpha_max;
        if (b->alpha_tex) {   /* no SetAlpha: Eval interpolates in alpha per query */
            b->rft2d = t2d;
            t2d = malloc(4ull * A * T);
        } else {
            rft_set_alpha(t, t2d, d1d, alpha, b->rft, &dsc);
        }
        if (d->type == HO_BSDF_ROUGH_PLASTIC) {
            float ksa = lum(par_average(s, d, 1, d->ks)), kda = lum(par_average(s, d, 0, d->kd));
            b->spec_w = ksa / (kda + ksa);
            /* m_pIntData: SetEta(1/eta) only; EvalDiffuse(alpha) is the 1D cubic over alpha */
            rft_set_eta(t, b->inv_eta, t2d, d1d);
            float wa = powf((alpha - t->alpha_min) / (t->alpha_max - t->alpha_min), 0.25f);
            float ed = clampf(cubic1d(wa, d1d, A, 0.0f, 1.0f), 0.0f, 1.0f);
            b->fdr_int = 1.0f - ed;
            if (b->alpha_tex) {
                b->rft_diff = d1d;
                d1d = malloc(4ull * A);
            }
        } else {
            float th = d->thickness;
            v3 sav = par_average(s, d, 3, d->sigma_a);
            float a0 = expf(sav.x * (-2.0f * th)), a1 = expf(sav.y * (-2.0f * th)),
                  a2 = expf(sav.z * (-2.0f * th));
            float avg = (a0 + a1 + a2) / 3.0f;
            b->spec_w = 1.0f / (avg + 1.0f);
            if (d->nested < 0 || d->nested >= s->nb) return fail("roughCoating needs a nested BSDF");
        }
        free(t2d); free(d1d);
    }
    if (d->type == HO_BSDF_CONDUCTOR)   /* ConductorBSDF ctor :17: m_Eta = Color3f(intIOR / extIOR) */
        for (int c = 0; c < 3; c++) b->eta_c[c] = b->eta;
    if (d->type == HO_BSDF_PLASTIC) {   /* PlasticBSDF ctor :25 and Activate :170 */
        float ksa = lum(par_average(s, d, 1, d->ks)), kda = lum(par_average(s, d, 0, d->kd));
        b->spec_w = ksa / (kda + ksa);
        b->fdr_int = approx_fresnel_diffuse(b->inv_eta);
    }
    if (d->type == HO_BSDF_TWO_SIDED) {   /* TwoSidedBSDF::Activate :98 */
        if (d->nested < 0 || d->nested >= s->nb) return fail("TwoSidedBSDF needs at least one nested BSDF!");
        if (d->nested2 >= s->nb) return fail("twoSided: invalid second nested BSDF");
        if (d->nested2 < 0) b->d.nested2 = d->nested;
        if (bsdf_transmits(s, d->nested, 0) || bsdf_transmits(s, b->d.nested2, 0))
            return fail("Only BSDF without transmission can be nested!");
    }
    if (d->type == HO_BSDF_COATING) {   /* CoatingBSDF::Activate :255 */
        float th = d->thickness;
        v3 sav = par_average(s, d, 3, d->sigma_a);
            float a0 = expf(sav.x * (-2.0f * th)), a1 = expf(sav.y * (-2.0f * th)),
              a2 = expf(sav.z * (-2.0f * th));
        b->spec_w = 1.0f / ((a0 + a1 + a2) / 3.0f + 1.0f);
        if (d->nested < 0 || d->nested >= s->nb) return fail("CoatingBSDF needs a nested BSDF!");
    }
    if (d->type == HO_BSDF_BUMP_MAP || d->type == HO_BSDF_NORMAL_MAP) {   /* BumpMapBSDF::Activate :138 */
        if (d->nested < 0 || d->nested >= s->nb) return fail("bumpMap / normalMap needs a nested BSDF");
        if (d->tex[0] <= 0) return fail("bumpMap / normalMap needs a map texture");
        int t = d->tex[0] - 1;
        while (s->tex[t].kind == HO_TEX_SCALE) t = s->tex[t].nested;
        if (s->tex[t].kind == HO_TEX_WIREFRAME || s->tex[t].kind == HO_TEX_CURVATURE)
            return fail("a wireframe or curvature texture as a bump / normal map is not supported");
    }
    if (d->type < HO_BSDF_DIFFUSE || d->type > HO_BSDF_NORMAL_MAP) return fail("unknown BSDF type");
    return 0;
}

/* Whether texture tid is (or scales) a wireframe or curvature texture; a
 * wireframe texture whose edgeWidth is 0 takes a tenth of the mean edge length
 * of mesh mi (WireframeTexture::Eval, src/texture/WireframeTexture.cpp:37-53:
 * the first mesh that evaluates it). */
static int tex_geo(ho_scene *s, int tid, int mi) {
    ho_texture_desc *t = &s->tex[tid];
    if (t->kind == HO_TEX_SCALE) return tex_geo(s, t->nested, mi);
    if (t->kind == HO_TEX_WIREFRAME && t->width == 0.0f) {
        const mesh_t *m = &s->meshes[mi];
        float ew = 0.0f;
        for (uint32_t i = 0; i < m->nt; i++) {
            const uint32_t *f = s->F + 3ull * (m->t0 + i);
            const v3 p0 = vload(s->P + 3ull * f[0]), p1 = vload(s->P + 3ull * f[1]), p2 = vload(s->P + 3ull * f[2]);
            const float l0 = norm(sub(p1, p0)), l1 = norm(sub(p2, p1)), l2 = norm(sub(p0, p2));
            ew += (l0 + l1) + l2;
        }
        t->width = 0.1f * ew / (float)(3u * m->nt);
    }
    return t->kind == HO_TEX_WIREFRAME || t->kind == HO_TEX_CURVATURE;
}
static int bsdf_geo(ho_scene *s, int bid, int mi, int depth) {
    if (bid < 0 || bid >= s->nb || depth > 4) return 0;
    const ho_bsdf_desc *d = &s->bsdfs[bid].d;
    int g = 0;
    for (int k = 0; k < 6; k++)
        if (d->tex[k] > 0) g |= tex_geo(s, d->tex[k] - 1, mi);
    if (d->type == HO_BSDF_ROUGH_COATING || d->type == HO_BSDF_COATING || d->type == HO_BSDF_TWO_SIDED ||
        d->type == HO_BSDF_BUMP_MAP || d->type == HO_BSDF_NORMAL_MAP)
        g |= bsdf_geo(s, d->nested, mi, depth + 1);
    if (d->type == HO_BSDF_TWO_SIDED) g |= bsdf_geo(s, d->nested2, mi, depth + 1);
    return g;
}

int ho_scene_finalize(ho_scene *s) {
    for (int i = 0; i < s->nb; i++) if (activate_bsdf(s, &s->bsdfs[i])) return -1;
    for (int i = 0; i < s->nm; i++) s->meshes[i].geo_tex = bsdf_geo(s, s->meshes[i].bsdf, i, 0);
    /* Mesh::Activate  src/core/Mesh.cpp:233 (area CDF) */
    for (int i = 0; i < s->nm; i++) {
        mesh_t *m = &s->meshes[i];
        float *areas = malloc(4ull * (m->nt ? m->nt : 1));
        float total = 0.0f;
        for (uint32_t t = 0; t < m->nt; t++) {
            const uint32_t *f = s->F + 3ull * (m->t0 + t);
            v3 p0 = vload(s->P + 3ull * f[0]), p1 = vload(s->P + 3ull * f[1]), p2 = vload(s->P + 3ull * f[2]);
            float a = 0.5f * norm(cross(sub(p1, p0), sub(p2, p0)));
            areas[t] = a; total += a;
        }
        m->inv_area = 1.0f / total;
        pdf1d p; pdf1d_build(&p, areas, (int)m->nt);
        m->cdf = p.cdf; m->func = p.func; m->func_int = p.integral;
        free(areas);
    }
    /* camera  src/camera/PerspectiveCamera.cpp:32 */
    s->aspect = (float)s->W / (float)s->H;
    s->cot = 1.0f / tanf((s->fov / 2.0f) * (PI_F / 180.0f));
    /* ImageBlock ctor  src/core/Block.cpp:9 */
    s->border = (int)ceilf(s->filt_r - 0.5f);
    for (int i = 0; i < 32; i++) s->ftab[i] = filter_eval(s, (s->filt_r * i) / 32);
    s->ftab[32] = 0.0f;
    s->lookup = 32 / s->filt_r;
    if (bvh_build(s)) return -1;
    s->finalized = 1;
    return 0;
}
void ho_scene_bbox(const ho_scene *s, float *o) { memcpy(o, s->bbox, 24); }
int ho_scene_num_emitters(const ho_scene *s) { return s->n_emit; }
int ho_film_border(const ho_scene *s) { return s->border; }

/* ------------------------------------------------------------ BSDF impl */
/* Texture2D::Eval(Isect) (src/core/Texture.cpp:211) of the procedural textures:
 * UV scaled and offset, then CheckerboardTexture::Eval (src/texture/
 * CheckerboardTexture.cpp:24) or GridTexture::Eval (src/texture/GridTexture.cpp:26);
 * ScaleTexture::Eval (src/texture/ScaleTexture.cpp:17) scales its nested texture. */
static inline int mod_positive(int a, int b) { int r = a % b; return r < 0 ? r + b : r; }
static v3 pattern_eval(const ho_texture_desc *t, float u, float v);
static float smooth_step(float lo, float hi, float x) {   /* SmoothStep (include/core/Common.hpp:994) */
    float v = (x - lo) / (hi - lo);
    v = v < 0.0f ? 0.0f : (v > 1.0f ? 1.0f : v);   /* Clamp (:752) */
    return v * v * (-2.0f * v + 3.0f);
}
/* WireframeTexture::Eval (src/texture/WireframeTexture.cpp:22) and
 * CurvatureTexture::Eval (src/texture/CurvatureTexture.cpp:34) from the hit's
 * edge distance and curvatures; without an intersection (record-level
 * queries) the interior colour and black */
static v3 geo_tex_eval(const ho_texture_desc *t, const isect_t *it) {
    if (t->kind == HO_TEX_WIREFRAME) {
        if (!it) return vload(t->a);
        const float w = t->width;
        const float al = smooth_step(w * (1.0f - t->scale), w, it->edge_d);
        return add(scl(vload(t->b), 1.0f - al), scl(vload(t->a), al));
    }
    const float val = !it ? 0.0f : (t->count ? it->curv_k : it->curv_h);
    if (val < 0.0f) {
        const float x = -val * t->scale;
        return scl(vload(t->b), 1.0f < x ? 1.0f : x);   /* std::min(x, 1) */
    }
    if (val > 0.0f) {
        const float x = val * t->scale;
        return scl(vload(t->a), 1.0f < x ? 1.0f : x);
    }
    return V(0, 0, 0);
}
/* duv NULL: Texture::Eval(Isect, bFilter = false); it: the record's
 * intersection (NULL in queries without one) */
static v3 tex_eval(const ho_texture_desc *T, mip_t *const *M, int id, const float *uvi, const float *duv,
                   const isect_t *it) {
    const ho_texture_desc *t = &T[id];
    if (t->kind == HO_TEX_SCALE) return scl(tex_eval(T, M, t->nested, uvi, duv, it), t->scale);
    if (t->kind == HO_TEX_BITMAP) return bitmap_eval(t, M[id], uvi, duv);
    if (t->kind == HO_TEX_WIREFRAME || t->kind == HO_TEX_CURVATURE) return geo_tex_eval(t, it);
    return pattern_eval(t, uvi[0] * t->uv_scale[0] + t->uv_offset[0], uvi[1] * t->uv_scale[1] + t->uv_offset[1]);
}
/* CheckerboardTexture / GridTexture::Eval(UV) at already scaled coordinates */
static v3 pattern_eval(const ho_texture_desc *t, float u, float v) {
    if (t->kind == HO_TEX_CHECKERBOARD) {
        int ex = mod_positive(mod_positive((int)(u * t->count), t->count), 2) == 0;
        int ey = mod_positive(mod_positive((int)(v * t->count), t->count), 2) == 0;
        return (ex ^ ey) ? vload(t->a) : vload(t->b);
    }
    float su = u * (float)(t->count - 1), sv = v * (float)(t->count - 1);
    float dx = su - floorf(su), dy = sv - floorf(sv);
    if (dx > 0.5f) dx -= 1.0f;
    if (dy > 0.5f) dy -= 1.0f;
    return (fabsf(dx) < t->width || fabsf(dy) < t->width) ? vload(t->a) : vload(t->b);
}
/* Texture::GetAverage of the procedural textures (used when BSDFs activate) */
/* Texture::EvalGradient(Isect) (src/core/Texture.cpp:227): the gradient at the
 * UNSCALED texture coordinates times the UV scale -- MipMap::EvalGradient at
 * level 0 for bitmaps (zero with nearest filtering, BitmapTexture.cpp:145),
 * forward differences of Eval(UV) with step Epsilon = 1e-4 for the
 * procedural ones (:235); ScaleTexture scales its nested gradient (:24). */
static void tex_gradient(const ho_texture_desc *T, mip_t *const *M, int id, const float *uv, v3 *g) {
    const ho_texture_desc *t = &T[id];
    if (t->kind == HO_TEX_SCALE) {
        tex_gradient(T, M, t->nested, uv, g);
        g[0] = scl(g[0], t->scale); g[1] = scl(g[1], t->scale);
        return;
    }
    if (t->kind == HO_TEX_BITMAP) {
        if (t->filter == HO_FILTER_NEAREST) g[0] = g[1] = V(0, 0, 0);
        else mip_gradient(M[id], 0, uv[0], uv[1], g);
    } else {
        const float eps = 1e-4f;
        v3 c = pattern_eval(t, uv[0], uv[1]), cu = pattern_eval(t, uv[0] + eps, uv[1]),
           cv = pattern_eval(t, uv[0], uv[1] + eps);
        g[0] = divs(sub(cu, c), eps);
        g[1] = divs(sub(cv, c), eps);
    }
    g[0] = scl(g[0], t->uv_scale[0]);
    g[1] = scl(g[1], t->uv_scale[1]);
}
static v3 tex_average(const ho_texture_desc *T, mip_t *const *M, int id) {
    const ho_texture_desc *t = &T[id];
    if (t->kind == HO_TEX_SCALE) return scl(tex_average(T, M, t->nested), t->scale);
    if (t->kind == HO_TEX_BITMAP) return vload(M[id]->avg);   /* BitmapTexture::GetAverage :176 */
    if (t->kind == HO_TEX_CHECKERBOARD) return scl(add(vload(t->a), vload(t->b)), 0.5f);
    if (t->kind == HO_TEX_WIREFRAME) return scl(add(vload(t->b), vload(t->a)), 0.5f);   /* :80 */
    if (t->kind == HO_TEX_CURVATURE) return V(0.5f, 0.5f, 0.5f);                       /* :61 */
    float iw = fmaxf(0.0f, 1.0f - 2.0f * t->width);    /* GridTexture::GetAverage :40 */
    float ia = iw * iw, la = 1.0f - ia;
    return add(scl(vload(t->a), la), scl(vload(t->b), ia));
}
/* A BSDF parameter at the query's intersection: its texture or its constant.
 * slot: 0 kd, 1 ks, 2 ksRefract, 3 sigmaA, 4 alpha(U), 5 alphaV */
static inline v3 par_rgb(const bsdf_t *b, int slot, const float *c, const brec *r) {
    int t = b->d.tex[slot];
    return t ? tex_eval(b->textures, b->mips, t - 1, r->uv, r->duv, r->it) : vload(c);
}
static inline float par_alpha(const bsdf_t *b, int slot, float c, const brec *r) {
    int t = b->d.tex[slot];
    return t ? tex_eval(b->textures, b->mips, t - 1, r->uv, r->duv, r->it).x : c;
}
void ho_texture_eval(const ho_scene *s, int id, const float *uv, const float *duv, float *out) {
    static const float zero[4] = {0, 0, 0, 0};
    vstore(out, tex_eval(s->tex, s->mips, id, uv, duv ? duv : zero, NULL));
}
int ho_texture_mip(const ho_scene *s, int id, int level, int *wh, float *texels) {
    if (id < 0 || id >= s->ntex || !s->mips[id]) return fail("not a bitmap texture");
    const mip_t *m = s->mips[id];
    if (level < 0 || level >= m->levels) return m->levels;
    wh[0] = m->w[level]; wh[1] = m->h[level];
    if (texels) {
        size_t n = (size_t)m->w[level] * m->h[level];
        for (size_t i = 0; i < n; i++)
            for (int c = 0; c < m->ch; c++) texels[i * m->ch + c] = m->lv[level][3 * i + c];
    }
    return m->levels;
}
static inline float alpha_u_of(const bsdf_t *b, const brec *r) { return clampf(par_alpha(b, 4, b->d.alpha_u, r), 5e-4f, 1.0f); }
/* the rough BSDFs' RoughTransmittance::Eval(c, Distribution.GetAlpha()) and
 * 1 - EvalDiffuse(alpha): the activated 1D table, or the 2D one per query
 * under a textured alpha (src/core/RoughTransmitance.cpp:48-87, :119-132) */
static inline float rft_b(const bsdf_t *b, float c, float alpha) {
    return b->alpha_tex ? rft_eval2d(b->rft2d, b->rft_n, b->rft_an, b->rft_amin, b->rft_amax, c, alpha)
                        : rft_eval1d(b->rft, b->rft_n, c);
}
static inline float fdr_b(const bsdf_t *b, float alpha) {
    if (!b->alpha_tex) return b->fdr_int;
    float wa = powf((alpha - b->rft_amin) / (b->rft_amax - b->rft_amin), 0.25f);
    return 1.0f - clampf(cubic1d(wa, b->rft_diff, b->rft_an, 0.0f, 1.0f), 0.0f, 1.0f);
}
static inline float alpha_v_of(const bsdf_t *b, const brec *r) {
    return b->d.anisotropic ? clampf(par_alpha(b, 5, b->d.alpha_v, r), 5e-4f, 1.0f) : alpha_u_of(b, r);
}

/* DiffuseBSDF  src/bsdf/DiffuseBSDF.cpp:20-67 */
static v3 diffuse_sample(const bsdf_t *b, brec *r, float ux, float uy) {
    if (r->wi.z <= 0) return V(0, 0, 0);
    r->measure = HO_MEASURE_SOLID_ANGLE;
    r->wo = square_to_cos_hemi(ux, uy);
    r->eta = 1.0f;
    return par_rgb(b, 0, b->d.kd, r);
}
static v3 diffuse_eval(const bsdf_t *b, const brec *r) {
    if (r->measure != HO_MEASURE_SOLID_ANGLE || r->wi.z <= 0 || r->wo.z <= 0) return V(0, 0, 0);
    return scl(par_rgb(b, 0, b->d.kd, r), (float)INV_PI_D);
}
static float diffuse_pdf(const brec *r) {
    if (r->measure != HO_MEASURE_SOLID_ANGLE || r->wi.z <= 0 || r->wo.z <= 0) return 0.0f;
    return (float)INV_PI_D * r->wo.z;
}

/* RoughConductorBSDF  src/bsdf/RoughConductorBSDF.cpp:54-154 */
static v3 conductor_sample(const bsdf_t *b, brec *r, float ux, float uy) {
    r->measure = HO_MEASURE_SOLID_ANGLE;
    float ci = r->wi.z;
    if (ci <= 0.0f) return V(0, 0, 0);
    mfd d = mfd_make(b->d.distribution, alpha_u_of(b, r), alpha_v_of(b, r));
    float pdf;
    v3 m = mfd_sample(&d, ux, uy, &pdf);
    if (pdf == 0.0f) return V(0, 0, 0);
    r->wo = reflect_m(r->wi, m);
    r->eta = 1.0f;
    if (r->wo.z < 0.0f) return V(0, 0, 0);
    float mdw = dot(m, r->wi);
    v3 F = fresnel_conductor(mdw, b->eta_c, b->k_c);
    float G = mfd_g(&d, r->wi, r->wo, m);
    float D = mfd_eval(&d, m);
    v3 ks = par_rgb(b, 1, b->d.ks, r);
    float den = pdf * r->wi.z;
    return V((((ks.x * F.x) * D) * G) * mdw / den, (((ks.y * F.y) * D) * G) * mdw / den,
             (((ks.z * F.z) * D) * G) * mdw / den);
}
static v3 conductor_eval(const bsdf_t *b, const brec *r) {
    float ci = r->wi.z, co = r->wo.z;
    if (r->measure != HO_MEASURE_SOLID_ANGLE || ci <= 0.0f || co <= 0.0f) return V(0, 0, 0);
    v3 h = normalize(add(r->wi, r->wo));
    mfd d = mfd_make(b->d.distribution, alpha_u_of(b, r), alpha_v_of(b, r));
    float D = mfd_eval(&d, h);
    if (D == 0.0f) return V(0, 0, 0);
    v3 F = mul(fresnel_conductor(dot(h, r->wi), b->eta_c, b->k_c), par_rgb(b, 1, b->d.ks, r));
    float G = mfd_g(&d, r->wi, r->wo, h);
    float dg = D * G, den = 4.0f * ci;
    return V(dg * F.x / den, dg * F.y / den, dg * F.z / den);
}
static float conductor_pdf(const bsdf_t *b, const brec *r) {
    float ci = r->wi.z, co = r->wo.z;
    if (r->measure != HO_MEASURE_SOLID_ANGLE || ci <= 0.0f || co <= 0.0f) return 0.0f;
    v3 h = normalize(add(r->wi, r->wo));
    mfd d = mfd_make(b->d.distribution, alpha_u_of(b, r), alpha_v_of(b, r));
    return mfd_pdf(&d, h) / (4.0f * fabsf(dot(h, r->wo)));
}

/* RoughDielectricBSDF  src/bsdf/RoughDielectricBSDF.cpp:57-281 */
static v3 dielectric_sample(const bsdf_t *b, brec *r, float ux, float uy, ho_pcg32 *rng, const float *u1f) {
    r->measure = HO_MEASURE_SOLID_ANGLE;
    float ci = r->wi.z;
    if (ci == 0.0f) return V(0, 0, 0);
    mfd d = mfd_make(b->d.distribution, alpha_u_of(b, r), alpha_v_of(b, r));
    mfd sd = d;
    float s = 1.2f - 0.2f * sqrtf(fabsf(ci));
    sd.au *= s; sd.av *= s;                                    /* ScaleAlpha */
    float pdf;
    v3 m = mfd_sample(&sd, ux, uy, &pdf);
    if (pdf == 0.0f) return V(0, 0, 0);
    float ct;
    float F = fresnel_dielectric(dot(r->wi, m), b->eta, b->inv_eta, &ct);
    float u1;
    if (u1f) u1 = *u1f;
    else if (rng) u1 = ho_pcg32_nextf(rng);
    else { ho_pcg32 t; pcg_default(&t); u1 = ho_pcg32_nextf(&t); }   /* :96-100 null sampler */
    int refl = !(u1 > F);
    v3 W = V(1, 1, 1);
    if (refl) {
        r->wo = reflect_m(r->wi, m);
        r->eta = 1.0f;
        float co = r->wo.z;
        if (co * ci <= 0.0f) return V(0, 0, 0);
        W = mul(W, par_rgb(b, 1, b->d.ks, r));
    } else {
        if (ct == 0.0f) return V(0, 0, 0);
        r->wo = refract_m(r->wi, m, ct, b->eta, b->inv_eta);
        r->eta = (ct < 0.0f ? b->eta : b->inv_eta);
        float co = r->wo.z;
        if (co * ci >= 0.0f) return V(0, 0, 0);
        float fac = (ct < 0.0f ? b->inv_eta : b->eta);
        W = mul(W, scl(par_rgb(b, 2, b->d.ks_refract, r), fac * fac));
    }
    float v = fabsf(mfd_eval(&d, m) * mfd_g(&d, r->wi, r->wo, m) * dot(r->wi, m) / (pdf * ci));
    return scl(W, v);
}
static v3 dielectric_eval(const bsdf_t *b, const brec *r) {
    float ci = r->wi.z, co = r->wo.z;
    if (r->measure != HO_MEASURE_SOLID_ANGLE || ci == 0.0f) return V(0, 0, 0);
    int refl = ci * co > 0.0f;
    v3 h;
    if (refl) h = normalize(add(r->wi, r->wo));
    else { float e = ci > 0.0f ? b->eta : b->inv_eta; h = normalize(add(r->wi, scl(r->wo, e))); }
    h = scl(h, signum(h.z));
    mfd d = mfd_make(b->d.distribution, alpha_u_of(b, r), alpha_v_of(b, r));
    float D = mfd_eval(&d, h);
    if (D == 0.0f) return V(0, 0, 0);
    float ct;
    float F = fresnel_dielectric(dot(r->wi, h), b->eta, b->inv_eta, &ct);
    float G = mfd_g(&d, r->wi, r->wo, h);
    if (refl) return scl(par_rgb(b, 1, b->d.ks, r), F * D * G / (4.0f * fabsf(ci)));
    float e = ci > 0.0f ? b->eta : b->inv_eta;
    float sd = dot(r->wi, h) + e * dot(r->wo, h);
    float val = ((1.0f - F) * D * G * e * e * dot(r->wi, h) * dot(r->wo, h)) / (ci * sd * sd);
    float fac = (ci < 0.0f ? b->inv_eta : b->eta);
    return scl(par_rgb(b, 2, b->d.ks_refract, r), fabsf(val * fac * fac));
}
static float dielectric_pdf(const bsdf_t *b, const brec *r) {
    if (r->measure != HO_MEASURE_SOLID_ANGLE) return 0.0f;
    float ci = r->wi.z, co = r->wo.z;
    if (ci == 0.0f || co == 0.0f) return 0.0f;
    int refl = ci * co > 0.0f;
    v3 h; float J;
    if (refl) { h = normalize(add(r->wi, r->wo)); J = 1.0f / (4.0f * dot(r->wo, h)); }
    else {
        float e = ci > 0.0f ? b->eta : b->inv_eta;
        h = normalize(add(r->wi, scl(r->wo, e)));
        float sd = dot(r->wi, h) + e * dot(r->wo, h);
        J = (e * e * dot(r->wo, h)) / (sd * sd);
    }
    h = scl(h, signum(h.z));
    mfd d = mfd_make(b->d.distribution, alpha_u_of(b, r), alpha_v_of(b, r));
    float s = 1.2f - 0.2f * sqrtf(fabsf(ci));
    d.au *= s; d.av *= s;
    float ct;
    float F = fresnel_dielectric(dot(r->wi, h), b->eta, b->inv_eta, &ct);
    float pdf = mfd_pdf(&d, h) * (refl ? F : (1.0f - F));
    return fabsf(pdf * J);
}

/* RoughPlasticBSDF  src/bsdf/RoughPlasticBSDF.cpp:66-192 */
static v3 plastic_eval(const bsdf_t *b, const brec *r) {
    float ci = r->wi.z, co = r->wo.z;
    if (r->measure == HO_MEASURE_UNKNOWN || ci <= 0.0f || co <= 0.0f) return V(0, 0, 0);
    float a = alpha_u_of(b, r);
    mfd d = mfd_make(b->d.distribution, a, a);
    float ct;
    v3 h = normalize(add(r->wi, r->wo));
    float D = mfd_eval(&d, h);
    float F = fresnel_dielectric(dot(r->wi, h), b->eta, b->inv_eta, &ct);
    float G = mfd_g(&d, r->wi, r->wi, h);                     /* G(Wi, Wi, H) as in :146 */
    float val = F * D * G / (4.0f * ci);
    v3 res = scl(par_rgb(b, 1, b->d.ks, r), val);
    v3 dif = par_rgb(b, 0, b->d.kd, r);
    float t12 = rft_b(b, ci, d.au);
    float t21 = rft_b(b, co, d.au);
    float fdr = fdr_b(b, d.au);
    if (b->d.nonlinear) dif = V(dif.x / (1.0f - dif.x * fdr), dif.y / (1.0f - dif.y * fdr), dif.z / (1.0f - dif.z * fdr));
    else dif = divs(dif, 1.0f - fdr);
    float k = (float)(INV_PI_D * co * t12 * t21 * b->inv_eta2);
    return add(res, scl(dif, k));
}
static float plastic_spec_pdf(const bsdf_t *b, float ci, float alpha) {
    float sp = 1.0f - rft_b(b, ci, alpha);
    return (sp * b->spec_w) / (sp * b->spec_w + (1.0f - sp) * (1.0f - b->spec_w));
}
static float plastic_pdf(const bsdf_t *b, const brec *r) {
    float ci = r->wi.z, co = r->wo.z;
    if (r->measure == HO_MEASURE_UNKNOWN || ci <= 0.0f || co <= 0.0f) return 0.0f;
    float a = alpha_u_of(b, r);
    mfd d = mfd_make(b->d.distribution, a, a);
    v3 h = normalize(add(r->wi, r->wo));
    float sp = plastic_spec_pdf(b, ci, d.au), dp = 1.0f - sp;
    float J = 1.0f / (4.0f * dot(r->wo, h));
    float res = mfd_pdf(&d, h) * J * sp;
    res += dp * cos_hemi_pdf(r->wo);
    return res;
}
static v3 plastic_sample(const bsdf_t *b, brec *r, float ux, float uy) {
    float ci = r->wi.z;
    if (ci <= 0.0f) return V(0, 0, 0);
    float a = alpha_u_of(b, r);
    mfd d = mfd_make(b->d.distribution, a, a);
    float sp = plastic_spec_pdf(b, ci, d.au), dp = 1.0f - sp;
    int spec;
    if (uy < sp) { uy /= sp; spec = 1; }
    else { uy = (uy - sp) / (1.0f - sp); spec = 0; }
    if (spec) {
        float pdf;
        v3 m = mfd_sample(&d, ux, uy, &pdf);
        r->wo = reflect_m(r->wi, m);
        r->measure = HO_MEASURE_DISCRETE;
    } else {
        r->wo = square_to_cos_hemi(ux, uy);
        r->measure = HO_MEASURE_SOLID_ANGLE;
    }
    r->eta = 1.0f;
    v3 h = normalize(add(r->wi, r->wo));
    float J = 1.0f / (4.0f * dot(r->wo, h));
    float P = mfd_pdf(&d, h) * J * sp + dp * cos_hemi_pdf(r->wo);
    if (P == 0.0f) return V(0, 0, 0);
    return divs(plastic_eval(b, r), P);
}

/* RoughCoatingBSDF  src/bsdf/RoughCoatingBSDF.cpp:62-385 */
static v3 coat_refract(v3 wi, float inv_eta) {   /* RefractIn :347 (RefractOut :367 with eta) */
    float ci = wi.z;
    int entering = ci > 0.0f;
    float st2 = inv_eta * inv_eta * sin_theta2(wi);
    if (st2 >= 1.0f) return V(0, 0, 0);
    float ct = sqrtf(1.0f - st2);
    return V(inv_eta * wi.x, inv_eta * wi.y, entering ? ct : -ct);
}
static v3 coating_eval(const ho_scene *s, const bsdf_t *b, const brec *r) {
    float ci = r->wi.z, co = r->wo.z;
    if (ci * co <= 0.0f) return V(0, 0, 0);
    float a = alpha_u_of(b, r);
    mfd d = mfd_make(b->d.distribution, a, a);
    v3 h = scl(normalize(add(r->wi, r->wo)), signum(r->wo.z));
    float ct;
    float D = mfd_eval(&d, h);
    float F = fresnel_dielectric(fabsf(dot(r->wi, h)), b->eta, b->inv_eta, &ct);
    float G = mfd_g(&d, r->wi, r->wo, h);
    v3 ks = par_rgb(b, 1, b->d.ks, r);
    float den = 4.0f * fabsf(ci);
    v3 res = V((((ks.x * F) * D) * G) / den, (((ks.y * F) * D) * G) / den, (((ks.z * F) * D) * G) / den);
    brec ri = *r;
    ri.wi = coat_refract(r->wi, b->inv_eta);
    ri.wo = coat_refract(r->wo, b->inv_eta);
    v3 nv = bsdf_eval(s, b->d.nested, &ri);
    float ti = rft_b(b, fabsf(ci), d.au), to = rft_b(b, fabsf(co), d.au);
    nv = V(nv.x * ti * to, nv.y * ti * to, nv.z * ti * to);
    v3 sa = scl(par_rgb(b, 3, b->d.sigma_a, r), b->d.thickness);
    if (!is_zero(sa)) {
        float q = 1.0f / fabsf(ri.wi.z) + 1.0f / fabsf(ri.wo.z);
        nv = mul(nv, V(expf(-sa.x * q), expf(-sa.y * q), expf(-sa.z * q)));
    }
    if (r->measure == HO_MEASURE_SOLID_ANGLE) nv = scl(nv, b->inv_eta * b->inv_eta * r->wo.z / ri.wo.z);
    return add(res, nv);
}
static float coating_pdf(const ho_scene *s, const bsdf_t *b, const brec *r) {
    v3 h = scl(normalize(add(r->wi, r->wo)), signum(r->wo.z));
    float a = alpha_u_of(b, r);
    mfd d = mfd_make(b->d.distribution, a, a);
    float ci = r->wi.z, co = r->wo.z;
    float r12 = 1.0f - rft_b(b, fabsf(ci), d.au);
    float sp = (r12 * b->spec_w) / (r12 * b->spec_w + (1.0f - r12) * (1.0f - b->spec_w));
    float np = 1.0f - sp;
    float res = 0.0f;
    if (ci * co > 0.0f) {
        float J = 1.0f / (4.0f * fabsf(dot(r->wo, h)));
        res = mfd_pdf(&d, h) * J * sp;
    }
    brec ri = *r;
    ri.wi = coat_refract(r->wi, b->inv_eta);
    ri.wo = coat_refract(r->wo, b->inv_eta);
    float p = bsdf_pdf(s, b->d.nested, &ri);
    if (ri.measure == HO_MEASURE_SOLID_ANGLE) p *= b->inv_eta * b->inv_eta * co / ri.wo.z;
    return res + p * np;
}
static v3 coating_sample(const ho_scene *s, const bsdf_t *b, brec *r, float ux, float uy, ho_pcg32 *rng,
                         const float *u1f) {
    float a = alpha_u_of(b, r);
    mfd d = mfd_make(b->d.distribution, a, a);
    float aci = fabsf(r->wi.z);
    float r12 = 1.0f - rft_b(b, aci, d.au);
    float sp = (r12 * b->spec_w) / (r12 * b->spec_w + (1.0f - r12) * (1.0f - b->spec_w));
    int spec;
    if (ux < sp) { spec = 1; ux /= sp; }
    else { spec = 0; ux = (ux - sp) / (1.0f - sp); }
    if (spec) {
        float pdf;
        v3 m = mfd_sample(&d, ux, uy, &pdf);
        r->wo = reflect_m(r->wi, m);
        r->measure = HO_MEASURE_DISCRETE;
        r->eta = 1.0f;
        if (r->wo.z * r->wo.z <= 0.0f) return V(0, 0, 0);
    } else {
        v3 wib = r->wi;
        r->wi = coat_refract(r->wi, b->inv_eta);
        v3 res = bsdf_sample(s, b->d.nested, r, ux, uy, rng, u1f);
        r->wi = wib;
        if (is_zero(res)) return V(0, 0, 0);
        r->wo = coat_refract(r->wo, b->eta);
        if (is_zero(r->wo)) return V(0, 0, 0);
    }
    float P = coating_pdf(s, b, r);
    if (P == 0.0f) return V(0, 0, 0);
    return divs(coating_eval(s, b, r), P);
}

/* ------------------------------------------------------- smooth BSDFs */
/* Delta-direction match |d . wo - 1| <= DeltaEpsilon (include/core/Common.hpp:46).
 * DeltaEpsilon is the double literal 1e-3: the comparison is made in double. */
static inline int delta_match(v3 d, v3 wo) { return (double)fabsf(dot(d, wo) - 1.0f) <= 1e-3; }
/* Reflect / Refract about the local normal  src/core/Common.cpp:606-615 */
static inline v3 reflect_n(v3 wi) { return V(-wi.x, -wi.y, wi.z); }
static inline v3 refract_n(v3 wi, float ct, float eta, float inv_eta) {
    float sc = -(ct < 0.0f ? inv_eta : eta);
    return V(sc * wi.x, sc * wi.y, ct);
}
/* ApproxFresnelDiffuseReflectance  src/core/Common.cpp:550: the published fits of
 * Egan & Hilgeman (1973) for eta < 1 and d'Eon & Irving (2011) otherwise. */
static float approx_fresnel_diffuse(float e) {
    if (e < 1.0f) return -1.4399f * (e * e) + 0.7099f * e + 0.6681f + 0.0636f / e;
    float i1 = 1.0f / e, i2 = i1 * i1, i3 = i2 * i1, i4 = i3 * i1, i5 = i4 * i1;
    return 0.919317f - 3.4793f * i1 + 6.75335f * i2 - 7.80989f * i3 + 4.98554f * i4 - 1.36881f * i5;
}

/* MirrorBSDF  src/bsdf/MirrorBSDF.cpp:15-55 (the measure is set only past the cosine test) */
static int mirror_match(const brec *r) {
    return r->wi.z > 0.0f && r->wo.z > 0.0f && r->measure == HO_MEASURE_DISCRETE && delta_match(reflect_n(r->wi), r->wo);
}
static v3 mirror_sample(brec *r) {
    if (r->wi.z <= 0) return V(0, 0, 0);
    r->wo = reflect_n(r->wi);
    r->measure = HO_MEASURE_DISCRETE;
    r->eta = 1.0f;
    return V(1, 1, 1);
}
static v3 mirror_eval(const brec *r) { return mirror_match(r) ? V(1, 1, 1) : V(0, 0, 0); }
static float mirror_pdf(const brec *r) { return mirror_match(r) ? 1.0f : 0.0f; }

/* ConductorBSDF  src/bsdf/ConductorBSDF.cpp:32-70 (eta = intIOR/extIOR on every channel) */
static v3 sconductor_sample(const bsdf_t *b, brec *r) {
    r->measure = HO_MEASURE_DISCRETE;
    float ci = r->wi.z;
    if (ci <= 0.0f) return V(0, 0, 0);
    v3 F = fresnel_conductor(ci, b->eta_c, b->k_c);
    r->wo = reflect_n(r->wi);
    r->eta = 1.0f;
    return mul(par_rgb(b, 1, b->d.ks, r), F);
}
static v3 sconductor_eval(const bsdf_t *b, const brec *r) {
    if (!mirror_match(r)) return V(0, 0, 0);
    return mul(par_rgb(b, 1, b->d.ks, r), fresnel_conductor(r->wi.z, b->eta_c, b->k_c));
}
static float sconductor_pdf(const brec *r) { return mirror_match(r) ? 1.0f : 0.0f; }

/* DielectricBSDF  src/bsdf/DielectricBSDF.cpp:33-110 (Eval and Pdf test no measure) */
static v3 sdielectric_sample(const bsdf_t *b, brec *r, float ux) {
    r->measure = HO_MEASURE_DISCRETE;
    float ct;
    float F = fresnel_dielectric(r->wi.z, b->eta, b->inv_eta, &ct);
    if (ux < F) {
        r->wo = reflect_n(r->wi);
        r->eta = 1.0f;
        return par_rgb(b, 1, b->d.ks, r);
    }
    r->wo = refract_n(r->wi, ct, b->eta, b->inv_eta);
    r->eta = ct < 0.0f ? b->eta : b->inv_eta;
    float f = ct < 0.0f ? b->inv_eta : b->eta;   /* radiance transport */
    return scl(par_rgb(b, 2, b->d.ks_refract, r), f * f);
}
static v3 sdielectric_eval(const bsdf_t *b, const brec *r) {
    float ci = r->wi.z, co = r->wo.z, ct;
    float F = fresnel_dielectric(ci, b->eta, b->inv_eta, &ct);
    if (ci * co >= 0.0f) {
        if (delta_match(reflect_n(r->wi), r->wo)) return scl(par_rgb(b, 1, b->d.ks, r), F);
    } else if (delta_match(refract_n(r->wi, ct, b->eta, b->inv_eta), r->wo)) {
        float f = ct < 0.0f ? b->inv_eta : b->eta;
        return scl(scl(par_rgb(b, 2, b->d.ks_refract, r), f * f), 1.0f - F);
    }
    return V(0, 0, 0);
}
static float sdielectric_pdf(const bsdf_t *b, const brec *r) {
    float ci = r->wi.z, co = r->wo.z, ct;
    float F = fresnel_dielectric(ci, b->eta, b->inv_eta, &ct);
    if (ci * co >= 0.0f) {
        if (delta_match(reflect_n(r->wi), r->wo)) return F;
    } else if (delta_match(refract_n(r->wi, ct, b->eta, b->inv_eta), r->wo)) {
        return 1.0f - F;
    }
    return 0.0f;
}

/* PlasticBSDF  src/bsdf/PlasticBSDF.cpp:33-142 */
static float splastic_spec_pdf(const bsdf_t *b, float Fi) {
    return (Fi * b->spec_w) / (Fi * b->spec_w + (1.0f - Fi) * (1.0f - b->spec_w));
}
static v3 splastic_diffuse(const bsdf_t *b, const brec *r) {
    v3 dif = par_rgb(b, 0, b->d.kd, r);
    float fdr = b->fdr_int;
    if (b->d.nonlinear) return V(dif.x / (1.0f - dif.x * fdr), dif.y / (1.0f - dif.y * fdr), dif.z / (1.0f - dif.z * fdr));
    return divs(dif, 1.0f - fdr);
}
static v3 splastic_sample(const bsdf_t *b, brec *r, float ux, float uy) {
    float ci = r->wi.z;
    if (ci <= 0.0f) return V(0, 0, 0);
    float ct;
    float Fi = fresnel_dielectric(ci, b->eta, b->inv_eta, &ct);
    float sp = splastic_spec_pdf(b, Fi);
    r->eta = 1.0f;
    if (ux < sp) {
        r->measure = HO_MEASURE_DISCRETE;
        r->wo = reflect_n(r->wi);
        return divs(scl(par_rgb(b, 1, b->d.ks, r), Fi), sp);
    }
    r->measure = HO_MEASURE_SOLID_ANGLE;
    r->wo = square_to_cos_hemi((ux - sp) / (1.0f - sp), uy);
    float Fo = fresnel_dielectric(r->wo.z, b->eta, b->inv_eta, &ct);
    return scl(splastic_diffuse(b, r), b->inv_eta2 * (1.0f - Fi) * (1.0f - Fo) / (1.0f - sp));
}
static v3 splastic_eval(const bsdf_t *b, const brec *r) {
    float ci = r->wi.z, co = r->wo.z;
    if (r->measure == HO_MEASURE_UNKNOWN || ci <= 0.0f || co <= 0.0f) return V(0, 0, 0);
    float ct;
    float Fi = fresnel_dielectric(ci, b->eta, b->inv_eta, &ct);
    if (r->measure == HO_MEASURE_DISCRETE)
        return delta_match(reflect_n(r->wi), r->wo) ? scl(par_rgb(b, 1, b->d.ks, r), Fi) : V(0, 0, 0);
    float Fo = fresnel_dielectric(co, b->eta, b->inv_eta, &ct);
    return scl(splastic_diffuse(b, r), cos_hemi_pdf(r->wo) * b->inv_eta2 * (1.0f - Fi) * (1.0f - Fo));
}
static float splastic_pdf(const bsdf_t *b, const brec *r) {
    float ci = r->wi.z, co = r->wo.z;
    if (r->measure == HO_MEASURE_UNKNOWN || ci <= 0.0f || co <= 0.0f) return 0.0f;
    float ct;
    float Fi = fresnel_dielectric(ci, b->eta, b->inv_eta, &ct);
    float sp = splastic_spec_pdf(b, Fi);
    if (r->measure == HO_MEASURE_DISCRETE)
        return delta_match(reflect_n(r->wi), r->wo) ? 1.0f - sp : 0.0f;   /* 1 - SpecularPDF, as :118 */
    return cos_hemi_pdf(r->wo) * (1.0f - sp);
}

/* CoatingBSDF  src/bsdf/CoatingBSDF.cpp:28-302: a smooth dielectric layer over a nested BSDF */
static v3 scoat_refract_in(const bsdf_t *b, v3 wi, float *R) {   /* RefractIn :290 */
    float ct;
    *R = fresnel_dielectric(fabsf(wi.z), b->eta, b->inv_eta, &ct);
    return V(b->inv_eta * wi.x, b->inv_eta * wi.y, -signum(wi.z) * ct);
}
static v3 scoat_refract_out(const bsdf_t *b, v3 wi, float *R) {   /* RefractOut :297 */
    float ct;
    *R = fresnel_dielectric(fabsf(wi.z), b->inv_eta, b->eta, &ct);
    return V(b->eta * wi.x, b->eta * wi.y, -signum(wi.z) * ct);
}
static v3 scoat_absorb(const bsdf_t *b, const brec *r, v3 res, v3 wi_int, v3 wo_int) {
    v3 sa = scl(par_rgb(b, 3, b->d.sigma_a, r), b->d.thickness);
    if (is_zero(sa)) return res;
    float q = 1.0f / fabsf(wi_int.z) + 1.0f / fabsf(wo_int.z);
    return mul(res, V(expf(-sa.x * q), expf(-sa.y * q), expf(-sa.z * q)));
}
static float scoat_spec_pdf(const bsdf_t *b, float R12) {
    return (R12 * b->spec_w) / (R12 * b->spec_w + (1.0f - R12) * (1.0f - b->spec_w));
}
static v3 scoating_sample(const ho_scene *s, const bsdf_t *b, brec *r, float ux, float uy, ho_pcg32 *rng,
                          const float *u1f) {
    float R12;
    v3 wip = scoat_refract_in(b, r->wi, &R12);
    float sp = scoat_spec_pdf(b, R12);
    if (ux < sp) {
        r->wo = reflect_n(r->wi);
        r->eta = 1.0f;
        r->measure = HO_MEASURE_DISCRETE;
        return scl(par_rgb(b, 1, b->d.ks, r), R12 / sp);
    }
    ux = (ux - sp) / (1.0f - sp);
    if (R12 == 1.0f) return V(0, 0, 0);
    v3 wib = r->wi;
    r->wi = wip;
    v3 res = bsdf_sample(s, b->d.nested, r, ux, uy, rng, u1f);
    r->wi = wib;
    if (is_zero(res)) return V(0, 0, 0);
    v3 wop = r->wo;
    res = scoat_absorb(b, r, res, wip, wop);
    float R21;
    r->wo = scoat_refract_out(b, wop, &R21);
    if (R21 == 1.0f) return V(0, 0, 0);
    res = divs(res, 1.0f - sp);
    return scl(res, (1.0f - R12) * (1.0f - R21));
}
static v3 scoating_eval(const ho_scene *s, const bsdf_t *b, const brec *r) {
    if (r->measure == HO_MEASURE_DISCRETE) {
        if (!delta_match(reflect_n(r->wi), r->wo)) return V(0, 0, 0);
        float ct;
        return scl(par_rgb(b, 1, b->d.ks, r), fresnel_dielectric(fabsf(r->wi.z), b->eta, b->inv_eta, &ct));
    }
    float R12, R21;
    brec ri = *r;
    ri.wi = scoat_refract_in(b, r->wi, &R12);
    ri.wo = scoat_refract_in(b, r->wo, &R21);
    if (R12 == 1.0f || R21 == 1.0f) return V(0, 0, 0);
    v3 res = scl(scl(bsdf_eval(s, b->d.nested, &ri), 1.0f - R12), 1.0f - R21);
    res = scoat_absorb(b, r, res, ri.wi, ri.wo);
    if (r->measure == HO_MEASURE_SOLID_ANGLE) res = scl(res, b->inv_eta * b->inv_eta * r->wo.z / ri.wo.z);
    return res;
}
static float scoating_pdf(const ho_scene *s, const bsdf_t *b, const brec *r) {
    float R12;
    v3 wip = scoat_refract_in(b, r->wi, &R12);
    float sp = scoat_spec_pdf(b, R12);
    if (r->measure == HO_MEASURE_DISCRETE) return delta_match(reflect_n(r->wi), r->wo) ? sp : 0.0f;
    float R21;
    brec ri = *r;
    ri.wi = wip;
    ri.wo = scoat_refract_in(b, r->wo, &R21);
    if (R12 == 1.0f || R21 == 1.0f) return 0.0f;
    float p = bsdf_pdf(s, b->d.nested, &ri);
    if (r->measure == HO_MEASURE_SOLID_ANGLE) p *= b->inv_eta * b->inv_eta * r->wo.z / ri.wo.z;
    return p * (1.0f - sp);
}

/* RoughDiffuseBSDF  src/bsdf/RoughDiffuseBSDF.cpp:19-140 (Oren-Nayar, full model or fast approximation) */
static inline float max_f(float a, float b) { return (a < b) ? b : a; }   /* std::max */
static inline float min_f(float a, float b) { return (b < a) ? b : a; }   /* std::min */
static inline float safe_acos(float v) { return acosf(min_f(1.0f, max_f(-1.0f, v))); }
static inline float safe_sqrt(float v) { return sqrtf(max_f(0.0f, v)); }
static inline float frame_sin_theta(v3 v) {   /* Frame::SinTheta  src/core/Frame.cpp:38 */
    float t = sin_theta2(v);
    return t <= 0.0f ? 0.0f : sqrtf(t);
}
static inline float frame_sin_phi(v3 v) {   /* :68 */
    float t = frame_sin_theta(v);
    return t == 0.0f ? 1.0f : clampf(v.y / t, -1.0f, 1.0f);
}
static inline float frame_cos_phi(v3 v) {   /* :78 */
    float t = frame_sin_theta(v);
    return t == 0.0f ? 1.0f : clampf(v.x / t, -1.0f, 1.0f);
}
static v3 roughdiffuse_eval(const bsdf_t *b, const brec *r) {
    float ci = r->wi.z, co = r->wo.z;
    if (ci <= 0.0f || co <= 0.0f || r->measure != HO_MEASURE_SOLID_ANGLE) return V(0, 0, 0);
    float sigma = clampf(par_alpha(b, 4, b->d.alpha_u, r), 5e-4f, 1.0f) * 0.70710678118655f;
    float s2 = sigma * sigma;
    float sti = frame_sin_theta(r->wi), sto = frame_sin_theta(r->wo);
    float cpd = 0.0f;
    if (sti > 1e-4f && sto > 1e-4f) {
        float spi = frame_sin_phi(r->wi), cpi = frame_cos_phi(r->wi);
        float spo = frame_sin_phi(r->wo), cpo = frame_cos_phi(r->wo);
        cpd = cpi * cpo + spi * spo;
    }
    const float inv_pi = (float)INV_PI_D;
    if (b->d.fast_approx) {
        float A = 1.0f - 0.5f * s2 / (s2 + 0.33f);
        float B = 0.45f * s2 / (s2 + 0.09f);
        float sa, tb;
        if (ci > co) { sa = sto; tb = sti / ci; }
        else { sa = sti; tb = sto / co; }
        return scl(par_rgb(b, 0, b->d.kd, r), inv_pi * co * (A + B * max_f(cpd, 0.0f) * sa * tb));
    }
    float thi = safe_acos(ci), tho = safe_acos(co);
    float al = max_f(thi, tho), be = min_f(thi, tho);
    float sa, sb, tb;
    if (ci > co) { sa = sto; sb = sti; tb = sti / ci; }
    else { sa = sti; sb = sto; tb = sto / co; }
    float t1 = s2 / (s2 + 0.09f);
    float t2 = (4.0f * (float)(INV_PI_D * INV_PI_D)) * al * be;
    float t3 = 2.0f * be * inv_pi;
    float C1 = 1.0f - 0.5f * s2 / (s2 + 0.33f);
    float C2 = 0.45f * t1;
    float C3 = 0.125f * t1 * t2 * t2;
    float C4 = 0.17f * s2 / (s2 + 0.13f);
    if (cpd > 0.0f) C2 *= sa;
    else C2 *= sa - t3 * t3 * t3;
    float th = (sa + sb) / (safe_sqrt(1.0f - sa * sa) + safe_sqrt(1.0f - sb * sb));
    if (isinf(th) || isnan(th)) return V(0, 0, 0);
    v3 rho = par_rgb(b, 0, b->d.kd, r);
    v3 lr1 = scl(rho, C1 + cpd * C2 * tb + (1.0f - fabsf(cpd)) * C3 * th);
    v3 lr2 = scl(mul(rho, rho), C4 * (1.0f - cpd * t3 * t3));
    return scl(add(lr1, lr2), inv_pi * co);
}
static float roughdiffuse_pdf(const brec *r) {
    if (r->wi.z <= 0.0f || r->wo.z <= 0.0f || r->measure != HO_MEASURE_SOLID_ANGLE) return 0.0f;
    return cos_hemi_pdf(r->wo);
}
static v3 roughdiffuse_sample(const bsdf_t *b, brec *r, float ux, float uy) {
    r->measure = HO_MEASURE_SOLID_ANGLE;
    if (r->wi.z <= 0.0f) return V(0, 0, 0);
    r->wo = square_to_cos_hemi(ux, uy);
    r->eta = 1.0f;
    float pdf = cos_hemi_pdf(r->wo);
    if (pdf == 0.0f) return V(0, 0, 0);
    return divs(roughdiffuse_eval(b, r), pdf);
}

/* TwoSidedBSDF  src/bsdf/TwoSidedBSDF.cpp:19-67: the back side mirrors z into the second BSDF */
static v3 twosided_sample(const ho_scene *s, const bsdf_t *b, brec *r, float ux, float uy, ho_pcg32 *rng,
                          const float *u1f) {
    int flip = r->wi.z < 0.0f;
    if (flip) r->wi.z *= -1.0f;
    v3 res = bsdf_sample(s, flip ? b->d.nested2 : b->d.nested, r, ux, uy, rng, u1f);
    if (flip) {
        r->wi.z *= -1.0f;
        if (!is_zero(res)) r->wo.z *= -1.0f;
    }
    return res;
}
static v3 twosided_eval(const ho_scene *s, const bsdf_t *b, const brec *r) {
    brec c = *r;
    if (c.wi.z > 0.0f) return bsdf_eval(s, b->d.nested, &c);
    c.wi.z *= -1.0f;
    c.wo.z *= -1.0f;
    return bsdf_eval(s, b->d.nested2, &c);
}
static float twosided_pdf(const ho_scene *s, const bsdf_t *b, const brec *r) {
    brec c = *r;
    if (c.wi.z > 0.0f) return bsdf_pdf(s, b->d.nested, &c);
    c.wi.z *= -1.0f;
    c.wo.z *= -1.0f;
    return bsdf_pdf(s, b->d.nested2, &c);
}

/* BumpMapBSDF::GetPerturbebFrame (src/bsdf/BumpMapBSDF.cpp:172) and
 * NormalMapBSDF::GetPerturbebFrame (src/bsdf/NormalMapBSDF.cpp:169) */
static frame perturbed_frame(const ho_scene *s, const bsdf_t *b, const isect_t *it) {
    frame f;
    const int tid = b->d.tex[0] - 1;
    if (b->d.type == HO_BSDF_BUMP_MAP) {
        v3 g[2];
        tex_gradient(s->tex, s->mips, tid, it->uv, g);
        float ddu = lum(g[0]), ddv = lum(g[1]);
        v3 n = it->sh.n;
        v3 dpdu = add(it->dpdu, scl(n, ddu - dot(n, it->dpdu)));
        v3 dpdv = add(it->dpdv, scl(n, ddv - dot(n, it->dpdv)));
        f.n = normalize(cross(dpdu, dpdv));
        f.s = normalize(sub(dpdu, scl(f.n, dot(f.n, dpdu))));
        f.t = cross(f.n, f.s);
        if (dot(f.n, it->geo.n) < 0.0f) f.n = scl(f.n, -1.0f);
    } else {
        v3 c = tex_eval(s->tex, s->mips, tid, it->uv, NULL, it);   /* Eval(Isect, false) */
        v3 nn = V(2.0f * c.x - 1.0f, 2.0f * c.y - 1.0f, 2.0f * c.z - 1.0f);
        f.n = normalize(to_world(&it->sh, nn));
        f.s = normalize(sub(it->dpdu, scl(f.n, dot(f.n, it->dpdu))));
        f.t = cross(f.n, f.s);
    }
    return f;
}
/* BumpMapBSDF / NormalMapBSDF Eval, Pdf (:56, :80): the record moved into the
 * perturbed frame, zero where a direction changes side */
static int perturb_record(const ho_scene *s, const bsdf_t *b, const brec *r, brec *q, frame *pf) {
    *pf = perturbed_frame(s, b, r->it);
    *q = *r;
    q->wi = to_local(pf, to_world(&r->it->sh, r->wi));
    q->wo = to_local(pf, to_world(&r->it->sh, r->wo));
    return !(r->wo.z * q->wo.z <= 0.0f || r->wi.z * q->wi.z <= 0.0f);
}
static v3 bump_eval(const ho_scene *s, const bsdf_t *b, const brec *r) {
    brec q; frame pf;
    if (!perturb_record(s, b, r, &q, &pf)) return V(0, 0, 0);
    return bsdf_eval(s, b->d.nested, &q);
}
static float bump_pdf(const ho_scene *s, const bsdf_t *b, const brec *r) {
    brec q; frame pf;
    if (!perturb_record(s, b, r, &q, &pf)) return 0.0f;
    return bsdf_pdf(s, b->d.nested, &q);
}
/* BumpMapBSDF::Sample (:22) */
static v3 bump_sample(const ho_scene *s, const bsdf_t *b, brec *r, float ux, float uy, ho_pcg32 *rng, const float *u1f) {
    frame pf = perturbed_frame(s, b, r->it);
    brec q = *r;
    q.wi = to_local(&pf, to_world(&r->it->sh, r->wi));
    q.wo = V(0, 0, 0);
    q.measure = HO_MEASURE_UNKNOWN;
    if (r->wi.z * q.wi.z <= 0.0f) return V(0, 0, 0);
    v3 res = bsdf_sample(s, b->d.nested, &q, ux, uy, rng, u1f);
    if (!is_zero(res)) {
        r->wo = to_local(&r->it->sh, to_world(&pf, q.wo));
        r->eta = q.eta;
        r->measure = q.measure;
        if (r->wo.z * q.wo.z <= 0.0f) return V(0, 0, 0);
    }
    return res;
}
static v3 bsdf_eval(const ho_scene *s, int id, const brec *r) {
    const bsdf_t *b = &s->bsdfs[id];
    switch (b->d.type) {
    case HO_BSDF_BUMP_MAP: case HO_BSDF_NORMAL_MAP: return bump_eval(s, b, r);
    case HO_BSDF_DIFFUSE: return diffuse_eval(b, r);
    case HO_BSDF_ROUGH_CONDUCTOR: return conductor_eval(b, r);
    case HO_BSDF_ROUGH_DIELECTRIC: return dielectric_eval(b, r);
    case HO_BSDF_ROUGH_PLASTIC: return plastic_eval(b, r);
    case HO_BSDF_ROUGH_COATING: return coating_eval(s, b, r);
    case HO_BSDF_MIRROR: return mirror_eval(r);
    case HO_BSDF_CONDUCTOR: return sconductor_eval(b, r);
    case HO_BSDF_DIELECTRIC: return sdielectric_eval(b, r);
    case HO_BSDF_PLASTIC: return splastic_eval(b, r);
    case HO_BSDF_COATING: return scoating_eval(s, b, r);
    case HO_BSDF_ROUGH_DIFFUSE: return roughdiffuse_eval(b, r);
    default: return twosided_eval(s, b, r);
    }
}
static float bsdf_pdf(const ho_scene *s, int id, const brec *r) {
    const bsdf_t *b = &s->bsdfs[id];
    switch (b->d.type) {
    case HO_BSDF_BUMP_MAP: case HO_BSDF_NORMAL_MAP: return bump_pdf(s, b, r);
    case HO_BSDF_DIFFUSE: return diffuse_pdf(r);
    case HO_BSDF_ROUGH_CONDUCTOR: return conductor_pdf(b, r);
    case HO_BSDF_ROUGH_DIELECTRIC: return dielectric_pdf(b, r);
    case HO_BSDF_ROUGH_PLASTIC: return plastic_pdf(b, r);
    case HO_BSDF_ROUGH_COATING: return coating_pdf(s, b, r);
    case HO_BSDF_MIRROR: return mirror_pdf(r);
    case HO_BSDF_CONDUCTOR: return sconductor_pdf(r);
    case HO_BSDF_DIELECTRIC: return sdielectric_pdf(b, r);
    case HO_BSDF_PLASTIC: return splastic_pdf(b, r);
    case HO_BSDF_COATING: return scoating_pdf(s, b, r);
    case HO_BSDF_ROUGH_DIFFUSE: return roughdiffuse_pdf(r);
    default: return twosided_pdf(s, b, r);
    }
}
static v3 bsdf_sample(const ho_scene *s, int id, brec *r, float ux, float uy, ho_pcg32 *rng, const float *u1f) {
    const bsdf_t *b = &s->bsdfs[id];
    switch (b->d.type) {
    case HO_BSDF_BUMP_MAP: case HO_BSDF_NORMAL_MAP: return bump_sample(s, b, r, ux, uy, rng, u1f);
    case HO_BSDF_DIFFUSE: return diffuse_sample(b, r, ux, uy);
    case HO_BSDF_ROUGH_CONDUCTOR: return conductor_sample(b, r, ux, uy);
    case HO_BSDF_ROUGH_DIELECTRIC: return dielectric_sample(b, r, ux, uy, rng, u1f);
    case HO_BSDF_ROUGH_PLASTIC: return plastic_sample(b, r, ux, uy);
    case HO_BSDF_ROUGH_COATING: return coating_sample(s, b, r, ux, uy, rng, u1f);
    case HO_BSDF_MIRROR: return mirror_sample(r);
    case HO_BSDF_CONDUCTOR: return sconductor_sample(b, r);
    case HO_BSDF_DIELECTRIC: return sdielectric_sample(b, r, ux);
    case HO_BSDF_PLASTIC: return splastic_sample(b, r, ux, uy);
    case HO_BSDF_COATING: return scoating_sample(s, b, r, ux, uy, rng, u1f);
    case HO_BSDF_ROUGH_DIFFUSE: return roughdiffuse_sample(b, r, ux, uy);
    default: return twosided_sample(s, b, r, ux, uy, rng, u1f);
    }
}

void ho_bsdf_sample(const ho_scene *s, int id, const float *wi, const float *u2, float u1, float *owo,
                    float *ow, int *om, float *oeta) {
    brec r; memset(&r, 0, sizeof r);
    r.wi = vload(wi); r.measure = HO_MEASURE_UNKNOWN; r.eta = 0.0f;
    v3 w = bsdf_sample(s, id, &r, u2[0], u2[1], NULL, &u1);
    vstore(owo, r.wo); vstore(ow, w); *om = r.measure; *oeta = r.eta;
}
void ho_bsdf_eval(const ho_scene *s, int id, const float *wi, const float *wo, int measure, float *o) {
    brec r; memset(&r, 0, sizeof r); r.wi = vload(wi); r.wo = vload(wo); r.measure = measure; r.eta = 0.0f;
    vstore(o, bsdf_eval(s, id, &r));
}
float ho_bsdf_pdf(const ho_scene *s, int id, const float *wi, const float *wo, int measure) {
    brec r; memset(&r, 0, sizeof r); r.wi = vload(wi); r.wo = vload(wo); r.measure = measure; r.eta = 0.0f;
    return bsdf_pdf(s, id, &r);
}
float ho_bsdf_rft_eval(const ho_scene *s, int id, float c) {
    const bsdf_t *b = &s->bsdfs[id];
    return rft_eval1d(b->rft, b->rft_n, c);
}
static void bsdf_batch_any(const ho_scene *s, int id, uint64_t n, const float *wi, const float *u2, const float *u1,
                           const float *wo, const float *uv, const float *duv, const float *isect, float *s_wo,
                           float *s_w, float *s_pdf, int32_t *s_m, float *e_rgb, float *p_pdf, int nthreads);
void ho_bsdf_batch(const ho_scene *s, int id, uint64_t n, const float *wi, const float *u2, const float *u1,
                   const float *wo, const float *uv, const float *duv, float *s_wo, float *s_w, float *s_pdf, int32_t *s_m,
                   float *e_rgb, float *p_pdf, int nthreads) {
    bsdf_batch_any(s, id, n, wi, u2, u1, wo, uv, duv, NULL, s_wo, s_w, s_pdf, s_m, e_rgb, p_pdf, nthreads);
}
void ho_bsdf_batch_isect(const ho_scene *s, int id, uint64_t n, const float *wi, const float *u2, const float *u1,
                         const float *wo, const float *isect, float *s_wo, float *s_w, float *s_pdf, int32_t *s_m,
                         float *e_rgb, float *p_pdf, int nthreads) {
    bsdf_batch_any(s, id, n, wi, u2, u1, wo, NULL, NULL, isect, s_wo, s_w, s_pdf, s_m, e_rgb, p_pdf, nthreads);
}
static void bsdf_batch_any(const ho_scene *s, int id, uint64_t n, const float *wi, const float *u2, const float *u1,
                           const float *wo, const float *uv, const float *duv, const float *isect, float *s_wo,
                           float *s_w, float *s_pdf, int32_t *s_m, float *e_rgb, float *p_pdf, int nthreads) {
#ifdef _OPENMP
    if (nthreads > 0) omp_set_num_threads(nthreads);
#pragma omp parallel for schedule(static)
#endif
    for (int64_t i = 0; i < (int64_t)n; i++) {
        isect_t it; memset(&it, 0, sizeof it);
        if (isect) {   /* S T N, geometric N, dPdU, dPdV, UV */
            const float *q = isect + 20 * i;
            it.sh.s = vload(q); it.sh.t = vload(q + 3); it.sh.n = vload(q + 6); it.geo.n = vload(q + 9);
            it.dpdu = vload(q + 12); it.dpdv = vload(q + 15); it.uv[0] = q[18]; it.uv[1] = q[19];
            it.has_uvp = 1;
        }
        brec r; memset(&r, 0, sizeof r);
        r.it = isect ? &it : NULL;
        if (isect) { r.uv[0] = it.uv[0]; r.uv[1] = it.uv[1]; }
        r.wi = vload(wi + 3 * i); r.measure = HO_MEASURE_UNKNOWN;
        if (uv) { r.uv[0] = uv[2 * i]; r.uv[1] = uv[2 * i + 1]; }
        if (duv) memcpy(r.duv, duv + 4 * i, 4 * sizeof(float));
        float uu = u1 ? u1[i] : 0.0f;
        v3 w = bsdf_sample(s, id, &r, u2[2 * i], u2[2 * i + 1], NULL, &uu);
        if (s_wo) vstore(s_wo + 3 * i, r.wo);
        if (s_w) vstore(s_w + 3 * i, w);
        if (s_m) s_m[i] = r.measure;
        if (s_pdf) s_pdf[i] = is_zero(w) && w.x == 0 && w.y == 0 && w.z == 0 ? 0.0f : bsdf_pdf(s, id, &r);
        brec q; memset(&q, 0, sizeof q);
        q.it = r.it;
        q.uv[0] = r.uv[0]; q.uv[1] = r.uv[1];
        q.wi = vload(wi + 3 * i); q.wo = vload(wo + 3 * i); q.measure = HO_MEASURE_SOLID_ANGLE; q.eta = 0;
        if (uv) { q.uv[0] = uv[2 * i]; q.uv[1] = uv[2 * i + 1]; }
        if (duv) memcpy(q.duv, duv + 4 * i, 4 * sizeof(float));
        if (e_rgb) vstore(e_rgb + 3 * i, bsdf_eval(s, id, &q));
        if (p_pdf) p_pdf[i] = bsdf_pdf(s, id, &q);
    }
}

/* ------------------------------------------------------------ geometry */
/* Mesh::RayIntersect  src/core/Mesh.cpp:340 (Moller-Trumbore) */
static int tri_intersect(const ho_scene *s, uint32_t t, v3 o, v3 d, float mint, float maxt, float *ou,
                         float *ov, float *ot) {
    const uint32_t *f = s->F + 3ull * t;
    v3 p0 = vload(s->P + 3ull * f[0]), p1 = vload(s->P + 3ull * f[1]), p2 = vload(s->P + 3ull * f[2]);
    v3 e1 = sub(p1, p0), e2 = sub(p2, p0);
    v3 pv = cross(d, e2);
    float det = dot(e1, pv);
    if (det > -1e-8f && det < 1e-8f) return 0;
    float inv = 1.0f / det;
    v3 tv = sub(o, p0);
    float u = dot(tv, pv) * inv;
    if (u < 0.0 || u > 1.0) return 0;
    v3 qv = cross(tv, e1);
    float v = dot(d, qv) * inv;
    if (v < 0.0 || u + v > 1.0) return 0;
    float tt = dot(e2, qv) * inv;
    *ou = u; *ov = v; *ot = tt;
    return tt >= mint && tt <= maxt;
}
/* BoundingBox::RayIntersect  include/core/BoundingBox.hpp:371 */
static int box_hit(const float *mn, const float *mx, const float *o, const float *d, const float *rd,
                   float mint, float maxt) {
    float nt = -INFINITY, ft = INFINITY;
    for (int i = 0; i < 3; i++) {
        if (d[i] == 0) { if (o[i] < mn[i] || o[i] > mx[i]) return 0; }
        else {
            float t1 = (mn[i] - o[i]) * rd[i], t2 = (mx[i] - o[i]) * rd[i];
            if (t1 > t2) { float tmp = t1; t1 = t2; t2 = tmp; }
            nt = fmaxf(t1, nt); ft = fminf(t2, ft);
            if (!(nt <= ft)) return 0;
        }
    }
    return mint <= ft && nt <= maxt;
}

typedef struct { float mn[3], mx[3]; } aabb;
static inline void aabb_empty(aabb *b) { for (int i = 0; i < 3; i++) { b->mn[i] = INFINITY; b->mx[i] = -INFINITY; } }
static inline void aabb_grow(aabb *b, const aabb *o) { for (int i = 0; i < 3; i++) { b->mn[i] = fminf(b->mn[i], o->mn[i]); b->mx[i] = fmaxf(b->mx[i], o->mx[i]); } }
static inline float aabb_area(const aabb *b) {
    float dx = b->mx[0] - b->mn[0], dy = b->mx[1] - b->mn[1], dz = b->mx[2] - b->mn[2];
    if (dx < 0) return 0;
    return 2.0f * (dx * dy + dy * dz + dz * dx);
}

typedef struct { aabb *tb; float *cent; uint32_t *ord; bnode *nodes; int nn, cap; } bctx;

static int bvh_rec(bctx *c, uint32_t b, uint32_t e) {
    if (c->nn == c->cap) { c->cap *= 2; c->nodes = realloc(c->nodes, c->cap * sizeof(bnode)); }
    int me = c->nn++;
    aabb bb, cb; aabb_empty(&bb); aabb_empty(&cb);
    for (uint32_t i = b; i < e; i++) {
        aabb_grow(&bb, &c->tb[c->ord[i]]);
        aabb pc; for (int k = 0; k < 3; k++) pc.mn[k] = pc.mx[k] = c->cent[3 * c->ord[i] + k];
        aabb_grow(&cb, &pc);
    }
    for (int k = 0; k < 3; k++) { c->nodes[me].bmin[k] = bb.mn[k]; c->nodes[me].bmax[k] = bb.mx[k]; }
    uint32_t n = e - b;
    int axis = 0; float ext = cb.mx[0] - cb.mn[0];
    for (int k = 1; k < 3; k++) if (cb.mx[k] - cb.mn[k] > ext) { ext = cb.mx[k] - cb.mn[k]; axis = k; }
    if (n <= 4 || ext <= 0.0f) {
        c->nodes[me].left_or_first = (int32_t)b; c->nodes[me].count = (int32_t)n; c->nodes[me].axis = axis; c->nodes[me].right = -1;
        return me;
    }
    /* 12-bucket binned SAH (the scheme of src/acceleration/BVHAcceleration.cpp:150) */
    enum { NB = 12 };
    aabb bk[NB]; uint32_t cnt[NB] = {0};
    for (int i = 0; i < NB; i++) aabb_empty(&bk[i]);
    float inv = 1.0f / ext;
    for (uint32_t i = b; i < e; i++) {
        int bi = (int)((NB - 1) * (c->cent[3 * c->ord[i] + axis] - cb.mn[axis]) * inv);
        bi = clampi(bi, 0, NB - 1);
        cnt[bi]++; aabb_grow(&bk[bi], &c->tb[c->ord[i]]);
    }
    float best = INFINITY; int bs = -1;
    for (int i = 0; i < NB - 1; i++) {
        aabb l, r; aabb_empty(&l); aabb_empty(&r); uint32_t nl = 0, nr = 0;
        for (int j = 0; j <= i; j++) { aabb_grow(&l, &bk[j]); nl += cnt[j]; }
        for (int j = i + 1; j < NB; j++) { aabb_grow(&r, &bk[j]); nr += cnt[j]; }
        if (!nl || !nr) continue;
        float cost = aabb_area(&l) * nl + aabb_area(&r) * nr;
        if (cost < best) { best = cost; bs = i; }
    }
    uint32_t mid = b;
    if (bs >= 0) {
        for (uint32_t i = b; i < e; i++) {
            int bi = (int)((NB - 1) * (c->cent[3 * c->ord[i] + axis] - cb.mn[axis]) * inv);
            bi = clampi(bi, 0, NB - 1);
            if (bi <= bs) { uint32_t t = c->ord[i]; c->ord[i] = c->ord[mid]; c->ord[mid] = t; mid++; }
        }
    }
    if (mid == b || mid == e) mid = b + n / 2;
    c->nodes[me].axis = axis; c->nodes[me].count = 0;
    int l = bvh_rec(c, b, mid);
    int r = bvh_rec(c, mid, e);
    c->nodes[me].left_or_first = l; c->nodes[me].right = r;
    return me;
}
static int bvh_build(ho_scene *s) {
    free(s->nodes); free(s->order); s->nodes = NULL; s->order = NULL; s->nnodes = 0;
    aabb all; aabb_empty(&all);
    for (uint64_t i = 0; i < s->nv; i++) {
        aabb p; for (int k = 0; k < 3; k++) p.mn[k] = p.mx[k] = s->P[3 * i + k];
        aabb_grow(&all, &p);
    }
    for (int k = 0; k < 3; k++) { s->bbox[k] = all.mn[k]; s->bbox[3 + k] = all.mx[k]; }
    if (s->nt == 0) return 0;
    bctx c; c.tb = malloc(sizeof(aabb) * s->nt); c.cent = malloc(12ull * s->nt); c.ord = malloc(4ull * s->nt);
    for (uint32_t t = 0; t < s->nt; t++) {
        const uint32_t *f = s->F + 3ull * t;
        aabb_empty(&c.tb[t]);
        for (int j = 0; j < 3; j++) { aabb p; for (int k = 0; k < 3; k++) p.mn[k] = p.mx[k] = s->P[3ull * f[j] + k]; aabb_grow(&c.tb[t], &p); }
        for (int k = 0; k < 3; k++) c.cent[3 * t + k] = (1.0f / 3.0f) * (s->P[3ull * f[0] + k] + s->P[3ull * f[1] + k] + s->P[3ull * f[2] + k]);
        c.ord[t] = t;
    }
    c.cap = 1024; c.nn = 0; c.nodes = malloc(c.cap * sizeof(bnode));
    bvh_rec(&c, 0, s->nt);
    s->nodes = c.nodes; s->nnodes = c.nn; s->order = c.ord;
    free(c.tb); free(c.cent);
    return 0;
}

typedef struct { float t, u, v; int32_t tri; } hit_t;
/* Closest/any hit.  Reference tie rule: accept T <= MaxT, so later-visited wins
 * (src/core/Acceleration.cpp:59-69, src/acceleration/HLBVHAcceleration.cpp:229-240). */
static int trace(const ho_scene *s, v3 o, v3 d, float mint, float maxt, int any, int use_bvh, hit_t *h) {
    int found = 0;
    h->tri = -1;
    if (!use_bvh || !s->nodes) {
        for (uint32_t t = 0; t < s->nt; t++) {
            float u, v, tt;
            if (tri_intersect(s, t, o, d, mint, maxt, &u, &v, &tt)) {
                if (any) { h->tri = (int32_t)t; return 1; }
                maxt = tt; h->t = tt; h->u = u; h->v = v; h->tri = (int32_t)t; found = 1;
            }
        }
        return found;
    }
    float of[3] = {o.x, o.y, o.z}, df[3] = {d.x, d.y, d.z}, rd[3] = {1.0f / d.x, 1.0f / d.y, 1.0f / d.z};
    int neg[3] = {rd[0] < 0, rd[1] < 0, rd[2] < 0};
    int stack[128]; int sp = 0; int cur = 0;
    for (;;) {
        const bnode *nd = &s->nodes[cur];
        if (box_hit(nd->bmin, nd->bmax, of, df, rd, mint, maxt)) {
            if (nd->count > 0) {
                for (int i = 0; i < nd->count; i++) {
                    uint32_t t = s->order[nd->left_or_first + i];
                    float u, v, tt;
                    if (tri_intersect(s, t, o, d, mint, maxt, &u, &v, &tt)) {
                        if (any) { h->tri = (int32_t)t; return 1; }
                        maxt = tt; h->t = tt; h->u = u; h->v = v; h->tri = (int32_t)t; found = 1;
                    }
                }
                if (sp == 0) break;
                cur = stack[--sp];
            } else {
                if (neg[nd->axis]) { stack[sp++] = nd->left_or_first; cur = nd->right; }
                else { stack[sp++] = nd->right; cur = nd->left_or_first; }
            }
        } else {
            if (sp == 0) break;
            cur = stack[--sp];
        }
    }
    return found;
}

void ho_trace(const ho_scene *s, uint64_t n, const float *rays, float *th, float *uh, float *vh, int32_t *tri,
              int any, int use_bvh, int nthreads) {
#ifdef _OPENMP
    if (nthreads > 0) omp_set_num_threads(nthreads);
#pragma omp parallel for schedule(dynamic, 256)
#endif
    for (int64_t i = 0; i < (int64_t)n; i++) {
        const float *r = rays + 8 * i;
        hit_t h; h.t = h.u = h.v = 0.0f;
        int f = trace(s, V(r[0], r[1], r[2]), V(r[3], r[4], r[5]), r[6], r[7], any, use_bvh, &h);
        if (any) { tri[i] = f; continue; }
        tri[i] = f ? h.tri : -1;
        if (th) th[i] = f ? h.t : 0.0f;
        if (uh) uh[i] = f ? h.u : 0.0f;
        if (vh) vh[i] = f ? h.v : 0.0f;
    }
}

/* normalized() of an expression over MatrixXf columns (dynamic size): Eigen
 * reduces the squared norm left to right, ((x*x + y*y) + z*z), where a
 * fixed-size Vector3f reduces x*x + (y*y + z*z) */
static inline v3 normalize_dyn(v3 a) {
    float z = (a.x * a.x + a.y * a.y) + a.z * a.z;
    return z > 0.0f ? divs(a, sqrtf(z)) : a;
}
/* Frame(N, dPdU)  src/core/Frame.cpp:7: tangent by Gram-Schmidt against N */
static frame frame_from_n_dpdu(v3 n, v3 dpdu) {
    frame f; f.n = n;
    f.s = normalize(sub(dpdu, scl(n, dot(n, dpdu))));
    f.t = cross(n, f.s);
    return f;
}
/* Triangle::PostIntersect  src/core/Mesh.cpp:67-172 (the UV partials of :137-156
 * are used only for the shading frame; dNdU / dNdV serve texture filtering) */

static void post_intersect(const ho_scene *s, const hit_t *h, isect_t *it) {
    const uint32_t *f = s->F + 3ull * h->tri;
    v3 p0 = vload(s->P + 3ull * f[0]), p1 = vload(s->P + 3ull * f[1]), p2 = vload(s->P + 3ull * f[2]);
    float b0 = 1 - (h->u + h->v), b1 = h->u, b2 = h->v;
    const mesh_t *m = &s->meshes[s->tri_mesh[h->tri]];
    it->p = add(add(scl(p0, b0), scl(p1, b1)), scl(p2, b2));
    it->uv[0] = it->uv[1] = 0.0f;
    const float *u0 = s->UV + 2ull * f[0], *u1 = s->UV + 2ull * f[1], *u2 = s->UV + 2ull * f[2];
    if (m->has_uv)
        for (int c = 0; c < 2; c++) it->uv[c] = (b0 * u0[c] + b1 * u1[c]) + b2 * u2[c];
    it->geo = frame_from_n(normalize(cross(sub(p1, p0), sub(p2, p0))));
    it->mesh = s->tri_mesh[h->tri];
    it->t = h->t;
    it->has_uvp = 0;
    it->dndu = it->dndv = V(0, 0, 0);
    it->edge_d = INFINITY;
    it->curv_h = it->curv_k = 0.0f;
    if (m->has_n && m->has_uv) {
        v3 dp1 = sub(p1, p0), dp2 = sub(p2, p0);
        float du1 = u1[0] - u0[0], dv1 = u1[1] - u0[1], du2 = u2[0] - u0[0], dv2 = u2[1] - u0[1];
        float len = norm(cross(dp1, dp2));
        v3 n0 = vload(s->N + 3ull * f[0]), n1 = vload(s->N + 3ull * f[1]), n2 = vload(s->N + 3ull * f[2]);
        if (len == 0.0f) {
            it->sh = it->geo;
        } else {
            float det = du1 * dv2 - dv1 * du2;
            it->has_uvp = 1;
            if (det == 0.0f) {
                it->sh = frame_from_n(normalize_dyn(add(add(scl(n0, b0), scl(n1, b1)), scl(n2, b2))));
                it->dpdu = it->sh.s; it->dpdv = it->sh.t;
            } else {
                float inv = 1.0f / det;
                v3 dpdu = scl(sub(scl(dp1, dv2), scl(dp2, dv1)), inv);
                it->dpdu = dpdu;
                it->dpdv = scl(add(scl(dp1, -du2), scl(dp2, du1)), inv);
                v3 ns = add(add(scl(n0, b0), scl(n1, b1)), scl(n2, b2));
                float ln = norm(ns);
                float inv_ln = 1.0f / ln;
                ns = scl(ns, inv_ln);
                it->sh = frame_from_n_dpdu(ns, dpdu);
                /* dN/du, dN/dv (:146-153) */
                v3 dnu = scl(sub(n1, n0), inv_ln);
                dnu = sub(dnu, scl(ns, dot(ns, dnu)));
                v3 dnv = scl(sub(n2, n0), inv_ln);
                dnv = sub(dnv, scl(ns, dot(ns, dnv)));
                it->dndu = scl(sub(scl(dnu, dv2), scl(dnv, dv1)), inv);
                it->dndv = scl(add(scl(dnu, -du2), scl(dnv, du1)), inv);
            }
        }
    } else if (m->has_n) {
        v3 n0 = vload(s->N + 3ull * f[0]), n1 = vload(s->N + 3ull * f[1]), n2 = vload(s->N + 3ull * f[2]);
        it->sh = frame_from_n(normalize_dyn(add(add(scl(n0, b0), scl(n1, b1)), scl(n2, b2))));
    } else {
        it->sh = it->geo;
    }
    if (m->geo_tex) {
        /* WireframeTexture::Eval (src/texture/WireframeTexture.cpp:22-77): the
         * distance from P to the nearest of the three edge lines */
        const v3 ps[3] = {p0, p1, p2};
        float min_d2 = FLT_MAX;
        for (int i = 0; i < 3; i++) {
            const v3 cur = ps[i], nxt = ps[(i + 1) % 3];
            const v3 d1 = normalize(sub(nxt, cur)), d2 = sub(it->p, cur);
            const v3 e = sub(add(cur, scl(d1, dot(d1, d2))), it->p);
            const float d2x = dot(e, e);
            min_d2 = d2x < min_d2 ? d2x : min_d2;   /* std::min */
        }
        it->edge_d = sqrtf(min_d2);
        /* Shape::ComputeCurvature (src/core/Shape.cpp:30-51) */
        if (it->has_uvp) {
            const float E = dot(it->dpdu, it->dpdu), F = dot(it->dpdu, it->dpdv), G = dot(it->dpdv, it->dpdv);
            const float L = -dot(it->dpdu, it->dndu), M = -dot(it->dpdv, it->dndu), N = -dot(it->dpdv, it->dndv);
            const float inv_denom = 1.0f / (E * G - F * F);
            it->curv_k = (L * N - M * M) * inv_denom;
            it->curv_h = 0.5f * ((L * G - 2.0f * M * F) + N * E) * inv_denom;
        }
    }
}
/* Texture::Eval(Isect, true) at the intersection of (triangle, barycentric u, v) */
void ho_texture_eval_hit(const ho_scene *s, int id, uint32_t tri, float u, float v, float *out) {
    static const float zero[4] = {0, 0, 0, 0};
    hit_t h; memset(&h, 0, sizeof h);
    h.tri = tri; h.u = u; h.v = v;
    isect_t it;
    post_intersect(s, &h, &it);
    vstore(out, tex_eval(s->tex, s->mips, id, it.uv, zero, &it));
}
/* Triangle::PostIntersect for (triangle, barycentric u, v): out p(3) s(3) t(3) n(3) uv(2) */
void ho_post_intersect(const ho_scene *s, uint32_t tri, float u, float v, float *out) {
    hit_t h; memset(&h, 0, sizeof h);
    h.tri = tri; h.u = u; h.v = v;
    isect_t it;
    post_intersect(s, &h, &it);
    vstore(out, it.p); vstore(out + 3, it.sh.s); vstore(out + 6, it.sh.t); vstore(out + 9, it.sh.n);
    out[12] = it.uv[0]; out[13] = it.uv[1];
}

/* ------------------------------------------------------------ emitters */
typedef struct { v3 ref, p, n, wi; float pdf, dist; } erec;

/* Mesh::SamplePosition  src/core/Mesh.cpp:273 */
static void mesh_sample(const ho_scene *s, const mesh_t *m, float u1, float ux, float uy, v3 *P, v3 *N) {
    int ti = cdf_find(m->cdf, (int)m->nt, u1);    /* DiscretePDF1D::SampleDiscrete :65 */
    float sq = sqrtf(1.0f - ux);
    float al = 1.0f - sq, be = uy * sq, ga = 1.0f - al - be;
    const uint32_t *f = s->F + 3ull * (m->t0 + ti);
    v3 p0 = vload(s->P + 3ull * f[0]), p1 = vload(s->P + 3ull * f[1]), p2 = vload(s->P + 3ull * f[2]);
    *P = add(add(scl(p0, ga), scl(p1, al)), scl(p2, be));
    if (m->has_n) {
        v3 n0 = vload(s->N + 3ull * f[0]), n1 = vload(s->N + 3ull * f[1]), n2 = vload(s->N + 3ull * f[2]);
        *N = add(add(scl(n0, ga), scl(n1, al)), scl(n2, be));
    } else {
        *N = normalize(cross(sub(p1, p0), sub(p2, p0)));
    }
}
/* AreaLight::Pdf / Eval  src/emitter/AreaLight.cpp:38,59 */
static float area_pdf(const mesh_t *m, const erec *r) {
    float gd = fabsf(dot(scl(r->wi, -1.0f), r->n));
    if (gd == 0.0f) return 0.0f;
    float gn = r->dist * r->dist;
    return m->inv_area * (gn / gd);
}
static v3 area_eval(const mesh_t *m, const erec *r) { return dot(r->n, r->wi) < 0.0f ? m->radiance : V(0, 0, 0); }
/* AreaLight::Sample  src/emitter/AreaLight.cpp:14 */
static v3 area_sample(const ho_scene *s, const mesh_t *m, erec *r, float ux, float uy, float u1) {
    mesh_sample(s, m, u1, ux, uy, &r->p, &r->n);
    v3 wi = sub(r->p, r->ref);
    r->dist = norm(wi);
    r->wi = normalize(wi);
    r->pdf = area_pdf(m, r);
    if (r->pdf == 0.0f || isinf(r->pdf)) return V(0, 0, 0);
    return divs(area_eval(m, r), r->pdf);
}
static inline v3 env_texel(const ho_scene *s, int y, int x) { return vload(s->env + 3ull * ((uint64_t)y * s->ew + x)); }
/* SphericalCoordinates  src/core/Common.cpp:481 */
static void spherical_coords(v3 d, float *th, float *ph) {
    *th = acosf(d.z); *ph = atan2f(d.y, d.x);
    if (*ph < 0) *ph += 2.0f * PI_F;
}
/* ConstantLight::Sample  src/emitter/ConstantLight.cpp:15 */
static v3 const_sample(const ho_scene *s, erec *r, float ux, float uy) {
    float th = uy * PI_F;
    float st = sinf(th);
    if (st != 0.0f) r->pdf = 1.0f / (2.0f * (float)(M_PI * M_PI) * st);
    else return V(0, 0, 0);
    float ph = ux * (float)(2.0 * M_PI);
    float ct = cosf(th), sp = sinf(ph), cp = cosf(ph);
    r->wi = V(st * cp, st * sp, ct);                  /* SphericalDirection :467 */
    r->n = scl(r->wi, -1.0f);
    r->p = add(r->ref, scl(scl(r->wi, r->dist), 2.0f));
    return divs(s->env_const, r->pdf);
}
/* ConstantLight::Pdf :36 */
static float const_pdf(const erec *r) {
    float th, ph;
    spherical_coords(r->wi, &th, &ph);
    float st = sinf(th);
    if (st == 0.0f) return 0.0f;
    return 1.0f / (2.0f * (float)(M_PI * M_PI) * st);
}
/* PointLight::Sample  src/emitter/PointLight.cpp:15; DirectionalLight::Sample  DirectionalLight.cpp:18 */
static v3 delta_sample(const ho_scene *s, int k, erec *r) {
    if (!s->delta[k].directional) {
        r->p = s->delta[k].vec;
        v3 wi = sub(r->p, r->ref);
        r->dist = norm(wi);
        r->wi = normalize(wi);
        r->n = scl(r->wi, -1.0f);
        r->pdf = 1.0f;
        return scl(s->delta[k].color, 1.0f / ((4.0f * PI_F) * (r->dist * r->dist)));
    }
    r->wi = scl(normalize(s->delta[k].vec), -1.0f);
    r->p = add(r->ref, scl(r->wi, 2.0f * r->dist));
    r->n = scl(r->wi, -1.0f);
    r->pdf = 1.0f;
    return s->delta[k].color;
}
/* EnvironmentLight::Sample  src/emitter/EnvironmentLight.cpp:41 */
static v3 env_sample(const ho_scene *s, erec *r, float ux, float uy) {
    if (s->env_const_on) return const_sample(s, r, ux, uy);
    float py, px; int iy, ix;
    float dy = pdf1d_sample_cont(&s->env_marg, uy, &py, &iy);
    float dx = pdf1d_sample_cont(&s->env_rows[iy], ux, &px, &ix);
    float mp = px * py;
    float th = dy * PI_F, st = sinf(th);
    if (mp == 0.0f) return V(0, 0, 0);
    if (st != 0.0f) r->pdf = mp / (2.0f * (float)(M_PI * M_PI) * st);
    else return V(0, 0, 0);
    float ph = dx * (float)(2.0 * M_PI);
    float sp = sinf(ph), cp = cosf(ph), ct = cosf(th);
    v3 dir = V(st * cp, st * sp, ct);                 /* SphericalDirection :467 */
    r->wi = mat3_mul(s->to_world, dir);
    r->n = scl(r->wi, -1.0f);
    r->p = add(r->ref, scl(scl(r->wi, r->dist), 2.0f));
    v3 rad = env_texel(s, iy, ix);
    if (!is_valid(rad)) return V(0, 0, 0);
    return divs(scl(rad, s->env_scale), r->pdf);
}
/* EnvironmentLight::Pdf :78 and DiscretePDF2D::Pdf  src/core/DiscretePDF.cpp:127 */
static float env_pdf(const ho_scene *s, const erec *r) {
    if (s->env_const_on) return const_pdf(r);
    float th, ph;
    spherical_coords(mat3_mul(s->to_local, r->wi), &th, &ph);
    float st = sinf(th);
    if (st == 0.0f) return 0.0f;
    float u = ph / (float)(2.0 * M_PI), v = th / (float)M_PI;
    int X = clampi((int)(u * s->ew), 0, (int)s->ew - 1), Y = clampi((int)(v * s->eh), 0, (int)s->eh - 1);
    float p = s->env_rows[Y].func[X] / s->env_marg.integral;
    return p / (2.0f * (float)(M_PI * M_PI) * st);
}
/* EnvironmentLight::Eval :92 */
static v3 env_eval(const ho_scene *s, v3 wi) {
    if (s->env_const_on) return s->env_const;   /* ConstantLight::Eval :47 */
    float th, ph;
    spherical_coords(mat3_mul(s->to_local, wi), &th, &ph);
    if (isnan(th) || isnan(ph)) return V(0, 0, 0);
    float X = clampf(ph / (float)(2.0 * M_PI) * (float)s->ew, 0.0f, (float)(s->ew - 1.0f));
    float Y = clampf(th / (float)M_PI * (float)s->eh, 0.0f, (float)(s->eh - 1.0f));
    v3 rad = env_texel(s, (int)Y, (int)X);
    if (!is_valid(rad)) return V(0, 0, 0);
    return scl(rad, s->env_scale);
}

/* ------------------------------------------------------------ camera */
/* PerspectiveCamera::SampleRay  src/camera/PerspectiveCamera.cpp:77.  The
 * sample->camera map inverted in closed form: near-plane point
 * (near(1-2u)/cot, near(1-2v)/(aspect cot), near). */
static void camera_ray(const ho_scene *s, float px, float py, v3 *o, v3 *d, float *mint, float *maxt) {
    float u = px * (1.0f / (float)s->W), v = py * (1.0f / (float)s->H);
    v3 np = V(s->near_c * (1.0f - 2.0f * u) / s->cot, s->near_c * (1.0f - 2.0f * v) / (s->aspect * s->cot), s->near_c);
    v3 dir = normalize(np);
    float invz = 1.0f / dir.z;
    const float *M = s->cam;
    float w = M[15];
    *o = V(M[3] / w, M[7] / w, M[11] / w);
    *d = V(M[0] * dir.x + M[1] * dir.y + M[2] * dir.z, M[4] * dir.x + M[5] * dir.y + M[6] * dir.z,
           M[8] * dir.x + M[9] * dir.y + M[10] * dir.z);
    *mint = s->near_c * invz;
    *maxt = s->far_c * invz;
}

/* The differential rays of PerspectiveCamera::SampleRay (:94-98): origins at
 * the camera, directions through the near-plane point offset by m_dX / m_dY
 * (:64, one pixel along x / y on the near plane; in closed form (near(1 - 2/W)
 * / cot - near / cot, 0, 0) and (0, near(1 - 2/H) / (aspect cot) - near /
 * (aspect cot), 0)). */
static void camera_diff(const ho_scene *s, float px, float py, v3 *rx, v3 *ry) {
    float iw = 1.0f / (float)s->W, ih = 1.0f / (float)s->H;
    float u = px * iw, v = py * ih;
    v3 np = V(s->near_c * (1.0f - 2.0f * u) / s->cot, s->near_c * (1.0f - 2.0f * v) / (s->aspect * s->cot), s->near_c);
    float dx = s->near_c * (1.0f - 2.0f * iw) / s->cot - s->near_c / s->cot;
    float dy = s->near_c * (1.0f - 2.0f * ih) / (s->aspect * s->cot) - s->near_c / (s->aspect * s->cot);
    const float *M = s->cam;
    v3 a = normalize(V(np.x + dx, np.y, np.z)), b = normalize(V(np.x, np.y + dy, np.z));
    *rx = V(M[0] * a.x + M[1] * a.y + M[2] * a.z, M[4] * a.x + M[5] * a.y + M[6] * a.z,
            M[8] * a.x + M[9] * a.y + M[10] * a.z);
    *ry = V(M[0] * b.x + M[1] * b.y + M[2] * b.z, M[4] * b.x + M[5] * b.y + M[6] * b.z,
            M[8] * b.x + M[9] * b.y + M[10] * b.z);
}
/* SolveLinearSystem2x2 (include/core/Common.hpp:881) */
static int solve2x2(const float A[2][2], const float B[2], float X[2]) {
    float det = A[0][0] * A[1][1] - A[0][1] * A[1][0];
    if (fabsf(det) <= 1.0f / FLT_MAX) return 0;
    float inv = 1.0f / det;
    X[0] = (A[1][1] * B[0] - A[0][1] * B[1]) * inv;
    X[1] = (A[0][0] * B[1] - A[1][0] * B[0]) * inv;
    return 1;
}
static inline float v3c(v3 a, int k) { return k == 0 ? a.x : (k == 1 ? a.y : a.z); }
/* Intersection::ComputeScreenSpacePartial (src/core/Intersection.cpp:30) for
 * a camera ray from o with differential directions rx, ry: out (dUdX, dVdX,
 * dUdY, dVdY), zero without UV partials. */
static void screen_partials(const isect_t *it, v3 o, v3 rx, v3 ry, float *out) {
    out[0] = out[1] = out[2] = out[3] = 0.0f;
    if (!it->has_uvp) return;
    if (is_zero(it->dpdu) && is_zero(it->dpdv)) return;
    v3 n = it->geo.n;
    float pp = dot(n, it->p), pro = dot(n, o);
    float prd = dot(n, rx), pyd = dot(n, ry);
    if (prd == 0.0f || pyd == 0.0f) return;
    float tx = (pp - pro) / prd, ty = (pp - pro) / pyd;
    float ax = fabsf(n.x), ay = fabsf(n.y), az = fabsf(n.z);
    int a0, a1;
    if (ax > ay && ax > az) { a0 = 1; a1 = 2; }
    else if (ay > az) { a0 = 0; a1 = 2; }
    else { a0 = 0; a1 = 1; }
    float A[2][2] = {{v3c(it->dpdu, a0), v3c(it->dpdv, a0)}, {v3c(it->dpdu, a1), v3c(it->dpdv, a1)}};
    v3 px = add(o, scl(rx, tx)), py = add(o, scl(ry, ty));
    float bx[2] = {v3c(px, a0) - v3c(it->p, a0), v3c(px, a1) - v3c(it->p, a1)};
    float by[2] = {v3c(py, a0) - v3c(it->p, a0), v3c(py, a1) - v3c(it->p, a1)};
    float X[2];
    if (solve2x2(A, bx, X)) { out[0] = X[0]; out[1] = X[1]; }
    else { out[0] = 1.0f; out[1] = 0.0f; }
    if (solve2x2(A, by, X)) { out[2] = X[0]; out[3] = X[1]; }
    else { out[2] = 0.0f; out[3] = 1.0f; }
}
void ho_screen_partials(const ho_scene *s, float px, float py, uint32_t tri, float u, float v, float *out4) {
    hit_t h; memset(&h, 0, sizeof h);
    h.tri = tri; h.u = u; h.v = v;
    isect_t it;
    post_intersect(s, &h, &it);
    v3 o, d, rx, ry; float mn, mx;
    camera_ray(s, px, py, &o, &d, &mn, &mx);
    camera_diff(s, px, py, &rx, &ry);
    screen_partials(&it, o, rx, ry, out4);
}

/* ------------------------------------------------------------ integrator */
typedef struct { uint64_t rays, shadow; } ctr_t;
static inline v3 emitter_sample_any(const ho_scene *s, int e, erec *r, float ux, float uy, float u1) {
    int mi = s->emit_mesh[e];
    if (mi == -1) return env_sample(s, r, ux, uy);
    if (mi < -1) return delta_sample(s, -2 - mi, r);
    return area_sample(s, &s->meshes[mi], r, ux, uy, u1);
}

/* PathMISIntegrator::Li  src/integrator/PathMISIntegrator.cpp:16-157 */
/* pxy: the camera sample's film position (its differential rays give the
 * first hit's screen-space UV partials; later hits have none) */
static v3 li_pathmis(const ho_scene *s, int depth_max, ho_pcg32 *rng, v3 ro, v3 rdir, float rmint, float rmaxt,
                     const float *pxy, ctr_t *ctr) {
    float duv[4] = {0, 0, 0, 0};
    hit_t hn; int found_next = 0;
    isect_t it, itn;
    v3 L = V(0, 0, 0), beta = V(1, 1, 1);
    uint32_t depth = 0;
    float w_ems = 1.0f, w_mats = 1.0f;
    int has_env = s->has_env;
    float radius = 0.5f * norm(V(s->bbox[3] - s->bbox[0], s->bbox[4] - s->bbox[1], s->bbox[5] - s->bbox[2]));
    while (depth < (uint32_t)depth_max) {
        if (depth == 0) {
            hit_t h;
            ctr->rays++;
            if (!trace(s, ro, rdir, rmint, rmaxt, 0, 1, &h)) {
                if (has_env && !s->force_bg) { L = add(L, mul(beta, env_eval(s, rdir))); break; }
                return s->background;
            }
            post_intersect(s, &h, &it);
            if (s->ray_diff && pxy) {
                v3 rx, ry;
                camera_diff(s, pxy[0], pxy[1], &rx, &ry);
                screen_partials(&it, ro, rx, ry, duv);
            }
        } else {
            duv[0] = duv[1] = duv[2] = duv[3] = 0.0f;
            if (found_next) it = itn;
            else {
                if (has_env) L = add(L, mul(beta, env_eval(s, rdir)));
                break;
            }
        }
        const mesh_t *m = &s->meshes[it.mesh];
        int bsdf = m->bsdf;
        if (m->emitter >= 0) {
            erec er; er.ref = ro; er.p = it.p; er.n = it.sh.n;
            v3 wi = sub(er.p, er.ref); er.dist = norm(wi); er.wi = divs(wi, er.dist);
            v3 le = area_eval(m, &er);
            L = add(L, mul(scl(beta, w_mats), le));
        }
        for (int e = 0; e < s->n_emit; e++) {
            erec er; memset(&er, 0, sizeof er); er.ref = it.p;
            if (s->emit_mesh[e] < 0) er.dist = radius;
            float u1 = ho_pcg32_nextf(rng);
            float ux = ho_pcg32_nextf(rng), uy = ho_pcg32_nextf(rng);
            if (s->swap2d) { float t_ = ux; ux = uy; uy = t_; }
            v3 ld = emitter_sample_any(s, e, &er, ux, uy, u1);
            float pl = er.pdf;
            if (!is_zero(ld)) {
                v3 sd = sub(er.p, it.p);
                ctr->shadow++;
                hit_t sh;
                if (!trace(s, it.p, sd, EPS_RAY, 1.0f - EPS_RAY, 1, 1, &sh)) {
                    brec br; br.wi = to_local(&it.sh, scl(rdir, -1.0f)); br.wo = to_local(&it.sh, er.wi);
                    br.uv[0] = it.uv[0]; br.uv[1] = it.uv[1];
                    memcpy(br.duv, duv, sizeof duv);
                    br.it = &it;
                    br.measure = HO_MEASURE_SOLID_ANGLE; br.eta = 0;
                    float pb = bsdf_pdf(s, bsdf, &br);
                    if (pl + pb != 0.0f) w_ems = pl / (pl + pb);
                    v3 f = bsdf_eval(s, bsdf, &br);
                    float c = fabsf(br.wo.z);
                    L = add(L, V((((beta.x * f.x) * c) * ld.x) * w_ems, (((beta.y * f.y) * c) * ld.y) * w_ems,
                                 (((beta.z * f.z) * c) * ld.z) * w_ems));
                }
            }
        }
        brec br; memset(&br, 0, sizeof br);
        br.uv[0] = it.uv[0]; br.uv[1] = it.uv[1];
        memcpy(br.duv, duv, sizeof duv);
        br.it = &it;
        br.wi = to_local(&it.sh, scl(rdir, -1.0f)); br.measure = HO_MEASURE_UNKNOWN;
        float sx = ho_pcg32_nextf(rng), sy = ho_pcg32_nextf(rng);
        if (s->swap2d) { float t_ = sx; sx = sy; sy = t_; }
        v3 F = bsdf_sample(s, bsdf, &br, sx, sy, rng, NULL);
        ro = it.p; rdir = to_world(&it.sh, br.wo);
        beta = mul(beta, F);
        if (is_zero(beta)) break;
        ctr->rays++;
        found_next = trace(s, ro, rdir, EPS_RAY, INFINITY, 0, 1, &hn);
        if (found_next) {
            post_intersect(s, &hn, &itn);
            const mesh_t *mn = &s->meshes[itn.mesh];
            if (mn->emitter >= 0) {
                erec er; er.ref = it.p; er.p = itn.p; er.n = itn.sh.n;
                v3 wi = sub(er.p, er.ref); er.dist = norm(wi); er.wi = divs(wi, er.dist);
                float plm = area_pdf(mn, &er);
                float pbm = bsdf_pdf(s, bsdf, &br);
                if (pbm + plm != 0.0f) w_mats = pbm / (pbm + plm);
            }
        }
        if (br.measure == HO_MEASURE_DISCRETE) { w_ems = 0.0f; w_mats = 1.0f; }
        if (ho_pcg32_nextf(rng) < 0.95f) beta = scl(beta, 1.0f / 0.95f);
        else break;
        depth++;
    }
    return L;
}

/* ImageBlock::Put(Point2f, Color3f)  src/core/Block.cpp:95 (whole image, double accum) */
static int film_put(const ho_scene *s, double *film, float px, float py, v3 val) {
    if (!is_valid(val)) return 1;
    int B = s->border, FW = (int)s->W + 2 * B, FH = (int)s->H + 2 * B;
    float cx = px - 0.5f - (0 - B), cy = py - 0.5f - (0 - B);
    int x0 = (int)ceilf(cx - s->filt_r), y0 = (int)ceilf(cy - s->filt_r);
    int x1 = (int)floorf(cx + s->filt_r), y1 = (int)floorf(cy + s->filt_r);
    x0 = x0 < 0 ? 0 : x0; y0 = y0 < 0 ? 0 : y0; x1 = x1 > FW - 1 ? FW - 1 : x1; y1 = y1 > FH - 1 ? FH - 1 : y1;
    float wx[16], wy[16];
    for (int x = x0, i = 0; x <= x1; ++x) wx[i++] = s->ftab[(int)(fabsf((float)x - cx) * s->lookup)];
    for (int y = y0, i = 0; y <= y1; ++y) wy[i++] = s->ftab[(int)(fabsf((float)y - cy) * s->lookup)];
    /* Color4f(Value) * WeightX * WeightY: each channel (v * wx) * wy in float,
     * the weight channel (1 * wx) * wy (Block.cpp:129-132) */
    for (int y = y0, yr = 0; y <= y1; ++y, ++yr)
        for (int x = x0, xr = 0; x <= x1; ++x, ++xr) {
            double *p = film + 4ull * ((uint64_t)y * FW + x);
            p[0] += (double)((val.x * wx[xr]) * wy[yr]);
            p[1] += (double)((val.y * wx[xr]) * wy[yr]);
            p[2] += (double)((val.z * wx[xr]) * wy[yr]);
            p[3] += (double)(wx[xr] * wy[yr]);
        }
    return 0;
}

int64_t ho_film_put_samples(const ho_scene *s, uint64_t n, const float *pos, const float *val, double *film) {
    int64_t dropped = 0;
    for (uint64_t i = 0; i < n; i++) {
        v3 c = {val[3 * i], val[3 * i + 1], val[3 * i + 2]};
        dropped += film_put(s, film, pos[2 * i], pos[2 * i + 1], c);
    }
    return dropped;
}

/* Render / RenderBlock  src/Main.cpp:11-44, 46-147 */
void ho_scene_set_reference_draw_order(ho_scene *s, int swap2d) { s->swap2d = swap2d != 0; }

int64_t ho_render(const ho_scene *s, int depth, int spp, const int32_t *blist, int nblk, double *film, int nthreads,
                  uint64_t *counters) {
    int BS = 32;
    int nbx = ((int)s->W + BS - 1) / BS, nby = ((int)s->H + BS - 1) / BS;
    int total = blist ? nblk : nbx * nby;
    int B = s->border;
    uint64_t FW = s->W + 2 * B, FH = s->H + 2 * B;
    int64_t dropped = 0; uint64_t rays = 0, shadow = 0;
#ifdef _OPENMP
    if (nthreads > 0) omp_set_num_threads(nthreads);
#pragma omp parallel reduction(+ : dropped, rays, shadow)
#endif
    {
        double *loc = calloc(FW * FH * 4, sizeof(double));
        ctr_t c = {0, 0};
#ifdef _OPENMP
#pragma omp for schedule(dynamic, 1)
#endif
        for (int bi = 0; bi < total; bi++) {
            int b = blist ? blist[bi] : bi;
            int ox = (b % nbx) * BS, oy = (b / nbx) * BS;
            ho_pcg32 rng; ho_pcg32_seed(&rng, (uint64_t)ox, (uint64_t)oy);   /* IndependentSampler::Prepare */
            int sx = ((int)s->W - ox) < BS ? ((int)s->W - ox) : BS, sy = ((int)s->H - oy) < BS ? ((int)s->H - oy) : BS;
            for (int y = 0; y < sy; ++y)
                for (int x = 0; x < sx; ++x)
                    for (int i = 0; i < spp; ++i) {
                        float jx = ho_pcg32_nextf(&rng), jy = ho_pcg32_nextf(&rng);
                        if (s->swap2d) { float t_ = jx; jx = jy; jy = t_; }
                        float px = (float)(x + ox) + jx, py = (float)(y + oy) + jy;
                        (void)ho_pcg32_nextf(&rng); (void)ho_pcg32_nextf(&rng);   /* aperture sample */
                        v3 o, d; float mn, mx;
                        camera_ray(s, px, py, &o, &d, &mn, &mx);
                        float pxy[2] = {px, py};
            v3 L = li_pathmis(s, depth, &rng, o, d, mn, mx, pxy, &c);
                        dropped += film_put(s, loc, px, py, L);
                    }
        }
#ifdef _OPENMP
#pragma omp critical
#endif
        for (uint64_t i = 0; i < FW * FH * 4; i++) film[i] += loc[i];
        free(loc);
        rays += c.rays; shadow += c.shadow;
    }
    if (counters) { counters[0] = (uint64_t)total; counters[1] = rays; counters[2] = shadow; counters[3] = 0; }
    return dropped;
}

void ho_pixel_stats(const ho_scene *s, int depth, int spp, uint64_t seed, int npix, const int32_t *pix, double *out,
                    int nthreads) {
#ifdef _OPENMP
    if (nthreads > 0) omp_set_num_threads(nthreads);
#pragma omp parallel for schedule(dynamic, 1)
#endif
    for (int k = 0; k < npix; k++) {
        int x = pix[2 * k], y = pix[2 * k + 1];
        ho_pcg32 rng; ho_pcg32_seed(&rng, seed, (uint64_t)y * s->W + x);
        double m[3] = {0, 0, 0}, v[3] = {0, 0, 0};
        ctr_t c = {0, 0};
        for (int i = 0; i < spp; i++) {
            float px = (float)x + ho_pcg32_nextf(&rng), py = (float)y + ho_pcg32_nextf(&rng);
            v3 o, d; float mn, mx;
            camera_ray(s, px, py, &o, &d, &mn, &mx);
            float pxy[2] = {px, py};
            v3 L = li_pathmis(s, depth, &rng, o, d, mn, mx, pxy, &c);
            double r[3] = {L.x, L.y, L.z};
            for (int ch = 0; ch < 3; ch++) { double dl = r[ch] - m[ch]; m[ch] += dl / (i + 1); v[ch] += dl * (r[ch] - m[ch]); }
        }
        for (int ch = 0; ch < 3; ch++) { out[6 * k + ch] = m[ch]; out[6 * k + 3 + ch] = spp > 1 ? v[ch] / (spp - 1) : 0; }
    }
}

/* One sample per listed pixel from the stream seeded (seed, pixel), as
 * ho_pixel_stats draws it: out npix x 5 floats (film x, film y, radiance rgb;
 * the radiance unfiltered and not checked for validity). */
void ho_pixel_samples(const ho_scene *s, int depth, uint64_t seed, int npix, const int32_t *pix, float *out,
                      int nthreads) {
#ifdef _OPENMP
    if (nthreads > 0) omp_set_num_threads(nthreads);
#pragma omp parallel for schedule(dynamic, 64)
#endif
    for (int k = 0; k < npix; k++) {
        int x = pix[2 * k], y = pix[2 * k + 1];
        ho_pcg32 rng; ho_pcg32_seed(&rng, seed, (uint64_t)y * s->W + x);
        ctr_t c = {0, 0};
        float px = (float)x + ho_pcg32_nextf(&rng), py = (float)y + ho_pcg32_nextf(&rng);
        v3 o, d; float mn, mx;
        camera_ray(s, px, py, &o, &d, &mn, &mx);
        float pxy[2] = {px, py};
        v3 L = li_pathmis(s, depth, &rng, o, d, mn, mx, pxy, &c);
        out[5 * k] = px; out[5 * k + 1] = py; out[5 * k + 2] = L.x; out[5 * k + 3] = L.y; out[5 * k + 4] = L.z;
    }
}

void ho_ttest_scene(const ho_scene *s, int depth, int n, double *mean, double *var) {
    ho_pcg32 rng; pcg_default(&rng);
    double m = 0, v = 0;
    ctr_t c = {0, 0};
    for (int k = 0; k < n; k++) {
        float a = ho_pcg32_nextf(&rng), b = ho_pcg32_nextf(&rng);
        if (s->swap2d) { float t_ = a; a = b; b = t_; }
        float px = a * (float)s->W, py = b * (float)s->H;
        (void)ho_pcg32_nextf(&rng); (void)ho_pcg32_nextf(&rng);
        v3 o, d; float mn, mx;
        camera_ray(s, px, py, &o, &d, &mn, &mx);
        float pxy[2] = {px, py};
            v3 L = li_pathmis(s, depth, &rng, o, d, mn, mx, pxy, &c);
        double r = lum(L);
        double dl = r - m; m += dl / (double)(k + 1); v += dl * (r - m);
    }
    *mean = m; *var = v / (n - 1);
}

void ho_film_resolve(const ho_scene *s, const double *film, float *out) {
    int B = s->border; uint64_t FW = s->W + 2 * B;
    for (uint32_t y = 0; y < s->H; y++)
        for (uint32_t x = 0; x < s->W; x++) {
            const double *p = film + 4 * ((uint64_t)(y + B) * FW + (x + B));
            float *o = out + 3ull * ((uint64_t)y * s->W + x);
            if (p[3] != 0.0) { o[0] = (float)(p[0] / p[3]); o[1] = (float)(p[1] / p[3]); o[2] = (float)(p[2] / p[3]); }
            else { o[0] = o[1] = o[2] = 0.0f; }
        }
}

/* ------------------------------------------------ emitter record queries */
/* Emitter::Sample for emitter e (Scene order) at reference point ref. out: p(3) n(3) wi(3) pdf dist value(3) */
void ho_emitter_sample(const ho_scene *s, int e, const float *ref, float ux, float uy, float u1, float *out) {
    erec r; memset(&r, 0, sizeof r); r.ref = vload(ref);
    float radius = 0.5f * norm(V(s->bbox[3] - s->bbox[0], s->bbox[4] - s->bbox[1], s->bbox[5] - s->bbox[2]));
    if (s->emit_mesh[e] < 0) r.dist = radius;
    v3 val = emitter_sample_any(s, e, &r, ux, uy, u1);
    vstore(out, r.p); vstore(out + 3, r.n); vstore(out + 6, r.wi); out[9] = r.pdf; out[10] = r.dist; vstore(out + 11, val);
}
/* Emitter::Pdf for a record built as EmitterQueryRecord(emitter, ref, p, n)  src/core/Emitter.cpp:16 */
float ho_emitter_pdf(const ho_scene *s, int e, const float *ref, const float *p, const float *n) {
    erec r; r.ref = vload(ref); r.p = vload(p); r.n = vload(n);
    v3 wi = sub(r.p, r.ref); r.dist = norm(wi); r.wi = divs(wi, r.dist);
    int mi = s->emit_mesh[e];
    if (mi < -1) return 0.0f;                                  /* point / directional: Pdf is 0 */
    if (mi < 0) { r.wi = vload(p); return env_pdf(s, &r); }   /* env: p carries the direction */
    return area_pdf(&s->meshes[mi], &r);
}
/* Environment Eval for a world direction. */
void ho_env_eval(const ho_scene *s, const float *wi, float *out) { vstore(out, env_eval(s, vload(wi))); }
/* Camera ray for a film position (px, py): out o(3) d(3) mint maxt */
void ho_camera_ray(const ho_scene *s, float px, float py, float *out) {
    v3 o, d; float mn, mx; camera_ray(s, px, py, &o, &d, &mn, &mx);
    vstore(out, o); vstore(out + 3, d); out[6] = mn; out[7] = mx;
}
/* Activated filter table (33 floats) and lookup factor. */
void ho_filter_table(const ho_scene *s, float *out33, float *lookup) { memcpy(out33, s->ftab, 33 * 4); *lookup = s->lookup; }
