// Host side of the B200 pathMIS core: scene assembly, object activation
// (BSDF tables, light CDFs, camera, filter), the BVH build and the C ABI of
// include/hikari_b200.h.
#include <cuda_runtime.h>

#include <algorithm>
#include <cfloat>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <memory>
#include <stdexcept>
#include <string>
#include <thread>
#include <vector>

#include "../../include/hikari_b200.h"
#include "hk_bvh.h"
#include "hk_hostutil.h"
#include "hk_device.h"
#include "hk_engine.h"
#include "hk_internal.h"
#include "hk_kernels.h"
#include "hk_lbvh.h"
#include "hk_mipmap.h"
#include "hk_wavefront.h"

extern "C" int hk_scene_load_xml_impl(const char *path, const char *data_dir, hk_scene **out, int32_t *depth,
                                      int32_t *spp, int build, std::string *err);
extern "C" int hk_exr_read_impl(const char *path, int *w, int *h, std::vector<float> *rgb, std::string *err);
extern "C" int hk_exr_write_impl(const char *path, int w, int h, const float *rgb, std::string *err);

namespace hk {
thread_local std::string g_error;
int set_error(int code, const std::string &msg) {
    g_error = msg;
    return code;
}
}  // namespace hk

using hk::DevBuf;
using hk::guarded;
using hk::HkError;
using hk::set_error;

namespace {

// ------------------------------------------------------------ float helpers
// Host 3-vectors in the reference's Eigen evaluation order: x + (y + z).
struct F3 {
    float x, y, z;
};
inline F3 f3sub(F3 a, F3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
inline F3 f3cross(F3 a, F3 b) { return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }
inline float f3dot(F3 a, F3 b) { return a.x * b.x + (a.y * b.y + a.z * b.z); }
inline float f3norm(F3 a) { return std::sqrt(f3dot(a, a)); }
inline float lum(const float *c) { return c[0] * 0.212671f + c[1] * 0.715160f + c[2] * 0.072169f; }
inline float clampf(float v, float lo, float hi) { return v < lo ? lo : (v > hi ? hi : v); }

// DiscretePDF1D ctor (src/core/DiscretePDF.cpp:5): cdf in float, normalised.
// Guide table of a CDF c[0..n] (the cutpoint method): g[k], k = 0..G, is the
// first index i with c[i] >= k / G (n + 1 if none).  A u in [k / G, (k+1) / G)
// has its lower bound in [g[k], g[k+1]], so a search there returns the index
// the search over the whole CDF returns.  G is a power of two, so k / G and
// u * G are exact in float.
constexpr int kCdfGuide = hk::kEnvGuide;
void cdf_guide(const float *c, int n, int32_t *g) {
    for (int k = 0; k <= kCdfGuide; ++k)
        g[k] = (int32_t)(std::lower_bound(c, c + n + 1, (float)k / (float)kCdfGuide) - c);
}

struct Pdf1D {
    std::vector<float> func, cdf;
    float integral = 0.0f;
    void build(const float *f, int n) {
        func.assign(f, f + n);
        cdf.assign(n + 1, 0.0f);
        for (int i = 1; i < n + 1; i++) cdf[i] = cdf[i - 1] + func[i - 1] / n;
        integral = cdf[n];
        if (integral == 0.0f) {
            for (int i = 1; i < n + 1; i++) cdf[i] = float(i) / float(n);
        } else {
            for (int i = 1; i < n + 1; i++) cdf[i] /= integral;
        }
    }
};

// ------------------------------------------------------------ RFT activation
// EvalCubicInterpolate1D/2D/3D (src/core/Common.cpp:230-464) restricted to
// the [0,1] domains the rough transmittance tables use.
float cubic1d(float x, const float *val, int size, float mn, float mx) {
    if (!(x >= mn && x <= mx)) return 0.0f;
    float t = ((x - mn) * (size - 1)) / (mx - mn);
    int k = std::max(0, std::min(int(t), size - 2));
    float f0 = val[k], f1 = val[k + 1];
    float d0 = (k > 0) ? 0.5f * (val[k + 1] - val[k - 1]) : val[k + 1] - val[k];
    float d1 = (k + 2 < size) ? 0.5f * (val[k + 2] - val[k]) : val[k + 1] - val[k];
    t = t - float(k);
    float t2 = t * t, t3 = t2 * t;
    return (2.0f * t3 - 3.0f * t2 + 1) * f0 + (-2.0f * t3 + 3.0f * t2) * f1 + (t3 - 2.0f * t2 + t) * d0 + (t3 - t2) * d1;
}
bool knot_weights(float p, int size, float *w, int &knot) {
    if (!(p >= 0.0f && p <= 1.0f)) return false;
    float t = ((p - 0.0f) * float(size - 1)) / (1.0f - 0.0f);
    knot = std::min(int(t), size - 2);
    t = t - float(knot);
    float t2 = t * t, t3 = t2 * t;
    w[0] = 0.0f;
    w[1] = 2.0f * t3 - 3.0f * t2 + 1;
    w[2] = -2.0f * t3 + 3.0f * t2;
    w[3] = 0.0f;
    float d0 = t3 - 2.0f * t2 + t, d1 = t3 - t2;
    if (knot > 0) { w[2] += 0.5f * d0; w[0] -= 0.5f * d0; }
    else { w[2] += d0; w[1] -= d0; }
    if (knot + 2 < size) { w[3] += 0.5f * d1; w[1] -= 0.5f * d1; }
    else { w[2] += d1; w[1] -= d1; }
    return true;
}
float cubic2d(float px, float py, const float *val, int sx, int sy) {
    float w[2][4];
    int k[2];
    if (!knot_weights(px, sx, w[0], k[0]) || !knot_weights(py, sy, w[1], k[1])) return 0.0f;
    float r = 0.0f;
    for (int y = -1; y <= 2; y++) {
        float wy = w[1][y + 1];
        for (int x = -1; x <= 2; x++) {
            float wxy = w[0][x + 1] * wy;
            if (wxy == 0) continue;
            r += val[(k[1] + y) * sx + k[0] + x] * wxy;
        }
    }
    return r;
}
float cubic3d(float px, float py, float pz, const float *val, int sx, int sy, int sz) {
    float w[3][4];
    int k[3];
    if (!knot_weights(px, sx, w[0], k[0]) || !knot_weights(py, sy, w[1], k[1]) || !knot_weights(pz, sz, w[2], k[2]))
        return 0.0f;
    float r = 0.0f;
    for (int z = -1; z <= 2; z++) {
        float wz = w[2][z + 1];
        for (int y = -1; y <= 2; y++) {
            float wyz = w[1][y + 1] * wz;
            for (int x = -1; x <= 2; x++) {
                float wxyz = w[0][x + 1] * wyz;
                if (wxyz == 0) continue;
                r += val[((k[2] + z) * sy + (k[1] + y)) * sx + k[0] + x] * wxyz;
            }
        }
    }
    return r;
}

struct RftTable {
    uint64_t eta_n = 0, alpha_n = 0, theta_n = 0, t_size = 0, d_size = 0;
    float eta_min = 0, eta_max = 0, alpha_min = 0, alpha_max = 0;
    std::vector<float> trans, diff;
    bool loaded = false;

    // RoughTransmittance ctor (src/core/RoughTransmitance.cpp:9): header then data
    void parse(const void *bytes, uint64_t n) {
        const unsigned char *b = (const unsigned char *)bytes;
        if (n < 56) throw HkError{HK_ERR_IO, "RFT table: short header"};
        uint64_t h[5];
        float f[4];
        std::memcpy(h, b, 40);
        std::memcpy(f, b + 40, 16);
        eta_n = h[0]; alpha_n = h[1]; theta_n = h[2]; t_size = h[3]; d_size = h[4];
        eta_min = f[0]; eta_max = f[1]; alpha_min = f[2]; alpha_max = f[3];
        if (theta_n > (uint64_t)hk::kRftThetaMax || theta_n < 2 || alpha_n < 2 || eta_n < 2)
            throw HkError{HK_ERR_IO, "RFT table: unsupported dimensions"};
        if (t_size != eta_n * alpha_n * theta_n * 2 || d_size != eta_n * alpha_n * 2)
            throw HkError{HK_ERR_IO, "RFT table: inconsistent sizes"};
        if (56 + 4 * (t_size + d_size) > n) throw HkError{HK_ERR_IO, "RFT table: short body"};
        trans.resize(t_size);
        diff.resize(d_size);
        std::memcpy(trans.data(), b + 56, 4 * t_size);
        std::memcpy(diff.data(), b + 56 + 4 * t_size, 4 * d_size);
        loaded = true;
    }
    // SetEta (src/core/RoughTransmitance.cpp:170)
    void set_eta(float eta, std::vector<float> &t2d, std::vector<float> &d1d) const {
        const float *pt = trans.data(), *pd = diff.data();
        int E = (int)eta_n, A = (int)alpha_n, T = (int)theta_n;
        if (eta < 1.0f) { pt += (uint64_t)E * A * T; pd += (uint64_t)E * A; eta = 1.0f / eta; }
        if (eta < eta_min) eta = eta_min;
        float we = std::pow((eta - eta_min) / (eta_max - eta_min), 0.25f);
        float da = 1.0f / (A - 1.0f), dt = 1.0f / (T - 1.0f);
        t2d.assign((size_t)A * T, 0.0f);
        d1d.assign(A, 0.0f);
        for (int i = 0; i < A; i++) {
            for (int j = 0; j < T; j++) t2d[i * T + j] = cubic3d(j * dt, i * da, we, pt, T, A, E);
            d1d[i] = cubic2d(i * da, we, pd, A, E);
        }
    }
    // SetAlpha (src/core/RoughTransmitance.cpp:237)
    void set_alpha(const std::vector<float> &t2d, const std::vector<float> &d1d, float alpha, float *t1d,
                   float &dscalar) const {
        int A = (int)alpha_n, T = (int)theta_n;
        float wa = std::pow((alpha - alpha_min) / (alpha_max - alpha_min), 0.25f);
        float dt = 1.0f / (T - 1.0f);
        for (int i = 0; i < T; i++) t1d[i] = cubic2d(i * dt, wa, t2d.data(), T, A);
        dscalar = cubic1d(wa, d1d.data(), A, 0.0f, 1.0f);
    }
};

struct MeshIn {
    std::vector<float> pos, nrm, uv;
    std::vector<uint32_t> idx;
    int32_t bsdf;
    bool emitter;
    float radiance[3];
};

}  // namespace

struct hk_scene {
    // inputs
    std::vector<hk_bsdf_desc> bsdfs;
    std::vector<int> bsdf_deep;   // per BSDF: dispatched through the deep layer dispatch (set by the build)
    std::vector<hk_texture_desc> textures;
    std::vector<std::shared_ptr<hk::MipPyramid>> bitmaps;   // per texture: the MIP pyramid of a bitmap, else null
    std::vector<MeshIn> meshes;
    std::vector<int> emitter_mesh;   // Scene order: mesh id, -1 environment, -2 - k delta_lights[k]
    struct DeltaLight { int directional; float color[3], vec[3]; };
    std::vector<DeltaLight> delta_lights;   // point / directional lights
    RftTable rft[2];
    bool has_env = false;
    bool env_constant = false;       // the environment is a ConstantLight
    float env_const[3] = {0, 0, 0};
    uint32_t env_w = 0, env_h = 0;
    std::vector<float> env_rgb;
    float env_to_world[16];
    float env_scale = 1.0f;
    uint32_t width = 1280, height = 720;
    float cam_to_world[16] = {1, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1};
    float fov = 30.0f, near_clip = 1e-4f, far_clip = 1e4f;
    int filt_kind = 2;
    float filt_r = 2.0f, filt_p0 = 0.5f, filt_p1 = 0.0f;
    float background[3] = {0, 0, 0};
    int force_background = 0;
    // built state
    bool built = false;
    hk::DevScene dev{};
    int32_t accel = HK_ACCEL_BVH8;
    DevBuf b_tris, b_nodes, b_wnodes, b_tri_normals, b_tri_uv, b_meshes, b_bsdfs, b_emitter_area, b_area, b_light_tris, b_light_normals,
        b_light_cdf, b_delta, b_textures, b_texels, b_env_rgb, b_env_marg_cdf, b_env_marg_func, b_env_cond_cdf, b_env_cond_func, b_env_cond_int, b_ftab,
        b_env_marg_guide, b_env_cond_guide, b_rft2d;
    DevBuf b_film, b_rgb, b_scratch;   // scratch: work counter + counters
    std::vector<std::unique_ptr<DevBuf>> batch_films;   // films of hk_render_batch_host
    hk_scene_info info{};
    int margin_lo = 0, margin_hi = 0;
    int sm_count = 148;
    int device = 0;   // CUDA device the scene was built on
    int image_form = HK_FORM_AUTO;             // form hk_render_image renders with
    int builder = HK_BUILDER_HOST;             // where hk_scene_build builds the trees
    double tree_build_s = 0.0;                 // seconds of the last tree build
    bool has_wf_cfg = false;                   // wf_cfg was set (autotuner or caller)
    hk_wavefront_config wf_cfg{};              // wavefront configuration of hk_render_image
    int occupancy = 1;        // resident megakernel CTAs per SM for the traversed tree
    int occupancy_of[2] = {1, 1};
    std::unique_ptr<hk::WfEngine> wf;   // wavefront engine (allocated on first use)
};

namespace {

float filter_eval(const hk_scene *s, float x) {   // src/filter/*.cpp Eval
    switch (s->filt_kind) {
    case 0: return 1.0f;
    case 1: return std::max(0.0f, 1.0f - std::abs(x));
    case 2: {
        float a = -1.0f / (2.0f * s->filt_p0 * s->filt_p0);
        return std::max(0.0f, std::exp(a * x * x) - std::exp(a * s->filt_r * s->filt_r));
    }
    default: {
        float B = s->filt_p0, C = s->filt_p1;
        x = std::abs(2.0f * x / s->filt_r);
        float x2 = x * x, x3 = x2 * x;
        if (x < 1.0f)
            return 1.0f / 6.0f * ((12.0f - 9.0f * B - 6.0f * C) * x3 + (-18.0f + 12.0f * B + 6.0f * C) * x2 + (6.0f - 2.0f * B));
        if (x < 2.0f)
            return 1.0f / 6.0f * ((-B - 6 * C) * x3 + (6.0f * B + 30.0f * C) * x2 + (-12.0f * B - 48.0f * C) * x + (8.0f * B + 24.0f * C));
        return 0.0f;
    }
    }
}

void mat3_inverse(const float *m, float *o) {
    double a = m[0], b = m[1], c = m[2], d = m[3], e = m[4], f = m[5], g = m[6], h = m[7], i = m[8];
    double det = a * (e * i - f * h) - b * (d * i - f * g) + c * (d * h - e * g);
    if (det == 0.0) throw HkError{HK_ERR_INVALID, "environment toWorld is singular"};
    o[0] = float((e * i - f * h) / det); o[1] = float((c * h - b * i) / det); o[2] = float((b * f - c * e) / det);
    o[3] = float((f * g - d * i) / det); o[4] = float((a * i - c * g) / det); o[5] = float((c * d - a * f) / det);
    o[6] = float((d * h - e * g) / det); o[7] = float((b * g - a * h) / det); o[8] = float((a * e - b * d) / det);
}

// Activation of one BSDF (RoughPlasticBSDF::Activate :261, RoughCoatingBSDF::Activate :315)
// ApproxFresnelDiffuseReflectance (src/core/Common.cpp:550): the published fits
// of Egan & Hilgeman (1973) for eta < 1 and of d'Eon & Irving (2011) otherwise.
float approx_fresnel_diffuse(float e) {
    if (e < 1.0f) return -1.4399f * (e * e) + 0.7099f * e + 0.6681f + 0.0636f / e;
    float i1 = 1.0f / e, i2 = i1 * i1, i3 = i2 * i1, i4 = i3 * i1, i5 = i4 * i1;
    return 0.919317f - 3.4793f * i1 + 6.75335f * i2 - 7.80989f * i3 + 4.98554f * i4 - 1.36881f * i5;
}

// Whether a BSDF has a transmission lobe; coatings inherit the nested BSDF's
// lobes (RoughCoatingBSDF.cpp:317).
bool bsdf_transmits(const hk_scene *s, int id, int depth) {
    if (id < 0 || id >= (int)s->bsdfs.size() || depth > 8) return false;
    const hk_bsdf_desc &d = s->bsdfs[id];
    switch (d.type) {
    case hk::kRoughDielectric:
    case hk::kDielectric: return true;
    case hk::kRoughCoating:
    case hk::kCoating: return bsdf_transmits(s, d.nested, depth + 1);
    case hk::kTwoSided: return bsdf_transmits(s, d.nested, depth + 1) || bsdf_transmits(s, d.nested2, depth + 1);
    case hk::kBumpMap:
    case hk::kNormalMap: return bsdf_transmits(s, d.nested, depth + 1);
    default: return false;
    }
}

// Texture::GetAverage of the procedural textures (CheckerboardTexture.cpp:30,
// GridTexture.cpp:40, ScaleTexture.cpp:28), used when BSDFs activate
F3 tex_average(const hk_scene *s, int id) {
    const hk_texture_desc &t = s->textures[id];
    if (t.kind == HK_TEX_SCALE) {
        F3 c = tex_average(s, t.nested);
        return {c.x * t.scale, c.y * t.scale, c.z * t.scale};
    }
    if (t.kind == HK_TEX_BITMAP) {   // BitmapTexture::GetAverage (src/texture/BitmapTexture.cpp:176)
        const float *a = s->bitmaps[id]->avg;
        return {a[0], a[1], a[2]};
    }
    if (t.kind == HK_TEX_CHECKERBOARD)
        return {(t.a[0] + t.b[0]) * 0.5f, (t.a[1] + t.b[1]) * 0.5f, (t.a[2] + t.b[2]) * 0.5f};
    if (t.kind == HK_TEX_WIREFRAME)   // (edge + interior) / 2 (src/texture/WireframeTexture.cpp:80)
        return {(t.b[0] + t.a[0]) * 0.5f, (t.b[1] + t.a[1]) * 0.5f, (t.b[2] + t.a[2]) * 0.5f};
    if (t.kind == HK_TEX_CURVATURE) return {0.5f, 0.5f, 0.5f};   // src/texture/CurvatureTexture.cpp:61
    float iw = std::max(0.0f, 1.0f - 2.0f * t.width);
    float ia = iw * iw, la = 1.0f - ia;
    return {t.a[0] * la + t.b[0] * ia, t.a[1] * la + t.b[1] * ia, t.a[2] * la + t.b[2] * ia};
}
// A parameter's average: its texture's or the constant
void par_average(const hk_scene *s, const hk_bsdf_desc &d, int slot, const float *c, float *out) {
    if (!d.tex[slot]) {
        for (int k = 0; k < 3; k++) out[k] = c[k];
        return;
    }
    F3 a = tex_average(s, d.tex[slot] - 1);
    out[0] = a.x; out[1] = a.y; out[2] = a.z;
}
// Whether texture id is (or scales) a wireframe or curvature texture
bool tex_geo(const hk_scene *s, int id) {
    while (s->textures[id].kind == HK_TEX_SCALE) id = s->textures[id].nested;
    return s->textures[id].kind == HK_TEX_WIREFRAME || s->textures[id].kind == HK_TEX_CURVATURE;
}
// The wireframe / curvature textures BSDF id reaches (its slots, nested BSDFs and
// maps), each once, through scale textures
void bsdf_geo_textures(const hk_scene *s, int id, int depth, std::vector<int> &out) {
    if (id < 0 || id >= (int)s->bsdfs.size() || depth > 8) return;
    const hk_bsdf_desc &d = s->bsdfs[id];
    for (int k = 0; k < 6; k++) {
        if (!d.tex[k]) continue;
        int t = d.tex[k] - 1;
        while (s->textures[t].kind == HK_TEX_SCALE) t = s->textures[t].nested;
        if ((s->textures[t].kind == HK_TEX_WIREFRAME || s->textures[t].kind == HK_TEX_CURVATURE) &&
            std::find(out.begin(), out.end(), t) == out.end())
            out.push_back(t);
    }
    const bool nests = d.type == hk::kRoughCoating || d.type == hk::kCoating || d.type == hk::kTwoSided ||
                       d.type == hk::kBumpMap || d.type == hk::kNormalMap;
    if (nests) bsdf_geo_textures(s, d.nested, depth + 1, out);
    if (d.type == hk::kTwoSided) bsdf_geo_textures(s, d.nested2, depth + 1, out);
}
bool bsdf_textured(const hk_scene *s, int id, int depth) {
    if (id < 0 || id >= (int)s->bsdfs.size() || depth > 8) return false;
    const hk_bsdf_desc &d = s->bsdfs[id];
    for (int k = 0; k < 6; k++)
        if (d.tex[k]) return true;
    return bsdf_textured(s, (d.type == hk::kRoughCoating || d.type == hk::kCoating || d.type == hk::kTwoSided) ? d.nested : -1, depth + 1) ||
           bsdf_textured(s, d.type == hk::kTwoSided ? d.nested2 : -1, depth + 1);
}

// Channel 0 of Texture::GetMinimum / GetMaximum, for the roughness range
// check of a textured alpha: checkerboard / grid / wireframe the smaller and
// larger colour, scale the nested range scaled, bitmaps their level-0
// texels, curvature [0, 1]
void tex_range0(const hk_scene *s, int id, float &lo, float &hi) {
    const hk_texture_desc &t = s->textures[id];
    if (t.kind == HK_TEX_SCALE) {
        tex_range0(s, t.nested, lo, hi);
        lo *= t.scale;
        hi *= t.scale;
        return;
    }
    if (t.kind == HK_TEX_CURVATURE) { lo = 0.0f; hi = 1.0f; return; }
    if (t.kind == HK_TEX_BITMAP) {
        const hk::MipPyramid &m = *s->bitmaps[id];
        lo = FLT_MAX;
        hi = -FLT_MAX;
        const std::vector<float> &L = m.lv[0];
        for (size_t i = 0; i < L.size(); i += (size_t)m.channels) {
            lo = std::min(lo, L[i]);
            hi = std::max(hi, L[i]);
        }
        return;
    }
    lo = std::min(t.a[0], t.b[0]);
    hi = std::max(t.a[0], t.b[0]);
}

bool is_layer(int type) { return type == hk::kRoughCoating || type == hk::kCoating || type == hk::kTwoSided; }

// Layers above the leaf BSDFs: 0 for a leaf, one more than the nested BSDF for
// a (rough) coating, one more than the deeper side for a twoSided; a cycle or
// an invalid index counts as too deep.
int layer_depth(const hk_scene *s, int id, int guard) {
    if (id < 0 || id >= (int)s->bsdfs.size() || guard > 2 * hk::kNestLevels) return 1 << 20;
    const hk_bsdf_desc &d = s->bsdfs[id];
    if (d.type == hk::kRoughCoating || d.type == hk::kCoating) return 1 + layer_depth(s, d.nested, guard + 1);
    if (d.type == hk::kTwoSided)
        return 1 + std::max(layer_depth(s, d.nested, guard + 1),
                            layer_depth(s, d.nested2 < 0 ? d.nested : d.nested2, guard + 1));
    return 0;
}

// Whether the one-level dispatch (a coating over a leaf; a twoSided over leaves
// or coatings over leaves) cannot evaluate the BSDF, so that it goes through
// the bounded-depth layer dispatch.
bool layer_deep(const hk_scene *s, const hk_bsdf_desc &d) {
    if (d.type == hk::kRoughCoating || d.type == hk::kCoating) return is_layer(s->bsdfs[d.nested].type);
    if (d.type != hk::kTwoSided) return false;
    for (int side : {d.nested, d.nested2 < 0 ? d.nested : d.nested2})
        if (s->bsdfs[side].type == hk::kTwoSided || layer_depth(s, side, 0) >= 2) return true;
    return false;
}

// rft_pool: where a textured alpha's 2D transmittance tables go (their
// offsets are kept in rft2d / rft_diff until the pool is on the device)
hk::DevBsdf activate_bsdf(const hk_scene *s, const hk_bsdf_desc &d, int n_bsdfs, std::vector<float> &rft_pool) {
    hk::DevBsdf b;
    std::memset(&b, 0, sizeof b);
    if (d.type < hk::kDiffuse || d.type > hk::kNormalMap) throw HkError{HK_ERR_INVALID, "unknown BSDF type"};
    for (int k = 0; k < 6; k++) {
        if (d.tex[k] < 0 || d.tex[k] > (int)s->textures.size()) throw HkError{HK_ERR_INVALID, "invalid texture id"};
        b.tex[k] = d.tex[k];
    }
    if (d.distribution != 0 && d.distribution != 1) throw HkError{HK_ERR_INVALID, "Unexpected distribution type"};
    b.type = d.type;
    b.distribution = d.distribution;
    b.anisotropic = d.anisotropic;
    b.nonlinear = d.nonlinear;
    b.alpha_u = clampf(d.alpha_u, 5e-4f, 1.0f);
    b.alpha_v = clampf(d.alpha_v, 5e-4f, 1.0f);
    b.eta = d.int_ior / d.ext_ior;
    b.inv_eta = 1.0f / b.eta;
    b.inv_eta2 = b.inv_eta * b.inv_eta;
    b.thickness = d.thickness;
    for (int c = 0; c < 3; c++) {
        b.eta_c[c] = d.eta[c];
        b.k_c[c] = d.k[c] / d.ext_ior;
        b.ks[c] = d.ks[c];
        b.ks_refract[c] = d.ks_refract[c];
        b.kd[c] = d.kd[c];
        b.sigma_a[c] = d.sigma_a[c];
    }
    b.nested = d.nested;
    b.nested2 = d.nested2;
    b.fast_approx = d.fast_approx;
    if (d.type == hk::kRoughPlastic || d.type == hk::kRoughCoating) {
        const RftTable &t = s->rft[d.distribution];
        if (!t.loaded) throw HkError{HK_ERR_INVALID, "RFT table for the BSDF's distribution was not set"};
        float alpha = b.alpha_u;
        float e = b.eta < 1.0f ? 1.0f / b.eta : b.eta;   // CheckEta / CheckAlpha (:315-345)
        if (e < t.eta_min || e > t.eta_max) throw HkError{HK_ERR_INVALID, "relative IOR outside the RFT table range"};
        b.alpha_tex = d.tex[4] ? 1 : 0;
        if (b.alpha_tex) {   // CheckAlpha(GetMinimum / GetMaximum) (RoughPlasticBSDF.cpp:268)
            float lo, hi;
            tex_range0(s, d.tex[4] - 1, lo, hi);
            if (lo < t.alpha_min || lo > t.alpha_max || hi < t.alpha_min || hi > t.alpha_max)
                throw HkError{HK_ERR_INVALID, "alpha texture outside the RFT range"};
        } else if (alpha < t.alpha_min || alpha > t.alpha_max) {
            throw HkError{HK_ERR_INVALID, "alpha outside the RFT range"};
        }
        std::vector<float> t2d, d1d;
        float dsc;
        t.set_eta(b.eta, t2d, d1d);
        b.rft_n = (int)t.theta_n;
        b.rft_an = (int)t.alpha_n;
        b.rft_amin = t.alpha_min;
        b.rft_amax = t.alpha_max;
        if (b.alpha_tex) {   // no SetAlpha: the 2D table is interpolated per query
            rft_pool.resize((rft_pool.size() + 3) & ~size_t(3));
            b.rft2d = reinterpret_cast<const float *>(rft_pool.size());
            rft_pool.insert(rft_pool.end(), t2d.begin(), t2d.end());
        } else {
            t.set_alpha(t2d, d1d, alpha, b.rft, dsc);
        }
        if (d.type == hk::kRoughPlastic) {
            float ksv[3], kdv[3];
            par_average(s, d, 1, d.ks, ksv);
            par_average(s, d, 0, d.kd, kdv);
            float ksa = lum(ksv), kda = lum(kdv);
            b.spec_w = ksa / (kda + ksa);
            t.set_eta(b.inv_eta, t2d, d1d);   // m_pIntData: SetEta(1/eta) only
            float wa = std::pow((alpha - t.alpha_min) / (t.alpha_max - t.alpha_min), 0.25f);
            b.fdr_int = 1.0f - clampf(cubic1d(wa, d1d.data(), (int)t.alpha_n, 0.0f, 1.0f), 0.0f, 1.0f);
            if (b.alpha_tex) {   // EvalDiffuse(alpha) per query
                rft_pool.resize((rft_pool.size() + 3) & ~size_t(3));
                b.rft_diff = reinterpret_cast<const float *>(rft_pool.size());
                rft_pool.insert(rft_pool.end(), d1d.begin(), d1d.end());
            }
        } else {
            float th = d.thickness;
            float sav[3];
            par_average(s, d, 3, d.sigma_a, sav);
            float a0 = std::exp(sav[0] * (-2.0f * th)), a1 = std::exp(sav[1] * (-2.0f * th)),
                  a2 = std::exp(sav[2] * (-2.0f * th));
            b.spec_w = 1.0f / ((a0 + a1 + a2) / 3.0f + 1.0f);
            if (d.nested < 0 || d.nested >= n_bsdfs) throw HkError{HK_ERR_INVALID, "RoughCoatingBSDF needs a nested BSDF!"};
            const int nt = s->bsdfs[d.nested].type;
            if (nt == hk::kBumpMap || nt == hk::kNormalMap)
                throw HkError{HK_ERR_INVALID, "roughCoating over a bumpMap or normalMap BSDF is not supported"};
        }
    }
    if (d.type == hk::kCoating) {   // CoatingBSDF::Activate (:255)
        float th = d.thickness;
        float sav[3];
            par_average(s, d, 3, d.sigma_a, sav);
            float a0 = std::exp(sav[0] * (-2.0f * th)), a1 = std::exp(sav[1] * (-2.0f * th)),
              a2 = std::exp(sav[2] * (-2.0f * th));
        b.spec_w = 1.0f / ((a0 + a1 + a2) / 3.0f + 1.0f);
        if (d.nested < 0 || d.nested >= n_bsdfs) throw HkError{HK_ERR_INVALID, "CoatingBSDF needs a nested BSDF!"};
        const int nt = s->bsdfs[d.nested].type;
        if (nt == hk::kBumpMap || nt == hk::kNormalMap)
            throw HkError{HK_ERR_INVALID, "coating over a bumpMap or normalMap BSDF is not supported"};
    }
    if (d.type == hk::kConductor)   // ConductorBSDF ctor (:17): m_Eta = Color3f(intIOR / extIOR)
        for (int c = 0; c < 3; c++) b.eta_c[c] = b.eta;
    if (d.type == hk::kPlastic) {   // PlasticBSDF ctor (:25) and Activate (:170)
        float ksv[3], kdv[3];
        par_average(s, d, 1, d.ks, ksv);
        par_average(s, d, 0, d.kd, kdv);
        float ksa = lum(ksv), kda = lum(kdv);
        b.spec_w = ksa / (kda + ksa);
        b.fdr_int = approx_fresnel_diffuse(b.inv_eta);
    }
    if (d.type == hk::kTwoSided) {   // TwoSidedBSDF::Activate (:98)
        if (d.nested < 0 || d.nested >= n_bsdfs) throw HkError{HK_ERR_INVALID, "TwoSidedBSDF needs at least one nested BSDF!"};
        if (d.nested2 >= n_bsdfs) throw HkError{HK_ERR_INVALID, "twoSided: invalid second nested BSDF"};
        if (d.nested2 < 0) b.nested2 = d.nested;
        for (int side : {b.nested, b.nested2}) {
            const int st = s->bsdfs[side].type;
            if (st == hk::kBumpMap || st == hk::kNormalMap)
                throw HkError{HK_ERR_INVALID, "twoSided over a bumpMap or normalMap BSDF is not supported"};
            if (bsdf_transmits(s, side, 0)) throw HkError{HK_ERR_INVALID, "Only BSDF without transmission can be nested!"};
        }
    }
    if (is_layer(d.type)) {
        if (layer_depth(s, (int)(&d - s->bsdfs.data()), 0) > hk::kNestLevels)
            throw HkError{HK_ERR_INVALID, "BSDF layers nested deeper than 4 (or in a cycle) are not supported"};
        b.deep = layer_deep(s, d) ? 1 : 0;
    }
    if (d.type == hk::kBumpMap || d.type == hk::kNormalMap) {   // BumpMapBSDF / NormalMapBSDF::Activate
        if (d.nested < 0 || d.nested >= n_bsdfs) throw HkError{HK_ERR_INVALID, "bumpMap / normalMap needs a nested BSDF"};
        if (d.tex[0] <= 0) throw HkError{HK_ERR_INVALID, "bumpMap / normalMap needs a map texture"};
        if (tex_geo(s, d.tex[0] - 1))
            throw HkError{HK_ERR_INVALID, "a wireframe or curvature texture as a bump / normal map is not supported"};
        const int nt = s->bsdfs[d.nested].type;
        if (nt == hk::kBumpMap || nt == hk::kNormalMap)
            throw HkError{HK_ERR_INVALID, "bumpMap / normalMap over another bumpMap / normalMap is not supported"};
    }
    return b;
}

void build_scene(hk_scene *s) {
    if (s->meshes.empty()) throw HkError{HK_ERR_INVALID, "scene has no meshes"};
    if (s->width == 0 || s->height == 0) throw HkError{HK_ERR_INVALID, "camera has an empty film"};
    // the perturbed frames need dP/du, dP/dv, which Triangle::PostIntersect sets
    // only with vertex normals and texture coordinates (the reference reads
    // stale or unset values otherwise)
    for (const MeshIn &m : s->meshes) {
        if (m.bsdf < 0 || m.bsdf >= (int)s->bsdfs.size()) continue;
        const int t = s->bsdfs[m.bsdf].type;
        if ((t == hk::kBumpMap || t == hk::kNormalMap) && (m.nrm.empty() || m.uv.empty()))
            throw HkError{HK_ERR_INVALID, "a mesh with a bumpMap / normalMap BSDF needs vertex normals and texture coordinates"};
    }
    s->wf.reset();   // the engine holds a copy of the device description that is rebuilt here
    hk::DevScene &D = s->dev;
    std::memset(&D, 0, sizeof D);
    size_t dev_bytes = 0;
    auto track = [&](DevBuf &b) { dev_bytes += b.bytes; };

    // BSDFs
    std::vector<hk::DevBsdf> bs;
    std::vector<hk::DevTexture> tex;
    // bitmap texels: one pool in HBM, the EWA weights first, then each
    // texture's levels (rgb as float4, 16-byte aligned; r as float)
    std::vector<float> pool(hk::kEwaLutSize);
    hk::ewa_weight_lut(pool.data());
    std::vector<size_t> base(s->textures.size(), 0);
    D.ray_diff = 0;
    for (size_t i = 0; i < s->textures.size(); ++i) {
        const hk::MipPyramid *m = s->bitmaps[i].get();
        if (!m) continue;
        pool.resize((pool.size() + 3) & ~size_t(3));
        base[i] = pool.size();
        for (auto &L : m->lv) {
            if (m->channels == 1) {
                pool.insert(pool.end(), L.begin(), L.end());
            } else {
                for (size_t k = 0; k < L.size(); k += 3) pool.insert(pool.end(), {L[k], L[k + 1], L[k + 2], 0.0f});
            }
        }
        if (pool.size() - base[i] >= (size_t)UINT32_MAX) throw HkError{HK_ERR_INVALID, "bitmap texture too large"};
        if (s->textures[i].filter >= HK_FILTER_TRILINEAR) D.ray_diff = 1;
    }
    if (pool.size() > hk::kEwaLutSize) { s->b_texels.upload(pool); track(s->b_texels); }
    const float *texels = s->b_texels.as<float>();
    // a wireframe texture's automatic edge width: a tenth of the mean edge
    // length of the first mesh (scene order) whose BSDF uses it (the reference
    // takes the first mesh that evaluates it, src/texture/WireframeTexture.cpp:37-53)
    std::vector<float> tex_width(s->textures.size());
    for (size_t i = 0; i < s->textures.size(); ++i) tex_width[i] = s->textures[i].width;
    std::vector<char> width_set(s->textures.size(), 0);
    for (const MeshIn &m : s->meshes) {
        std::vector<int> used;
        bsdf_geo_textures(s, m.bsdf, 0, used);
        for (int t : used) {
            if (s->textures[t].kind != HK_TEX_WIREFRAME || s->textures[t].width != 0.0f || width_set[t]) continue;
            float ew = 0.0f;
            const size_t nt = m.idx.size() / 3;
            for (size_t f = 0; f < nt; ++f) {
                const float *p0 = &m.pos[3 * (size_t)m.idx[3 * f]], *p1 = &m.pos[3 * (size_t)m.idx[3 * f + 1]],
                            *p2 = &m.pos[3 * (size_t)m.idx[3 * f + 2]];
                const float l0 = f3norm(F3{p1[0] - p0[0], p1[1] - p0[1], p1[2] - p0[2]});
                const float l1 = f3norm(F3{p2[0] - p1[0], p2[1] - p1[1], p2[2] - p1[2]});
                const float l2 = f3norm(F3{p0[0] - p2[0], p0[1] - p2[1], p0[2] - p2[2]});
                ew += (l0 + l1) + l2;
            }
            tex_width[t] = 0.1f * ew / (float)(3u * (uint32_t)nt);
            width_set[t] = 1;
        }
    }
    for (size_t i = 0; i < s->textures.size(); ++i) {
        const hk_texture_desc &t = s->textures[i];
        hk::DevTexture x;
        std::memset(&x, 0, sizeof x);
        x.kind = t.kind; x.nested = t.nested; x.count = t.count; x.width = tex_width[i]; x.scale = t.scale;
        for (int k = 0; k < 2; k++) { x.uv_scale[k] = t.uv_scale[k]; x.uv_offset[k] = t.uv_offset[k]; }
        for (int k = 0; k < 3; k++) { x.a[k] = t.a[k]; x.b[k] = t.b[k]; }
        if (const hk::MipPyramid *m = s->bitmaps[i].get()) {
            x.filter = t.filter;
            x.channels = m->channels;
            x.levels = m->levels; x.lw = m->lw; x.lh = m->lh;
            x.black = (t.wrap_u == HK_WRAP_BLACK || t.wrap_v == HK_WRAP_BLACK) ? 1 : 0;
            x.max_aniso = t.max_anisotropy;
            x.texels = texels + base[i];
            x.lut = texels;
            uint32_t off = 0;
            for (int l = 0; l < m->levels; ++l) {
                x.lvl_off[l] = off;
                off += (uint32_t)(m->lv[(size_t)l].size() / (size_t)m->channels);
            }
        }
        tex.push_back(x);
    }
    s->b_textures.upload(tex); track(s->b_textures);
    std::vector<float> rft_pool;
    for (auto &d : s->bsdfs) bs.push_back(activate_bsdf(s, d, (int)s->bsdfs.size(), rft_pool));
    s->bsdf_deep.clear();
    for (const hk::DevBsdf &b : bs) s->bsdf_deep.push_back(b.deep);
    if (!rft_pool.empty()) { s->b_rft2d.upload(rft_pool); track(s->b_rft2d); }
    for (size_t i = 0; i < bs.size(); ++i) {
        if (bs[i].alpha_tex) {   // pool offsets -> device pointers
            const float *base = s->b_rft2d.as<float>();
            bs[i].rft2d = base + reinterpret_cast<size_t>(bs[i].rft2d);
            if (bs[i].type == hk::kRoughPlastic) bs[i].rft_diff = base + reinterpret_cast<size_t>(bs[i].rft_diff);
        }
        bs[i].textures = s->b_textures.as<hk::DevTexture>();
        bs[i].textured = bsdf_textured(s, (int)i, 0) ? 1 : 0;
        std::vector<int> geo;
        bsdf_geo_textures(s, (int)i, 0, geo);
        bs[i].geo_tex = geo.empty() ? 0 : 1;
        D.textured |= bs[i].textured;
    }
    s->b_bsdfs.upload(bs); track(s->b_bsdfs);
    D.bsdfs = s->b_bsdfs.as<hk::DevBsdf>();
    D.nbsdfs = (int)bs.size();

    // meshes, global triangles
    std::vector<hk::DevMesh> dm;
    uint64_t ntris = 0;
    bool any_normals = false;
    for (auto &m : s->meshes) ntris += m.idx.size() / 3;
    if (ntris >= (1ull << hk::kLeafCountShift)) throw HkError{HK_ERR_INVALID, "too many triangles"};
    std::vector<float> P;       // 9 floats per triangle (original order)
    std::vector<int32_t> tmesh;
    P.reserve(ntris * 9);
    tmesh.reserve(ntris);
    std::vector<float> tri_normals;   // 12 floats per triangle (3 float4) if any normals
    std::vector<float> tri_uv;        // 6 floats per triangle (3 float2) if any texture coordinates
    bool any_uv = false;
    for (auto &m : s->meshes) {
        any_normals |= !m.nrm.empty();
        any_uv |= !m.uv.empty();
    }
    if (any_normals) tri_normals.resize(ntris * 12, 0.0f);
    if (any_uv) tri_uv.resize(ntris * 6, 0.0f);
    float bb[6] = {INFINITY, INFINITY, INFINITY, -INFINITY, -INFINITY, -INFINITY};
    std::vector<int> mesh_emitter(s->meshes.size(), -1);
    for (size_t e = 0; e < s->emitter_mesh.size(); ++e)
        if (s->emitter_mesh[e] >= 0) mesh_emitter[s->emitter_mesh[e]] = (int)e;
    uint64_t t = 0;
    for (size_t mi = 0; mi < s->meshes.size(); ++mi) {
        auto &m = s->meshes[mi];
        hk::DevMesh d;
        std::memset(&d, 0, sizeof d);
        if (m.bsdf < 0 || m.bsdf >= (int)bs.size()) throw HkError{HK_ERR_INVALID, "mesh has an invalid BSDF id"};
        d.bsdf = m.bsdf;
        d.emitter = mesh_emitter[mi];
        d.has_normals = !m.nrm.empty();
        d.has_uv = !m.uv.empty();
        for (int c = 0; c < 3; c++) d.radiance[c] = m.radiance[c];
        dm.push_back(d);
        size_t nv = m.pos.size() / 3;
        for (size_t v = 0; v < nv; ++v)
            for (int c = 0; c < 3; c++) {
                bb[c] = std::min(bb[c], m.pos[3 * v + c]);
                bb[3 + c] = std::max(bb[3 + c], m.pos[3 * v + c]);
            }
        for (size_t f = 0; f < m.idx.size() / 3; ++f, ++t) {
            for (int k = 0; k < 3; k++) {
                uint32_t vi = m.idx[3 * f + k];
                for (int c = 0; c < 3; c++) P.push_back(m.pos[3 * vi + c]);
                if (any_normals && !m.nrm.empty())
                    for (int c = 0; c < 3; c++) tri_normals[t * 12 + 4 * k + c] = m.nrm[3 * vi + c];
                if (any_uv && !m.uv.empty())
                    for (int c = 0; c < 2; c++) tri_uv[t * 6 + 2 * k + c] = m.uv[2 * vi + c];
            }
            tmesh.push_back((int32_t)mi);
        }
    }
    s->b_meshes.upload(dm); track(s->b_meshes);
    D.meshes = s->b_meshes.as<hk::DevMesh>();
    D.nmeshes = (int)dm.size();
    if (any_normals) { s->b_tri_normals.upload(tri_normals); track(s->b_tri_normals); }
    D.tri_normals = s->b_tri_normals.as<float4>();
    if (any_uv) { s->b_tri_uv.upload(tri_uv); track(s->b_tri_uv); }
    D.tri_uv = s->b_tri_uv.as<float2>();

    const auto t_tree = std::chrono::steady_clock::now();
    uint32_t tree_depth2 = 0, tree_depth8 = 0;
    if (s->builder == HK_BUILDER_GPU) {
        // the 8-wide tree built on the device (no binary tree)
        if (s->accel != HK_ACCEL_BVH8) throw HkError{HK_ERR_INVALID, "the device builder makes the 8-wide tree only"};
        DevBuf dP, dmesh;
        dP.upload(P);
        dmesh.upload(tmesh);
        hk::GpuBvh8 G;
        hk::build_bvh8_gpu(dP.as<float>(), (uint32_t)ntris, nullptr, G);
        s->b_tris.alloc((size_t)ntris * 48);
        hk::gather_tri_records(dP.as<float>(), dmesh.as<int32_t>(), G.order.as<uint32_t>(), (uint32_t)ntris,
                               s->b_tris.as<float>(), nullptr);
        HK_CUDA(cudaDeviceSynchronize());
        track(s->b_tris);
        s->b_nodes.release();
        s->b_wnodes.take(G.nodes);
        track(s->b_wnodes);
        D.tris = s->b_tris.as<float4>();
        D.nodes = nullptr;
        D.nnodes = 0;
        D.ntris = (uint32_t)ntris;
        D.wnodes = s->b_wnodes.as<uint4>();
        D.nwnodes = G.nnodes;
        tree_depth8 = G.depth;
        D.postpone = 2 * (int)G.depth + 2 <= hk::kStackSize ? 1 : 0;
        if ((int)G.depth + 1 > hk::kStackSize) throw HkError{HK_ERR_INVALID, "8-wide BVH too deep"};
        D.accel = s->accel;
        s->tree_build_s = std::chrono::duration<double>(std::chrono::steady_clock::now() - t_tree).count();
    } else {
    // BVH: one binned-SAH build, packed as the binary tree and collapsed into
    // the compressed 8-wide tree over one triangle order
    hk::BvhPair pair = hk::build_bvh_pair(P.data(), (uint32_t)ntris);
    const hk::Bvh2 &bvh = pair.bvh2;
    std::vector<float> recs(bvh.tri_order.size() * 12);
    for (size_t i = 0; i < bvh.tri_order.size(); ++i) {
        uint32_t o = bvh.tri_order[i];
        float *r = &recs[i * 12];
        for (int k = 0; k < 3; k++)
            for (int c = 0; c < 3; c++) r[4 * k + c] = P[9 * o + 3 * k + c];
        int32_t oi = (int32_t)o, mm = tmesh[o];
        std::memcpy(&r[3], &oi, 4);
        std::memcpy(&r[7], &mm, 4);
        r[11] = 0.0f;
    }
    s->b_tris.upload(recs); track(s->b_tris);
    s->b_nodes.upload(bvh.nodes); track(s->b_nodes);
    D.tris = s->b_tris.as<float4>();
    D.nodes = s->b_nodes.as<float4>();
    D.ntris = (uint32_t)ntris;
    D.nnodes = (uint32_t)(bvh.nodes.size() / 16);
    s->b_wnodes.upload(pair.bvh8.nodes); track(s->b_wnodes);
    D.wnodes = s->b_wnodes.as<uint4>();
    D.nwnodes = (uint32_t)(pair.bvh8.nodes.size() / 20);
    // the traversal stack holds at most one node group and one postponed
    // triangle group per level (plus the root)
    tree_depth2 = bvh.depth;
    tree_depth8 = pair.bvh8.depth;
    D.postpone = 2 * (int)pair.bvh8.depth + 2 <= hk::kStackSize ? 1 : 0;
    if ((int)pair.bvh8.depth + 1 > hk::kStackSize) throw HkError{HK_ERR_INVALID, "8-wide BVH too deep"};
    D.accel = s->accel;
    s->tree_build_s = std::chrono::duration<double>(std::chrono::steady_clock::now() - t_tree).count();
    }

    // emitters (Scene order)
    std::vector<int32_t> emitter_area;
    std::vector<hk::DevAreaLight> area;
    std::vector<float> ltris, lnorms, lcdf;
    D.env_index = -1;
    for (size_t e = 0; e < s->emitter_mesh.size(); ++e) {
        int mi = s->emitter_mesh[e];
        if (mi == -1) { emitter_area.push_back(-1); D.env_index = (int)e; continue; }
        if (mi < -1) { emitter_area.push_back(mi); continue; }   // point / directional light -2 - k
        auto &m = s->meshes[mi];
        hk::DevAreaLight L;
        std::memset(&L, 0, sizeof L);
        L.tri0 = (uint32_t)(ltris.size() / 12);
        L.ntri = (uint32_t)(m.idx.size() / 3);
        L.cdf0 = (uint32_t)lcdf.size();
        L.mesh = mi;
        std::vector<float> areas(L.ntri);
        float total = 0.0f;
        for (uint32_t f = 0; f < L.ntri; ++f) {   // Mesh::Activate / SurfaceArea (src/core/Mesh.cpp:233,311)
            F3 p[3];
            for (int k = 0; k < 3; k++) {
                uint32_t vi = m.idx[3 * f + k];
                p[k] = {m.pos[3 * vi], m.pos[3 * vi + 1], m.pos[3 * vi + 2]};
                for (int c = 0; c < 3; c++) ltris.push_back(c == 0 ? p[k].x : (c == 1 ? p[k].y : p[k].z));
                ltris.push_back(0.0f);
                if (!m.nrm.empty()) {
                    for (int c = 0; c < 3; c++) lnorms.push_back(m.nrm[3 * vi + c]);
                    lnorms.push_back(1.0f);
                } else {
                    for (int c = 0; c < 4; c++) lnorms.push_back(0.0f);
                }
            }
            float a = 0.5f * f3norm(f3cross(f3sub(p[1], p[0]), f3sub(p[2], p[0])));
            areas[f] = a;
            total += a;
        }
        L.inv_area = 1.0f / total;
        Pdf1D pdf;
        pdf.build(areas.data(), (int)L.ntri);
        lcdf.insert(lcdf.end(), pdf.cdf.begin(), pdf.cdf.end());
        for (int c = 0; c < 3; c++) L.radiance[c] = m.radiance[c];
        emitter_area.push_back((int32_t)area.size());
        area.push_back(L);
    }
    s->b_emitter_area.upload(emitter_area); track(s->b_emitter_area);
    s->b_area.upload(area); track(s->b_area);
    s->b_light_tris.upload(ltris); track(s->b_light_tris);
    s->b_light_normals.upload(lnorms); track(s->b_light_normals);
    s->b_light_cdf.upload(lcdf); track(s->b_light_cdf);
    D.nemitters = (int)emitter_area.size();
    D.emitter_area = s->b_emitter_area.as<int32_t>();
    D.area_lights = s->b_area.as<hk::DevAreaLight>();
    D.light_tris = s->b_light_tris.as<float4>();
    D.light_normals = s->b_light_normals.as<float4>();
    D.light_cdf = s->b_light_cdf.as<float>();

    // point / directional lights: (position or direction, kind), (power or irradiance, 0)
    std::vector<float> delta;
    for (auto &l : s->delta_lights) {
        for (int c = 0; c < 3; c++) delta.push_back(l.vec[c]);
        delta.push_back((float)l.directional);
        for (int c = 0; c < 3; c++) delta.push_back(l.color[c]);
        delta.push_back(0.0f);
    }
    s->b_delta.upload(delta); track(s->b_delta);
    D.delta_lights = s->b_delta.as<float4>();
    D.env_kind = s->has_env ? (s->env_constant ? hk::kEnvConstant : hk::kEnvMap) : 0;
    for (int c = 0; c < 3; c++) D.env_const[c] = s->env_const[c];

    // environment (EnvironmentLight ctor, src/emitter/EnvironmentLight.cpp:8-31)
    if (s->has_env && !s->env_constant) {
        uint32_t W = s->env_w, H = s->env_h;
        std::vector<float> rgb4((size_t)W * H * 4), lumv((size_t)W * H);
        for (uint32_t y = 0; y < H; y++) {
            float th = float(y + 0.5f) / H * float(M_PI);
            float st = std::sin(th);
            for (uint32_t x = 0; x < W; x++) {
                const float *c = &s->env_rgb[3 * ((size_t)y * W + x)];
                float *o = &rgb4[4 * ((size_t)y * W + x)];
                o[0] = c[0]; o[1] = c[1]; o[2] = c[2]; o[3] = 0.0f;
                lumv[(size_t)y * W + x] = lum(c) * st;
            }
        }
        std::vector<float> ccdf((size_t)H * (W + 1)), cfunc((size_t)H * W), cint(H), marg(H);
        std::vector<int32_t> cguide((size_t)H * (kCdfGuide + 1)), mguide(kCdfGuide + 1);
        for (uint32_t y = 0; y < H; y++) {
            Pdf1D r;
            r.build(&lumv[(size_t)y * W], (int)W);
            std::copy(r.cdf.begin(), r.cdf.end(), ccdf.begin() + (size_t)y * (W + 1));
            std::copy(r.func.begin(), r.func.end(), cfunc.begin() + (size_t)y * W);
            cint[y] = r.integral;
            marg[y] = r.integral;
            cdf_guide(r.cdf.data(), (int)W, &cguide[(size_t)y * (kCdfGuide + 1)]);
        }
        Pdf1D mp;
        mp.build(marg.data(), (int)H);
        cdf_guide(mp.cdf.data(), (int)H, mguide.data());
        s->b_env_marg_guide.upload(mguide); track(s->b_env_marg_guide);
        s->b_env_cond_guide.upload(cguide); track(s->b_env_cond_guide);
        D.env_marg_guide = s->b_env_marg_guide.as<int32_t>();
        D.env_cond_guide = s->b_env_cond_guide.as<int32_t>();
        s->b_env_rgb.upload(rgb4); track(s->b_env_rgb);
        s->b_env_marg_cdf.upload(mp.cdf); track(s->b_env_marg_cdf);
        s->b_env_marg_func.upload(mp.func); track(s->b_env_marg_func);
        s->b_env_cond_cdf.upload(ccdf); track(s->b_env_cond_cdf);
        s->b_env_cond_func.upload(cfunc); track(s->b_env_cond_func);
        s->b_env_cond_int.upload(cint); track(s->b_env_cond_int);
        D.env_rgb = s->b_env_rgb.as<float4>();
        D.env_marg_cdf = s->b_env_marg_cdf.as<float>();
        D.env_marg_func = s->b_env_marg_func.as<float>();
        D.env_cond_cdf = s->b_env_cond_cdf.as<float>();
        D.env_cond_func = s->b_env_cond_func.as<float>();
        D.env_cond_int = s->b_env_cond_int.as<float>();
        D.env_marg_int = mp.integral;
        D.env_w = W;
        D.env_h = H;
        D.env_scale = s->env_scale;
        for (int r = 0; r < 3; r++)
            for (int c = 0; c < 3; c++) D.env_to_world[3 * r + c] = s->env_to_world[4 * r + c];
        mat3_inverse(D.env_to_world, D.env_to_local);
    }
    // BoundingBox::GetRadius of the accel bbox (include/core/BoundingBox.hpp:453)
    D.scene_radius = f3norm(F3{bb[3] - bb[0], bb[4] - bb[1], bb[5] - bb[2]}) * 0.5f;

    // camera (PerspectiveCamera::Activate, src/camera/PerspectiveCamera.cpp:32)
    D.width = s->width;
    D.height = s->height;
    D.cam_aspect = float(s->width) / float(s->height);
    D.cam_cot = 1.0f / std::tan((s->fov / 2.0f) * (float(M_PI) / 180.0f));
    D.cam_near = s->near_clip;
    D.cam_far = s->far_clip;
    const float *M = s->cam_to_world;
    float w = M[15];
    for (int r = 0; r < 3; r++) {
        for (int c = 0; c < 3; c++) D.cam[4 * r + c] = M[4 * r + c];
        D.cam[4 * r + 3] = M[4 * r + 3] / w;
    }
    // filter table (ImageBlock ctor, src/core/Block.cpp:9-30)
    std::vector<float> ftab(33);
    for (int i = 0; i < 32; i++) ftab[i] = filter_eval(s, (s->filt_r * i) / 32);
    ftab[32] = 0.0f;
    s->b_ftab.upload(ftab); track(s->b_ftab);
    D.ftab = s->b_ftab.as<float>();
    D.filt_radius = s->filt_r;
    D.filt_lookup = 32 / s->filt_r;
    D.border = (int)std::ceil(s->filt_r - 0.5f);
    if (D.border > 8) throw HkError{HK_ERR_INVALID, "reconstruction filter radius too large (max 8.5)"};
    for (int c = 0; c < 3; c++) D.background[c] = s->background[c];
    D.force_background = s->force_background;
    s->margin_lo = (int)std::ceil(D.border - 0.5f - s->filt_r);
    s->margin_hi = (int)std::floor(D.border + 0.5f + s->filt_r);

    // scratch: [0] work counter (u32 in a u64 slot), [1..3] counters
    s->b_scratch.alloc(16 * sizeof(unsigned long long));
    HK_CUDA(cudaMemset(s->b_scratch.p, 0, s->b_scratch.bytes));
    track(s->b_scratch);

    int dev = 0;
    HK_CUDA(cudaGetDevice(&dev));
    s->device = dev;
    HK_CUDA(cudaDeviceGetAttribute(&s->sm_count, cudaDevAttrMultiProcessorCount, dev));
    for (int a = 0; a < 2; ++a) s->occupancy_of[a] = std::max(1, hk::render_occupancy(s->margin_lo, s->margin_hi, a, D.textured != 0));
    s->occupancy = s->occupancy_of[D.accel];
    HK_CUDA(cudaGetLastError());

    hk_scene_info &I = s->info;
    I.n_meshes = (uint32_t)s->meshes.size();
    I.n_triangles = (uint32_t)ntris;
    I.n_bsdfs = (uint32_t)bs.size();
    I.n_emitters = (uint32_t)emitter_area.size();
    I.n_bvh_nodes = D.nnodes;
    I.bvh_depth = tree_depth2;
    I.n_wide_nodes = D.nwnodes;
    I.wide_depth = tree_depth8;
    I.accel = D.accel;
    I.postpone = D.postpone;
    I.env_index = D.env_index;
    I.film_border = D.border;
    std::memcpy(I.bbox, bb, sizeof bb);
    I.device_bytes = dev_bytes;
    s->built = true;
}

void require_built(const hk_scene *s) {
    if (!s) throw HkError{HK_ERR_INVALID, "null scene"};
    if (!s->built) throw HkError{HK_ERR_INVALID, "scene is not built (call hk_scene_build)"};
}
// The megakernel entry points render at the scene camera's size only.
void require_scene_size(const hk_scene *s, const hk_render_desc &d) {
    if ((d.width != 0 && (uint32_t)d.width != s->width) || (d.height != 0 && (uint32_t)d.height != s->height))
        throw HkError{HK_ERR_INVALID, "this entry point renders at the scene camera's resolution only"};
}

// ------------------------------------------------------------ wavefront engine
hk::WfEngine &wf_ensure(hk_scene *s, const hk::WfEngineConfig &c) {
    if (s->wf) {
        const hk::WfEngineConfig &o = s->wf->config();
        if (o.capacity == c.capacity && o.threads_extend == c.threads_extend && o.threads_shade == c.threads_shade &&
            o.fetch_steps == c.fetch_steps && o.fetch_min_idle == c.fetch_min_idle &&
            o.fetch_steps_shadow == c.fetch_steps_shadow && o.fetch_min_idle_shadow == c.fetch_min_idle_shadow &&
            o.reg_lean == c.reg_lean && o.shadow_tests == c.shadow_tests && o.closest_tests == c.closest_tests)
            return *s->wf;
        s->wf.reset();
    }
    s->wf.reset(new hk::WfEngine(s->dev, s->sm_count, c));
    return *s->wf;
}

}  // namespace

namespace hk {

SceneView scene_view(hk_scene *s) {
    require_built(s);
    SceneView v;
    v.dev = &s->dev;
    v.sm_count = s->sm_count;
    v.width = s->width;
    v.height = s->height;
    v.cfg = &s->wf_cfg;
    v.has_cfg = &s->has_wf_cfg;
    return v;
}

JobSize job_size(const hk_scene *s, const hk_render_desc &d) {
    if (d.width < 0 || d.height < 0) throw HkError{HK_ERR_INVALID, "negative image size"};
    JobSize z;
    z.width = d.width > 0 ? (uint32_t)d.width : s->width;
    z.height = d.height > 0 ? (uint32_t)d.height : s->height;
    if (z.width > 16384 || z.height > 16384) throw HkError{HK_ERR_INVALID, "image larger than 16384 x 16384"};
    const size_t FW = z.width + 2 * (size_t)s->dev.border, FH = z.height + 2 * (size_t)s->dev.border;
    z.film_bytes = FW * FH * 4 * sizeof(float);
    z.rgb_bytes = (size_t)z.width * z.height * 3 * sizeof(float);
    return z;
}

WfJob make_wf_job(const hk_scene *s, const hk_render_desc &d) {
    if (d.spp <= 0 || d.depth < 0) throw HkError{HK_ERR_INVALID, "bad job: spp must be > 0 and depth >= 0"};
    const JobSize z = job_size(s, d);
    WfJob o;
    std::memset(&o, 0, sizeof o);
    std::memcpy(o.cam, s->dev.cam, sizeof o.cam);
    if (d.use_camera) {
        const float *M = d.camera_to_world;
        if (M[15] == 0.0f) throw HkError{HK_ERR_INVALID, "camera_to_world has w = 0"};
        for (int r = 0; r < 3; r++) {
            for (int c = 0; c < 3; c++) o.cam[4 * r + c] = M[4 * r + c];
            o.cam[4 * r + 3] = M[4 * r + 3] / M[15];
        }
    }
    const uint32_t tiles_x = (z.width + kWfTileSide - 1) / kWfTileSide;
    const uint32_t tiles_y = (z.height + kWfTileSide - 1) / kWfTileSide;
    o.seed = d.seed;
    o.spp = (uint32_t)d.spp;
    o.sample_offset = (uint32_t)d.sample_offset;
    o.image_index = (uint32_t)d.image_index;
    o.tiles_x = tiles_x;
    o.width = z.width;
    o.height = z.height;
    o.cam_aspect = float(z.width) / float(z.height);   // PerspectiveCamera::Activate aspect
    o.depth = d.depth;
    o.rr_start = d.rr_start;
    o.work_count = (uint64_t)tiles_x * tiles_y * (uint64_t)d.spp * kWfTilePixels;
    return o;
}

}  // namespace hk

extern "C" {

const char *hk_last_error(void) { return hk::g_error.c_str(); }
int hk_version(void) { return 1; }

int hk_scene_create(hk_scene **out) {
    return guarded([&] {
        if (!out) throw HkError{HK_ERR_INVALID, "null output pointer"};
        *out = new hk_scene();
        return HK_OK;
    });
}
int hk_scene_destroy(hk_scene *s) {
    return guarded([&] {
        delete s;
        return HK_OK;
    });
}
int hk_scene_set_rft(hk_scene *s, int distribution, const void *bytes, uint64_t nbytes) {
    return guarded([&] {
        if (!s || !bytes || (distribution != 0 && distribution != 1)) throw HkError{HK_ERR_INVALID, "bad arguments"};
        s->rft[distribution].parse(bytes, nbytes);
        s->built = false;
        return HK_OK;
    });
}
int hk_scene_add_texture(hk_scene *s, const hk_texture_desc *d, int32_t *out_id) {
    return guarded([&] {
        if (!s || !d) throw HkError{HK_ERR_INVALID, "bad arguments"};
        const bool geo = d->kind == HK_TEX_WIREFRAME || d->kind == HK_TEX_CURVATURE;
        if ((d->kind < HK_TEX_CHECKERBOARD || d->kind > HK_TEX_SCALE) && !geo)
            throw HkError{HK_ERR_INVALID, "unknown texture kind"};
        if (d->kind == HK_TEX_SCALE && (d->nested < 0 || d->nested >= (int)s->textures.size()))
            throw HkError{HK_ERR_INVALID, "scale texture needs a nested texture"};
        if (d->kind != HK_TEX_SCALE && !geo && d->count <= 0)
            throw HkError{HK_ERR_INVALID, "texture block / line count must be positive"};
        s->textures.push_back(*d);
        s->bitmaps.push_back(nullptr);
        if (out_id) *out_id = (int32_t)s->textures.size() - 1;
        s->built = false;
        return HK_OK;
    });
}
int hk_scene_add_bitmap(hk_scene *s, const hk_texture_desc *d, const uint8_t *pixels, int32_t width, int32_t height,
                        int32_t *out_id) {
    return guarded([&] {
        if (!s || !d) throw HkError{HK_ERR_INVALID, "bad arguments"};
        if (d->kind != HK_TEX_BITMAP) throw HkError{HK_ERR_INVALID, "bitmap texture expected"};
        std::shared_ptr<hk::MipPyramid> m;
        try {
            m = std::make_shared<hk::MipPyramid>(hk::build_bitmap(*d, pixels, width, height));
        } catch (const std::invalid_argument &e) {
            throw HkError{HK_ERR_INVALID, e.what()};
        }
        s->textures.push_back(*d);
        s->bitmaps.push_back(std::move(m));
        if (out_id) *out_id = (int32_t)s->textures.size() - 1;
        s->built = false;
        return HK_OK;
    });
}
int hk_scene_add_bsdf(hk_scene *s, const hk_bsdf_desc *d, int32_t *out_id) {
    return guarded([&] {
        if (!s || !d) throw HkError{HK_ERR_INVALID, "bad arguments"};
        const int nb = (int)s->bsdfs.size();
        if (d->type < HK_BSDF_DIFFUSE || d->type > HK_BSDF_NORMAL_MAP) throw HkError{HK_ERR_INVALID, "unknown BSDF type"};
        if (d->type == HK_BSDF_ROUGH_COATING && (d->nested < 0 || d->nested >= nb))
            throw HkError{HK_ERR_INVALID, "RoughCoatingBSDF needs a nested BSDF!"};
        if (d->type == HK_BSDF_COATING && (d->nested < 0 || d->nested >= nb))
            throw HkError{HK_ERR_INVALID, "CoatingBSDF needs a nested BSDF!"};
        if (d->type == HK_BSDF_TWO_SIDED && (d->nested < 0 || d->nested >= nb || d->nested2 >= nb))
            throw HkError{HK_ERR_INVALID, "TwoSidedBSDF needs at least one nested BSDF!"};
        s->bsdfs.push_back(*d);
        if (out_id) *out_id = (int32_t)s->bsdfs.size() - 1;
        s->built = false;
        return HK_OK;
    });
}
int hk_scene_add_mesh(hk_scene *s, const float *pos, uint32_t nv, const uint32_t *idx, uint32_t nt, const float *nrm,
                      int32_t bsdf, const float *rad, int32_t *out_id) {
    return guarded([&] {
        if (!s || !pos || !idx || nv == 0 || nt == 0) throw HkError{HK_ERR_INVALID, "mesh needs vertices and faces"};
        MeshIn m;
        m.pos.assign(pos, pos + 3 * (size_t)nv);
        m.idx.assign(idx, idx + 3 * (size_t)nt);
        for (uint32_t v : m.idx)
            if (v >= nv) throw HkError{HK_ERR_INVALID, "mesh index out of range"};
        if (nrm) m.nrm.assign(nrm, nrm + 3 * (size_t)nv);
        m.bsdf = bsdf;
        m.emitter = rad != nullptr;
        for (int c = 0; c < 3; c++) m.radiance[c] = rad ? rad[c] : 0.0f;
        s->meshes.push_back(std::move(m));
        if (rad) s->emitter_mesh.push_back((int)s->meshes.size() - 1);
        if (out_id) *out_id = (int32_t)s->meshes.size() - 1;
        s->built = false;
        return HK_OK;
    });
}
int hk_scene_set_mesh_uv(hk_scene *s, int32_t mesh, const float *uv) {
    return guarded([&] {
        if (!s || !uv || mesh < 0 || mesh >= (int)s->meshes.size()) throw HkError{HK_ERR_INVALID, "bad arguments"};
        MeshIn &m = s->meshes[mesh];
        m.uv.assign(uv, uv + m.pos.size() / 3 * 2);
        s->built = false;
        return HK_OK;
    });
}
int hk_scene_set_envmap(hk_scene *s, const float *rgb, uint32_t w, uint32_t h, const float *tw16, float scale) {
    return guarded([&] {
        if (!s || !rgb || !tw16 || w == 0 || h == 0) throw HkError{HK_ERR_INVALID, "bad arguments"};
        if (s->has_env) throw HkError{HK_ERR_INVALID, "Only one environment emitter is allowed for the entire scene"};
        s->has_env = true;
        s->env_w = w;
        s->env_h = h;
        s->env_rgb.assign(rgb, rgb + 3 * (size_t)w * h);
        std::memcpy(s->env_to_world, tw16, 64);
        s->env_scale = scale;
        s->emitter_mesh.push_back(-1);
        s->built = false;
        return HK_OK;
    });
}
int hk_scene_set_constant_light(hk_scene *s, const float *radiance) {
    return guarded([&] {
        if (!s || !radiance) throw HkError{HK_ERR_INVALID, "bad arguments"};
        if (s->has_env) throw HkError{HK_ERR_INVALID, "Only one environment emitter is allowed for the entire scene"};
        s->has_env = true;
        s->env_constant = true;
        for (int c = 0; c < 3; c++) s->env_const[c] = radiance[c];
        s->emitter_mesh.push_back(-1);
        s->built = false;
        return HK_OK;
    });
}
static int add_delta_light(hk_scene *s, int directional, const float *color, const float *vec) {
    return guarded([&] {
        if (!s || !color || !vec) throw HkError{HK_ERR_INVALID, "bad arguments"};
        hk_scene::DeltaLight l;
        l.directional = directional;
        for (int c = 0; c < 3; c++) { l.color[c] = color[c]; l.vec[c] = vec[c]; }
        s->emitter_mesh.push_back(-2 - (int)s->delta_lights.size());
        s->delta_lights.push_back(l);
        s->built = false;
        return HK_OK;
    });
}
int hk_scene_add_point_light(hk_scene *s, const float *power, const float *position) {
    return add_delta_light(s, 0, power, position);
}
int hk_scene_add_directional_light(hk_scene *s, const float *irradiance, const float *direction) {
    return add_delta_light(s, 1, irradiance, direction);
}
int hk_scene_set_camera(hk_scene *s, uint32_t w, uint32_t h, const float *tw16, float fov, float n, float f) {
    return guarded([&] {
        if (!s || w == 0 || h == 0) throw HkError{HK_ERR_INVALID, "bad camera"};
        s->width = w;
        s->height = h;
        if (tw16) std::memcpy(s->cam_to_world, tw16, 64);
        s->fov = fov;
        s->near_clip = n;
        s->far_clip = f;
        s->built = false;
        return HK_OK;
    });
}
int hk_scene_set_filter(hk_scene *s, int kind, float r, float p0, float p1) {
    return guarded([&] {
        if (!s || kind < 0 || kind > 3 || !(r > 0.0f)) throw HkError{HK_ERR_INVALID, "bad filter"};
        s->filt_kind = kind;
        s->filt_r = r;
        s->filt_p0 = p0;
        s->filt_p1 = p1;
        s->built = false;
        return HK_OK;
    });
}
int hk_scene_set_background(hk_scene *s, const float *rgb, int force) {
    return guarded([&] {
        if (!s || !rgb) throw HkError{HK_ERR_INVALID, "bad arguments"};
        std::memcpy(s->background, rgb, 12);
        s->force_background = force;
        s->built = false;
        return HK_OK;
    });
}
int hk_scene_build(hk_scene *s) {
    return guarded([&] {
        if (!s) throw HkError{HK_ERR_INVALID, "null scene"};
        build_scene(s);
        return HK_OK;
    });
}
int hk_bvh_check(const float *tris, uint32_t n, uint32_t *n_bvh_nodes, uint32_t *n_wide_nodes, uint32_t *wide_depth) {
    return guarded([&] {
        if (!tris || n == 0) throw HkError{HK_ERR_INVALID, "bad arguments"};
        hk::BvhPair P = hk::build_bvh_pair(tris, n);
        std::string err = hk::check_bvh_pair(P, tris, n);
        if (!err.empty()) throw HkError{HK_ERR_INVALID, err};
        if (n_bvh_nodes) *n_bvh_nodes = (uint32_t)(P.bvh2.nodes.size() / 16);
        if (n_wide_nodes) *n_wide_nodes = (uint32_t)(P.bvh8.nodes.size() / 20);
        if (wide_depth) *wide_depth = P.bvh8.depth;
        return HK_OK;
    });
}
int hk_scene_set_builder(hk_scene *s, int32_t builder) {
    return guarded([&] {
        if (!s || (builder != HK_BUILDER_HOST && builder != HK_BUILDER_GPU)) throw HkError{HK_ERR_INVALID, "bad arguments"};
        s->builder = builder;
        s->built = false;
        return HK_OK;
    });
}
int hk_scene_tree_build_seconds(const hk_scene *s, double *seconds) {
    return guarded([&] {
        if (!s || !seconds) throw HkError{HK_ERR_INVALID, "bad arguments"};
        *seconds = s->tree_build_s;
        return HK_OK;
    });
}
int hk_wavefront_launch_log(hk_scene *s, int32_t which, uint32_t *rays_host, int32_t max, int32_t *launches) {
    return guarded([&] {
        require_built(s);
        if ((which != 0 && which != 1) || max < 0 || (max > 0 && !rays_host) || !launches)
            throw HkError{HK_ERR_INVALID, "bad arguments"};
        if (!s->wf) throw HkError{HK_ERR_INVALID, "the scene has not rendered with the wavefront integrator"};
        *launches = s->wf->launch_log(which, rays_host, max);
        return HK_OK;
    });
}
int hk_bvh_check_gpu(const float *tris, uint32_t n, uint32_t *n_wide_nodes, uint32_t *wide_depth) {
    return guarded([&] {
        if (!tris || n == 0) throw HkError{HK_ERR_INVALID, "bad arguments"};
        DevBuf dP;
        dP.alloc((size_t)n * 9 * sizeof(float));
        HK_CUDA(cudaMemcpy(dP.p, tris, dP.bytes, cudaMemcpyHostToDevice));
        hk::GpuBvh8 G;
        hk::build_bvh8_gpu(dP.as<float>(), n, nullptr, G);
        std::vector<uint32_t> nodes((size_t)G.nnodes * 20), order(n);
        HK_CUDA(cudaMemcpy(nodes.data(), G.nodes.p, nodes.size() * 4, cudaMemcpyDeviceToHost));
        HK_CUDA(cudaMemcpy(order.data(), G.order.p, order.size() * 4, cudaMemcpyDeviceToHost));
        const std::string err = hk::check_bvh8(nodes, order, tris, n);
        if (!err.empty()) throw HkError{HK_ERR_INVALID, err};
        if (n_wide_nodes) *n_wide_nodes = G.nnodes;
        if (wide_depth) *wide_depth = G.depth;
        return HK_OK;
    });
}
int hk_scene_set_accel(hk_scene *s, int32_t accel) {
    return guarded([&] {
        if (!s || (accel != HK_ACCEL_BVH2 && accel != HK_ACCEL_BVH8)) throw HkError{HK_ERR_INVALID, "bad arguments"};
        if (accel == HK_ACCEL_BVH2 && s->built && s->dev.nnodes == 0)
            throw HkError{HK_ERR_INVALID, "the scene was built on the device: it has the 8-wide tree only"};
        s->accel = accel;
        s->dev.accel = accel;
        s->info.accel = accel;
        s->occupancy = s->occupancy_of[accel];
        s->wf.reset();   // the engine holds a copy of the device description
        return HK_OK;
    });
}
int hk_scene_get_info(const hk_scene *s, hk_scene_info *info) {
    return guarded([&] {
        if (!s || !info) throw HkError{HK_ERR_INVALID, "bad arguments"};
        if (s->built) {
            *info = s->info;
            return HK_OK;
        }
        // host-side view of an unbuilt scene (no BVH / device fields yet)
        hk_scene_info I{};
        I.n_meshes = (uint32_t)s->meshes.size();
        float bb[6] = {INFINITY, INFINITY, INFINITY, -INFINITY, -INFINITY, -INFINITY};
        for (auto &m : s->meshes) {
            I.n_triangles += (uint32_t)(m.idx.size() / 3);
            for (size_t v = 0; v < m.pos.size() / 3; ++v)
                for (int c = 0; c < 3; c++) {
                    bb[c] = std::min(bb[c], m.pos[3 * v + c]);
                    bb[3 + c] = std::max(bb[3 + c], m.pos[3 * v + c]);
                }
        }
        I.n_bsdfs = (uint32_t)s->bsdfs.size();
        I.n_emitters = (uint32_t)s->emitter_mesh.size();
        I.env_index = -1;
        for (size_t e = 0; e < s->emitter_mesh.size(); ++e)
            if (s->emitter_mesh[e] == -1) I.env_index = (int32_t)e;
        I.film_border = (int32_t)std::ceil(s->filt_r - 0.5f);
        std::memcpy(I.bbox, bb, sizeof bb);
        *info = I;
        return HK_OK;
    });
}

int hk_render(hk_scene *s, const hk_render_desc *d, float *film, unsigned long long *counters, void *stream) {
    return guarded([&] {
        require_built(s);
        if (!d || !film) throw HkError{HK_ERR_INVALID, "bad arguments"};
        if (d->spp <= 0 || d->depth < 0) throw HkError{HK_ERR_INVALID, "spp must be > 0 and depth >= 0"};
        require_scene_size(s, *d);
        cudaStream_t st = (cudaStream_t)stream;
        hk::RenderLaunch P;
        std::memset(&P, 0, sizeof P);
        P.film = film;
        P.work_counter = (unsigned int *)s->b_scratch.p;
        P.counters = counters;
        P.seed = d->seed;
        P.spp = d->spp;
        P.sample_offset = d->sample_offset;
        P.depth = d->depth;
        P.rr_start = d->rr_start;
        P.image_index = d->image_index;
        P.tiles_x = ((int)s->width + hk::kTile - 1) / hk::kTile;
        P.tiles_y = ((int)s->height + hk::kTile - 1) / hk::kTile;
        const int tiles = P.tiles_x * P.tiles_y;
        const int resident = s->sm_count * s->occupancy;
        int per_item = d->spp_per_item;
        if (per_item <= 0) {
            int chunks = std::max(1, std::min(d->spp, (4 * resident + tiles - 1) / tiles));
            per_item = (d->spp + chunks - 1) / chunks;
        }
        P.spp_per_item = per_item;
        P.n_chunks = (d->spp + per_item - 1) / per_item;
        P.n_items = tiles * P.n_chunks;
        P.margin_lo = s->margin_lo;
        P.margin_hi = s->margin_hi;
        HK_CUDA(cudaMemsetAsync(s->b_scratch.p, 0, sizeof(unsigned long long), st));
        int grid = std::min(P.n_items, resident);
        if (d->use_camera) {
            hk::DevScene D = s->dev;   // per-call camera pose (passed by value with the launch)
            const float *M = d->camera_to_world;
            float w = M[15];
            if (w == 0.0f) throw HkError{HK_ERR_INVALID, "camera_to_world has w = 0"};
            for (int r = 0; r < 3; r++) {
                for (int c = 0; c < 3; c++) D.cam[4 * r + c] = M[4 * r + c];
                D.cam[4 * r + 3] = M[4 * r + 3] / w;
            }
            HK_CUDA(hk::launch_render(D, P, grid, st));
        } else {
            HK_CUDA(hk::launch_render(s->dev, P, grid, st));
        }
        return HK_OK;
    });
}
int hk_film_resolve(hk_scene *s, const float *film, float *rgb, void *stream) {
    return guarded([&] {
        require_built(s);
        if (!film || !rgb) throw HkError{HK_ERR_INVALID, "bad arguments"};
        HK_CUDA(hk::launch_resolve(film, rgb, (int)s->width, (int)s->height, s->dev.border, (cudaStream_t)stream));
        return HK_OK;
    });
}
// Whether hk_render_image renders this call with the wavefront: always for
// HK_FORM_WAVEFRONT; for HK_FORM_AUTO once the image has at least 256 x 256
// pixels and 2^22 paths (below that a pool of path slots cannot fill the GPU
// better than the megakernel's persistent tiles).
static bool image_uses_wavefront(const hk_scene *s, const hk_render_desc &d) {
    if (s->image_form == HK_FORM_WAVEFRONT) return true;
    if (s->image_form == HK_FORM_MEGAKERNEL) return false;
    const uint64_t px = (uint64_t)s->width * s->height;
    return px >= 65536 && px * (uint64_t)std::max(d.spp, 0) >= (1ull << 22);
}
int hk_render_image(hk_scene *s, const hk_render_desc *d, float *rgb_host, unsigned long long *counters, void *stream) {
    return guarded([&] {
        require_built(s);
        if (!d || !rgb_host) throw HkError{HK_ERR_INVALID, "bad arguments"};
        if (d->spp <= 0 || d->depth < 0) throw HkError{HK_ERR_INVALID, "spp must be > 0 and depth >= 0"};
        require_scene_size(s, *d);
        cudaStream_t st = (cudaStream_t)stream;
        size_t FW = s->width + 2 * s->dev.border, FH = s->height + 2 * s->dev.border;
        size_t film_bytes = FW * FH * 4 * sizeof(float), rgb_bytes = (size_t)s->width * s->height * 3 * sizeof(float);
        if (s->b_film.bytes < film_bytes) s->b_film.alloc(film_bytes);
        if (s->b_rgb.bytes < rgb_bytes) s->b_rgb.alloc(rgb_bytes);
        // counters: [1..5] the megakernel's, [8..14] the wavefront's 7
        unsigned long long *ctr = (unsigned long long *)s->b_scratch.p + 1;
        unsigned long long *ctr7 = (unsigned long long *)s->b_scratch.p + 8;
        HK_CUDA(cudaMemsetAsync(s->b_film.p, 0, film_bytes, st));
        const bool wave = image_uses_wavefront(s, *d);
        int rc;
        if (wave) {
            HK_CUDA(cudaMemsetAsync(ctr7, 0, 7 * sizeof(unsigned long long), st));
            hk_render_job job;
            job.film_dev = s->b_film.as<float>();
            job.desc = *d;
            job.desc.width = job.desc.height = 0;
            rc = hk_render_batch(s, &job, 1, s->has_wf_cfg ? &s->wf_cfg : nullptr, ctr7, stream);
        } else {
            HK_CUDA(cudaMemsetAsync(ctr, 0, 5 * sizeof(unsigned long long), st));
            rc = hk_render(s, d, s->b_film.as<float>(), ctr, stream);
        }
        if (rc != HK_OK) return rc;
        HK_CUDA(hk::launch_resolve(s->b_film.as<float>(), s->b_rgb.as<float>(), (int)s->width, (int)s->height,
                                   s->dev.border, st));
        HK_CUDA(cudaMemcpyAsync(rgb_host, s->b_rgb.p, rgb_bytes, cudaMemcpyDeviceToHost, st));
        unsigned long long c7[7] = {0, 0, 0, 0, 0, 0, 0};
        if (counters) {
            if (wave) HK_CUDA(cudaMemcpyAsync(c7, ctr7, sizeof c7, cudaMemcpyDeviceToHost, st));
            else HK_CUDA(cudaMemcpyAsync(counters, ctr, 5 * sizeof(unsigned long long), cudaMemcpyDeviceToHost, st));
        }
        HK_CUDA(cudaStreamSynchronize(st));
        if (counters && wave) {   // the megakernel's five: traversal totals over both ray kinds
            counters[0] = c7[0];
            counters[1] = c7[1];
            counters[2] = c7[2];
            counters[3] = c7[3] + c7[5];
            counters[4] = c7[4] + c7[6];
        }
        return HK_OK;
    });
}
int hk_scene_set_image_form(hk_scene *s, int32_t form) {
    return guarded([&] {
        if (!s || form < HK_FORM_AUTO || form > HK_FORM_WAVEFRONT) throw HkError{HK_ERR_INVALID, "bad arguments"};
        s->image_form = form;
        return HK_OK;
    });
}
int hk_scene_set_wavefront_config(hk_scene *s, const hk_wavefront_config *cfg) {
    return guarded([&] {
        if (!s) throw HkError{HK_ERR_INVALID, "bad arguments"};
        s->has_wf_cfg = cfg != nullptr;
        if (cfg) {
            s->wf_cfg = *cfg;
            s->wf_cfg.kernel_ms = nullptr;
            s->wf_cfg.kernel_launches = nullptr;
        }
        return HK_OK;
    });
}
// Render without any device allocation: the work counter, the counters and the
// film accumulator live in the library's static scratch (hk_kernels.cu); the
// caller supplies the output image.  Asynchronous on `stream`.
int hk_render_image_static(hk_scene *s, const hk_render_desc *d, float *rgb_dev, unsigned long long *counters_dev,
                           void *stream) {
    return guarded([&] {
        require_built(s);
        if (!d || !rgb_dev) throw HkError{HK_ERR_INVALID, "bad arguments"};
        if (d->spp <= 0 || d->depth < 0) throw HkError{HK_ERR_INVALID, "spp must be > 0 and depth >= 0"};
        require_scene_size(s, *d);
        const size_t FW = s->width + 2 * s->dev.border, FH = s->height + 2 * s->dev.border;
        const size_t film_floats = FW * FH * 4;
        if (film_floats > hk::kStaticFilmFloats)
            throw HkError{HK_ERR_INVALID, "image of " + std::to_string(s->width) + "x" + std::to_string(s->height) +
                                              " with filter border " + std::to_string(s->dev.border) + " needs " +
                                              std::to_string(film_floats) + " film floats; the static scratch holds " +
                                              std::to_string(hk::kStaticFilmFloats) +
                                              " (up to 512x512 pixels at border 4); use hk_render"};
        // the scratch address is per device: the scene's device must be current
        int cur = 0;
        HK_CUDA(cudaGetDevice(&cur));
        if (cur != s->device)
            throw HkError{HK_ERR_INVALID, "the scene was built on device " + std::to_string(s->device) +
                                              " but device " + std::to_string(cur) + " is current"};
        void *scratch = nullptr;
        HK_CUDA(hk::static_render_scratch(&scratch));
        cudaStream_t st = (cudaStream_t)stream;
        unsigned long long *hdr = (unsigned long long *)scratch;
        float *film = (float *)(hdr + hk::kStaticHeaderWords);
        // the array keeps the previous call's contents: clear what must start at zero
        HK_CUDA(cudaMemsetAsync(hdr, 0, hk::kStaticHeaderWords * sizeof(unsigned long long), st));
        HK_CUDA(cudaMemsetAsync(film, 0, film_floats * sizeof(float), st));
        hk::RenderLaunch P;
        std::memset(&P, 0, sizeof P);
        P.film = film;
        P.work_counter = (unsigned int *)hdr;
        P.counters = hdr + 1;
        P.seed = d->seed;
        P.spp = d->spp;
        P.sample_offset = d->sample_offset;
        P.depth = d->depth;
        P.rr_start = d->rr_start;
        P.image_index = d->image_index;
        P.tiles_x = ((int)s->width + hk::kTile - 1) / hk::kTile;
        P.tiles_y = ((int)s->height + hk::kTile - 1) / hk::kTile;
        const int tiles = P.tiles_x * P.tiles_y;
        const int resident = s->sm_count * s->occupancy;
        int per_item = d->spp_per_item;
        if (per_item <= 0) {
            int chunks = std::max(1, std::min(d->spp, (4 * resident + tiles - 1) / tiles));
            per_item = (d->spp + chunks - 1) / chunks;
        }
        P.spp_per_item = per_item;
        P.n_chunks = (d->spp + per_item - 1) / per_item;
        P.n_items = tiles * P.n_chunks;
        P.margin_lo = s->margin_lo;
        P.margin_hi = s->margin_hi;
        const int grid = std::min(P.n_items, resident);
        hk::DevScene D = s->dev;
        if (d->use_camera) {
            const float *M = d->camera_to_world;
            if (M[15] == 0.0f) throw HkError{HK_ERR_INVALID, "camera_to_world has w = 0"};
            for (int r = 0; r < 3; r++) {
                for (int c = 0; c < 3; c++) D.cam[4 * r + c] = M[4 * r + c];
                D.cam[4 * r + 3] = M[4 * r + 3] / M[15];
            }
        }
        HK_CUDA(hk::launch_render(D, P, grid, st));
        HK_CUDA(hk::launch_resolve(film, rgb_dev, (int)s->width, (int)s->height, s->dev.border, st));
        if (counters_dev)
            HK_CUDA(cudaMemcpyAsync(counters_dev, hdr + 1, 5 * sizeof(unsigned long long), cudaMemcpyDeviceToDevice, st));
        return HK_OK;
    });
}
int hk_render_batch(hk_scene *s, const hk_render_job *jobs, int njobs, const hk_wavefront_config *cfg,
                    unsigned long long *counters_dev, void *stream) {
    return guarded([&] {
        require_built(s);
        if (!jobs || njobs <= 0 || njobs > hk::kWfMaxJobs) throw HkError{HK_ERR_INVALID, "need 1..1024 jobs"};
        hk_wavefront_config c{};
        if (cfg) c = *cfg;
        hk::WfEngineConfig ec;
        ec.capacity = std::max(1024, std::min(c.capacity > 0 ? c.capacity : (1 << 21), 1 << 26));
        ec.threads_extend = c.threads_extend > 0 ? c.threads_extend : 128;
        ec.threads_shade = c.threads_shade > 0 ? c.threads_shade : 128;
        ec.fetch_steps = std::max(0, std::min(1024, c.fetch_steps));
        ec.fetch_min_idle = c.fetch_min_idle > 0 ? std::min(32, c.fetch_min_idle) : 1;
        ec.fetch_steps_shadow = std::max(0, std::min(1024, c.fetch_steps_shadow));
        ec.fetch_min_idle_shadow = c.fetch_min_idle_shadow > 0 ? std::min(32, c.fetch_min_idle_shadow) : 0;
        ec.reg_lean = c.reg_lean & 7;
        ec.shadow_tests = c.shadow_tests >= 0 && c.shadow_tests <= 2 ? c.shadow_tests : 0;
        ec.closest_tests = c.closest_tests == 2 ? 2 : 0;
        hk::WfEngine &E = wf_ensure(s, ec);
        cudaStream_t user = (cudaStream_t)stream, st = E.stream();
        // order after the caller's stream (the films may have been cleared there)
        cudaEvent_t ev;
        HK_CUDA(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
        struct EvGuard {
            cudaEvent_t e;
            ~EvGuard() { cudaEventDestroy(e); }
        } guard{ev};
        HK_CUDA(cudaEventRecord(ev, user));
        HK_CUDA(cudaStreamWaitEvent(st, ev, 0));
        std::vector<hk::WfSeg> plan(njobs);
        uint64_t total = 0;
        E.reset();
        for (int j = 0; j < njobs; ++j) {
            if (!jobs[j].film_dev) throw HkError{HK_ERR_INVALID, "bad job: null film"};
            hk::WfJob J = hk::make_wf_job(s, jobs[j].desc);
            J.sample_major = c.sample_major ? 1 : 0;
            J.film = jobs[j].film_dev;
            E.set_job(j, J);
            plan[j] = hk::WfSeg{total, 0, j, 0};
            total += J.work_count;
        }
        E.set_plan(plan, total);
        const bool profile = c.kernel_ms != nullptr;
        const bool use_graph = c.no_graph == 0 && !profile;
        const int per_check = c.iterations_per_check > 0 ? c.iterations_per_check : 16;
        uint64_t iters = 0;
        const uint64_t max_iters = 1ull << 40;
        for (;;) {
            E.run(per_check, use_graph, c.kernel_ms, c.kernel_launches);
            iters += per_check;
            E.fetch_status();
            HK_CUDA(cudaEventSynchronize(E.done_event()));
            const hk::WfCounters &h = E.status();
            if (h.active == 0 && h.next_work >= h.total_work) break;
            if (iters > max_iters) throw HkError{HK_ERR_CUDA, "wavefront did not terminate"};
        }
        if (counters_dev) E.add_counters(counters_dev);
        // the caller's stream continues after the engine's work
        HK_CUDA(cudaEventRecord(ev, st));
        HK_CUDA(cudaStreamWaitEvent(user, ev, 0));
        return HK_OK;
    });
}
int hk_render_batch_host(hk_scene *s, const hk_render_desc *descs, int n, const hk_wavefront_config *cfg,
                         float *const *rgb_host, unsigned long long *counters_host, void *stream) {
    return guarded([&] {
        require_built(s);
        if (!descs || !rgb_host || n <= 0 || n > hk::kWfMaxJobs) throw HkError{HK_ERR_INVALID, "bad arguments"};
        cudaStream_t st = (cudaStream_t)stream;
        std::vector<hk::JobSize> sz(n);
        size_t rgb_max = 0;
        for (int j = 0; j < n; ++j) {
            sz[j] = hk::job_size(s, descs[j]);
            rgb_max = std::max(rgb_max, sz[j].rgb_bytes);
        }
        while ((int)s->batch_films.size() < n) s->batch_films.emplace_back(new DevBuf());
        if (s->b_rgb.bytes < rgb_max) s->b_rgb.alloc(rgb_max);
        unsigned long long *ctr = (unsigned long long *)s->b_scratch.p + 1;   // 7 slots
        HK_CUDA(cudaMemsetAsync(ctr, 0, 7 * sizeof(unsigned long long), st));
        std::vector<hk_render_job> jobs(n);
        for (int j = 0; j < n; ++j) {
            if (s->batch_films[j]->bytes < sz[j].film_bytes) s->batch_films[j]->alloc(sz[j].film_bytes);
            HK_CUDA(cudaMemsetAsync(s->batch_films[j]->p, 0, sz[j].film_bytes, st));
            jobs[j].film_dev = s->batch_films[j]->as<float>();
            jobs[j].desc = descs[j];
        }
        int rc = hk_render_batch(s, jobs.data(), n, cfg, ctr, stream);
        if (rc != HK_OK) return rc;
        for (int j = 0; j < n; ++j) {
            HK_CUDA(hk::launch_resolve(jobs[j].film_dev, s->b_rgb.as<float>(), (int)sz[j].width, (int)sz[j].height,
                                       s->dev.border, st));
            HK_CUDA(cudaMemcpyAsync(rgb_host[j], s->b_rgb.p, sz[j].rgb_bytes, cudaMemcpyDeviceToHost, st));
        }
        if (counters_host)
            HK_CUDA(cudaMemcpyAsync(counters_host, ctr, 7 * sizeof(unsigned long long), cudaMemcpyDeviceToHost, st));
        HK_CUDA(cudaStreamSynchronize(st));
        return HK_OK;
    });
}
int hk_wavefront_autotune(hk_scene *s, const hk_render_desc *probe, hk_wavefront_config *best, float *best_ms) {
    return guarded([&] {
        require_built(s);
        if (!probe || !best) throw HkError{HK_ERR_INVALID, "bad arguments"};
        // probe film (the tuner allocates; rendering afterwards does not need it)
        size_t FW = s->width + 2 * s->dev.border, FH = s->height + 2 * s->dev.border;
        DevBuf film;
        film.alloc(FW * FH * 4 * sizeof(float));
        hk_render_job job;
        job.film_dev = film.as<float>();
        job.desc = *probe;
        cudaEvent_t e0, e1;
        HK_CUDA(cudaEventCreate(&e0));
        HK_CUDA(cudaEventCreate(&e1));
        float best_t = INFINITY;
        hk_wavefront_config bc{};
        const int caps[] = {1 << 20, 1 << 21, 1 << 22};
        const int threads[] = {64, 128, 256};
        const int checks[] = {16, 64};
        const int steps8[] = {2, 3, 6}, steps2[] = {4, 8, 16};
        const int min_idle[] = {1, 8, 16};
        // a configuration's time: the better of two timed renders after a warm one
        // (one timed render lets run-to-run noise of a few percent pick the configuration)
        auto run = [&](const hk_wavefront_config &c) {
            HK_CUDA(cudaMemset(film.p, 0, film.bytes));
            int rc = hk_render_batch(s, &job, 1, &c, nullptr, nullptr);   // warm (allocation, graph)
            if (rc != HK_OK) throw HkError{rc, hk_last_error()};
            float best_ms = INFINITY;
            for (int rep = 0; rep < 2; ++rep) {
                HK_CUDA(cudaEventRecord(e0, nullptr));
                rc = hk_render_batch(s, &job, 1, &c, nullptr, nullptr);
                if (rc != HK_OK) throw HkError{rc, hk_last_error()};
                HK_CUDA(cudaEventRecord(e1, nullptr));
                HK_CUDA(cudaEventSynchronize(e1));
                float ms = 0;
                HK_CUDA(cudaEventElapsedTime(&ms, e0, e1));
                best_ms = std::min(best_ms, ms);
            }
            return best_ms;
        };
        // coordinate descent: capacity, then block sizes, then the check interval
        hk_wavefront_config c{};
        c.threads_extend = 128; c.threads_shade = 128; c.iterations_per_check = 16;
        for (int cap : caps) {
            c.capacity = cap;
            float ms = run(c);
            if (ms < best_t) { best_t = ms; bc = c; }
        }
        c = bc;
        for (int te : threads)
            for (int ts : threads) {
                c.threads_extend = te; c.threads_shade = ts;
                float ms = run(c);
                if (ms < best_t) { best_t = ms; bc = c; }
            }
        c = bc;
        for (int k : checks) {
            c.iterations_per_check = k;
            float ms = run(c);
            if (ms < best_t) { best_t = ms; bc = c; }
        }
        // dynamic ray fetch: node visits between refills, idle lanes before a refill
        c = bc;
        for (int k : (s->dev.accel == hk::kAccelBvh8 ? steps8 : steps2)) {
            c.fetch_steps = k;
            float ms = run(c);
            if (ms < best_t) { best_t = ms; bc = c; }
        }
        c = bc;
        for (int k : min_idle) {
            c.fetch_min_idle = k;
            float ms = run(c);
            if (ms < best_t) { best_t = ms; bc = c; }
        }
        // register budgets of the extend and shadow kernels, then of the shade kernels
        c = bc;
        for (int k : {1, 2, 3}) {
            c.reg_lean = k;
            float ms = run(c);
            if (ms < best_t) { best_t = ms; bc = c; }
        }
        c = bc;
        c.reg_lean |= 4;
        {
            float ms = run(c);
            if (ms < best_t) { best_t = ms; bc = c; }
        }
        // the shadow rays' own refill interval and idle-lane threshold
        c = bc;
        for (int k : (s->dev.accel == hk::kAccelBvh8 ? steps8 : steps2)) {
            c.fetch_steps_shadow = k;
            float ms = run(c);
            if (ms < best_t) { best_t = ms; bc = c; }
        }
        c = bc;
        for (int k : min_idle) {
            c.fetch_min_idle_shadow = k;
            float ms = run(c);
            if (ms < best_t) { best_t = ms; bc = c; }
        }
        // the shadow rays' triangle tests postponed or shared out over the warp (8-wide tree only)
        if (s->dev.accel == hk::kAccelBvh8) {
            c = bc;
            for (int k : {1, 2}) {
                if (k == 1 && !s->dev.postpone) continue;
                c.shadow_tests = k;
                float ms = run(c);
                if (ms < best_t) { best_t = ms; bc = c; }
            }
            // and the closest-hit rays' shared out
            c = bc;
            c.closest_tests = 2;
            float ms = run(c);
            if (ms < best_t) { best_t = ms; bc = c; }
        }
        // work items sample by sample
        c = bc;
        c.sample_major = 1;
        {
            float ms = run(c);
            if (ms < best_t) { best_t = ms; bc = c; }
        }
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        *best = bc;
        if (best_ms) *best_ms = best_t;
        s->wf_cfg = bc;   // hk_render_image renders its wavefront calls with it
        s->has_wf_cfg = true;
        return HK_OK;
    });
}
int hk_trace(hk_scene *s, uint64_t n, const float *rays, int32_t *tri, float *t, float *u, float *v, int any_hit,
             unsigned long long *visits, void *stream) {
    return guarded([&] {
        require_built(s);
        if (n == 0) return HK_OK;
        if (!rays || !tri) throw HkError{HK_ERR_INVALID, "bad arguments"};
        HK_CUDA(hk::launch_trace(s->dev, n, rays, tri, t, u, v, any_hit, visits, (cudaStream_t)stream));
        return HK_OK;
    });
}
int hk_bsdf_batch(hk_scene *s, int32_t bsdf, uint64_t n, const float *wi, const float *u2, const float *u1,
                  const float *wo, const float *uv, const float *duv, float *s_wo, float *s_w, float *s_pdf, int32_t *s_m,
                  float *e_rgb, float *p_pdf, void *stream) {
    return guarded([&] {
        require_built(s);
        if (bsdf < 0 || bsdf >= s->dev.nbsdfs) throw HkError{HK_ERR_INVALID, "invalid BSDF id"};
        if (n == 0) return HK_OK;
        if (!wi || !u2 || !wo) throw HkError{HK_ERR_INVALID, "bad arguments"};
        HK_CUDA(hk::launch_bsdf_batch(s->dev, bsdf, s->bsdf_deep[bsdf] ? -1 : s->bsdfs[bsdf].type, n, wi, u2, u1, wo, uv, duv, s_wo, s_w, s_pdf,
                                      s_m, e_rgb, p_pdf, (cudaStream_t)stream));
        return HK_OK;
    });
}
int hk_texture_eval(hk_scene *s, int32_t tex, uint64_t n, const float *uv, const float *duv, float *out, void *stream) {
    return guarded([&] {
        require_built(s);
        if (tex < 0 || tex >= (int)s->textures.size()) throw HkError{HK_ERR_INVALID, "invalid texture id"};
        if (n == 0) return HK_OK;
        if (!uv || !out) throw HkError{HK_ERR_INVALID, "bad arguments"};
        HK_CUDA(hk::launch_texture_eval(s->dev, s->b_textures.as<hk::DevTexture>(), tex, n, uv, duv, out,
                                        (cudaStream_t)stream));
        return HK_OK;
    });
}
int hk_emitter_sample(hk_scene *s, int32_t e, uint64_t n, const float *in, float *out, void *stream) {
    return guarded([&] {
        require_built(s);
        if (e < 0 || e >= s->dev.nemitters) throw HkError{HK_ERR_INVALID, "invalid emitter index"};
        if (n == 0) return HK_OK;
        HK_CUDA(hk::launch_emitter_sample(s->dev, e, n, in, out, (cudaStream_t)stream));
        return HK_OK;
    });
}
int hk_camera_rays(hk_scene *s, uint64_t n, const float *pos, float *rays, void *stream) {
    return guarded([&] {
        require_built(s);
        if (n == 0) return HK_OK;
        HK_CUDA(hk::launch_camera_rays(s->dev, n, pos, rays, (cudaStream_t)stream));
        return HK_OK;
    });
}
int hk_env_eval(hk_scene *s, uint64_t n, const float *wi, float *rgb, float *pdf, void *stream) {
    return guarded([&] {
        require_built(s);
        if (s->dev.env_index < 0) throw HkError{HK_ERR_INVALID, "scene has no environment emitter"};
        if (n == 0) return HK_OK;
        HK_CUDA(hk::launch_env_eval(s->dev, n, wi, rgb, pdf, (cudaStream_t)stream));
        return HK_OK;
    });
}

int hk_scene_load_xml(const char *path, const char *data_dir, hk_scene **out, int32_t *depth, int32_t *spp) {
    return guarded([&] {
        if (!path || !out) throw HkError{HK_ERR_INVALID, "bad arguments"};
        std::string err;
        int rc = hk_scene_load_xml_impl(path, data_dir, out, depth, spp, 1, &err);
        if (rc != HK_OK && !err.empty()) return set_error(rc, err);
        return rc;
    });
}
int hk_scene_parse_xml(const char *path, const char *data_dir, hk_scene **out, int32_t *depth, int32_t *spp) {
    return guarded([&] {
        if (!path || !out) throw HkError{HK_ERR_INVALID, "bad arguments"};
        std::string err;
        int rc = hk_scene_load_xml_impl(path, data_dir, out, depth, spp, 0, &err);
        if (rc != HK_OK && !err.empty()) return set_error(rc, err);
        return rc;
    });
}
int hk_exr_read(const char *path, int32_t *w, int32_t *h, float *rgb, uint64_t capacity) {
    return guarded([&] {
        if (!path || !w || !h) throw HkError{HK_ERR_INVALID, "bad arguments"};
        std::vector<float> buf;
        std::string err;
        int W = 0, H = 0;
        int rc = hk_exr_read_impl(path, &W, &H, &buf, &err);
        if (rc != HK_OK) return set_error(rc, err);
        *w = W;
        *h = H;
        if (rgb) {
            if (capacity < buf.size()) throw HkError{HK_ERR_INVALID, "output buffer too small"};
            std::memcpy(rgb, buf.data(), buf.size() * sizeof(float));
        }
        return HK_OK;
    });
}
int hk_exr_write(const char *path, int32_t w, int32_t h, const float *rgb) {
    return guarded([&] {
        if (!path || !rgb || w <= 0 || h <= 0) throw HkError{HK_ERR_INVALID, "bad arguments"};
        std::string err;
        int rc = hk_exr_write_impl(path, w, h, rgb, &err);
        if (rc != HK_OK) return set_error(rc, err);
        return HK_OK;
    });
}

}  // extern "C"
