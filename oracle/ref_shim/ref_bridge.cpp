/* C entry points over the reference's own BSDF classes, compiled from the
 * reference sources by oracle/ref_build.py.  Used by tests only, to pin the
 * oracle restatement (oracle/hk_oracle.c) record by record. */
#include <core\Common.hpp>
#include <core\Object.hpp>
#include <core\PropertyList.hpp>
#include <core\BSDF.hpp>
#include <core\Sampler.hpp>
#include <core\Intersection.hpp>
#include <core\Color.hpp>
#include <core\Vector.hpp>
#include <core\Emitter.hpp>
#include <core\Mesh.hpp>
#include <core\Texture.hpp>
#include <core\Camera.hpp>
#include <core\Transform.hpp>
#include <core\Acceleration.hpp>
#include <core\ReconstructionFilter.hpp>
#include <core\Block.hpp>
#include <stb_image.h>

#include <vector>

using namespace Hikari;

namespace {
/* Sampler whose Next1D returns a value set per query (roughDielectric draws
 * its reflect/refract choice from the record's sampler). */
class FixedSampler : public Sampler {
public:
    float u1 = 0.0f;
    std::unique_ptr<Sampler> Clone() const override { return std::unique_ptr<Sampler>(new FixedSampler(*this)); }
    void Prepare(const ImageBlock &) override {}
    void Generate() override {}
    void Advance() override {}
    float Next1D() override { return u1; }
    Point2f Next2D() override { return Point2f(u1, u1); }
    std::string ToString() const override { return "FixedSampler"; }
};
thread_local FixedSampler g_sampler;
const Intersection &null_isect() { static const Intersection I; return I; }
/* the intersection of the current query: only its texture coordinates matter */
thread_local Intersection g_isect;
const Intersection &query_isect() { return g_isect; }
}

extern "C" {

void hr_init(const char *search_dir) { GetFileResolver()->prepend(filesystem::path(search_dir)); }

/* type: 0 diffuse, 1 roughConductor, 2 roughDielectric, 3 roughPlastic, 4 roughCoating,
 * 5 mirror, 6 conductor, 7 dielectric, 8 plastic, 9 twoSided (nested, then nested2 if given),
 * 10 coating, 11 roughDiffuse */
void *hr_bsdf_create(int type, int ggx, float alpha, float int_ior, float ext_ior, const float *k,
                     const float *ks, const float *kd, const float *sigma_a, float thickness, void *nested,
                     void *nested2, const float *ks_refract, int nonlinear, int fast_approx, void **tex,
                     int anisotropic) {
    static const char *names[] = {"diffuse", "roughConductor", "roughDielectric", "roughPlastic", "roughCoating",
                                  "mirror", "conductor", "dielectric", "plastic", "twoSided", "coating",
                                  "roughDiffuse", "bumpMap", "normalMap"};
    auto col = [](const float *c) { return Color3f(c[0], c[1], c[2]); };
    try {
        PropertyList pl;
        if (type == 0) {
            pl.SetColor("albedo", col(kd));
        } else if (type <= 4) {
            pl.SetString("type", ggx ? "ggx" : "beckmann");
            pl.SetFloat("alpha", alpha);
            if (anisotropic && (type == 1 || type == 2)) {
                pl.SetBoolean("as", true);
                pl.SetFloat("alphaU", alpha);
                pl.SetFloat("alphaV", alpha);
            }
            pl.SetFloat("intIOR", int_ior);
            pl.SetFloat("extIOR", ext_ior);
            if (type == 1) { pl.SetColor("k", col(k)); pl.SetColor("ks", col(ks)); }
            if (type == 2) { pl.SetColor("ksReflect", col(ks)); pl.SetColor("ksRefract", col(ks_refract)); }
            if (type == 3) { pl.SetColor("ks", col(ks)); pl.SetColor("kd", col(kd)); pl.SetBoolean("nonlinear", nonlinear != 0); }
            if (type == 4) { pl.SetColor("ks", col(ks)); pl.SetColor("sigmaA", col(sigma_a)); pl.SetFloat("thickness", thickness); }
        } else if (type >= 6 && type <= 8) {
            pl.SetFloat("intIOR", int_ior);
            pl.SetFloat("extIOR", ext_ior);
            if (type == 6) { pl.SetColor("k", col(k)); pl.SetColor("ks", col(ks)); }
            if (type == 7) { pl.SetColor("ksReflect", col(ks)); pl.SetColor("ksRefract", col(ks_refract)); }
            if (type == 8) { pl.SetColor("ks", col(ks)); pl.SetColor("kd", col(kd)); pl.SetBoolean("nonlinear", nonlinear != 0); }
        } else if (type == 10) {
            pl.SetFloat("intIOR", int_ior);
            pl.SetFloat("extIOR", ext_ior);
            pl.SetColor("ks", col(ks));
            pl.SetColor("sigmaA", col(sigma_a));
            pl.SetFloat("thickness", thickness);
        } else if (type == 11) {
            pl.SetColor("albedo", col(kd));
            pl.SetFloat("alpha", alpha);
            pl.SetBoolean("fastApprox", fast_approx != 0);
        }
        BSDF *b = (BSDF *)ObjectFactory::CreateInstance(names[type], pl);
        if (nested) b->AddChild((Object *)nested, "");
        if (nested2) b->AddChild((Object *)nested2, "");
        /* textures by their XML names: kd / albedo, ks / ksReflect, ksRefract, sigmaA, alpha(U), alphaV */
        for (int k = 0; k < 6 && tex; k++) {
            if (!tex[k]) continue;
            const bool refl = type == 2 || type == 7, albedo = type == 0 || type == 11;
            const char *names[6] = {albedo ? "albedo" : "kd", refl ? "ksReflect" : "ks", "ksRefract", "sigmaA",
                                    anisotropic ? "alphaU" : "alpha", "alphaV"};
            b->AddChild((Object *)tex[k], names[k]);
        }
        b->Activate();
        return b;
    } catch (const std::exception &e) {
        fprintf(stderr, "hr_bsdf_create: %s\n", e.what());
        return nullptr;
    }
}

void hr_bsdf_sample(void *h, const float *wi, const float *u2, float u1, float *wo, float *w, int *measure, float *eta) {
    g_sampler.u1 = u1;
    BSDFQueryRecord r(Vector3f(wi[0], wi[1], wi[2]), ETransportMode::ERadiance, &g_sampler, query_isect());
    r.Wo = Vector3f(0.0f); r.Eta = 0.0f;
    Color3f c = ((BSDF *)h)->Sample(r, Point2f(u2[0], u2[1]));
    wo[0] = r.Wo.x(); wo[1] = r.Wo.y(); wo[2] = r.Wo.z();
    w[0] = c[0]; w[1] = c[1]; w[2] = c[2];
    *measure = int(r.Measure); *eta = r.Eta;
}

void hr_bsdf_eval(void *h, const float *wi, const float *wo, int measure, float *out) {
    BSDFQueryRecord r(Vector3f(wi[0], wi[1], wi[2]), Vector3f(wo[0], wo[1], wo[2]), EMeasure(measure),
                      ETransportMode::ERadiance, &g_sampler, query_isect());
    Color3f c = ((BSDF *)h)->Eval(r);
    out[0] = c[0]; out[1] = c[1]; out[2] = c[2];
}

float hr_bsdf_pdf(void *h, const float *wi, const float *wo, int measure) {
    BSDFQueryRecord r(Vector3f(wi[0], wi[1], wi[2]), Vector3f(wo[0], wo[1], wo[2]), EMeasure(measure),
                      ETransportMode::ERadiance, &g_sampler, query_isect());
    return ((BSDF *)h)->Pdf(r);
}

namespace {
/* A Mesh whose buffers are filled from arrays (the OBJ reader's result). */
class ArrayMesh : public Mesh {
public:
    ArrayMesh(const float *P, uint32_t nv, const float *N, const float *UV, const uint32_t *F, uint32_t nt) {
        m_V.resize(3, nv);
        for (uint32_t i = 0; i < nv; i++) m_V.col(i) = Vector3f(P[3 * i], P[3 * i + 1], P[3 * i + 2]);
        if (N) {
            m_N.resize(3, nv);
            for (uint32_t i = 0; i < nv; i++) m_N.col(i) = Vector3f(N[3 * i], N[3 * i + 1], N[3 * i + 2]);
        }
        if (UV) {
            m_UV.resize(2, nv);
            for (uint32_t i = 0; i < nv; i++) m_UV.col(i) = Vector2f(UV[2 * i], UV[2 * i + 1]);
        }
        m_F.resize(3, nt);
        for (uint32_t i = 0; i < nt; i++)
            for (int c = 0; c < 3; c++) m_F(c, i) = F[3 * i + c];
        /* the mesh box over every vertex, as WavefrontObjMesh computes it */
        for (uint32_t i = 0; i < nv; i++) m_BBox.ExpandBy(Point3f(m_V.col(i)));
    }
    uint32_t *facet(uint32_t i) { return m_F.data() + 3 * i; }
};
}

void *hr_mesh_create(const float *P, uint32_t nv, const float *N, const float *UV, const uint32_t *F, uint32_t nt) {
    return new ArrayMesh(P, nv, N, UV, F, nt);
}

/* Triangle::PostIntersect at barycentric (u, v) of triangle tri: out p(3) s(3) t(3) n(3) uv(2) */
void hr_post_intersect(void *h, uint32_t tri, float u, float v, float *out) {
    ArrayMesh *m = (ArrayMesh *)h;
    Triangle T(m, m->facet(tri), tri);
    Intersection I;
    I.pShape = &T;
    I.UV = Point2f(u, v);
    T.PostIntersect(I);
    const Frame &F = I.ShadingFrame;
    for (int c = 0; c < 3; c++) {
        out[c] = I.P[c]; out[3 + c] = F.S[c]; out[6 + c] = F.T[c]; out[9 + c] = F.N[c];
    }
    out[12] = I.UV.x(); out[13] = I.UV.y();
}

/* texture coordinates of the single-record queries (hr_bsdf_sample / eval / pdf) */
void hr_set_uv(float u, float v) { g_isect.UV = Point2f(u, v); }

/* kind 1 checkerboard, 2 grid, 3 scale (of nested), 5 wireframe (a interiorColor,
 * b edgeColor, width edgeWidth, scale transitionWidth), 6 curvature (a
 * positiveColor, b negativeColor, scale, count 1 gaussian / 0 mean) */
void *hr_texture_create(int kind, int count, float width, float scale, const float *uv_scale, const float *uv_offset,
                        const float *a, const float *b, void *nested) {
    try {
        PropertyList pl;
        Color3f ca(a[0], a[1], a[2]), cb(b[0], b[1], b[2]);
        const char *name = kind == 1 ? "checkerboard"
                                     : (kind == 2 ? "grid" : (kind == 5 ? "wireframe" : (kind == 6 ? "curvature" : "scale")));
        if (kind == 5) {
            pl.SetColor("interiorColor", ca);
            pl.SetColor("edgeColor", cb);
            pl.SetFloat("edgeWidth", width);
            pl.SetFloat("transitionWidth", scale);
        } else if (kind == 6) {
            pl.SetColor("positiveColor", ca);
            pl.SetColor("negativeColor", cb);
            pl.SetFloat("scale", scale);
            pl.SetString("curvatureType", count ? "gaussian" : "mean");
        } else if (kind == 1 || kind == 2) {
            pl.SetInteger(kind == 1 ? "blocks" : "lines", count);
            pl.SetColor(kind == 1 ? "colorA" : "lineColor", ca);
            pl.SetColor(kind == 1 ? "colorB" : "backgroundColor", cb);
            if (kind == 2) pl.SetFloat("lineWidth", width);
            pl.SetFloat("uScale", uv_scale[0]);
            pl.SetFloat("vScale", uv_scale[1]);
            pl.SetFloat("uOffset", uv_offset[0]);
            pl.SetFloat("vOffset", uv_offset[1]);
        } else {
            pl.SetFloat("scale", scale);
        }
        Object *t = ObjectFactory::CreateInstance(name, pl);
        if (nested) t->AddChild((Object *)nested, "");
        t->Activate();
        return t;
    } catch (const std::exception &e) {
        fprintf(stderr, "hr_texture_create: %s\n", e.what());
        return nullptr;
    }
}

/* kind: 0 point (power, position), 1 directional (irradiance, direction), 2 constant (radiance) */
void *hr_emitter_create(int kind, const float *color, const float *vec) {
    static const char *names[] = {"point", "directional", "constant"};
    try {
        PropertyList pl;
        Color3f c(color[0], color[1], color[2]);
        if (kind == 0) { pl.SetColor("power", c); pl.SetPoint("position", Point3f(vec[0], vec[1], vec[2])); }
        if (kind == 1) { pl.SetColor("irradiance", c); pl.SetVector("direction", Vector3f(vec[0], vec[1], vec[2])); }
        if (kind == 2) pl.SetColor("radiance", c);
        Emitter *e = (Emitter *)ObjectFactory::CreateInstance(names[kind], pl);
        e->Activate();
        return e;
    } catch (const std::exception &ex) {
        fprintf(stderr, "hr_emitter_create: %s\n", ex.what());
        return nullptr;
    }
}

/* Emitter::Sample for n references: in ref(3) u2(2) u1 distance; out p(3) n(3) wi(3) pdf dist value(3) */
void hr_emitter_sample(void *h, uint64_t n, const float *in, float *out) {
    for (uint64_t i = 0; i < n; i++) {
        const float *q = in + 7 * i;
        EmitterQueryRecord r(Point3f(q[0], q[1], q[2]));
        r.Distance = q[6];
        r.Pdf = 0.0f;
        Color3f v = ((Emitter *)h)->Sample(r, Point2f(q[3], q[4]), q[5]);
        float *o = out + 14 * i;
        o[0] = r.P.x(); o[1] = r.P.y(); o[2] = r.P.z(); o[3] = r.N.x(); o[4] = r.N.y(); o[5] = r.N.z();
        o[6] = r.Wi.x(); o[7] = r.Wi.y(); o[8] = r.Wi.z(); o[9] = r.Pdf; o[10] = r.Distance;
        o[11] = v[0]; o[12] = v[1]; o[13] = v[2];
    }
}

/* Emitter::Eval / Pdf for world directions (the environment emitters): out value(3) pdf */
void hr_emitter_eval_dir(void *h, uint64_t n, const float *wi, float *out) {
    for (uint64_t i = 0; i < n; i++) {
        EmitterQueryRecord r;
        r.Wi = Vector3f(wi[3 * i], wi[3 * i + 1], wi[3 * i + 2]);
        Color3f v = ((Emitter *)h)->Eval(r);
        out[4 * i] = v[0]; out[4 * i + 1] = v[1]; out[4 * i + 2] = v[2];
        out[4 * i + 3] = ((Emitter *)h)->Pdf(r);
    }
}

/* BitmapTexture (src/texture/BitmapTexture.cpp) of `filename` found under
 * search_dir: filter 0 nearest 1 bilinear 2 trilinear 3 ewa; wrap 0 repeat 1
 * clamp 2 black; channels 1 (r) or 3 (rgb). */
void *hr_bitmap_create(const char *search_dir, const char *filename, int filter, int wrap_u, int wrap_v,
                       int channels, float gamma, float max_aniso, const float *uv_scale, const float *uv_offset) {
    static const char *filters[] = {"nearest", "bilinear", "trilinear", "ewa"};
    static const char *wraps[] = {"repeat", "clamp", "black"};
    try {
        GetFileResolver()->prepend(filesystem::path(search_dir));
        PropertyList pl;
        pl.SetString("filename", filename);
        pl.SetString("filterType", filters[filter]);
        pl.SetString("uWrapMode", wraps[wrap_u]);
        pl.SetString("vWrapMode", wraps[wrap_v]);
        pl.SetString("channel", channels == 1 ? "r" : "rgb");
        pl.SetFloat("gamma", gamma);
        pl.SetFloat("maxAnisotropy", max_aniso);
        pl.SetFloat("uScale", uv_scale[0]);
        pl.SetFloat("vScale", uv_scale[1]);
        pl.SetFloat("uOffset", uv_offset[0]);
        pl.SetFloat("vOffset", uv_offset[1]);
        Object *t = ObjectFactory::CreateInstance("bitmap", pl);
        t->Activate();
        return t;
    } catch (const std::exception &e) {
        fprintf(stderr, "hr_bitmap_create: %s\n", e.what());
        return nullptr;
    }
}

/* Texture::Eval(Isect, bFilter = true) at n texture coordinates uv (2 each)
 * with screen-space partials duv (dUdX, dVdX, dUdY, dVdY each, or NULL): out rgb */
void hr_texture_eval(void *t, uint64_t n, const float *uv, const float *duv, float *out) {
    for (uint64_t i = 0; i < n; i++) {
        Intersection I;
        I.UV = Point2f(uv[2 * i], uv[2 * i + 1]);
        if (duv) { I.dUdX = duv[4 * i]; I.dVdX = duv[4 * i + 1]; I.dUdY = duv[4 * i + 2]; I.dVdY = duv[4 * i + 3]; }
        Color3f c = ((Texture *)t)->Eval(I, true);
        out[3 * i] = c[0]; out[3 * i + 1] = c[1]; out[3 * i + 2] = c[2];
    }
}
/* Texture::Eval(Isect, true) at the intersection Triangle::PostIntersect
 * makes of barycentric (u, v) on triangle tri[i] of mesh: out rgb per record */
void hr_texture_eval_hit(void *t, void *mesh, uint64_t n, const uint32_t *tri, const float *uv, float *out) {
    ArrayMesh *m = (ArrayMesh *)mesh;
    for (uint64_t i = 0; i < n; i++) {
        Triangle T(m, m->facet(tri[i]), tri[i]);
        Intersection I;
        I.pShape = &T;
        I.UV = Point2f(uv[2 * i], uv[2 * i + 1]);
        T.PostIntersect(I);
        Color3f c = ((Texture *)t)->Eval(I, true);
        out[3 * i] = c[0]; out[3 * i + 1] = c[1]; out[3 * i + 2] = c[2];
    }
}
/* Texture::GetAverage: out rgb */
void hr_texture_average(void *t, float *out) {
    Color3f c = ((Texture *)t)->GetAverage();
    out[0] = c[0]; out[1] = c[1]; out[2] = c[2];
}

/* stbi_load as LoadImageFromFileR / RGB (src/core/Texture.cpp:28, :90) call
 * it: returns width * height * req bytes (copied to out when not NULL), 0 on failure. */
uint64_t hr_image_load(const char *path, int req, int *w, int *h, unsigned char *out) {
    int c = 0;
    unsigned char *p = stbi_load(path, w, h, &c, req);
    if (!p) return 0;
    uint64_t n = (uint64_t)(*w) * (uint64_t)(*h) * (uint64_t)req;
    if (out) memcpy(out, p, n);
    stbi_image_free(p);
    return n;
}

/* PerspectiveCamera (src/camera/PerspectiveCamera.cpp) with its default filter */
void *hr_camera_create(int width, int height, const float *to_world16, float fov, float near_clip, float far_clip) {
    try {
        PropertyList pl;
        pl.SetInteger("width", width);
        pl.SetInteger("height", height);
        Eigen::Matrix4f M;
        for (int r = 0; r < 4; r++)
            for (int c = 0; c < 4; c++) M(r, c) = to_world16[4 * r + c];
        pl.SetTransform("toWorld", Transform(M));
        pl.SetFloat("fov", fov);
        pl.SetFloat("nearClip", near_clip);
        pl.SetFloat("farClip", far_clip);
        Object *c = ObjectFactory::CreateInstance("perspective", pl);
        c->Activate();
        return c;
    } catch (const std::exception &e) {
        fprintf(stderr, "hr_camera_create: %s\n", e.what());
        return nullptr;
    }
}
/* Camera::SampleRay at film position (px, py): out o(3) d(3) rx_o(3) rx_d(3) ry_o(3) ry_d(3) mint maxt */
void hr_camera_ray(void *c, float px, float py, float *out) {
    Ray3f R;
    ((Camera *)c)->SampleRay(R, Point2f(px, py), Point2f(0.5f, 0.5f));
    for (int k = 0; k < 3; k++) {
        out[k] = R.Origin[k]; out[3 + k] = R.Direction[k]; out[6 + k] = R.RxOrigin[k];
        out[9 + k] = R.RxDirection[k]; out[12 + k] = R.RyOrigin[k]; out[15 + k] = R.RyDirection[k];
    }
    out[18] = R.MinT; out[19] = R.MaxT;
}
/* Triangle::PostIntersect then Intersection::ComputeScreenSpacePartial for the
 * camera ray through (px, py): out (dUdX, dVdX, dUdY, dVdY) */
void hr_screen_partials(void *cam, void *mesh, uint32_t tri, float u, float v, float px, float py, float *out) {
    Ray3f R;
    ((Camera *)cam)->SampleRay(R, Point2f(px, py), Point2f(0.5f, 0.5f));
    ArrayMesh *m = (ArrayMesh *)mesh;
    Triangle T(m, m->facet(tri), tri);
    Intersection I;
    I.pShape = &T;
    I.UV = Point2f(u, v);
    T.PostIntersect(I);
    I.ComputeScreenSpacePartial(R);
    out[0] = I.dUdX; out[1] = I.dVdX; out[2] = I.dUdY; out[3] = I.dVdY;
}

/* hr_bsdf_batch with each record's intersection: n x 20 floats (shading frame
 * S T N, geometric N, dPdU, dPdV, UV) -- for bumpMap / normalMap */
void hr_bsdf_batch_isect(void *h, uint64_t n, const float *wi, const float *u2, const float *u1, const float *wo,
                         const float *isect, float *s_wo, float *s_w, float *s_pdf, int *s_m, float *e_rgb,
                         float *p_pdf) {
    for (uint64_t i = 0; i < n; i++) {
        const float *q = isect + 20 * i;
        Intersection I;
        I.ShadingFrame = Frame(Vector3f(q[0], q[1], q[2]), Vector3f(q[3], q[4], q[5]), Vector3f(q[6], q[7], q[8]));
        I.GeometricFrame = Frame(Vector3f(q[9], q[10], q[11]));
        I.dPdU = Vector3f(q[12], q[13], q[14]);
        I.dPdV = Vector3f(q[15], q[16], q[17]);
        I.UV = Point2f(q[18], q[19]);
        I.bHasUVPartial = true;
        g_isect = I;
        float eta; int m;
        hr_bsdf_sample(h, wi + 3 * i, u2 + 2 * i, u1 ? u1[i] : 0.0f, s_wo + 3 * i, s_w + 3 * i, &m, &eta);
        s_m[i] = m;
        bool zero = s_w[3 * i] == 0.0f && s_w[3 * i + 1] == 0.0f && s_w[3 * i + 2] == 0.0f;
        s_pdf[i] = zero ? 0.0f : hr_bsdf_pdf(h, wi + 3 * i, s_wo + 3 * i, m);
        hr_bsdf_eval(h, wi + 3 * i, wo + 3 * i, 1, e_rgb + 3 * i);
        p_pdf[i] = hr_bsdf_pdf(h, wi + 3 * i, wo + 3 * i, 1);
    }
}

/* batched over n AoS records (same layout as ho_bsdf_batch) */
void hr_bsdf_batch(void *h, uint64_t n, const float *wi, const float *u2, const float *u1, const float *wo,
                   const float *uv, const float *duv,
                   float *s_wo, float *s_w, float *s_pdf, int *s_m, float *e_rgb, float *p_pdf) {
    for (uint64_t i = 0; i < n; i++) {
        g_isect.UV = uv ? Point2f(uv[2 * i], uv[2 * i + 1]) : Point2f(0.0f, 0.0f);
        g_isect.dUdX = duv ? duv[4 * i] : 0.0f;
        g_isect.dVdX = duv ? duv[4 * i + 1] : 0.0f;
        g_isect.dUdY = duv ? duv[4 * i + 2] : 0.0f;
        g_isect.dVdY = duv ? duv[4 * i + 3] : 0.0f;
        float eta; int m;
        hr_bsdf_sample(h, wi + 3 * i, u2 + 2 * i, u1 ? u1[i] : 0.0f, s_wo + 3 * i, s_w + 3 * i, &m, &eta);
        s_m[i] = m;
        bool zero = s_w[3 * i] == 0.0f && s_w[3 * i + 1] == 0.0f && s_w[3 * i + 2] == 0.0f;
        s_pdf[i] = zero ? 0.0f : hr_bsdf_pdf(h, wi + 3 * i, s_wo + 3 * i, m);
        hr_bsdf_eval(h, wi + 3 * i, wo + 3 * i, 1, e_rgb + 3 * i);
        p_pdf[i] = hr_bsdf_pdf(h, wi + 3 * i, wo + 3 * i, 1);
    }
}

/* ---- acceleration structures (src/core/Acceleration.cpp, src/acceleration/*.cpp) ---- */
namespace {
struct RefAccel {
    Acceleration *accel = nullptr;
    std::vector<Mesh *> meshes;
    std::vector<uint32_t> base;   /* global index of each mesh's first triangle */
};
}

/* kind 0 "bruto" (the reference's brute-force loop), 1 "bvh", 2 "hlbvh" over
 * the meshes (hr_mesh_create handles, in order); triangle ids are global in
 * that order. */
void *hr_accel_create(int kind, int leaf_size, void *const *meshes, int n) {
    static const char *names[] = {"bruto", "bvh", "hlbvh"};
    try {
        PropertyList pl;
        if (kind > 0) pl.SetInteger("leafSize", leaf_size);
        RefAccel *r = new RefAccel;
        r->accel = (Acceleration *)ObjectFactory::CreateInstance(names[kind], pl);
        uint32_t b = 0;
        for (int i = 0; i < n; i++) {
            Mesh *m = (Mesh *)meshes[i];
            r->meshes.push_back(m);
            r->base.push_back(b);
            b += m->GetTriangleCount();
            r->accel->AddMesh(m);
        }
        r->accel->Build();
        return r;
    } catch (const std::exception &e) {
        fprintf(stderr, "hr_accel_create: %s\n", e.what());
        return nullptr;
    }
}

/* Acceleration::RayIntersect for n rays of 8 floats (o, d, minT, maxT).
 * any_hit: tri[i] = 1 / 0.  Otherwise tri[i] = global triangle id or -1 and
 * t, u, v of the hit; u, v are the barycentrics Mesh::RayIntersect returns for
 * the hit triangle (PostIntersect replaces Isect.UV by texture coordinates). */
void hr_accel_trace(void *h, uint64_t n, const float *rays, int any_hit, int32_t *tri, float *t, float *u, float *v) {
    RefAccel *r = (RefAccel *)h;
    for (uint64_t i = 0; i < n; i++) {
        const float *q = rays + 8 * i;
        Ray3f R(Point3f(q[0], q[1], q[2]), Vector3f(q[3], q[4], q[5]), q[6], q[7]);
        Intersection I;
        const bool f = r->accel->RayIntersect(R, I, any_hit != 0);
        if (any_hit) { tri[i] = f ? 1 : 0; continue; }
        if (!f) { tri[i] = -1; t[i] = u[i] = v[i] = 0.0f; continue; }
        const Mesh *m = I.pShape->GetMesh();
        const uint32_t facet = I.pShape->GetFacetIndex();
        size_t k = 0;
        while (k < r->meshes.size() && r->meshes[k] != m) k++;
        tri[i] = (int32_t)(r->base[k] + facet);
        float U = 0.0f, V = 0.0f, T = 0.0f;
        m->RayIntersect(facet, R, U, V, T);
        t[i] = I.T; u[i] = U; v[i] = V;
    }
}

void hr_accel_free(void *h) {
    RefAccel *r = (RefAccel *)h;
    delete r->accel;
    delete r;
}

/* ---- EnvironmentLight (src/emitter/EnvironmentLight.cpp) ---- */
/* The "env" emitter of an EXR file (read through the oracle's Bitmap
 * stand-in), toWorld a row-major 4x4.  Sample / Eval / Pdf go through
 * hr_emitter_sample and hr_emitter_eval_dir. */
void *hr_env_create(const char *exr_path, const float *to_world16, float scale) {
    try {
        PropertyList pl;
        pl.SetString("filename", exr_path);
        Eigen::Matrix4f M;
        for (int r = 0; r < 4; r++)
            for (int c = 0; c < 4; c++) M(r, c) = to_world16[4 * r + c];
        pl.SetTransform("toWorld", Transform(M));
        pl.SetFloat("scale", scale);
        Emitter *e = (Emitter *)ObjectFactory::CreateInstance("env", pl);
        e->Activate();
        return e;
    } catch (const std::exception &ex) {
        fprintf(stderr, "hr_env_create: %s\n", ex.what());
        return nullptr;
    }
}

void hr_object_free(void *o) { delete (Object *)o; }

/* ---- reconstruction filters and ImageBlock::Put (src/filter/*.cpp, src/core/Block.cpp) ---- */
/* kind 0 box, 1 tent, 2 gaussian (radius, stddev = p0), 3 mitchell (radius, B = p0, C = p1) */
void *hr_filter_create(int kind, float radius, float p0, float p1) {
    static const char *names[] = {"box", "tent", "gaussian", "mitchell"};
    try {
        PropertyList pl;
        if (kind == 2) { pl.SetFloat("radius", radius); pl.SetFloat("stddev", p0); }
        if (kind == 3) { pl.SetFloat("radius", radius); pl.SetFloat("B", p0); pl.SetFloat("C", p1); }
        Object *f = ObjectFactory::CreateInstance(names[kind], pl);
        f->Activate();
        return f;
    } catch (const std::exception &e) {
        fprintf(stderr, "hr_filter_create: %s\n", e.what());
        return nullptr;
    }
}

/* ReconstructionFilter::Eval at n offsets; returns the filter radius */
float hr_filter_eval(void *f, uint64_t n, const float *x, float *out) {
    const ReconstructionFilter *F = (const ReconstructionFilter *)f;
    for (uint64_t i = 0; i < n; i++) out[i] = F->Eval(x[i]);
    return F->GetRadius();
}

/* ImageBlock(W x H, filter) with offset (0, 0): Clear, then Put every sample
 * (pos n x 2 film coordinates, val n x 3) in order; film_rgbw receives the
 * (H+2B) x (W+2B) x 4 result.  Returns the border B. */
int hr_block_put(void *f, int W, int H, uint64_t n, const float *pos, const float *val, float *film_rgbw) {
    ImageBlock B(Vector2i(W, H), (const ReconstructionFilter *)f);
    B.Clear();
    for (uint64_t i = 0; i < n; i++)
        B.Put(Point2f(pos[2 * i], pos[2 * i + 1]), Color3f(val[3 * i], val[3 * i + 1], val[3 * i + 2]));
    if (film_rgbw) {
        const int rows = (int)B.rows(), cols = (int)B.cols();
        for (int y = 0; y < rows; y++)
            for (int x = 0; x < cols; x++)
                for (int c = 0; c < 4; c++) film_rgbw[4 * ((size_t)y * cols + x) + c] = B.coeff(y, x)(c);
    }
    return B.GetBorderSize();
}
}

extern "C" {
/* The reference IndependentSampler prepared for a block at (ox, oy): n calls
 * of Next2D (out 2n floats), then n of Next1D (out n floats) -- shows the
 * order in which this build's Next2D consumes its two draws (the argument
 * evaluation order of Point2f(nextFloat(), nextFloat()) is unspecified in C++). */
void hr_sampler_draws(int ox, int oy, int n, float *out2d, float *out1d) {
    PropertyList pl;
    pl.SetInteger("sampleCount", 1);
    std::unique_ptr<Sampler> S((Sampler *)ObjectFactory::CreateInstance("independent", pl));
    ImageBlock B(Vector2i(1, 1), nullptr);
    B.SetOffset(Point2i(ox, oy));
    S->Prepare(B);
    for (int i = 0; i < n; i++) {
        Point2f p = S->Next2D();
        out2d[2 * i] = p.x();
        out2d[2 * i + 1] = p.y();
    }
    for (int i = 0; i < n; i++) out1d[i] = S->Next1D();
}
}
