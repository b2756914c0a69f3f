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
                                  "roughDiffuse"};
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

/* kind 1 checkerboard, 2 grid, 3 scale (of nested) */
void *hr_texture_create(int kind, int count, float width, float scale, const float *uv_scale, const float *uv_offset,
                        const float *a, const float *b, void *nested) {
    try {
        PropertyList pl;
        Color3f ca(a[0], a[1], a[2]), cb(b[0], b[1], b[2]);
        const char *name = kind == 1 ? "checkerboard" : (kind == 2 ? "grid" : "scale");
        if (kind == 1 || kind == 2) {
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

/* batched over n AoS records (same layout as ho_bsdf_batch) */
void hr_bsdf_batch(void *h, uint64_t n, const float *wi, const float *u2, const float *u1, const float *wo,
                   const float *uv,
                   float *s_wo, float *s_w, float *s_pdf, int *s_m, float *e_rgb, float *p_pdf) {
    for (uint64_t i = 0; i < n; i++) {
        g_isect.UV = uv ? Point2f(uv[2 * i], uv[2 * i + 1]) : Point2f(0.0f, 0.0f);
        float eta; int m;
        hr_bsdf_sample(h, wi + 3 * i, u2 + 2 * i, u1 ? u1[i] : 0.0f, s_wo + 3 * i, s_w + 3 * i, &m, &eta);
        s_m[i] = m;
        bool zero = s_w[3 * i] == 0.0f && s_w[3 * i + 1] == 0.0f && s_w[3 * i + 2] == 0.0f;
        s_pdf[i] = zero ? 0.0f : hr_bsdf_pdf(h, wi + 3 * i, s_wo + 3 * i, m);
        hr_bsdf_eval(h, wi + 3 * i, wo + 3 * i, 1, e_rgb + 3 * i);
        p_pdf[i] = hr_bsdf_pdf(h, wi + 3 * i, wo + 3 * i, 1);
    }
}
}
