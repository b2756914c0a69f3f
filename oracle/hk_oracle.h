/*
 * hk_oracle.h -- CPU restatement of Hikari's pathMIS hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the checker for the CUDA
 * renderer in hikari_b200/: only tests/, __graft_entry__.smoke() and the
 * cpu_baseline leg of bench.py may load it.  It is never linked into, or
 * called by, the product path.
 *
 * Every function restates the reference algorithm in plain C99 (float
 * arithmetic, in the reference's operation order where that order is
 * observable) and cites the reference file:line it follows.  Parity pins:
 * the golden Student-t scenes of scene/pa5/tests/test-direct.xml and
 * test-furnace.xml, and record-wise comparison against the reference BSDF
 * sources compiled under oracle/_ref (see oracle/ref_build.py).
 */
#ifndef HK_ORACLE_H
#define HK_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* BSDF kinds (XML type names of the reference, include/core/Common.hpp). */
enum {
    HO_BSDF_DIFFUSE = 0,          /* "diffuse"          src/bsdf/DiffuseBSDF.cpp        */
    HO_BSDF_ROUGH_CONDUCTOR = 1,  /* "roughConductor"   src/bsdf/RoughConductorBSDF.cpp */
    HO_BSDF_ROUGH_DIELECTRIC = 2, /* "roughDielectric"  src/bsdf/RoughDielectricBSDF.cpp*/
    HO_BSDF_ROUGH_PLASTIC = 3,    /* "roughPlastic"     src/bsdf/RoughPlasticBSDF.cpp   */
    HO_BSDF_ROUGH_COATING = 4,    /* "roughCoating"     src/bsdf/RoughCoatingBSDF.cpp   */
    HO_BSDF_MIRROR = 5,           /* "mirror"           src/bsdf/MirrorBSDF.cpp         */
    HO_BSDF_CONDUCTOR = 6,        /* "conductor"        src/bsdf/ConductorBSDF.cpp      */
    HO_BSDF_DIELECTRIC = 7,       /* "dielectric"       src/bsdf/DielectricBSDF.cpp     */
    HO_BSDF_PLASTIC = 8,          /* "plastic"          src/bsdf/PlasticBSDF.cpp        */
    HO_BSDF_TWO_SIDED = 9,        /* "twoSided"         src/bsdf/TwoSidedBSDF.cpp       */
    HO_BSDF_COATING = 10,         /* "coating"          src/bsdf/CoatingBSDF.cpp        */
    HO_BSDF_ROUGH_DIFFUSE = 11,   /* "roughDiffuse"     src/bsdf/RoughDiffuseBSDF.cpp   */
    HO_BSDF_BUMP_MAP = 12,        /* "bumpMap"          src/bsdf/BumpMapBSDF.cpp        */
    HO_BSDF_NORMAL_MAP = 13       /* "normalMap"        src/bsdf/NormalMapBSDF.cpp      */
    /* bumpMap / normalMap: the map texture in tex[0], the wrapped BSDF in nested */
};
enum { HO_BECKMANN = 0, HO_GGX = 1 };
enum { HO_MEASURE_UNKNOWN = 0, HO_MEASURE_SOLID_ANGLE = 1, HO_MEASURE_DISCRETE = 2 };

/* Flat BSDF description: the XML properties of the in-scope BSDFs. */
typedef struct {
    int32_t type;          /* HO_BSDF_* */
    int32_t distribution;  /* HO_BECKMANN / HO_GGX */
    int32_t anisotropic;   /* "as" */
    int32_t nonlinear;     /* roughPlastic "nonlinear" */
    float alpha_u, alpha_v;
    float int_ior, ext_ior;
    float eta[3];          /* roughConductor: intIOR/extIOR per channel */
    float k[3];            /* roughConductor: extinction k (divided by extIOR internally) */
    float ks[3];           /* ks / ksReflect */
    float ks_refract[3];   /* roughDielectric ksRefract */
    float kd[3];           /* roughPlastic kd, diffuse albedo */
    float sigma_a[3];      /* roughCoating sigmaA */
    float thickness;       /* roughCoating thickness */
    int32_t nested;        /* roughCoating / twoSided (front): index of the nested BSDF, else -1 */
    int32_t nested2;       /* twoSided (back): index of the second nested BSDF, -1 = the front one */
    int32_t fast_approx;   /* roughDiffuse "fastApprox" */
    /* textures of kd, ks / ksReflect, ksRefract, sigmaA, alpha / alphaU, alphaV:
     * 1 + texture id (ho_scene_add_texture), 0 = the constant value above */
    int32_t tex[6];
} ho_bsdf_desc;

/* Procedural textures (src/texture/{Checkerboard,Grid,Scale}Texture.cpp) and
 * bitmap textures (src/texture/BitmapTexture.cpp over include/core/MipMap.hpp). */
enum { HO_TEX_CHECKERBOARD = 1, HO_TEX_GRID = 2, HO_TEX_SCALE = 3, HO_TEX_BITMAP = 4, HO_TEX_WIREFRAME = 5,
       HO_TEX_CURVATURE = 6 };
enum { HO_FILTER_NEAREST = 0, HO_FILTER_BILINEAR = 1, HO_FILTER_TRILINEAR = 2, HO_FILTER_EWA = 3 };
enum { HO_WRAP_REPEAT = 0, HO_WRAP_CLAMP = 1, HO_WRAP_BLACK = 2 };
typedef struct {
    int32_t kind;          /* HO_TEX_* */
    int32_t nested;        /* scale: the scaled texture's id */
    int32_t count;         /* checkerboard "blocks", grid "lines" */
    float width;           /* grid "lineWidth" */
    float scale;           /* scale "scale" */
    float uv_scale[2], uv_offset[2];   /* "uScale" "vScale", "uOffset" "vOffset" */
    float a[3], b[3];      /* checkerboard colorA / colorB; grid lineColor / backgroundColor;
                              wireframe interiorColor / edgeColor; curvature positiveColor / negativeColor */
    /* wireframe: width "edgeWidth" (0: a tenth of the mean edge length of the
     * first mesh whose BSDF uses it), scale "transitionWidth"; curvature:
     * scale "scale", count 1 "gaussian" / 0 "mean" ("curvatureType") */
    /* bitmap: "filterType", "uWrapMode" / "vWrapMode", "channel" (1 = r, 3 = rgb),
     * "gamma", "maxAnisotropy" */
    int32_t filter, wrap_u, wrap_v, channels;
    float gamma, max_anisotropy;
} ho_texture_desc;

typedef struct ho_scene ho_scene;

/* --- RNG (pcg32, ext/pcg32/pcg32.h) ------------------------------------ */
typedef struct { uint64_t state, inc; } ho_pcg32;
void     ho_pcg32_seed(ho_pcg32 *r, uint64_t initstate, uint64_t initseq);
uint32_t ho_pcg32_next(ho_pcg32 *r);
float    ho_pcg32_nextf(ho_pcg32 *r);

/* --- scene construction ------------------------------------------------- */
ho_scene *ho_scene_create(void);
void      ho_scene_destroy(ho_scene *s);
/* Raw RFT table file bytes (data/{Beckmann,GGX}RFTData.bin), index = distribution. */
int  ho_scene_set_rft(ho_scene *s, int distribution, const void *bytes, uint64_t nbytes);
int  ho_scene_add_bsdf(ho_scene *s, const ho_bsdf_desc *d);   /* returns id or <0 */
int  ho_scene_add_texture(ho_scene *s, const ho_texture_desc *d);   /* returns id or <0 */
/* Bitmap texture from 8-bit pixels as stbi_load returns them (row 0 = the top
 * row, d->channels bytes per pixel).  Returns id or <0. */
int  ho_scene_add_bitmap(ho_scene *s, const ho_texture_desc *d, const uint8_t *pixels, int width, int height);
/* Texture2D::Eval(Isect, filter = true) at texture coordinates uv (2) with the
 * screen-space partials duv = (dUdX, dVdX, dUdY, dVdY) or NULL (zero): out rgb (3). */
void ho_texture_eval(const ho_scene *s, int id, const float *uv, const float *duv, float *out);
/* The MIP pyramid of a bitmap texture: level count, or, for 0 <= level <
 * levels, the level's size (out wh[2]) and texels (channels floats each,
 * row-major, row 0 = v 0) when texels != NULL. */
int  ho_texture_mip(const ho_scene *s, int id, int level, int *wh, float *texels);
/* Texture::Eval(Isect, true) at the intersection Triangle::PostIntersect makes
 * of barycentric (u, v) on triangle tri (scene order): out rgb (3).  The form
 * the wireframe and curvature textures need (they read the hit's triangle,
 * position and UV partials). */
void ho_texture_eval_hit(const ho_scene *s, int id, uint32_t tri, float u, float v, float *out);
/* positions 3*nv, indices 3*nt (mesh-local), normals 3*nv or NULL,
 * radiance 3 or NULL (area light).  Returns mesh id or <0. */
int  ho_scene_add_mesh(ho_scene *s, const float *positions, uint32_t nv,
                       const uint32_t *indices, uint32_t nt, const float *normals,
                       int32_t bsdf, const float *radiance);
/* rgb H*W*3 row-major (row 0 = theta 0); to_world row-major 4x4. */
int  ho_scene_set_envmap(ho_scene *s, const float *rgb, uint32_t w, uint32_t h,
                         const float *to_world16, float scale);
/* Texture coordinates of a mesh: 2 floats per vertex. */
int  ho_scene_set_mesh_uv(ho_scene *s, int mesh, const float *uv);
/* Triangle::PostIntersect of a finalized scene: out p(3) s(3) t(3) n(3) uv(2). */
void ho_post_intersect(const ho_scene *s, uint32_t tri, float u, float v, float *out);
/* ConstantLight radiance (one environment emitter per scene); point / directional lights. */
int  ho_scene_set_constant_light(ho_scene *s, const float *radiance);
int  ho_scene_add_point_light(ho_scene *s, const float *power, const float *position);
int  ho_scene_add_directional_light(ho_scene *s, const float *irradiance, const float *direction);
/* camera: to_world row-major 4x4, horizontal fov degrees, clip planes. */
int  ho_scene_set_camera(ho_scene *s, uint32_t width, uint32_t height, const float *to_world16,
                         float fov_deg, float near_clip, float far_clip);
/* filter: 0 box, 1 tent, 2 gaussian(radius, stddev), 3 mitchell(radius, B, C) */
int  ho_scene_set_filter(ho_scene *s, int kind, float radius, float p0, float p1);
int  ho_scene_set_background(ho_scene *s, const float *rgb, int force_background);
int  ho_scene_finalize(ho_scene *s);     /* activate BSDFs, light CDFs, BVH */
const char *ho_last_error(void);
void ho_scene_bbox(const ho_scene *s, float *out6);
int  ho_scene_num_emitters(const ho_scene *s);

/* --- single-record BSDF queries (local frame) ------------------------- */
/* Sample: wi in, u2 (2 floats), u1 = the Next1D draw of roughDielectric.
 * out_wo (3), returns weight in out_w (3), out_measure, out_eta. */
void  ho_bsdf_sample(const ho_scene *s, int bsdf, const float *wi, const float *u2, float u1,
                     float *out_wo, float *out_w, int *out_measure, float *out_eta);
void  ho_bsdf_eval(const ho_scene *s, int bsdf, const float *wi, const float *wo, int measure,
                   float *out_rgb);
float ho_bsdf_pdf(const ho_scene *s, int bsdf, const float *wi, const float *wo, int measure);
/* batched over n records, 2^k friendly; records are AoS float3 */
void  ho_bsdf_batch(const ho_scene *s, int bsdf, uint64_t n, const float *wi, const float *u2,
                    const float *u1, const float *wo, const float *uv, const float *duv, float *s_wo,
                    float *s_w, float *s_pdf, int32_t *s_measure, float *e_rgb, float *p_pdf, int nthreads);
/* (uv: n x 2 texture coordinates of the records' intersections, or NULL;
 *  duv: n x 4 screen-space partials (dUdX, dVdX, dUdY, dVdY), or NULL) */
/* Intersection::ComputeScreenSpacePartial (src/core/Intersection.cpp:30) of
 * the camera ray through film position (px, py) hitting (tri, u, v):
 * out duv (4) = (dUdX, dVdX, dUdY, dVdY). */
/* ho_bsdf_batch with each record's intersection (n x 20 floats: shading
 * frame S T N, geometric N, dPdU, dPdV, UV) -- the records of bumpMap /
 * normalMap, whose frames perturb the shading frame. */
void  ho_bsdf_batch_isect(const ho_scene *s, int bsdf, uint64_t n, const float *wi, const float *u2,
                          const float *u1, const float *wo, const float *isect, float *s_wo, float *s_w,
                          float *s_pdf, int32_t *s_measure, float *e_rgb, float *p_pdf, int nthreads);
void  ho_screen_partials(const ho_scene *s, float px, float py, uint32_t tri, float u, float v, float *out4);
/* RFT 1D eval after activation (for table parity tests). */
float ho_bsdf_rft_eval(const ho_scene *s, int bsdf, float cos_theta);

/* --- ray queries ------------------------------------------------------- */
/* rays: n x 8 floats (ox,oy,oz,dx,dy,dz,mint,maxt).  hits: n x {t,u,v} floats
 * and tri (global triangle index, -1 for miss).  any_hit != 0: shadow query,
 * returns 1/0 in tri.  use_bvh selects the SAH BVH, else the reference's
 * brute-force loop (src/core/Acceleration.cpp:45). */
void ho_trace(const ho_scene *s, uint64_t n, const float *rays, float *thit, float *uhit, float *vhit,
              int32_t *tri, int any_hit, int use_bvh, int nthreads);

/* --- rendering ---------------------------------------------------------- */
/* Full render like src/Main.cpp:46 (32x32 blocks, per-block pcg32 seeded with
 * the block offset), accumulating RGBW in double.  film_rgbw has
 * (H+2B)*(W+2B)*4 doubles where B = ceil(radius-0.5).  If block_list is
 * non-NULL only those block indices (row-major over the block grid) render.
 * depth: the integrator's "depth".  Returns number of dropped samples. */
/* swap2d != 0: every two-dimensional draw (pixel jitter, emitter and BSDF
 * sample pairs) takes (second, first) uniform, as the reference's Next2D does
 * when built with right-to-left argument evaluation (GCC); default (first,
 * second), the CUDA kernels' order.  Only path-level comparisons against the
 * compiled reference need it. */
void ho_scene_set_reference_draw_order(ho_scene *s, int swap2d);
int64_t ho_render(const ho_scene *s, int depth, int spp, const int32_t *block_list, int nblocks,
                  double *film_rgbw, int nthreads, uint64_t *counters /* 4: paths, rays, shadow, 0 */);
/* Per-pixel per-sample statistics: sample 'spp' paths per pixel of the listed
 * pixels with streams seeded from (seed, pixel), store the mean and variance
 * of each channel of Li (no filter). pix: npix*2 ints. out: npix*6 doubles. */
void ho_pixel_stats(const ho_scene *s, int depth, int spp, uint64_t seed, int npix,
                    const int32_t *pix, double *out, int nthreads);
/* One sample per listed pixel from the stream (seed, pixel): out npix x 5
 * floats (film x, film y, radiance rgb). */
void ho_pixel_samples(const ho_scene *s, int depth, uint64_t seed, int npix, const int32_t *pix, float *out,
                      int nthreads);
/* StudentTTest scene mode (src/core/StudentTTest.cpp:143-174): n paths with
 * a default-seeded independent sampler; mean and variance of luminance. */
void ho_ttest_scene(const ho_scene *s, int depth, int n, double *mean, double *var);
/* Resolve the bordered film to an H*W*3 float image (Block.cpp:61). */
void ho_film_resolve(const ho_scene *s, const double *film_rgbw, float *out_rgb);
int  ho_film_border(const ho_scene *s);
/* ImageBlock::Put (src/core/Block.cpp:95-134) of n samples (film positions
 * n x 2, values n x 3) into a bordered film of doubles; returns the number
 * dropped as invalid. */
int64_t ho_film_put_samples(const ho_scene *s, uint64_t n, const float *pos, const float *val, double *film);

/* --- emitter / camera / filter record queries -------------------------- */
void  ho_emitter_sample(const ho_scene *s, int e, const float *ref, float ux, float uy, float u1, float *out14);
float ho_emitter_pdf(const ho_scene *s, int e, const float *ref, const float *p, const float *n);
void  ho_env_eval(const ho_scene *s, const float *wi, float *out3);
void  ho_camera_ray(const ho_scene *s, float px, float py, float *out8);
void  ho_filter_table(const ho_scene *s, float *out33, float *lookup);

#ifdef __cplusplus
}
#endif
#endif
