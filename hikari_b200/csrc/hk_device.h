// Device-resident scene layout shared by the host builder (hk_host.cpp) and the
// sm_100a kernels.  Everything here lives in HBM and is read through the
// read-only path; record sizes are multiples of 16 bytes so every fetch is a
// 128-bit load.
#pragma once
#include <cstdint>
#include <vector_types.h>

namespace hk {

enum BsdfType : int32_t {
    kDiffuse = 0, kRoughConductor = 1, kRoughDielectric = 2, kRoughPlastic = 3, kRoughCoating = 4,
    kMirror = 5, kConductor = 6, kDielectric = 7, kPlastic = 8, kTwoSided = 9, kCoating = 10, kRoughDiffuse = 11,
    kBumpMap = 12, kNormalMap = 13   // wrap `nested`; the map texture is tex[0]
};
enum Distribution : int32_t { kBeckmann = 0, kGGX = 1 };
enum Measure : int32_t { kMeasureUnknown = 0, kMeasureSolidAngle = 1, kMeasureDiscrete = 2 };

enum EnvKind : int32_t { kEnvMap = 1, kEnvConstant = 2 };

constexpr int kRftThetaMax = 100;   // data/*RFTData.bin hold 100 theta samples

// One activated BSDF: constant-texture parameters plus the 1D rough
// transmittance table reduced at activation (RoughTransmittance::SetEta then
// SetAlpha, src/core/RoughTransmitance.cpp:170,237).
struct DevTexture;
// Layers (coatings, twoSided) a BSDF may stack above its leaf BSDFs: the
// device walks at most this many layers of a stack (deep_* in hk_bsdf.cuh)
constexpr int kNestLevels = 4;
struct alignas(16) DevBsdf {
    int32_t type, distribution, anisotropic, nonlinear;
    float alpha_u, alpha_v;          // clamped to [MIN_ALPHA, MAX_ALPHA]
    float eta, inv_eta;              // intIOR / extIOR and its inverse
    float inv_eta2;
    float spec_w;                    // m_SpecularSamplingWeight
    float fdr_int;                   // roughPlastic: 1 - IntData.EvalDiffuse(alpha)
    float thickness;
    float eta_c[3], k_c[3];          // conductor eta and k/extIOR per channel
    float ks[3], ks_refract[3], kd[3], sigma_a[3];
    int32_t nested;                  // (rough)coating nested BSDF / twoSided front BSDF index, -1 otherwise
    int32_t rft_n;                   // theta samples in rft[]
    int32_t nested2;                 // twoSided back BSDF index (the front one when only one is given)
    int32_t fast_approx;             // roughDiffuse: the fast Oren-Nayar approximation
    // textures of kd, ks, ks_refract, sigma_a, alpha_u, alpha_v: 1 + index into
    // textures, 0 = the constant above; textured: any slot here or in a nested BSDF
    int32_t tex[6];
    const DevTexture *textures;
    int32_t textured;
    int32_t geo_tex;                 // a wireframe or curvature texture in a slot here or in a nested BSDF
    int32_t alpha_tex;               // roughPlastic / roughCoating with a textured alpha: rft2d / rft_diff below
    int32_t rft_an;                  // alpha samples of rft2d / rft_diff
    float rft[kRftThetaMax];
    // a textured alpha: the transmittance left 2D by SetEta ([alpha][theta],
    // rft_an x rft_n) and roughPlastic's diffuse one over alpha (rft_an)
    const float *rft2d;
    const float *rft_diff;
    float rft_amin, rft_amax;
    // a layered BSDF nested deeper than one (rough) coating over a leaf, or a
    // twoSided over such a layer or over a twoSided: dispatched through the
    // deep_* functions of hk_bsdf.cuh, never by per-type kernels (kept at the
    // end so that the fields above keep their offsets and vector loads)
    int32_t deep;
    int32_t pad6;
};

// cutpoints per CDF in the environment map's guide tables (a power of two)
constexpr int kEnvGuide = 1024;
// Procedural texture (src/texture/{Checkerboard,Grid,Scale}Texture.cpp),
// bitmap (src/texture/BitmapTexture.cpp over include/core/MipMap.hpp) or a
// texture of the hit's geometry (src/texture/{Wireframe,Curvature}Texture.cpp:
// a interior / positive colour, b edge / negative colour, width the edge
// width, scale the transition width / curvature scale, count 1 for Gaussian
// curvature, 0 for mean curvature).
enum TexKind : int32_t { kTexCheckerboard = 1, kTexGrid = 2, kTexScale = 3, kTexBitmap = 4, kTexWireframe = 5,
                         kTexCurvature = 6 };
enum TexFilter : int32_t { kFilterNearest = 0, kFilterBilinear = 1, kFilterTrilinear = 2, kFilterEwa = 3 };
constexpr int kMipMaxLevels = 16;   // level 0 up to 32768 texels a side
constexpr int kEwaLutSize = 128;
struct alignas(16) DevTexture {
    int32_t kind, nested, count;     // nested: the scaled texture; count: blocks / lines
    float width, scale;              // grid line width; scale factor
    float uv_scale[2], uv_offset[2];
    float a[3], b[3];                // colorA / lineColor, colorB / backgroundColor
    // bitmap: MIP levels of power-of-two sizes, level l is (1 << max(0, lw - l)) x
    // (1 << max(0, lh - l)) texels, row-major from v = 0; rgb texels are float4
    // (w unused), r texels one float
    int32_t filter;                  // TexFilter
    int32_t channels, levels, lw, lh;
    int32_t black;                   // a wrap mode is "black": every texel reads black
    float max_aniso;
    int32_t pad0, pad1;
    const float *texels;             // level 0 first
    const float *lut;                // EWA weights (kEwaLutSize)
    uint32_t lvl_off[kMipMaxLevels]; // first texel of each level
};

// Per-mesh shading data.
struct alignas(16) DevMesh {
    int32_t bsdf;          // DevBsdf index
    int32_t emitter;       // emitter index or -1
    int32_t has_normals;   // vertex normals present -> interpolated shading frame
    int32_t has_uv;        // texture coordinates present (with normals: the frame follows dP/du)
    float radiance[3];     // area emitter radiance
    float pad1;
};

// Area emitter: triangles of its mesh in mesh order with the area CDF
// (DiscretePDF1D over triangle areas, src/core/Mesh.cpp:233).
struct alignas(16) DevAreaLight {
    uint32_t tri0;         // first record in DevScene::light_tris (3 float4 per triangle)
    uint32_t ntri;
    uint32_t cdf0;         // first entry in DevScene::light_cdf (ntri+1 floats)
    int32_t mesh;
    float inv_area;
    float radiance[3];
};

// BVH2 node: both children's boxes, 64 bytes = 4 x 128-bit loads.
//   a = (c0.lo.x, c0.hi.x, c0.lo.y, c0.hi.y)
//   b = (c1.lo.x, c1.hi.x, c1.lo.y, c1.hi.y)
//   c = (c0.lo.z, c0.hi.z, c1.lo.z, c1.hi.z)
//   d = (child0, child1, -, -) as int; child < 0 -> leaf ~(start | count << 27)
constexpr int kStackSize = 64;   // traversal stack entries per ray (tree depth is capped below it)
constexpr int kAccelBvh2 = 0;
constexpr int kAccelBvh8 = 1;
constexpr int kLeafCountShift = 27;
constexpr uint32_t kLeafStartMask = (1u << kLeafCountShift) - 1u;

struct DevScene {
    // geometry: triangle records in BVH leaf order, 3 float4 each:
    //   v0.xyz, bits(original triangle index); v1.xyz, bits(mesh); v2.xyz, 0
    const float4 *tris;
    const float4 *nodes;          // 4 float4 per BVH2 node
    const uint4 *wnodes;          // 5 uint4 per compressed 8-wide node (hk_bvh.h)
    const float4 *tri_normals;    // 3 float4 per ORIGINAL triangle (only if any mesh has normals)
    const float2 *tri_uv;         // 3 float2 per ORIGINAL triangle (only if any mesh has texture coordinates)
    uint32_t ntris, nnodes, nwnodes;
    int32_t accel;                // kAccelBvh2 or kAccelBvh8: the tree the kernels traverse
    int32_t postpone;             // 8-wide traversal may postpone triangle tests (stack bound allows it)
    int32_t postpone_any;         // ... and does so for any-hit rays too (set per launch, 0 in the scene)
    int32_t textured;             // some material has textures (the megakernel compiles lookups in)
    int32_t ray_diff;             // a bitmap filters with the camera ray's differentials (first hits)
    const DevMesh *meshes;
    const DevBsdf *bsdfs;
    int32_t nmeshes, nbsdfs;
    // emitters in Scene order; env is the one with area index -1
    int32_t nemitters;
    int32_t env_index;            // position of the environment emitter, -1 if none
    // per emitter: index into area_lights, -1 the environment, -2 - k delta_lights[k]
    const int32_t *emitter_area;
    const float4 *delta_lights;   // point / directional: (position or direction, kind), (power or irradiance, 0)
    int32_t env_kind;             // kEnvMap or kEnvConstant when env_index >= 0
    float env_const[3];           // ConstantLight radiance
    const DevAreaLight *area_lights;
    const float4 *light_tris;     // emitter triangles, 3 float4 each (v0, v1, v2)
    const float4 *light_normals;  // matching vertex normals (w = has normals)
    const float *light_cdf;
    // environment map
    const float4 *env_rgb;        // H*W texels (rgb, 0)
    const float *env_marg_cdf;    // H+1
    const float *env_marg_func;   // H
    const float *env_cond_cdf;    // H*(W+1)
    const float *env_cond_func;   // H*W
    const float *env_cond_int;    // H row integrals
    const int32_t *env_marg_guide;   // kEnvGuide + 1 cutpoints of the marginal CDF
    const int32_t *env_cond_guide;   // H * (kEnvGuide + 1) cutpoints of the row CDFs
    float env_marg_int;
    uint32_t env_w, env_h;
    float env_scale;
    float env_to_world[9], env_to_local[9];
    float scene_radius;           // BoundingBox::GetRadius of the accel bbox
    // camera (PerspectiveCamera, src/camera/PerspectiveCamera.cpp:32-100)
    float cam[12];                // row-major 3x4 camera-to-world (rows of the 4x4 divided by w)
    float cam_cot, cam_aspect, cam_near, cam_far;
    uint32_t width, height;
    // reconstruction filter table (ImageBlock ctor, src/core/Block.cpp:9)
    const float *ftab;            // 33 entries in HBM (dynamic index)
    float filt_radius, filt_lookup;
    int32_t border;
    float background[3];
    int32_t force_background;
};

}  // namespace hk
