/*
 * hikari_b200.h -- C ABI of the B200 pathMIS renderer core.
 *
 * The drop-in boundary for Hikari's path-tracing hot path.  In the reference
 * the per-sample virtual call Integrator::Li (include/core/Integrator.hpp:35)
 * is driven by RenderBlock (src/Main.cpp:11-44) over TBB blocks
 * (src/Main.cpp:46-147); here a scene is uploaded once (the Preprocess hook,
 * include/core/Integrator.hpp:21) and whole images are rendered by one call.
 *
 * Conventions: every function returns an int status (HK_OK = 0, negative on
 * error) and never throws; hk_last_error() returns a thread-local message.
 * Pointers named *_dev are device (HBM) pointers; all others are host
 * pointers.  `stream` is a cudaStream_t (NULL = legacy default stream).
 * Handles are owned by the library and are not thread-safe per handle.
 */
#ifndef HIKARI_B200_H
#define HIKARI_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define HK_OK 0
#define HK_ERR_INVALID (-1)   /* bad argument / scene state (HikariException) */
#define HK_ERR_CUDA (-2)      /* CUDA runtime error */
#define HK_ERR_NOMEM (-3)     /* device allocation failed */
#define HK_ERR_IO (-4)        /* file could not be read or parsed */

typedef struct hk_scene hk_scene;

/* BSDF kinds: XML type names of the reference (include/core/Common.hpp:229-272) */
#define HK_BSDF_DIFFUSE 0          /* "diffuse"         src/bsdf/DiffuseBSDF.cpp        */
#define HK_BSDF_ROUGH_CONDUCTOR 1  /* "roughConductor"  src/bsdf/RoughConductorBSDF.cpp */
#define HK_BSDF_ROUGH_DIELECTRIC 2 /* "roughDielectric" src/bsdf/RoughDielectricBSDF.cpp*/
#define HK_BSDF_ROUGH_PLASTIC 3    /* "roughPlastic"    src/bsdf/RoughPlasticBSDF.cpp   */
#define HK_BSDF_ROUGH_COATING 4    /* "roughCoating"    src/bsdf/RoughCoatingBSDF.cpp   */
#define HK_BSDF_MIRROR 5           /* "mirror"          src/bsdf/MirrorBSDF.cpp         */
#define HK_BSDF_CONDUCTOR 6        /* "conductor"       src/bsdf/ConductorBSDF.cpp      */
#define HK_BSDF_DIELECTRIC 7       /* "dielectric"      src/bsdf/DielectricBSDF.cpp     */
#define HK_BSDF_PLASTIC 8          /* "plastic"         src/bsdf/PlasticBSDF.cpp        */
#define HK_BSDF_TWO_SIDED 9        /* "twoSided"        src/bsdf/TwoSidedBSDF.cpp       */
#define HK_BSDF_COATING 10         /* "coating"         src/bsdf/CoatingBSDF.cpp        */
#define HK_BSDF_ROUGH_DIFFUSE 11   /* "roughDiffuse"    src/bsdf/RoughDiffuseBSDF.cpp   */
#define HK_BSDF_BUMP_MAP 12        /* "bumpMap"         src/bsdf/BumpMapBSDF.cpp        */
#define HK_BSDF_NORMAL_MAP 13      /* "normalMap"       src/bsdf/NormalMapBSDF.cpp      */
/* bumpMap / normalMap wrap the BSDF `nested`; their map texture is tex[0] */
#define HK_BECKMANN 0
#define HK_GGX 1

/* XML properties of one BSDF (the reference's PropertyList for that type).
 * Replaces the BSDF plugin constructors, e.g. RoughConductorBSDF ctor
 * (src/bsdf/RoughConductorBSDF.cpp:11). */
typedef struct {
    int32_t type;          /* HK_BSDF_* */
    int32_t distribution;  /* HK_BECKMANN / HK_GGX ("type" property) */
    int32_t anisotropic;   /* "as" */
    int32_t nonlinear;     /* roughPlastic "nonlinear" */
    float alpha_u, alpha_v;/* "alpha" (or "alphaU", "alphaV") */
    float int_ior, ext_ior;
    float eta[3];          /* roughConductor relative IOR per channel (intIOR/extIOR) */
    float k[3];            /* roughConductor "k" */
    float ks[3];           /* "ks" / "ksReflect" */
    float ks_refract[3];   /* roughDielectric "ksRefract" */
    float kd[3];           /* roughPlastic "kd", diffuse "albedo" */
    float sigma_a[3];      /* roughCoating "sigmaA" */
    float thickness;       /* roughCoating "thickness" */
    int32_t nested;        /* roughCoating / twoSided front: id of the nested BSDF (added first), else -1;
                              coatings and twoSided stack up to four layers above a leaf BSDF (deeper
                              stacks fail hk_scene_build); a bumpMap / normalMap may wrap a stack but
                              not sit inside one */
    int32_t nested2;       /* twoSided back: id of the second nested BSDF, -1 = the front one */
    int32_t fast_approx;   /* roughDiffuse "fastApprox" */
    /* textures of kd / albedo, ks / ksReflect, ksRefract, sigmaA, alpha / alphaU,
     * alphaV: 1 + texture id (hk_scene_add_texture), 0 = the constant above */
    int32_t tex[6];
} hk_bsdf_desc;

typedef struct {
    uint32_t n_meshes, n_triangles, n_bsdfs, n_emitters;
    uint32_t n_bvh_nodes, bvh_depth;        /* binary tree: 64-byte nodes */
    int32_t env_index;
    int32_t film_border;
    float bbox[6];
    uint64_t device_bytes;
    uint32_t n_wide_nodes, wide_depth;      /* compressed 8-wide tree: 80-byte nodes */
    int32_t accel;                          /* HK_ACCEL_* the kernels traverse */
    int32_t postpone;                       /* 8-wide traversal postpones triangle tests */
} hk_scene_info;

/* Acceleration structures (both are built; hk_scene_set_accel picks the one
 * traversed).  The reference's accel plugins (src/acceleration/*.cpp: bruto,
 * bvh, hlbvh) all answer the same closest-hit query. */
#define HK_ACCEL_BVH2 0   /* binary binned-SAH tree, 64-byte nodes */
#define HK_ACCEL_BVH8 1   /* compressed 8-wide tree, 80-byte quantised nodes (default) */

const char *hk_last_error(void);
int hk_version(void);

/* ---- scene construction (Scene::AddChild src/core/Scene.cpp:167 order) ---- */
int hk_scene_create(hk_scene **out);
int hk_scene_destroy(hk_scene *s);
/* Procedural textures (src/texture/{Checkerboard,Grid,Scale}Texture.cpp) and
 * bitmaps (src/texture/BitmapTexture.cpp over include/core/MipMap.hpp). */
#define HK_TEX_CHECKERBOARD 1
#define HK_TEX_GRID 2
#define HK_TEX_SCALE 3
#define HK_TEX_BITMAP 4
/* Textures of the hit's geometry (src/texture/{Wireframe,Curvature}Texture.cpp):
 * wireframe: a interiorColor, b edgeColor, width edgeWidth (0: a tenth of the
 * mean edge length of the first mesh, in scene order, whose BSDF uses it),
 * scale transitionWidth; curvature: a positiveColor, b negativeColor, scale,
 * count 1 "gaussian" / 0 "mean" curvatureType.  Neither may be the map of a
 * bumpMap or normalMap. */
#define HK_TEX_WIREFRAME 5
#define HK_TEX_CURVATURE 6
/* bitmap "filterType" */
#define HK_FILTER_NEAREST 0
#define HK_FILTER_BILINEAR 1
#define HK_FILTER_TRILINEAR 2
#define HK_FILTER_EWA 3
/* bitmap "uWrapMode" / "vWrapMode" */
#define HK_WRAP_REPEAT 0
#define HK_WRAP_CLAMP 1
#define HK_WRAP_BLACK 2
typedef struct {
    int32_t kind;          /* HK_TEX_* */
    int32_t nested;        /* scale: id of the scaled texture (added first) */
    int32_t count;         /* checkerboard "blocks", grid "lines" */
    float width;           /* grid "lineWidth" */
    float scale;           /* scale "scale" */
    float uv_scale[2], uv_offset[2];   /* "uScale" "vScale", "uOffset" "vOffset" */
    float a[3], b[3];      /* checkerboard colorA / colorB; grid lineColor / backgroundColor */
    /* bitmap: "filterType" (HK_FILTER_*), "uWrapMode" / "vWrapMode" (HK_WRAP_*),
     * "channel" (1 = r, 3 = rgb), "gamma", "maxAnisotropy" */
    int32_t filter, wrap_u, wrap_v, channels;
    float gamma, max_anisotropy;
} hk_texture_desc;
int hk_scene_add_texture(hk_scene *s, const hk_texture_desc *desc, int32_t *out_id);
/* A bitmap texture (desc->kind HK_TEX_BITMAP) from 8-bit pixels as stbi_load
 * returns them to LoadImageFromFileR / RGB (src/core/Texture.cpp:12, :74):
 * row 0 is the image's top row, desc->channels bytes per pixel.  The gamma
 * correction, the resampling to power-of-two sizes and the MIP pyramid
 * (include/core/MipMap.hpp:67) are built on the host when the scene is added
 * to; the pyramid lives in HBM from hk_scene_build on. */
int hk_scene_add_bitmap(hk_scene *s, const hk_texture_desc *desc, const uint8_t *pixels, int32_t width,
                        int32_t height, int32_t *out_id);
/* Decode an 8-bit image file (PNG, binary PGM / PPM, baseline JPEG) into
 * `channels` (1 or 3) bytes per pixel, row 0 = top, like stbi_load with that
 * request.  *out is allocated by the library (hk_image_free). */
int hk_image_load(const char *path, int32_t channels, int32_t *width, int32_t *height, uint8_t **out);
void hk_image_free(uint8_t *p);
/* Raw bytes of data/BeckmannRFTData.bin (distribution 0) or GGXRFTData.bin (1),
 * the RoughTransmittance table file (src/core/RoughTransmitance.cpp:9). */
int hk_scene_set_rft(hk_scene *s, int distribution, const void *bytes, uint64_t nbytes);
int hk_scene_add_bsdf(hk_scene *s, const hk_bsdf_desc *desc, int32_t *out_id);
/* Mesh (WavefrontObjMesh, src/mesh/WavefrontObjMesh.cpp:10) in world space:
 * positions 3*nv floats, indices 3*nt, normals 3*nv or NULL, radiance 3 floats
 * for an attached area emitter (src/emitter/AreaLight.cpp:8) or NULL. */
int hk_scene_add_mesh(hk_scene *s, const float *positions, uint32_t nv, const uint32_t *indices, uint32_t nt,
                      const float *normals, int32_t bsdf, const float *radiance, int32_t *out_id);
/* Texture coordinates of a mesh (the OBJ "vt" of each vertex): 2*nv floats.
 * With vertex normals they orient the shading frame along dP/du
 * (Triangle::PostIntersect, src/core/Mesh.cpp:107-158). */
int hk_scene_set_mesh_uv(hk_scene *s, int32_t mesh, const float *uv);
/* Environment emitter (EnvironmentLight ctor, src/emitter/EnvironmentLight.cpp:8):
 * rgb is H*W*3 floats, row 0 at theta = 0; to_world row-major 4x4. */
int hk_scene_set_envmap(hk_scene *s, const float *rgb, uint32_t width, uint32_t height, const float *to_world16,
                        float scale);
/* Constant environment emitter (ConstantLight, src/emitter/ConstantLight.cpp:8):
 * radiance 3 floats.  One environment emitter per scene (map or constant). */
int hk_scene_set_constant_light(hk_scene *s, const float *radiance);
/* Point light (PointLight, src/emitter/PointLight.cpp:8): power and position, 3 floats each. */
int hk_scene_add_point_light(hk_scene *s, const float *power, const float *position);
/* Directional light (DirectionalLight, src/emitter/DirectionalLight.cpp:8):
 * irradiance and direction of travel, 3 floats each. */
int hk_scene_add_directional_light(hk_scene *s, const float *irradiance, const float *direction);
/* OBJ ingest (WavefrontObjMesh, src/mesh/WavefrontObjMesh.cpp:10-152), parsed
 * in parallel: positions (3*nv) transformed by to_world16 (row-major 4x4, NULL =
 * identity), normals (3*nv) by its inverse transpose, texture coordinates
 * (2*nv), indices (3*nt), quads split and vertices de-duplicated in first-use
 * order like the reference.  Call with positions == NULL to get nv / nt, then
 * with arrays of that size; attrs bit 0: normals present, bit 1: uv present. */
int hk_obj_load(const char *path, const float *to_world16, uint32_t *nv, uint32_t *nt, float *positions,
                float *normals, float *uv, uint32_t *indices, int32_t *attrs);
/* PerspectiveCamera (src/camera/PerspectiveCamera.cpp:13): to_world row-major 4x4. */
int hk_scene_set_camera(hk_scene *s, uint32_t width, uint32_t height, const float *to_world16, float fov_deg,
                        float near_clip, float far_clip);
/* Reconstruction filter (src/filter/*.cpp): kind 0 box, 1 tent, 2 gaussian
 * (p0 = stddev), 3 mitchell (p0 = B, p1 = C). */
int hk_scene_set_filter(hk_scene *s, int kind, float radius, float p0, float p1);
int hk_scene_set_background(hk_scene *s, const float *rgb3, int force_background);
/* Activate every object and upload (Scene::Activate src/core/Scene.cpp:128 +
 * Integrator::Preprocess): BSDF tables, light CDFs, the BVH, device buffers. */
int hk_scene_build(hk_scene *s);
/* Where hk_scene_build builds the trees.  HK_BUILDER_HOST (default): the
 * binned-SAH binary tree and its SAH-optimal 8-wide collapse on the host
 * threads (the reference builds its HLBVH on the host too,
 * src/acceleration/HLBVHAcceleration.cpp:81).  HK_BUILDER_GPU: the 8-wide tree
 * only, built on the device from Morton-ordered triangles (a linear BVH
 * collapsed greedily): milliseconds instead of seconds for millions of
 * triangles, for scenes that must become renderable fast, at some cost in
 * traversal work; the scene then traverses the 8-wide tree only. */
enum { HK_BUILDER_HOST = 0, HK_BUILDER_GPU = 1 };
int hk_scene_set_builder(hk_scene *s, int32_t builder);
/* Seconds the last hk_scene_build spent building (and uploading) its trees. */
int hk_scene_tree_build_seconds(const hk_scene *s, double *seconds);
/* Profiling aid, no counterpart in the reference: the rays each launch of the
 * closest-hit (which 0) or shadow (which 1) traversal kernel traced in the
 * scene's last hk_render_batch, in launch order.  Up to max counts go to
 * rays_host (the first 1024 launches are kept); *launches gets the number of
 * launches.  Waits for the scene's wavefront work to finish. */
int hk_wavefront_launch_log(hk_scene *s, int32_t which, uint32_t *rays_host, int32_t max, int32_t *launches);
/* Build the device 8-wide tree over n triangles (9 floats each, host) and run
 * hk_bvh_check's structural check of the 8-wide tree on it (HK_ERR_INVALID
 * with the first problem found). */
int hk_bvh_check_gpu(const float *tris, uint32_t n, uint32_t *n_wide_nodes, uint32_t *wide_depth);
/* Select the tree the render and trace kernels traverse (takes effect
 * immediately on a built scene; both trees share one triangle order; a scene
 * built with HK_BUILDER_GPU has the 8-wide tree only). */
int hk_scene_set_accel(hk_scene *s, int32_t accel);
/* Counts and bbox; before hk_scene_build the BVH and device fields are 0. */
int hk_scene_get_info(const hk_scene *s, hk_scene_info *info);
/* Parse a Hikari scene XML file through the C++ plugin layer (LoadFromXML,
 * src/core/Parser.cpp:9) and build it.  data_dir holds the RFT tables.
 * Returns the pathMIS depth and sampler sampleCount in *depth / *spp. */
int hk_scene_load_xml(const char *path, const char *data_dir, hk_scene **out, int32_t *depth, int32_t *spp);
/* Same parse without the build/upload step (host only; hk_scene_build later). */
int hk_scene_parse_xml(const char *path, const char *data_dir, hk_scene **out, int32_t *depth, int32_t *spp);

/* OpenEXR I/O of the output path (Bitmap, src/core/Bitmap.cpp:14,76): read an
 * RGB(A) scanline EXR (NONE/ZIPS/ZIP, HALF/FLOAT) -- call with rgb = NULL to
 * get the size, then with a buffer of capacity >= w*h*3 floats; write an
 * uncompressed FLOAT RGB EXR from h*w*3 floats. */
int hk_exr_read(const char *path, int32_t *width, int32_t *height, float *rgb, uint64_t capacity);
int hk_exr_write(const char *path, int32_t width, int32_t height, const float *rgb);

/* ---- rendering (replaces the Render / RenderBlock loop, src/Main.cpp:11-147) ---- */
typedef struct {
    int32_t spp;            /* samples per pixel of this call */
    int32_t depth;          /* pathMIS "depth" (src/integrator/PathMISIntegrator.cpp:13) */
    int32_t rr_start;       /* first depth with Russian roulette; 0 = reference behaviour */
    int32_t sample_offset;  /* index of the first sample (progressive accumulation) */
    uint64_t seed;
    int32_t image_index;    /* decorrelates streams of several images of one scene */
    int32_t spp_per_item;   /* 0 = automatic work split */
    int32_t use_camera;     /* 1: render from camera_to_world instead of the scene camera */
    float camera_to_world[16];
    int32_t width, height;  /* image size; 0 = the scene camera's (wavefront and serving only:
                               hk_render rejects any other size) */
} hk_render_desc;

/* Accumulate spp samples per pixel into film_dev ((H+2B)*(W+2B)*4 floats of
 * RGB*w and w, B = ceil(radius - 0.5)); counters_dev (optional, 5 x u64) gets
 * closest-hit rays, shadow rays, dropped (invalid) samples, BVH node visits
 * and triangle tests added. */
int hk_render(hk_scene *s, const hk_render_desc *desc, float *film_dev, unsigned long long *counters_dev,
              void *stream);
/* film -> H*W*3 RGB (ImageBlock::ToBitmap, src/core/Block.cpp:61) */
int hk_film_resolve(hk_scene *s, const float *film_dev, float *rgb_dev, void *stream);
/* End-to-end call, the whole-image render a pathMISCuda plugin's RenderImage
 * makes in place of Render's block loop (src/Main.cpp:46-147): render into
 * the scene's own film, resolve and copy the H*W*3 float image to host memory
 * rgb_host.  counters (host, 5) optional: as hk_render's (node visits and
 * triangle tests summed over closest-hit and shadow rays).  The image is
 * rendered with the wavefront integrator (hk_render_batch, one job) when the
 * scene's image form says so -- by default once it has at least 256 x 256
 * pixels and 2^22 paths -- else with the megakernel (hk_render).  Both run the
 * same estimator on the same per-sample streams: the images agree up to the
 * order of the film's float additions. */
int hk_render_image(hk_scene *s, const hk_render_desc *desc, float *rgb_host, unsigned long long *counters,
                    void *stream);
enum { HK_FORM_AUTO = 0, HK_FORM_MEGAKERNEL = 1, HK_FORM_WAVEFRONT = 2 };
/* The form hk_render_image renders with (HK_FORM_AUTO by default). */
int hk_scene_set_image_form(hk_scene *s, int32_t form);

/* ---- wavefront rendering (the batched form) ---- */
/* One image of a batch: accumulate desc.spp samples into film_dev (film layout
 * of hk_render).  desc.use_camera selects a per-image camera pose. */
typedef struct {
    float *film_dev;
    hk_render_desc desc;
} hk_render_job;

typedef struct {
    int32_t capacity;              /* path slots in flight (0 = 2^21) */
    int32_t threads_extend;        /* block size of the extend/shadow kernels (0 = 128) */
    int32_t threads_shade;         /* block size of the shade kernels (0 = 128) */
    int32_t iterations_per_check;  /* iterations between host termination checks (0 = 16) */
    int32_t no_graph;              /* 1: launch kernels directly instead of replaying a CUDA graph */
    float *kernel_ms;              /* optional host float[4]: adds the device time of the regen, extend,
                                      shade and shadow phases (timed with events, no graph) */
    int32_t *kernel_launches;      /* optional host int32[4]: adds the kernel launches per phase */
    int32_t fetch_steps;           /* node visits of a ray between refills of the traversal lanes
                                      (0 = 8 for the binary tree, 3 for the 8-wide tree) */
    int32_t fetch_min_idle;        /* idle lanes of a warp before it refills while others still
                                      traverse (0 = 1: refill at once) */
    int32_t fetch_steps_shadow;    /* the same two for the shadow (any-hit) rays; 0 = the closest-hit */
    int32_t fetch_min_idle_shadow; /*   rays' values */
    int32_t reg_lean;              /* bit 0 / bit 1: the extend / shadow kernel with a register budget of
                                      48 (five resident blocks of 256 threads) instead of the compiler's;
                                      bit 2: the shade kernels of untextured materials with 64 (four
                                      resident blocks of 256 threads) */
    int32_t shadow_tests;          /* triangle tests of the shadow rays (8-wide tree): 0 each lane tests
                                      its own; 1 the same, postponed like closest-hit rays' while few
                                      lanes of the warp have triangles; 2 shared out over the warp, 32
                                      at a time */
    int32_t closest_tests;         /* triangle tests of the closest-hit rays (8-wide tree): 0 each lane
                                      tests its own, postponed while few lanes of the warp have
                                      triangles; 2 shared out over the warp, 32 at a time, the least t
                                      of each ray kept (the later test on equal t, as the serial loop) */
    int32_t sample_major;          /* 0: each image's work is dealt tile by tile (all samples of a 16 x 16
                                      tile, then the next); 1: sample by sample over the whole image.
                                      Images agree up to the order of the film's float additions */
} hk_wavefront_config;

/* Render every job of the batch with the wavefront integrator: a pool of path
 * slots shared by all images, compacted ray queues, one shading kernel per
 * material type, and iterations replayed from a CUDA graph.  Same estimator
 * as hk_render (PathMISIntegrator::Li, src/integrator/PathMISIntegrator.cpp:16).
 * Returns when every job is done; counters_dev (optional, 7 x u64) gets rays,
 * shadow rays, dropped samples, node visits and triangle tests of the
 * closest-hit traversal, node visits and triangle tests of the shadow rays
 * added (as hk_render adds its 5). */
int hk_render_batch(hk_scene *s, const hk_render_job *jobs, int njobs, const hk_wavefront_config *cfg,
                    unsigned long long *counters_dev, void *stream);

/* End-to-end batch: render n images with the wavefront into films owned by the
 * scene, resolve them and copy each H*W*3 float image to host memory
 * rgb_host[i].  counters_host (optional, 7 x u64) as hk_render_batch. */
int hk_render_batch_host(hk_scene *s, const hk_render_desc *descs, int n, const hk_wavefront_config *cfg,
                         float *const *rgb_host, unsigned long long *counters_host, void *stream);

/* Autotuner: render `probe` (one image) under candidate configurations --
 * slot capacity 2^20..2^22, block sizes 64/128/256, termination-check
 * interval 16/64, traversal refill interval and idle-lane threshold -- by
 * coordinate descent and return the fastest. */
int hk_wavefront_autotune(hk_scene *s, const hk_render_desc *probe, hk_wavefront_config *best, float *best_ms);
/* The wavefront configuration hk_render_image uses (NULL: the defaults of
 * hk_render_batch).  hk_wavefront_autotune sets it to the configuration it
 * finds, so a plugin that tunes once in Preprocess renders every image with it. */
int hk_scene_set_wavefront_config(hk_scene *s, const hk_wavefront_config *cfg);

/* Render into a caller-provided device image without allocating any device
 * memory.  This entry point has no counterpart in the reference.  It is for
 * callers that cannot call cudaMalloc while rendering -- a host application
 * whose device memory is owned by its own allocator or held to a fixed
 * budget, or a plugin that may not grow the process's footprint after
 * start-up.  The scene must already be built (hk_scene_build allocates the
 * scene itself).  Scratch (work counter, counters, film accumulator) lives in
 * one static device array of about 4.3 MB that every GPU loading the library
 * holds until exit; films are limited to (W+2B)*(H+2B) <= 520*520 pixels
 * (512x512 at a filter border of 4) and larger images are rejected with
 * HK_ERR_INVALID.  The first call on a device looks up the array's device
 * address (cudaGetSymbolAddress) and caches it for the life of the process;
 * make that first call before any stream capture.  The scene's device must be
 * the current device (HK_ERR_INVALID otherwise).  A device reset
 * (cudaDeviceReset, or a reset of the primary context) while the library is
 * loaded is not supported: the cached address would be stale.  All calls share
 * the array and each call clears it: calls that overlap on the GPU (other
 * streams, other threads) race, and the caller must serialise them.
 * rgb_dev: H*W*3 floats; counters_dev (optional): 5 x u64 as hk_render. */
int hk_render_image_static(hk_scene *s, const hk_render_desc *desc, float *rgb_dev, unsigned long long *counters_dev,
                           void *stream);

/* ---- serving: continuous batching of render jobs ---- */
/* No counterpart in the reference (its renderer runs one scene file per
 * process, src/Main.cpp:150).  A server keeps registered scenes resident and
 * renders jobs -- (scene, image size, spp, camera) -- as they arrive: a job
 * is admitted when its film and image fit the device-memory budget (the
 * first job of a scene also charges the scene's path-slot pool), its paths
 * join the scene's wavefront pool between iterations, and its image is
 * copied to the caller's host buffer when its last path is done.  Jobs of
 * one scene share one pool; scenes run on separate streams.  A job's image
 * is the same whether it runs alone or among others: each path's random
 * stream depends only on (seed, sample, pixel, image_index), so results
 * differ only in the order of the film's float additions.  One host thread
 * per server drives the device; the functions below are thread-safe. */
typedef struct hk_server hk_server;

#define HK_ERR_TIMEOUT (-5)   /* hk_job_wait: the job did not finish in time */

#define HK_SERVE_SRPT 0   /* dispatch the job with the least undispensed work first */
#define HK_SERVE_FIFO 1   /* dispatch jobs in arrival order */
/* SRPT within and across scenes: a scene's engine runs only while its job
 * with the least remaining work (undispensed plus in flight) has at most
 * HK_SERVE_GATE times the remaining work of the least job of any scene, so a
 * small job is not slowed by large jobs of other scenes sharing the GPU. */
#define HK_SERVE_SRPT_ACROSS 2
#define HK_SERVE_GATE 4
/* SRPT within a scene; across scenes the gate of HK_SERVE_SRPT_ACROSS holds
 * only while the least job of any scene has at most `small_work` paths left
 * (hk_server_config; default HK_SERVE_SMALL_WORK): a small job gets the GPU
 * nearly to itself for the few milliseconds it needs, while large jobs of
 * different scenes keep overlapping. */
#define HK_SERVE_SRPT_SMALL 3
#define HK_SERVE_SMALL_WORK (1ull << 22)

#define HK_JOB_QUEUED 0
#define HK_JOB_RUNNING 1
#define HK_JOB_DONE 2
#define HK_JOB_CANCELLED 3
#define HK_JOB_FAILED 4      /* the server hit a device error; hk_job_wait returns it */

typedef struct {
    int32_t capacity;             /* path slots of each scene's pool (0 = 2^19) */
    int32_t threads_extend;       /* 0 = 128 */
    int32_t threads_shade;        /* 0 = 128 */
    int32_t iterations_per_poll;  /* wavefront iterations between host polls (0 = 4) */
    int32_t policy;               /* HK_SERVE_SRPT, HK_SERVE_FIFO or HK_SERVE_SRPT_ACROSS */
    int32_t max_jobs;             /* jobs admitted at once per scene (0 = 256, max 1024) */
    uint64_t hbm_budget;          /* device bytes for pools, films and images (0 = 90% of free at create) */
    uint64_t small_work;          /* HK_SERVE_SRPT_SMALL: paths left below which a job gates the other
                                     scenes (0 = HK_SERVE_SMALL_WORK) */
} hk_server_config;

typedef struct {
    int32_t state;                /* HK_JOB_* */
    int32_t scene;
    uint32_t width, height;
    uint64_t paths;               /* width * height * spp */
    uint64_t device_bytes;        /* film + image charged while admitted */
    double submit_s, admit_s, done_s;   /* server clock (seconds since hk_server_create) */
    double latency_s;             /* done_s - submit_s (0 until done) */
} hk_job_status;

typedef struct {
    uint64_t jobs_submitted, jobs_done, jobs_cancelled, jobs_queued, jobs_running;
    uint64_t paths_done;          /* paths of finished jobs */
    uint64_t rays, shadow_rays;   /* traced by all pools */
    uint64_t bytes_in_use, hbm_budget;
    double busy_s;                /* time with at least one job admitted */
    double now_s;
} hk_server_stats;

int hk_server_create(const hk_server_config *cfg, hk_server **out);
/* Cancels queued jobs, finishes the running ones and frees everything. */
int hk_server_destroy(hk_server *srv);
/* Register a built scene (not owned; keep it alive and unchanged while the server lives).
 * The scene's pool is sized by the server's configuration; its traversal
 * settings (ray-fetch intervals, register budgets, triangle-test modes) come
 * from the scene's wavefront configuration (hk_wavefront_autotune or
 * hk_scene_set_wavefront_config) when the scene has one at its first job. */
int hk_server_add_scene(hk_server *srv, hk_scene *scene, int32_t *scene_id);
/* Queue a job.  rgb_host receives height*width*3 floats (pinned memory is
 * copied into directly, other memory through a pinned staging buffer); it
 * must stay valid until the job is done or cancelled. */
int hk_job_submit(hk_server *srv, int32_t scene_id, const hk_render_desc *desc, float *rgb_host, uint64_t *job_id);
int hk_job_poll(hk_server *srv, uint64_t job_id, hk_job_status *status);
/* Block until the job is done or cancelled, or timeout_s passes (HK_ERR_TIMEOUT). */
int hk_job_wait(hk_server *srv, uint64_t job_id, double timeout_s, hk_job_status *status);
/* A queued job is dropped; a running job stops dispatching and ends when its
 * paths in flight are done (its image is not written). */
int hk_job_cancel(hk_server *srv, uint64_t job_id);
/* Progressive preview (the headless replacement of the reference's preview
 * window): the job's film accumulated so far, resolved into rgb_host
 * (width*height*3 floats, row-major), and the fraction of its paths finished.
 * A queued, cancelled or failed job gives zeros, a finished job its final image.
 * Waits at most timeout_s (< 0: no limit) for the server to reach a point
 * between iterations. */
int hk_job_preview(hk_server *srv, uint64_t job_id, float *rgb_host, double timeout_s, double *fraction);
int hk_server_get_stats(hk_server *srv, hk_server_stats *stats);

/* Host-only check of the tree builder (no counterpart in the reference; used
 * by the tests): builds both trees over ntris triangles (9 floats each) and
 * verifies that every triangle sits in exactly one leaf of each tree and that
 * every quantised 8-wide child box contains its triangles.  Returns HK_OK and
 * the tree sizes, or HK_ERR_INVALID with the first problem in hk_last_error(). */
int hk_bvh_check(const float *tris, uint32_t ntris, uint32_t *n_bvh_nodes, uint32_t *n_wide_nodes,
                 uint32_t *wide_depth);

/* ---- record-level entry points (parity tests and the BSDF batch) ---- */
/* Ray queries against the scene accel (Acceleration::RayIntersect,
 * include/core/Acceleration.hpp:57).  rays_dev: n x 8 floats (o, d, mint,
 * maxt).  tri_dev: original triangle index or -1 (any_hit: 1/0).
 * node_visits_dev (optional, 2 x u64): node visits and triangle tests added. */
int hk_trace(hk_scene *s, uint64_t n, const float *rays_dev, int32_t *tri_dev, float *t_dev, float *u_dev, float *v_dev,
             int any_hit, unsigned long long *node_visits_dev, void *stream);
/* BSDF::Sample/Eval/Pdf (include/core/BSDF.hpp:67,78,94) over n records in
 * the local frame: inputs wi (n x 3), u2 (n x 2), u1 (n, roughDielectric's
 * Next1D draw, may be NULL), wo (n x 3), uv (n x 2 texture coordinates of the
 * records' intersection, for textured parameters; NULL = (0, 0)); outputs (any
 * may be NULL): sampled wo, weight, pdf of the sample, measure; Eval and Pdf at
 * wo (ESolidAngle). */
int hk_bsdf_batch(hk_scene *s, int32_t bsdf, uint64_t n, const float *wi_dev, const float *u2_dev, const float *u1_dev,
                  const float *wo_dev, const float *uv_dev, const float *duv_dev, float *s_wo_dev, float *s_w_dev,
                  float *s_pdf_dev, int32_t *s_measure_dev, float *e_rgb_dev, float *p_pdf_dev, void *stream);
/* (duv: n x 4 screen-space partials of the texture coordinates, (dUdX, dVdX,
 * dUdY, dVdY) per record, or NULL = 0; used by filtered bitmap lookups) */
/* Texture2D::Eval(Isect, filter = true) (src/core/Texture.cpp:211) of texture
 * `tex` at n texture coordinates uv (n x 2) with partials duv (n x 4 or NULL):
 * out n x 3. */
int hk_texture_eval(hk_scene *s, int32_t tex, uint64_t n, const float *uv_dev, const float *duv_dev, float *out_dev,
                    void *stream);
/* Emitter::Sample (include/core/Emitter.hpp:77) for emitter e: in n x 8
 * (ref xyz, u2, u1, -, -), out n x 16 (p, n, wi, pdf, distance, value, -). */
int hk_emitter_sample(hk_scene *s, int32_t e, uint64_t n, const float *in_dev, float *out_dev, void *stream);
/* Camera::SampleRay (include/core/Camera.hpp:38): pos n x 2 -> rays n x 8 */
int hk_camera_rays(hk_scene *s, uint64_t n, const float *pos_dev, float *rays_dev, void *stream);
/* EnvironmentLight::Eval/Pdf for world directions: n x 3 -> n x 3, n */
int hk_env_eval(hk_scene *s, uint64_t n, const float *wi_dev, float *rgb_dev, float *pdf_dev, void *stream);

#ifdef __cplusplus
}
#endif
#endif
