// Launch interface between the host library (hk_host.cpp) and the kernels.
#pragma once
#include <cuda_runtime.h>

#include "hk_device.h"

namespace hk {

constexpr int kTile = 16;                  // render tile: 16 x 16 pixels
constexpr int kTileThreads = kTile * kTile;

struct RenderLaunch {
    float *film;                          // (H+2B) x (W+2B) x 4 floats, accumulated
    unsigned int *work_counter;           // zeroed before launch
    unsigned long long *counters;         // [rays, shadow rays, dropped samples, node visits, triangle tests]
    uint64_t seed;
    int spp;                              // samples per pixel in this launch
    int sample_offset;                    // first sample index (progressive rendering)
    int spp_per_item;                     // samples per thread per work item
    int n_chunks;                         // work items per tile
    int tiles_x, tiles_y, n_items;
    int depth, rr_start;
    int image_index;
    int margin_lo, margin_hi;             // film footprint offsets of a tile pixel
};

// Static scratch of hk_render_image_static: a 256-byte header ([0] work
// counter, [1..5] ray/sample counters) followed by the film accumulator, sized
// for films of up to 512 x 512 pixels with a filter border of up to 4.
constexpr size_t kStaticHeaderWords = 32;
constexpr size_t kStaticFilmFloats = 4ull * 520 * 520;
constexpr size_t kStaticScratchWords = kStaticHeaderWords + kStaticFilmFloats / 2;
constexpr int kStaticMaxDevices = 64;
// Device address of the static scratch on the current device (looked up once
// per device with cudaGetSymbolAddress, then cached).
cudaError_t static_render_scratch(void **out);

cudaError_t launch_render(const DevScene &S, const RenderLaunch &P, int grid, cudaStream_t st);
cudaError_t launch_resolve(const float *film, float *rgb, int W, int H, int B, cudaStream_t st);
cudaError_t launch_trace(const DevScene &S, uint64_t n, const float *rays, int32_t *tri, float *t, float *u, float *v,
                         int any_hit, unsigned long long *visits, cudaStream_t st);
// type: top-level BSDF type of id `bsdf` (HK_BSDF_*)
cudaError_t launch_bsdf_batch(const DevScene &S, int bsdf, int type, uint64_t n, const float *wi, const float *u2,
                              const float *u1, const float *wo, const float *uv, const float *duv, float *s_wo, float *s_w,
                              float *s_pdf, int32_t *s_m, float *e_rgb, float *p_pdf, cudaStream_t st);
cudaError_t launch_texture_eval(const DevScene &S, const DevTexture *T, int tex, uint64_t n, const float *uv,
                                const float *duv, float *out, cudaStream_t st);
cudaError_t launch_emitter_sample(const DevScene &S, int e, uint64_t n, const float *in, float *out, cudaStream_t st);
cudaError_t launch_camera_rays(const DevScene &S, uint64_t n, const float *pos, float *out, cudaStream_t st);
cudaError_t launch_env_eval(const DevScene &S, uint64_t n, const float *wi, float *out, float *pdf, cudaStream_t st);
int render_occupancy(int margin_lo, int margin_hi, int accel, bool textured);

// Per-instantiation launchers behind the functions above, each compiled in its
// own translation unit (megakernel: hk_render_*.cu; BSDF batch: hk_batch_*.cu).
template <int kAccel, bool kTex>
cudaError_t launch_render_t(const DevScene &S, const RenderLaunch &P, int grid, cudaStream_t st);
template <int kAccel, bool kTex>
int render_occupancy_t(int margin_lo, int margin_hi);
template <int BT>
cudaError_t launch_bsdf_batch_t(const DevScene &S, int bsdf, uint64_t n, const float *wi, const float *u2, const float *u1,
                                const float *wo, const float *uv, const float *duv, float *s_wo, float *s_w, float *s_pdf,
                                int32_t *s_m, float *e_rgb, float *p_pdf, int grid, cudaStream_t st);

}  // namespace hk
