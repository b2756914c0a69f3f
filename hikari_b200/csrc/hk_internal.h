// What the serving loop needs from a built scene (defined in hk_host.cpp).
#pragma once
#include <cstddef>
#include <cstdint>

#include "../../include/hikari_b200.h"
#include "hk_device.h"
#include "hk_wavefront.h"

namespace hk {

struct SceneView {
    const DevScene *dev;   // device description; valid while the scene lives and is not rebuilt
    int sm_count;
    uint32_t width, height;   // scene camera's image size
    // the scene's wavefront configuration (autotuner or caller) when *has_cfg;
    // both point into the scene and stay valid while it lives
    const hk_wavefront_config *cfg;
    const bool *has_cfg;
};
// Throws HkError when the scene is null or not built.
SceneView scene_view(hk_scene *s);

// Image size of a render request and the device bytes of its film and RGB image.
struct JobSize {
    uint32_t width, height;
    size_t film_bytes, rgb_bytes;
};
JobSize job_size(const hk_scene *s, const hk_render_desc &d);

// Job-table entry of a request (film and finished counter left for the caller).
WfJob make_wf_job(const hk_scene *s, const hk_render_desc &d);

}  // namespace hk
