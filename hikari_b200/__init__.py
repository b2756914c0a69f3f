"""hikari_b200: a B200-native core for Hikari's pathMIS path-tracing hot path.

The product is the sm_100a CUDA library ``_build/libhikari_b200.so`` behind
the C ABI of ``include/hikari_b200.h``.  This module binds that ABI with
ctypes; torch is used only to hold device buffers and streams.  There is no
CPU fallback: every entry point raises if the CUDA library is missing.
"""
from __future__ import annotations

import ctypes as C
import os
from typing import Optional

import numpy as np

from . import scenedesc
from .scenedesc import TEX_BITMAP, TEX_SLOTS, BSDFDesc, SceneDesc

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "libhikari_b200.so")
DATA_DIR = os.path.join(HERE, "data")

HK_OK = 0
ACCEL_BVH2, ACCEL_BVH8 = 0, 1
# where Scene.from_desc builds the trees (HK_BUILDER_*)
BUILDER_HOST, BUILDER_GPU = 0, 1
# forms of Scene.render_image (HK_FORM_*)
FORM_AUTO, FORM_MEGAKERNEL, FORM_WAVEFRONT = 0, 1, 2


class HikariError(RuntimeError):
    """A non-zero status from the C ABI (the reference raises HikariException)."""


class BsdfDesc(C.Structure):
    _fields_ = [
        ("type", C.c_int32), ("distribution", C.c_int32), ("anisotropic", C.c_int32), ("nonlinear", C.c_int32),
        ("alpha_u", C.c_float), ("alpha_v", C.c_float), ("int_ior", C.c_float), ("ext_ior", C.c_float),
        ("eta", C.c_float * 3), ("k", C.c_float * 3), ("ks", C.c_float * 3), ("ks_refract", C.c_float * 3),
        ("kd", C.c_float * 3), ("sigma_a", C.c_float * 3), ("thickness", C.c_float), ("nested", C.c_int32),
        ("nested2", C.c_int32), ("fast_approx", C.c_int32), ("tex", C.c_int32 * 6),
    ]


class TextureDesc(C.Structure):
    _fields_ = [
        ("kind", C.c_int32), ("nested", C.c_int32), ("count", C.c_int32), ("width", C.c_float),
        ("scale", C.c_float), ("uv_scale", C.c_float * 2), ("uv_offset", C.c_float * 2), ("a", C.c_float * 3),
        ("b", C.c_float * 3), ("filter", C.c_int32), ("wrap_u", C.c_int32), ("wrap_v", C.c_int32),
        ("channels", C.c_int32), ("gamma", C.c_float), ("max_anisotropy", C.c_float),
    ]


class SceneInfo(C.Structure):
    _fields_ = [
        ("n_meshes", C.c_uint32), ("n_triangles", C.c_uint32), ("n_bsdfs", C.c_uint32), ("n_emitters", C.c_uint32),
        ("n_bvh_nodes", C.c_uint32), ("bvh_depth", C.c_uint32), ("env_index", C.c_int32), ("film_border", C.c_int32),
        ("bbox", C.c_float * 6), ("device_bytes", C.c_uint64), ("n_wide_nodes", C.c_uint32),
        ("wide_depth", C.c_uint32), ("accel", C.c_int32), ("postpone", C.c_int32),
    ]


class RenderDesc(C.Structure):
    _fields_ = [
        ("spp", C.c_int32), ("depth", C.c_int32), ("rr_start", C.c_int32), ("sample_offset", C.c_int32),
        ("seed", C.c_uint64), ("image_index", C.c_int32), ("spp_per_item", C.c_int32),
        ("use_camera", C.c_int32), ("camera_to_world", C.c_float * 16), ("width", C.c_int32), ("height", C.c_int32),
    ]


class RenderJob(C.Structure):
    _fields_ = [("film_dev", C.c_void_p), ("desc", RenderDesc)]


class WavefrontConfig(C.Structure):
    _fields_ = [("capacity", C.c_int32), ("threads_extend", C.c_int32), ("threads_shade", C.c_int32),
                ("iterations_per_check", C.c_int32), ("no_graph", C.c_int32), ("kernel_ms", C.c_void_p),
                ("kernel_launches", C.c_void_p), ("fetch_steps", C.c_int32), ("fetch_min_idle", C.c_int32),
                ("fetch_steps_shadow", C.c_int32), ("fetch_min_idle_shadow", C.c_int32), ("reg_lean", C.c_int32),
                ("shadow_tests", C.c_int32), ("closest_tests", C.c_int32), ("sample_major", C.c_int32)]


class ServerConfig(C.Structure):
    _fields_ = [("capacity", C.c_int32), ("threads_extend", C.c_int32), ("threads_shade", C.c_int32),
                ("iterations_per_poll", C.c_int32), ("policy", C.c_int32), ("max_jobs", C.c_int32),
                ("hbm_budget", C.c_uint64), ("small_work", C.c_uint64)]


class JobStatus(C.Structure):
    _fields_ = [("state", C.c_int32), ("scene", C.c_int32), ("width", C.c_uint32), ("height", C.c_uint32),
                ("paths", C.c_uint64), ("device_bytes", C.c_uint64), ("submit_s", C.c_double),
                ("admit_s", C.c_double), ("done_s", C.c_double), ("latency_s", C.c_double)]


class ServerStats(C.Structure):
    _fields_ = [("jobs_submitted", C.c_uint64), ("jobs_done", C.c_uint64), ("jobs_cancelled", C.c_uint64),
                ("jobs_queued", C.c_uint64), ("jobs_running", C.c_uint64), ("paths_done", C.c_uint64),
                ("rays", C.c_uint64), ("shadow_rays", C.c_uint64), ("bytes_in_use", C.c_uint64),
                ("hbm_budget", C.c_uint64), ("busy_s", C.c_double), ("now_s", C.c_double)]


def render_desc(spp, depth, seed=0, sample_offset=0, rr_start=0, image_index=0, spp_per_item=0,
                camera=None, width=0, height=0) -> RenderDesc:
    d = RenderDesc(spp, depth, rr_start, sample_offset, seed, image_index, spp_per_item, 0)
    d.width, d.height = int(width), int(height)
    if camera is not None:
        d.use_camera = 1
        d.camera_to_world[:] = [float(x) for x in np.asarray(camera, np.float32).reshape(16)]
    return d


_lib = None


def lib():
    """Load the CUDA library (raises HikariError when it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise HikariError(f"CUDA library not built: {LIB_PATH} (run hikari_b200.build.build())")
    L = C.CDLL(LIB_PATH)
    P, U64, I32, F = C.c_void_p, C.c_uint64, C.c_int32, C.c_float
    sig = {
        "hk_last_error": ([], C.c_char_p),
        "hk_version": ([], C.c_int),
        "hk_scene_create": ([C.POINTER(P)], C.c_int),
        "hk_scene_destroy": ([P], C.c_int),
        "hk_scene_set_rft": ([P, C.c_int, C.c_char_p, U64], C.c_int),
        "hk_scene_add_bsdf": ([P, C.POINTER(BsdfDesc), C.POINTER(I32)], C.c_int),
        "hk_scene_add_mesh": ([P, P, C.c_uint32, P, C.c_uint32, P, I32, P, C.POINTER(I32)], C.c_int),
        "hk_scene_set_envmap": ([P, P, C.c_uint32, C.c_uint32, P, F], C.c_int),
        "hk_scene_set_constant_light": ([P, P], C.c_int),
        "hk_scene_add_texture": ([P, C.POINTER(TextureDesc), C.POINTER(I32)], C.c_int),
        "hk_scene_add_bitmap": ([P, C.POINTER(TextureDesc), P, I32, I32, C.POINTER(I32)], C.c_int),
        "hk_image_load": ([C.c_char_p, I32, C.POINTER(I32), C.POINTER(I32), C.POINTER(C.POINTER(C.c_uint8))],
                          C.c_int),
        "hk_image_free": ([C.POINTER(C.c_uint8)], None),
        "hk_texture_eval": ([P, I32, U64, P, P, P, P], C.c_int),
        "hk_scene_set_mesh_uv": ([P, I32, P], C.c_int),
        "hk_obj_load": ([C.c_char_p, P, C.POINTER(C.c_uint32), C.POINTER(C.c_uint32), P, P, P, P, C.POINTER(I32)],
                        C.c_int),
        "hk_scene_add_point_light": ([P, P, P], C.c_int),
        "hk_scene_add_directional_light": ([P, P, P], C.c_int),
        "hk_scene_set_camera": ([P, C.c_uint32, C.c_uint32, P, F, F, F], C.c_int),
        "hk_scene_set_filter": ([P, C.c_int, F, F, F], C.c_int),
        "hk_scene_set_background": ([P, P, C.c_int], C.c_int),
        "hk_scene_build": ([P], C.c_int),
        "hk_scene_set_accel": ([P, I32], C.c_int),
        "hk_scene_set_image_form": ([P, I32], C.c_int),
        "hk_scene_set_wavefront_config": ([P, C.POINTER(WavefrontConfig)], C.c_int),
        "hk_scene_set_builder": ([P, I32], C.c_int),
        "hk_scene_tree_build_seconds": ([P, C.POINTER(C.c_double)], C.c_int),
        "hk_wavefront_launch_log": ([P, I32, P, I32, C.POINTER(I32)], C.c_int),
        "hk_bvh_check_gpu": ([P, C.c_uint32, C.POINTER(C.c_uint32), C.POINTER(C.c_uint32)], C.c_int),
        "hk_bvh_check": ([P, C.c_uint32, C.POINTER(C.c_uint32), C.POINTER(C.c_uint32), C.POINTER(C.c_uint32)],
                         C.c_int),
        "hk_scene_get_info": ([P, C.POINTER(SceneInfo)], C.c_int),
        "hk_scene_load_xml": ([C.c_char_p, C.c_char_p, C.POINTER(P), C.POINTER(I32), C.POINTER(I32)], C.c_int),
        "hk_scene_parse_xml": ([C.c_char_p, C.c_char_p, C.POINTER(P), C.POINTER(I32), C.POINTER(I32)], C.c_int),
        "hk_exr_read": ([C.c_char_p, C.POINTER(I32), C.POINTER(I32), P, U64], C.c_int),
        "hk_exr_write": ([C.c_char_p, I32, I32, P], C.c_int),
        "hk_render": ([P, C.POINTER(RenderDesc), P, P, P], C.c_int),
        "hk_film_resolve": ([P, P, P, P], C.c_int),
        "hk_render_image": ([P, C.POINTER(RenderDesc), P, P, P], C.c_int),
        "hk_render_image_static": ([P, C.POINTER(RenderDesc), P, P, P], C.c_int),
        "hk_render_batch": ([P, C.POINTER(RenderJob), C.c_int, C.POINTER(WavefrontConfig), P, P], C.c_int),
        "hk_render_batch_host": ([P, C.POINTER(RenderDesc), C.c_int, C.POINTER(WavefrontConfig),
                                  C.POINTER(C.c_void_p), P, P], C.c_int),
        "hk_wavefront_autotune": ([P, C.POINTER(RenderDesc), C.POINTER(WavefrontConfig), C.POINTER(C.c_float)],
                                  C.c_int),
        "hk_server_create": ([C.POINTER(ServerConfig), C.POINTER(P)], C.c_int),
        "hk_server_destroy": ([P], C.c_int),
        "hk_server_add_scene": ([P, P, C.POINTER(I32)], C.c_int),
        "hk_job_submit": ([P, I32, C.POINTER(RenderDesc), P, C.POINTER(U64)], C.c_int),
        "hk_job_poll": ([P, U64, C.POINTER(JobStatus)], C.c_int),
        "hk_job_wait": ([P, U64, C.c_double, C.POINTER(JobStatus)], C.c_int),
        "hk_job_cancel": ([P, U64], C.c_int),
        "hk_job_preview": ([P, U64, P, C.c_double, C.POINTER(C.c_double)], C.c_int),
        "hk_server_get_stats": ([P, C.POINTER(ServerStats)], C.c_int),
        "hk_trace": ([P, U64, P, P, P, P, P, C.c_int, P, P], C.c_int),
        "hk_bsdf_batch": ([P, I32, U64, P, P, P, P, P, P, P, P, P, P, P, P, P], C.c_int),
        "hk_emitter_sample": ([P, I32, U64, P, P, P], C.c_int),
        "hk_camera_rays": ([P, U64, P, P, P], C.c_int),
        "hk_env_eval": ([P, U64, P, P, P, P], C.c_int),
    }
    for name, (args, res) in sig.items():
        if not hasattr(L, name):
            raise HikariError(f"{LIB_PATH} does not export {name}; rebuild the library")
        fn = getattr(L, name)
        fn.argtypes = args
        fn.restype = res
    _lib = L
    return L


def check(rc: int) -> None:
    if rc != HK_OK:
        raise HikariError(f"hikari_b200 error {rc}: {lib().hk_last_error().decode()}")


def _p(a) -> Optional[int]:
    """Raw pointer of a numpy array or a torch tensor (None passes NULL)."""
    if a is None:
        return None
    if isinstance(a, np.ndarray):
        return a.ctypes.data
    return a.data_ptr()


def _f32(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.float32)


def _stream(stream) -> Optional[int]:
    if stream is None:
        import torch

        return torch.cuda.current_stream().cuda_stream
    return getattr(stream, "cuda_stream", stream)


def texture_desc_c(t, nested_id: int = -1) -> TextureDesc:
    c = TextureDesc()
    c.kind, c.nested, c.count, c.width, c.scale = t.kind, nested_id, t.count, t.width, t.scale
    c.uv_scale[:], c.uv_offset[:], c.a[:], c.b[:] = t.uv_scale, t.uv_offset, t.a, t.b
    c.filter, c.wrap_u, c.wrap_v = t.filter, t.wrap_u, t.wrap_v
    c.channels, c.gamma, c.max_anisotropy = t.channels, t.gamma, t.max_anisotropy
    return c


def image_load(path: str, channels: int = 3) -> np.ndarray:
    """Decode an 8-bit image file (PNG, PGM / PPM, baseline JPEG) like
    stbi_load with `channels` (1 or 3): height x width x channels uint8, row 0
    = the top row."""
    L = lib()
    w, h = C.c_int32(), C.c_int32()
    buf = C.POINTER(C.c_uint8)()
    check(L.hk_image_load(os.fsencode(path), channels, C.byref(w), C.byref(h), C.byref(buf)))
    try:
        a = np.ctypeslib.as_array(buf, shape=(h.value, w.value, channels)).copy()
    finally:
        L.hk_image_free(buf)
    return a


def bsdf_desc_c(d: BSDFDesc, nested_id: int = -1, nested2_id: int = -1, tex_ids=None) -> BsdfDesc:
    c = BsdfDesc()
    c.type, c.distribution = d.type, d.distribution
    c.anisotropic, c.nonlinear = int(d.anisotropic), int(d.nonlinear)
    c.alpha_u, c.alpha_v, c.int_ior, c.ext_ior = d.alpha_u, d.alpha_v, d.int_ior, d.ext_ior
    c.eta[:] = d.conductor_eta()
    c.k[:], c.ks[:], c.ks_refract[:], c.kd[:], c.sigma_a[:] = d.k, d.ks, d.ks_refract, d.kd, d.sigma_a
    c.thickness, c.nested, c.nested2 = d.thickness, nested_id, nested2_id
    c.fast_approx = int(getattr(d, "fast_approx", False))
    for k, t in enumerate(tex_ids or [-1] * 6):
        c.tex[k] = t + 1
    return c


def read_rft(distribution: int) -> bytes:
    name = "GGXRFTData.bin" if distribution == scenedesc.GGX else "BeckmannRFTData.bin"
    with open(os.path.join(DATA_DIR, name), "rb") as f:
        return f.read()


class Scene:
    """A device-resident scene (hk_scene handle)."""

    def __init__(self, handle, desc: Optional[SceneDesc] = None, bsdf_ids=None):
        self.h = handle
        self.desc = desc
        self.bsdf_ids = bsdf_ids or {}
        info = SceneInfo()
        check(lib().hk_scene_get_info(self.h, C.byref(info)))
        self.info = info
        self._film = None

    # ------------------------------------------------------------ construction
    @classmethod
    def from_desc(cls, desc: SceneDesc, builder: int = BUILDER_HOST) -> "Scene":
        L = lib()
        h = C.c_void_p()
        check(L.hk_scene_create(C.byref(h)))
        try:
            for dist in (0, 1):
                b = read_rft(dist)
                check(L.hk_scene_set_rft(h, dist, b, len(b)))
            ids = {}

            tids = {}

            def add_texture(t) -> int:
                if id(t) in tids:
                    return tids[id(t)]
                nested = add_texture(t.nested) if t.nested is not None else -1
                c = texture_desc_c(t, nested)
                out = C.c_int32()
                if t.kind == TEX_BITMAP:
                    px = np.ascontiguousarray(t.pixels, dtype=np.uint8)
                    check(L.hk_scene_add_bitmap(h, C.byref(c), _p(px), px.shape[1], px.shape[0], C.byref(out)))
                else:
                    check(L.hk_scene_add_texture(h, C.byref(c), C.byref(out)))
                tids[id(t)] = out.value
                return out.value

            def add_bsdf(d: BSDFDesc) -> int:
                if id(d) in ids:
                    return ids[id(d)]
                nested = add_bsdf(d.nested) if d.nested is not None else -1
                nested2 = add_bsdf(d.nested2) if d.nested2 is not None else -1
                tex = d.textures or {}
                c = bsdf_desc_c(d, nested, nested2, [add_texture(tex[k]) if k in tex else -1 for k in TEX_SLOTS])
                out = C.c_int32()
                check(L.hk_scene_add_bsdf(h, C.byref(c), C.byref(out)))
                ids[id(d)] = out.value
                return out.value

            mesh_bsdf = [add_bsdf(m.bsdf) for m in desc.meshes]
            for kind, i in desc.build_steps():   # emitters in Scene::AddChild order
                if kind == "env" and desc.env_constant is not None:
                    rad = _f32(desc.env_constant)
                    check(L.hk_scene_set_constant_light(h, _p(rad)))
                elif kind == "env":
                    e = desc.env
                    rgb, tw = _f32(e.rgb), _f32(e.to_world)
                    check(L.hk_scene_set_envmap(h, rgb.ctypes.data, rgb.shape[1], rgb.shape[0], tw.ctypes.data,
                                                e.scale))
                elif kind == "light":
                    l = desc.lights[i]
                    add = L.hk_scene_add_point_light if l.kind == "point" else L.hk_scene_add_directional_light
                    col, vec = _f32(l.color), _f32(l.vector)
                    check(add(h, _p(col), _p(vec)))
                else:
                    m = desc.meshes[i]
                    pos = _f32(m.positions)
                    idx = np.ascontiguousarray(m.indices, dtype=np.uint32)
                    nrm = _f32(m.normals) if m.normals is not None else None
                    rad = _f32(m.radiance) if m.radiance is not None else None
                    mid = C.c_int32()
                    check(L.hk_scene_add_mesh(h, _p(pos), pos.shape[0], _p(idx), idx.shape[0], _p(nrm), mesh_bsdf[i],
                                              _p(rad), C.byref(mid)))
                    if getattr(m, "uv", None) is not None:
                        uv = _f32(m.uv)
                        check(L.hk_scene_set_mesh_uv(h, mid.value, _p(uv)))
            cam = desc.camera
            tw = _f32(cam.to_world)
            check(L.hk_scene_set_camera(h, cam.width, cam.height, tw.ctypes.data, cam.fov, cam.near_clip, cam.far_clip))
            f = desc.filter
            check(L.hk_scene_set_filter(h, f.kind, f.radius, f.p0, f.p1))
            bg = _f32(desc.background)
            check(L.hk_scene_set_background(h, bg.ctypes.data, int(desc.force_background)))
            check(L.hk_scene_set_builder(h, builder))
            check(L.hk_scene_build(h))
        except Exception:
            L.hk_scene_destroy(h)
            raise
        sc = cls(h, desc, ids)
        sc.tex_ids = tids
        return sc

    @classmethod
    def from_xml(cls, path: str) -> "Scene":
        """Load through the C++ plugin layer (LoadFromXML mirror)."""
        L = lib()
        h = C.c_void_p()
        depth, spp = C.c_int32(), C.c_int32()
        check(L.hk_scene_load_xml(path.encode(), DATA_DIR.encode(), C.byref(h), C.byref(depth), C.byref(spp)))
        s = cls(h)
        s.xml_depth, s.xml_spp = depth.value, spp.value
        return s

    def close(self):
        if self.h:
            lib().hk_scene_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # ------------------------------------------------------------ rendering
    @property
    def width(self):
        return self.desc.camera.width if self.desc else None

    def set_image_form(self, form: int) -> None:
        """The form render_image renders with: FORM_AUTO (the wavefront for
        images of at least 256 x 256 pixels and 2^22 paths), FORM_MEGAKERNEL
        or FORM_WAVEFRONT."""
        check(lib().hk_scene_set_image_form(self.h, form))

    def set_wavefront_config(self, cfg: Optional[dict]) -> None:
        """The wavefront configuration of render_image's wavefront calls (a dict
        as autotune returns; None: the defaults).  autotune sets it too."""
        if cfg is None:
            check(lib().hk_scene_set_wavefront_config(self.h, None))
            return
        c = WavefrontConfig(cfg.get("capacity", 0), cfg.get("threads_extend", 0), cfg.get("threads_shade", 0),
                            cfg.get("iterations_per_check", 0), 0, None, None, cfg.get("fetch_steps", 0),
                            cfg.get("fetch_min_idle", 0), cfg.get("fetch_steps_shadow", 0),
                            cfg.get("fetch_min_idle_shadow", 0), cfg.get("reg_lean", 0),
                            cfg.get("shadow_tests", 0), cfg.get("closest_tests", 0), cfg.get("sample_major", 0))
        check(lib().hk_scene_set_wavefront_config(self.h, C.byref(c)))

    def tree_build_seconds(self) -> float:
        """Seconds the scene's last build spent on its trees."""
        s = C.c_double()
        check(lib().hk_scene_tree_build_seconds(self.h, C.byref(s)))
        return s.value

    def wavefront_launch_log(self, which: int) -> np.ndarray:
        """Rays of each launch of the closest-hit (which 0) or shadow (which 1)
        traversal kernel in the scene's last render_batch, in launch order."""
        buf = np.zeros(1024, np.uint32)
        n = C.c_int32()
        check(lib().hk_wavefront_launch_log(self.h, which, buf.ctypes.data, len(buf), C.byref(n)))
        return buf[:min(n.value, len(buf))].copy()

    def set_accel(self, accel: int) -> None:
        """Traverse the binary tree (ACCEL_BVH2) or the compressed 8-wide tree (ACCEL_BVH8)."""
        check(lib().hk_scene_set_accel(self.h, accel))
        check(lib().hk_scene_get_info(self.h, C.byref(self.info)))

    def film_shape(self, width: int = 0, height: int = 0):
        """Film (RGBW accumulator) shape at the scene camera's size or at width x height."""
        B = self.info.film_border
        cam = self.desc.camera
        w, h = (width or cam.width), (height or cam.height)
        return (h + 2 * B, w + 2 * B, 4)

    def render(self, film, spp: int, depth: int, seed: int = 0, sample_offset: int = 0, rr_start: int = 0,
               image_index: int = 0, counters=None, spp_per_item: int = 0, camera=None, stream=None) -> None:
        """Accumulate into a device film tensor ((H+2B, W+2B, 4) float32).
        counters: optional device int64 tensor of 5 (rays, shadow rays,
        dropped samples, node visits, triangle tests)."""
        d = render_desc(spp, depth, seed, sample_offset, rr_start, image_index, spp_per_item, camera)
        check(lib().hk_render(self.h, C.byref(d), _p(film), _p(counters), _stream(stream)))

    def resolve(self, film, rgb, stream=None) -> None:
        check(lib().hk_film_resolve(self.h, _p(film), _p(rgb), _stream(stream)))

    def render_progressive(self, passes: int, spp_per_pass: int, depth: int, seed: int = 0, exr_path=None,
                           capacity: int = 0):
        """Progressive rendering into one film (the headless replacement of
        the reference's preview window): pass k renders samples
        [k * spp_per_pass, (k + 1) * spp_per_pass) of every pixel, so after n
        passes the film equals an n * spp_per_pass render of the same seed up
        to float addition order.  Yields (pass, H x W x 3 image) after each
        pass; with exr_path the current image is also written there."""
        import torch

        cam = self.desc.camera
        film = torch.zeros(self.film_shape(), dtype=torch.float32, device="cuda")
        rgb = torch.empty((cam.height, cam.width, 3), dtype=torch.float32, device="cuda")
        for k in range(passes):
            self.render_batch([film], spp=spp_per_pass, depth=depth, seeds=[seed], image_indices=[0],
                              sample_offset=k * spp_per_pass, capacity=capacity)
            self.resolve(film, rgb)
            img = rgb.cpu().numpy()
            if exr_path is not None:
                exr_write(exr_path, img)
            yield k, img

    def render_image(self, spp: int, depth: int, seed: int = 0, rr_start: int = 0, out: Optional[np.ndarray] = None,
                     camera=None, image_index: int = 0, stream=None):
        """End-to-end: render, resolve and return the H x W x 3 float32 image on the host."""
        cam = self.desc.camera
        if out is None:
            out = np.empty((cam.height, cam.width, 3), np.float32)
        ctr = np.zeros(5, np.uint64)
        d = render_desc(spp, depth, seed, 0, rr_start, image_index, 0, camera)
        check(lib().hk_render_image(self.h, C.byref(d), out.ctypes.data, ctr.ctypes.data, _stream(stream)))
        return out, ctr

    def render_batch(self, films, spp: int, depth: int, seeds=None, cameras=None, image_indices=None,
                     sample_offset: int = 0, rr_start: int = 0, counters=None, capacity: int = 0,
                     threads_extend: int = 0, threads_shade: int = 0, iterations_per_check: int = 0,
                     no_graph: bool = False, kernel_ms=None, kernel_launches=None, sizes=None,
                     fetch_steps: int = 0, fetch_min_idle: int = 0, fetch_steps_shadow: int = 0,
                     fetch_min_idle_shadow: int = 0, reg_lean: int = 0, shadow_tests: int = 0,
                     closest_tests: int = 0, sample_major: int = 0, stream=None) -> None:
        """Wavefront render of several images at once: films[i] (device
        tensors of film_shape(), or of film_shape(*sizes[i]) with per-image
        sizes (width, height)) accumulate spp samples of view cameras[i].
        counters: device int64 tensor of 7 that the statistics are added to
        (see hk_render_batch).  kernel_ms /
        kernel_launches: host float32[4] / int32[4] arrays that receive the
        per-phase device time and launch counts (profiling; no graph)."""
        n = len(films)
        jobs = (RenderJob * n)()
        for i, f in enumerate(films):
            cam = cameras[i] if cameras is not None else None
            seed = seeds[i] if seeds is not None else i
            idx = image_indices[i] if image_indices is not None else i
            jobs[i].film_dev = _p(f)
            w, h = sizes[i] if sizes is not None else (0, 0)
            jobs[i].desc = render_desc(spp, depth, seed, sample_offset, rr_start, idx, 0, cam, w, h)
        cfg = WavefrontConfig(capacity, threads_extend, threads_shade, iterations_per_check, int(no_graph),
                              _p(kernel_ms), _p(kernel_launches), fetch_steps, fetch_min_idle, fetch_steps_shadow,
                              fetch_min_idle_shadow, reg_lean, shadow_tests, closest_tests, sample_major)
        check(lib().hk_render_batch(self.h, jobs, n, C.byref(cfg), _p(counters), _stream(stream)))

    def render_batch_host(self, outs, spp: int, depth: int, seeds=None, cameras=None, image_indices=None,
                          rr_start: int = 0, capacity: int = 0, threads_extend: int = 0, threads_shade: int = 0,
                          iterations_per_check: int = 0, fetch_steps: int = 0, fetch_min_idle: int = 0,
                          fetch_steps_shadow: int = 0, fetch_min_idle_shadow: int = 0, reg_lean: int = 0,
                          shadow_tests: int = 0, closest_tests: int = 0, sample_major: int = 0, stream=None):
        """End-to-end wavefront batch into host images outs[i] (H x W x 3 float32)."""
        n = len(outs)
        descs = (RenderDesc * n)()
        for i in range(n):
            cam = cameras[i] if cameras is not None else None
            seed = seeds[i] if seeds is not None else i
            idx = image_indices[i] if image_indices is not None else i
            descs[i] = render_desc(spp, depth, seed, 0, rr_start, idx, 0, cam)
        ptrs = (C.c_void_p * n)(*[o.ctypes.data for o in outs])
        ctr = np.zeros(7, np.uint64)
        cfg = WavefrontConfig(capacity, threads_extend, threads_shade, iterations_per_check, 0, None, None,
                              fetch_steps, fetch_min_idle, fetch_steps_shadow, fetch_min_idle_shadow, reg_lean,
                              shadow_tests, closest_tests, sample_major)
        check(lib().hk_render_batch_host(self.h, descs, n, C.byref(cfg), ptrs, ctr.ctypes.data, _stream(stream)))
        return ctr

    def autotune(self, spp: int, depth: int, camera=None):
        """Pick the wavefront configuration (slot capacity, block sizes, check
        interval) that renders one probe image fastest; returns (config dict, ms)."""
        d = render_desc(spp, depth, 1, 0, 0, 0, 0, camera)
        cfg = WavefrontConfig()
        ms = C.c_float()
        check(lib().hk_wavefront_autotune(self.h, C.byref(d), C.byref(cfg), C.byref(ms)))
        return dict(capacity=cfg.capacity, threads_extend=cfg.threads_extend, threads_shade=cfg.threads_shade,
                    iterations_per_check=cfg.iterations_per_check, fetch_steps=cfg.fetch_steps,
                    fetch_min_idle=cfg.fetch_min_idle, fetch_steps_shadow=cfg.fetch_steps_shadow,
                    fetch_min_idle_shadow=cfg.fetch_min_idle_shadow, reg_lean=cfg.reg_lean,
                    shadow_tests=cfg.shadow_tests, closest_tests=cfg.closest_tests,
                    sample_major=cfg.sample_major), ms.value

    def render_image_static(self, out, spp: int, depth: int, seed: int = 0, rr_start: int = 0, counters=None,
                            camera=None, image_index: int = 0, stream=None) -> None:
        """Render into the device tensor `out` (H x W x 3 float32) through the
        entry point that allocates no device memory (static scratch; films up
        to 520 x 520 including the filter border).

        The C side cannot check the buffers it is given, so they are checked
        here: `out` a contiguous float32 CUDA tensor of shape (H, W, 3),
        `counters` (optional) a contiguous 8-byte integer CUDA tensor of at
        least 5 elements, both on the current device."""
        import torch

        cam = self.desc.camera if self.desc is not None else None
        dev = torch.cuda.current_device()

        def on_device(t, what):
            if not isinstance(t, torch.Tensor) or not t.is_cuda:
                raise TypeError(f"{what} must be a CUDA tensor")
            if t.device.index != dev:
                raise ValueError(f"{what} is on cuda:{t.device.index}, the current device is cuda:{dev}")
            if not t.is_contiguous():
                raise ValueError(f"{what} must be contiguous")

        on_device(out, "out")
        if out.dtype != torch.float32 or out.dim() != 3 or out.shape[2] != 3:
            raise ValueError(f"out must be float32 of shape (H, W, 3), got {out.dtype} {tuple(out.shape)}")
        if cam is not None and (out.shape[0], out.shape[1]) != (cam.height, cam.width):
            raise ValueError(f"out is {tuple(out.shape[:2])}, the image is ({cam.height}, {cam.width})")
        if counters is not None:
            on_device(counters, "counters")
            if counters.element_size() != 8 or counters.dtype.is_floating_point or counters.numel() < 5:
                raise ValueError("counters must hold at least 5 64-bit integers")
        d = render_desc(spp, depth, seed, 0, rr_start, image_index, 0, camera)
        check(lib().hk_render_image_static(self.h, C.byref(d), _p(out), _p(counters), _stream(stream)))

    # ------------------------------------------------------------ record queries
    def trace(self, rays, any_hit: bool = False, stream=None):
        import torch

        n = rays.shape[0]
        dev = rays.device
        tri = torch.empty(n, dtype=torch.int32, device=dev)
        t = torch.empty(n, dtype=torch.float32, device=dev)
        u = torch.empty_like(t)
        v = torch.empty_like(t)
        visits = torch.zeros(2, dtype=torch.int64, device=dev)
        check(lib().hk_trace(self.h, n, _p(rays), _p(tri), _p(t), _p(u), _p(v), int(any_hit), _p(visits),
                             _stream(stream)))
        return tri, t, u, v, visits

    def bsdf_batch(self, bsdf_id: int, wi, u2, u1, wo, stream=None, uv=None, duv=None):
        import torch

        n = wi.shape[0]
        dev = wi.device
        out = dict(
            s_wo=torch.empty((n, 3), dtype=torch.float32, device=dev),
            s_w=torch.empty((n, 3), dtype=torch.float32, device=dev),
            s_pdf=torch.empty(n, dtype=torch.float32, device=dev),
            s_measure=torch.empty(n, dtype=torch.int32, device=dev),
            e_rgb=torch.empty((n, 3), dtype=torch.float32, device=dev),
            p_pdf=torch.empty(n, dtype=torch.float32, device=dev),
        )
        check(lib().hk_bsdf_batch(self.h, bsdf_id, n, _p(wi), _p(u2), _p(u1), _p(wo), _p(uv), _p(duv), _p(out["s_wo"]),
                                  _p(out["s_w"]), _p(out["s_pdf"]), _p(out["s_measure"]), _p(out["e_rgb"]),
                                  _p(out["p_pdf"]), _stream(stream)))
        return out

    def texture_eval(self, tex_id: int, uv, duv=None, stream=None):
        """Texture2D::Eval(Isect, filter) of texture `tex_id` at device texture
        coordinates uv (n x 2) with partials duv (n x 4, or None): n x 3."""
        import torch

        out = torch.empty((uv.shape[0], 3), dtype=torch.float32, device=uv.device)
        check(lib().hk_texture_eval(self.h, tex_id, uv.shape[0], _p(uv), _p(duv), _p(out), _stream(stream)))
        return out

    def emitter_sample(self, e: int, inp, stream=None):
        import torch

        out = torch.empty((inp.shape[0], 16), dtype=torch.float32, device=inp.device)
        check(lib().hk_emitter_sample(self.h, e, inp.shape[0], _p(inp), _p(out), _stream(stream)))
        return out

    def camera_rays(self, pos, stream=None):
        import torch

        out = torch.empty((pos.shape[0], 8), dtype=torch.float32, device=pos.device)
        check(lib().hk_camera_rays(self.h, pos.shape[0], _p(pos), _p(out), _stream(stream)))
        return out

    def env_eval(self, wi, stream=None):
        import torch

        rgb = torch.empty((wi.shape[0], 3), dtype=torch.float32, device=wi.device)
        pdf = torch.empty(wi.shape[0], dtype=torch.float32, device=wi.device)
        check(lib().hk_env_eval(self.h, wi.shape[0], _p(wi), _p(rgb), _p(pdf), _stream(stream)))
        return rgb, pdf


def exr_read(path: str) -> np.ndarray:
    """Read an RGB OpenEXR image (H x W x 3 float32) through the library."""
    L = lib()
    w, h = C.c_int32(), C.c_int32()
    check(L.hk_exr_read(path.encode(), C.byref(w), C.byref(h), None, 0))
    out = np.empty((h.value, w.value, 3), np.float32)
    check(L.hk_exr_read(path.encode(), C.byref(w), C.byref(h), out.ctypes.data, out.size))
    return out


def exr_write(path: str, rgb: np.ndarray) -> None:
    """Write an H x W x 3 float image as an uncompressed FLOAT RGB OpenEXR."""
    a = np.ascontiguousarray(rgb, np.float32)
    check(lib().hk_exr_write(path.encode(), a.shape[1], a.shape[0], a.ctypes.data))


def bvh_check(tris: np.ndarray):
    """Build both trees over tris (n x 3 x 3 float32) on the host and check
    them; returns (binary nodes, 8-wide nodes, 8-wide depth)."""
    t = np.ascontiguousarray(tris, np.float32).reshape(-1, 9)
    a, b, c = C.c_uint32(), C.c_uint32(), C.c_uint32()
    check(lib().hk_bvh_check(t.ctypes.data, t.shape[0], C.byref(a), C.byref(b), C.byref(c)))
    return a.value, b.value, c.value


def bvh_check_gpu(tris: np.ndarray):
    """Build the 8-wide tree over tris (n x 3 x 3 float32) on the device and
    check it; returns (8-wide nodes, 8-wide depth)."""
    t = np.ascontiguousarray(tris, np.float32).reshape(-1, 9)
    a, b = C.c_uint32(), C.c_uint32()
    check(lib().hk_bvh_check_gpu(t.ctypes.data, t.shape[0], C.byref(a), C.byref(b)))
    return a.value, b.value


def obj_load(path: str, to_world=None):
    """Load an OBJ through the library's parallel reader: (positions (nv, 3),
    indices (nt, 3), normals (nv, 3) or None, uv (nv, 2) or None)."""
    L = lib()
    tw = None if to_world is None else np.ascontiguousarray(to_world, dtype=np.float32)
    nv, nt, attrs = C.c_uint32(), C.c_uint32(), C.c_int32()
    check(L.hk_obj_load(path.encode(), _p(tw), C.byref(nv), C.byref(nt), None, None, None, None, C.byref(attrs)))
    pos = np.empty((nv.value, 3), np.float32)
    nrm = np.empty((nv.value, 3), np.float32)
    uv = np.empty((nv.value, 2), np.float32)
    idx = np.empty((nt.value, 3), np.uint32)
    check(L.hk_obj_load(path.encode(), _p(tw), C.byref(nv), C.byref(nt), _p(pos), _p(nrm), _p(uv), _p(idx),
                        C.byref(attrs)))
    return pos, idx, (nrm if attrs.value & 1 else None), (uv if attrs.value & 2 else None)


def parse_xml_info(path: str):
    """Parse a scene through the C++ plugin layer without building it (no GPU needed)."""
    L = lib()
    h = C.c_void_p()
    depth, spp = C.c_int32(), C.c_int32()
    check(L.hk_scene_parse_xml(path.encode(), DATA_DIR.encode(), C.byref(h), C.byref(depth), C.byref(spp)))
    info = SceneInfo()
    try:
        check(L.hk_scene_get_info(h, C.byref(info)))
    finally:
        L.hk_scene_destroy(h)
    return info, depth.value, spp.value


__all__ = ["Scene", "SceneDesc", "BSDFDesc", "HikariError", "lib", "scenedesc"]
