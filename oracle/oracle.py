"""ctypes binding of the CPU oracle (oracle/hk_oracle.c).

TEST INFRASTRUCTURE: imported only by tests/, __graft_entry__.smoke() and
bench.py's cpu_baseline leg, as the checker.  The product never imports it.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "libhk_oracle.so")
RFT_DIR = os.path.join(os.path.dirname(HERE), "hikari_b200", "data")


def build(force: bool = False) -> str:
    """Compile the oracle (gcc, -ffp-contract=off keeps the reference's float rounding)."""
    src = os.path.join(HERE, "hk_oracle.c")
    if force or not os.path.exists(LIB_PATH) or os.path.getmtime(LIB_PATH) < max(
        os.path.getmtime(src), os.path.getmtime(os.path.join(HERE, "hk_oracle.h"))
    ):
        os.makedirs(os.path.dirname(LIB_PATH), exist_ok=True)
        subprocess.check_call(
            ["gcc", "-O2", "-fopenmp", "-ffp-contract=off", "-fPIC", "-shared", "-o", LIB_PATH, src, "-lm"]
        )
    return LIB_PATH


class BsdfDescC(C.Structure):
    _fields_ = [
        ("type", C.c_int32), ("distribution", C.c_int32), ("anisotropic", C.c_int32), ("nonlinear", C.c_int32),
        ("alpha_u", C.c_float), ("alpha_v", C.c_float), ("int_ior", C.c_float), ("ext_ior", C.c_float),
        ("eta", C.c_float * 3), ("k", C.c_float * 3), ("ks", C.c_float * 3), ("ks_refract", C.c_float * 3),
        ("kd", C.c_float * 3), ("sigma_a", C.c_float * 3), ("thickness", C.c_float), ("nested", C.c_int32),
        ("nested2", C.c_int32), ("fast_approx", C.c_int32), ("tex", C.c_int32 * 6),
    ]


class TextureDescC(C.Structure):
    _fields_ = [
        ("kind", C.c_int32), ("nested", C.c_int32), ("count", C.c_int32), ("width", C.c_float),
        ("scale", C.c_float), ("uv_scale", C.c_float * 2), ("uv_offset", C.c_float * 2), ("a", C.c_float * 3),
        ("b", C.c_float * 3), ("filter", C.c_int32), ("wrap_u", C.c_int32), ("wrap_v", C.c_int32),
        ("channels", C.c_int32), ("gamma", C.c_float), ("max_anisotropy", C.c_float),
    ]


def texture_desc_c(t, nested_index=-1) -> TextureDescC:
    c = TextureDescC()
    c.kind, c.nested, c.count, c.width, c.scale = t.kind, nested_index, t.count, t.width, t.scale
    c.uv_scale[:], c.uv_offset[:], c.a[:], c.b[:] = t.uv_scale, t.uv_offset, t.a, t.b
    c.filter, c.wrap_u, c.wrap_v = t.filter, t.wrap_u, t.wrap_v
    c.channels, c.gamma, c.max_anisotropy = t.channels, t.gamma, t.max_anisotropy
    return c


def bitmap_pixels(t) -> np.ndarray:
    """The bitmap's 8-bit pixels as a contiguous height x width x channels array."""
    px = np.ascontiguousarray(t.pixels, dtype=np.uint8)
    if px.ndim == 2:
        px = px[:, :, None]
    if px.ndim != 3 or px.shape[2] != t.channels:
        raise ValueError(f"bitmap pixels must be height x width x {t.channels}")
    return px


_lib = None


def lib():
    global _lib
    if _lib is None:
        _lib = C.CDLL(build())
        L = _lib
        P = C.c_void_p
        L.ho_scene_create.restype = P
        L.ho_scene_destroy.argtypes = [P]
        L.ho_scene_set_rft.argtypes = [P, C.c_int, C.c_char_p, C.c_uint64]
        L.ho_scene_add_bsdf.argtypes = [P, C.POINTER(BsdfDescC)]
        L.ho_scene_add_mesh.argtypes = [P, P, C.c_uint32, P, C.c_uint32, P, C.c_int32, P]
        L.ho_scene_set_envmap.argtypes = [P, P, C.c_uint32, C.c_uint32, P, C.c_float]
        L.ho_scene_set_constant_light.argtypes = [P, P]
        L.ho_scene_set_mesh_uv.argtypes = [P, C.c_int, P]
        L.ho_post_intersect.argtypes = [P, C.c_uint32, C.c_float, C.c_float, P]
        L.ho_scene_add_point_light.argtypes = [P, P, P]
        L.ho_scene_add_directional_light.argtypes = [P, P, P]
        L.ho_scene_set_camera.argtypes = [P, C.c_uint32, C.c_uint32, P, C.c_float, C.c_float, C.c_float]
        L.ho_scene_set_filter.argtypes = [P, C.c_int, C.c_float, C.c_float, C.c_float]
        L.ho_scene_set_background.argtypes = [P, P, C.c_int]
        L.ho_scene_finalize.argtypes = [P]
        L.ho_last_error.restype = C.c_char_p
        L.ho_scene_bbox.argtypes = [P, P]
        L.ho_bsdf_sample.argtypes = [P, C.c_int, P, P, C.c_float, P, P, P, P]
        L.ho_bsdf_eval.argtypes = [P, C.c_int, P, P, C.c_int, P]
        L.ho_bsdf_pdf.argtypes = [P, C.c_int, P, P, C.c_int]
        L.ho_bsdf_pdf.restype = C.c_float
        L.ho_bsdf_batch.argtypes = [P, C.c_int, C.c_uint64, P, P, P, P, P, P, P, P, P, P, P, P, C.c_int]
        L.ho_scene_add_texture.argtypes = [P, C.POINTER(TextureDescC)]
        L.ho_bsdf_batch_isect.argtypes = [P, C.c_int, C.c_uint64, P, P, P, P, P, P, P, P, P, P, P, C.c_int]
        L.ho_scene_add_bitmap.argtypes = [P, C.POINTER(TextureDescC), P, C.c_int, C.c_int]
        L.ho_texture_eval.argtypes = [P, C.c_int, P, P, P]
        L.ho_texture_eval_hit.argtypes = [P, C.c_int, C.c_uint32, C.c_float, C.c_float, P]
        L.ho_texture_mip.argtypes = [P, C.c_int, C.c_int, P, P]
        L.ho_screen_partials.argtypes = [P, C.c_float, C.c_float, C.c_uint32, C.c_float, C.c_float, P]
        L.ho_bsdf_rft_eval.argtypes = [P, C.c_int, C.c_float]
        L.ho_bsdf_rft_eval.restype = C.c_float
        L.ho_trace.argtypes = [P, C.c_uint64, P, P, P, P, P, C.c_int, C.c_int, C.c_int]
        L.ho_render.argtypes = [P, C.c_int, C.c_int, P, C.c_int, P, C.c_int, P]
        L.ho_render.restype = C.c_int64
        L.ho_scene_set_reference_draw_order.argtypes = [P, C.c_int]
        L.ho_film_put_samples.argtypes = [P, C.c_uint64, P, P, P]
        L.ho_pixel_samples.argtypes = [P, C.c_int, C.c_uint64, C.c_int, P, P, C.c_int]
        L.ho_film_put_samples.restype = C.c_int64
        L.ho_pixel_stats.argtypes = [P, C.c_int, C.c_int, C.c_uint64, C.c_int, P, P, C.c_int]
        L.ho_ttest_scene.argtypes = [P, C.c_int, C.c_int, P, P]
        L.ho_film_resolve.argtypes = [P, P, P]
        L.ho_film_border.argtypes = [P]
        L.ho_emitter_sample.argtypes = [P, C.c_int, P, C.c_float, C.c_float, C.c_float, P]
        L.ho_emitter_pdf.argtypes = [P, C.c_int, P, P, P]
        L.ho_emitter_pdf.restype = C.c_float
        L.ho_env_eval.argtypes = [P, P, P]
        L.ho_camera_ray.argtypes = [P, C.c_float, C.c_float, P]
        L.ho_filter_table.argtypes = [P, P, P]
    return _lib


def _p(a):
    return a.ctypes.data_as(C.c_void_p) if a is not None else None


def _f32(a):
    return np.ascontiguousarray(a, dtype=np.float32)


def bsdf_desc_c(d, nested_index=-1, nested2_index=-1, tex_ids=None) -> BsdfDescC:
    c = BsdfDescC()
    c.type, c.distribution = d.type, d.distribution
    c.anisotropic, c.nonlinear = int(d.anisotropic), int(d.nonlinear)
    c.alpha_u, c.alpha_v, c.int_ior, c.ext_ior = d.alpha_u, d.alpha_v, d.int_ior, d.ext_ior
    c.eta[:] = d.conductor_eta()
    c.k[:], c.ks[:], c.ks_refract[:], c.kd[:], c.sigma_a[:] = d.k, d.ks, d.ks_refract, d.kd, d.sigma_a
    c.thickness, c.nested, c.nested2 = d.thickness, nested_index, nested2_index
    c.fast_approx = int(getattr(d, "fast_approx", False))
    for k, t in enumerate(tex_ids or [-1] * 6):
        c.tex[k] = t + 1
    return c


def read_rft(dist: int) -> bytes:
    name = "GGXRFTData.bin" if dist == 1 else "BeckmannRFTData.bin"
    with open(os.path.join(RFT_DIR, name), "rb") as f:
        return f.read()


class OracleScene:
    """A finalized oracle scene built from a :class:`hikari_b200.scenedesc.SceneDesc`."""

    def __init__(self, desc):
        L = lib()
        self.desc = desc
        self.h = L.ho_scene_create()
        self._keep = []
        for dist in (0, 1):
            b = read_rft(dist)
            L.ho_scene_set_rft(self.h, dist, b, len(b))
        self.bsdf_ids = {}
        self.mesh_bsdf = []
        for m in desc.meshes:
            self.mesh_bsdf.append(self.add_bsdf(m.bsdf))
        for kind, i in desc.build_steps():   # emitters in Scene::AddChild order
            if kind == "env":
                self._set_env()
            elif kind == "light":
                l = desc.lights[i]
                col, vec = _f32(l.color), _f32(l.vector)
                self._keep += [col, vec]
                add = L.ho_scene_add_point_light if l.kind == "point" else L.ho_scene_add_directional_light
                if add(self.h, _p(col), _p(vec)) < 0:
                    raise RuntimeError(L.ho_last_error().decode())
            else:
                m = desc.meshes[i]
                pos = _f32(m.positions)
                idx = np.ascontiguousarray(m.indices, dtype=np.uint32)
                nrm = _f32(m.normals) if m.normals is not None else None
                rad = _f32(m.radiance) if m.radiance is not None else None
                self._keep += [pos, idx, nrm, rad]
                r = L.ho_scene_add_mesh(self.h, _p(pos), pos.shape[0], _p(idx), idx.shape[0], _p(nrm),
                                        self.mesh_bsdf[i], _p(rad))
                if r < 0:
                    raise RuntimeError(L.ho_last_error().decode())
                if getattr(m, "uv", None) is not None:
                    uv = _f32(m.uv)
                    self._keep.append(uv)
                    L.ho_scene_set_mesh_uv(self.h, r, _p(uv))
        cam = desc.camera
        tw = _f32(cam.to_world)
        L.ho_scene_set_camera(self.h, cam.width, cam.height, _p(tw), cam.fov, cam.near_clip, cam.far_clip)
        f = desc.filter
        L.ho_scene_set_filter(self.h, f.kind, f.radius, f.p0, f.p1)
        bg = _f32(desc.background)
        L.ho_scene_set_background(self.h, _p(bg), int(desc.force_background))
        if L.ho_scene_finalize(self.h) < 0:
            raise RuntimeError(L.ho_last_error().decode())

    def _set_env(self):
        if self.desc.env_constant is not None:
            c = _f32(self.desc.env_constant)
            self._keep.append(c)
            if lib().ho_scene_set_constant_light(self.h, _p(c)) < 0:
                raise RuntimeError(lib().ho_last_error().decode())
            return
        e = self.desc.env
        rgb = _f32(e.rgb)
        tw = _f32(e.to_world)
        self._keep += [rgb, tw]
        if lib().ho_scene_set_envmap(self.h, _p(rgb), rgb.shape[1], rgb.shape[0], _p(tw), e.scale) < 0:
            raise RuntimeError(lib().ho_last_error().decode())

    def add_bsdf(self, d) -> int:
        key = id(d)
        if key in self.bsdf_ids:
            return self.bsdf_ids[key]
        nested = self.add_bsdf(d.nested) if d.nested is not None else -1
        nested2 = self.add_bsdf(d.nested2) if getattr(d, "nested2", None) is not None else -1
        from hikari_b200.scenedesc import TEX_SLOTS
        tex = getattr(d, "textures", {}) or {}
        c = bsdf_desc_c(d, nested, nested2, [self.add_texture(tex[k]) if k in tex else -1 for k in TEX_SLOTS])
        self._keep.append(c)
        i = lib().ho_scene_add_bsdf(self.h, C.byref(c))
        self.bsdf_ids[key] = i
        return i

    def add_texture(self, t) -> int:
        if not hasattr(self, "tex_ids"):
            self.tex_ids = {}
        if id(t) in self.tex_ids:
            return self.tex_ids[id(t)]
        nested = self.add_texture(t.nested) if t.nested is not None else -1
        c = texture_desc_c(t, nested)
        self._keep.append(c)
        if t.kind == 4:   # bitmap
            px = bitmap_pixels(t)
            i = lib().ho_scene_add_bitmap(self.h, C.byref(c), _p(px), px.shape[1], px.shape[0])
        else:
            i = lib().ho_scene_add_texture(self.h, C.byref(c))
        if i < 0:
            raise RuntimeError(lib().ho_last_error().decode())
        self.tex_ids[id(t)] = i
        if not hasattr(self, "_tex_channels"):
            self._tex_channels = {}
        self._tex_channels[id(t)] = t.channels if t.kind == 4 else 3
        return i

    def __del__(self):
        try:
            lib().ho_scene_destroy(self.h)
        except Exception:
            pass

    # ---- queries
    def bbox(self):
        o = np.zeros(6, np.float32)
        lib().ho_scene_bbox(self.h, _p(o))
        return o

    def bsdf_batch(self, bsdf, wi, u2, u1, wo, nthreads=0, uv=None, duv=None):
        n = wi.shape[0]
        wi, u2, wo = _f32(wi), _f32(u2), _f32(wo)
        u1 = _f32(u1) if u1 is not None else None
        uv = _f32(uv) if uv is not None else None
        duv = _f32(duv) if duv is not None else None
        out = dict(
            s_wo=np.zeros((n, 3), np.float32), s_w=np.zeros((n, 3), np.float32), s_pdf=np.zeros(n, np.float32),
            s_measure=np.zeros(n, np.int32), e_rgb=np.zeros((n, 3), np.float32), p_pdf=np.zeros(n, np.float32),
        )
        lib().ho_bsdf_batch(self.h, bsdf, n, _p(wi), _p(u2), _p(u1), _p(wo), _p(uv), _p(duv), _p(out["s_wo"]), _p(out["s_w"]),
                            _p(out["s_pdf"]), _p(out["s_measure"]), _p(out["e_rgb"]), _p(out["p_pdf"]), nthreads)
        return out

    def bsdf_batch_isect(self, bsdf, wi, u2, u1, wo, isect, nthreads=0):
        """bsdf_batch with each record's intersection: isect n x 20 (shading
        frame S T N, geometric N, dPdU, dPdV, UV)."""
        n = wi.shape[0]
        wi, u2, wo, isect = _f32(wi), _f32(u2), _f32(wo), _f32(isect)
        u1 = _f32(u1) if u1 is not None else None
        out = dict(
            s_wo=np.zeros((n, 3), np.float32), s_w=np.zeros((n, 3), np.float32), s_pdf=np.zeros(n, np.float32),
            s_measure=np.zeros(n, np.int32), e_rgb=np.zeros((n, 3), np.float32), p_pdf=np.zeros(n, np.float32),
        )
        lib().ho_bsdf_batch_isect(self.h, bsdf, n, _p(wi), _p(u2), _p(u1), _p(wo), _p(isect), _p(out["s_wo"]),
                                  _p(out["s_w"]), _p(out["s_pdf"]), _p(out["s_measure"]), _p(out["e_rgb"]),
                                  _p(out["p_pdf"]), nthreads)
        return out

    def texture_eval(self, tex, uv, duv=None):
        """Texture2D::Eval(Isect) of texture `tex` (an id or a TextureDesc added
        with a BSDF) at n x 2 texture coordinates, n x 4 partials or None."""
        tid = tex if isinstance(tex, int) else self.tex_ids[id(tex)]
        uv = _f32(uv)
        duv = _f32(duv) if duv is not None else None
        out = np.zeros((uv.shape[0], 3), np.float32)
        for k in range(uv.shape[0]):
            lib().ho_texture_eval(self.h, tid, _p(uv[k]), _p(duv[k]) if duv is not None else None, _p(out[k]))
        return out

    def texture_eval_hit(self, tex, tri, u, v):
        """Texture::Eval(Isect, true) of texture `tex` at the intersections of
        triangles tri (scene order) at barycentric (u, v): n x 3."""
        tid = tex if isinstance(tex, int) else self.tex_ids[id(tex)]
        out = np.zeros((len(tri), 3), np.float32)
        for k in range(len(tri)):
            lib().ho_texture_eval_hit(self.h, tid, int(tri[k]), float(u[k]), float(v[k]), _p(out[k]))
        return out

    def texture_mip(self, tex):
        """The MIP pyramid of a bitmap texture: a list of height x width x channels float arrays."""
        tid = tex if isinstance(tex, int) else self.tex_ids[id(tex)]
        wh = np.zeros(2, np.int32)
        n = lib().ho_texture_mip(self.h, tid, -1, _p(wh), None)
        if n < 0:
            raise RuntimeError(lib().ho_last_error().decode())
        out = []
        for l in range(n):
            lib().ho_texture_mip(self.h, tid, l, _p(wh), None)
            ch = self.desc_channels(tid)
            a = np.zeros((wh[1], wh[0], ch), np.float32)
            lib().ho_texture_mip(self.h, tid, l, _p(wh), _p(a))
            out.append(a)
        return out

    def desc_channels(self, tid):
        for key, i in self.tex_ids.items():
            if i == tid:
                return self._tex_channels[key]
        return 3

    def screen_partials(self, px, py, tri, u, v):
        out = np.zeros(4, np.float32)
        lib().ho_screen_partials(self.h, px, py, tri, u, v, _p(out))
        return out

    def bsdf_sample(self, bsdf, wi, u2, u1=0.0):
        wo = np.zeros(3, np.float32); w = np.zeros(3, np.float32)
        m = C.c_int(0); eta = C.c_float(0)
        wi, u2 = _f32(wi), _f32(u2)
        lib().ho_bsdf_sample(self.h, bsdf, _p(wi), _p(u2), u1, _p(wo), _p(w), C.byref(m), C.byref(eta))
        return wo, w, m.value, eta.value

    def bsdf_pdf(self, bsdf, wi, wo, measure=1):
        return lib().ho_bsdf_pdf(self.h, bsdf, _p(_f32(wi)), _p(_f32(wo)), measure)

    def bsdf_eval(self, bsdf, wi, wo, measure=1):
        o = np.zeros(3, np.float32)
        lib().ho_bsdf_eval(self.h, bsdf, _p(_f32(wi)), _p(_f32(wo)), measure, _p(o))
        return o

    def trace(self, rays, any_hit=False, use_bvh=True, nthreads=0):
        rays = _f32(rays)
        n = rays.shape[0]
        t = np.zeros(n, np.float32); u = np.zeros(n, np.float32); v = np.zeros(n, np.float32)
        tri = np.zeros(n, np.int32)
        lib().ho_trace(self.h, n, _p(rays), _p(t), _p(u), _p(v), _p(tri), int(any_hit), int(use_bvh), nthreads)
        return tri, t, u, v

    def set_reference_draw_order(self, on: bool = True):
        """Two-dimensional draws as the compiled reference's Next2D takes them
        (second uniform first); for path-level comparisons with the reference."""
        lib().ho_scene_set_reference_draw_order(self.h, int(on))

    def render(self, spp, depth=None, blocks=None, nthreads=0):
        L = lib()
        B = L.ho_film_border(self.h)
        W, H = self.desc.camera.width, self.desc.camera.height
        film = np.zeros((H + 2 * B, W + 2 * B, 4), np.float64)
        bl = np.ascontiguousarray(blocks, dtype=np.int32) if blocks is not None else None
        ctr = np.zeros(4, np.uint64)
        dropped = L.ho_render(self.h, depth or self.desc.depth, spp, _p(bl), 0 if bl is None else len(bl),
                              _p(film), nthreads, _p(ctr))
        return film, int(dropped), ctr

    def film_put(self, pos, val):
        """ImageBlock::Put of samples into an empty bordered film (double)."""
        B = lib().ho_film_border(self.h)
        W, H = self.desc.camera.width, self.desc.camera.height
        film = np.zeros((H + 2 * B, W + 2 * B, 4), np.float64)
        pos, val = _f32(pos), _f32(val)
        dropped = lib().ho_film_put_samples(self.h, pos.shape[0], _p(pos), _p(val), _p(film))
        return film, int(dropped)

    def resolve(self, film):
        W, H = self.desc.camera.width, self.desc.camera.height
        out = np.zeros((H, W, 3), np.float32)
        lib().ho_film_resolve(self.h, _p(np.ascontiguousarray(film)), _p(out))
        return out

    def pixel_stats(self, pixels, spp, seed=0, depth=None, nthreads=0):
        pix = np.ascontiguousarray(pixels, dtype=np.int32)
        out = np.zeros((pix.shape[0], 6), np.float64)
        lib().ho_pixel_stats(self.h, depth or self.desc.depth, spp, seed, pix.shape[0], _p(pix), _p(out), nthreads)
        return out[:, :3], out[:, 3:]

    def pixel_samples(self, pixels, seed, depth=None, nthreads=0):
        """One path per pixel from the stream (seed, pixel): (film positions n x 2, radiance n x 3)."""
        pix = np.ascontiguousarray(pixels, dtype=np.int32)
        out = np.zeros((pix.shape[0], 5), np.float32)
        lib().ho_pixel_samples(self.h, depth or self.desc.depth, seed, pix.shape[0], _p(pix), _p(out), nthreads)
        return out[:, :2].copy(), out[:, 2:].copy()

    def ttest_scene(self, n, depth=None):
        m = C.c_double(0); v = C.c_double(0)
        lib().ho_ttest_scene(self.h, depth or self.desc.depth, n, C.byref(m), C.byref(v))
        return m.value, v.value

    def camera_ray(self, px, py):
        o = np.zeros(8, np.float32)
        lib().ho_camera_ray(self.h, px, py, _p(o))
        return o

    def emitter_sample(self, e, ref, u):
        o = np.zeros(14, np.float32)
        lib().ho_emitter_sample(self.h, e, _p(_f32(ref)), float(u[0]), float(u[1]), float(u[2]), _p(o))
        return o

    def emitter_pdf(self, e, ref, p, n):
        return lib().ho_emitter_pdf(self.h, e, _p(_f32(ref)), _p(_f32(p)), _p(_f32(n)))

    def env_eval(self, wi):
        o = np.zeros(3, np.float32)
        lib().ho_env_eval(self.h, _p(_f32(wi)), _p(o))
        return o


# ------------------------------------------------------------ statistics
def students_t_test(mean, variance, reference, n, alpha, num_tests):
    """hypothesis::students_t_test (ext/hypothesis/hypothesis.h:319), restated with scipy."""
    from scipy import stats

    t = abs(mean - reference) * np.sqrt(n / max(variance, 1e-5))
    pval = 2 * (1 - stats.t.cdf(t, n - 1))
    a = 1.0 - (1.0 - alpha) ** (1.0 / num_tests)
    return pval >= a, pval


def chi2_test(obs, exp, sample_count, min_exp_freq, alpha, num_tests):
    """hypothesis::chi2_test (ext/hypothesis/hypothesis.h:140): cells sorted by
    expected frequency, low-frequency cells pooled, Sidak-corrected level."""
    from scipy import stats

    obs = np.asarray(obs, np.float64).ravel()
    exp = np.asarray(exp, np.float64).ravel()
    order = np.argsort(exp, kind="stable")
    pooled_f = pooled_e = chsq = 0.0
    dof = 0
    for i in order:
        e, o = exp[i], obs[i]
        if e < 0:
            return False, 0.0, "negative expected frequency"
        if e == 0:
            if o > sample_count * 1e-5:
                return False, 0.0, f"{o} samples in a cell with expected frequency 0"
        elif e < min_exp_freq:
            pooled_f += o; pooled_e += e
        elif pooled_e > 0 and pooled_e < min_exp_freq:
            pooled_f += o; pooled_e += e
        else:
            chsq += (o - e) ** 2 / e
            dof += 1
    if pooled_e > 0 or pooled_f > 0:
        chsq += (pooled_f - pooled_e) ** 2 / pooled_e
        dof += 1
    dof -= 1
    if dof <= 0:
        return False, 0.0, "too few degrees of freedom"
    pval = 1 - stats.chi2.cdf(chsq, dof)
    a = 1.0 - (1.0 - alpha) ** (1.0 / num_tests)
    return (pval >= a and np.isfinite(pval)), pval, f"chi2={chsq:.2f} dof={dof}"
