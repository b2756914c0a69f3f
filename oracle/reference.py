"""ctypes access to the reference renderer compiled from its own sources
(oracle/ref_build.py -> oracle/_ref/libhikari_ref.so).

Test infrastructure and the timed CPU baseline only: tests use it to pin the
oracle restatement (oracle/hk_oracle.c) against the reference's own classes,
and bench.py's reference arm times the reference's pathMIS renderer through
it.  Nothing in the library imports this module.
"""
from __future__ import annotations

import ctypes as C
import os
from typing import Optional, Sequence

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "_ref", "libhikari_ref.so")
_lib = None


class ReferenceUnavailable(RuntimeError):
    pass


def lib(build_if_possible: bool = True):
    """The loaded library; rebuilt first when the reference checkout is
    present (the build is incremental), else the prebuilt file is used."""
    global _lib
    if _lib is not None:
        return _lib
    if build_if_possible:
        from oracle import ref_build

        try:
            ref_build.build()
        except FileNotFoundError:
            pass   # no checkout here: use the prebuilt library
    if not os.path.exists(LIB):
        raise ReferenceUnavailable(f"{LIB} is not built (the reference checkout is needed to build it)")
    R = C.CDLL(LIB)
    P, F, I, U64 = C.c_void_p, C.c_float, C.c_int, C.c_uint64
    sig = {
        "hr_init": ([C.c_char_p], None),
        "hr_last_error": ([], C.c_char_p),
        "hr_scene_load": ([C.c_char_p], P),
        "hr_scene_free": ([P], None),
        "hr_scene_info": ([P, P], None),
        "hr_render": ([P, I, I, P, I, P], C.c_double),
        "hr_mesh_create": ([P, C.c_uint32, P, P, P, C.c_uint32], P),
        "hr_accel_create": ([I, I, P, I], P),
        "hr_accel_trace": ([P, U64, P, I, P, P, P, P], None),
        "hr_accel_free": ([P], None),
        "hr_env_create": ([C.c_char_p, P, F], P),
        "hr_object_free": ([P], None),
        "hr_emitter_sample": ([P, U64, P, P], None),
        "hr_emitter_eval_dir": ([P, U64, P, P], None),
        "hr_filter_create": ([I, F, F, F], P),
        "hr_filter_eval": ([P, U64, P, P], F),
        "hr_block_put": ([P, I, I, U64, P, P, P], I),
    }
    for name, (args, res) in sig.items():
        fn = getattr(R, name)
        fn.argtypes = args
        fn.restype = res
    R.hr_init(os.path.dirname(LIB).encode())
    _lib = R
    return R


def _p(a):
    return None if a is None else a.ctypes.data


class RefScene:
    """A scene XML loaded by the reference parser (LoadFromXML)."""

    def __init__(self, xml_path: str):
        R = lib()
        self.h = R.hr_scene_load(os.fsencode(xml_path))
        if not self.h:
            raise RuntimeError("reference parse failed: " + R.hr_last_error().decode())
        info = np.zeros(4, np.int32)
        R.hr_scene_info(self.h, _p(info))
        self.width, self.height, self.spp, self.border = (int(x) for x in info)

    def render(self, nthreads: int = 0, max_blocks: int = 0, blocks: Optional[Sequence[int]] = None):
        """Render like src/Main.cpp's Render; returns (film RGBW (H+2B, W+2B, 4), seconds)."""
        R = lib()
        film = np.zeros((self.height + 2 * self.border, self.width + 2 * self.border, 4), np.float32)
        bl = None if blocks is None else np.ascontiguousarray(blocks, dtype=np.int32)
        secs = R.hr_render(self.h, int(nthreads), int(max_blocks), _p(bl), 0 if bl is None else len(bl), _p(film))
        if secs < 0:
            raise RuntimeError("reference render failed: " + R.hr_last_error().decode())
        return film, secs

    def resolve(self, film: np.ndarray) -> np.ndarray:
        """ImageBlock::ToBitmap: interior pixels divided by their weight."""
        B = self.border
        c = film[B:B + self.height, B:B + self.width].astype(np.float32)
        w = c[..., 3:4]
        with np.errstate(divide="ignore", invalid="ignore"):
            return np.where(w != 0, c[..., :3] / w, 0.0).astype(np.float32)

    # No destructor: the reference's scene teardown is not safe to run.
    # HLBVHAcceleration::Build releases its memory arena
    # (src/acceleration/HLBVHAcceleration.cpp:200), which also holds the
    # Triangle shapes Acceleration::AddMesh allocated from it
    # (src/core/Acceleration.cpp:20), and deleting a loaded scene crashed
    # here; loaded scenes live until the process exits.


class RefAccel:
    """A reference acceleration structure ("bruto", "bvh", "hlbvh") over meshes."""

    KINDS = {"bruto": 0, "bvh": 1, "hlbvh": 2}

    def __init__(self, meshes, kind: str = "hlbvh", leaf_size: int = 10):
        R = lib()
        self._keep = []
        hs = []
        for m in meshes:
            P = np.ascontiguousarray(m.positions, np.float32)
            Fi = np.ascontiguousarray(m.indices, np.uint32)
            N = None if m.normals is None else np.ascontiguousarray(m.normals, np.float32)
            self._keep += [P, Fi, N]
            hs.append(R.hr_mesh_create(_p(P), P.shape[0], _p(N), None, _p(Fi), Fi.shape[0]))
        arr = (C.c_void_p * len(hs))(*hs)
        self.h = R.hr_accel_create(self.KINDS[kind], leaf_size, arr, len(hs))
        if not self.h:
            raise RuntimeError("reference accel build failed")

    def trace(self, rays: np.ndarray, any_hit: bool = False):
        rays = np.ascontiguousarray(rays, np.float32)
        n = rays.shape[0]
        tri = np.zeros(n, np.int32)
        t, u, v = (np.zeros(n, np.float32) for _ in range(3))
        lib().hr_accel_trace(self.h, n, _p(rays), int(any_hit), _p(tri), _p(t), _p(u), _p(v))
        return tri, t, u, v

    def __del__(self):
        try:
            if self.h:
                lib().hr_accel_free(self.h)
        except Exception:
            pass


def env_light(exr_path: str, to_world: np.ndarray, scale: float = 1.0):
    """EnvironmentLight of an EXR file (its directory joins the reference's
    file resolver, which resolves relative names only)."""
    tw = np.ascontiguousarray(to_world, np.float32).reshape(16)
    lib().hr_init(os.fsencode(os.path.dirname(os.path.abspath(exr_path))))
    h = lib().hr_env_create(os.fsencode(os.path.basename(exr_path)), _p(tw), float(scale))
    if not h:
        raise RuntimeError("reference env light failed")
    return h


def emitter_sample(h, ref_u_dist: np.ndarray) -> np.ndarray:
    """Emitter::Sample over n records (ref xyz, u2, u1, distance): n x 14
    (p, n, wi, pdf, distance, value)."""
    q = np.ascontiguousarray(ref_u_dist, np.float32)
    out = np.zeros((q.shape[0], 14), np.float32)
    lib().hr_emitter_sample(h, q.shape[0], _p(q), _p(out))
    return out


def emitter_eval_dir(h, wi: np.ndarray) -> np.ndarray:
    """Emitter::Eval and Pdf for world directions: n x 4 (value, pdf)."""
    wi = np.ascontiguousarray(wi, np.float32)
    out = np.zeros((wi.shape[0], 4), np.float32)
    lib().hr_emitter_eval_dir(h, wi.shape[0], _p(wi), _p(out))
    return out


def filter_create(kind: int, radius: float, p0: float, p1: float):
    h = lib().hr_filter_create(kind, radius, p0, p1)
    if not h:
        raise RuntimeError("reference filter failed")
    return h


def block_put(filt, W: int, H: int, pos: np.ndarray, val: np.ndarray):
    """ImageBlock::Put of every sample into a cleared W x H block: (film, border)."""
    pos = np.ascontiguousarray(pos, np.float32)
    val = np.ascontiguousarray(val, np.float32)
    R = lib()
    probe = R.hr_block_put(filt, 1, 1, 0, None, None, None)
    film = np.zeros((H + 2 * probe, W + 2 * probe, 4), np.float32)
    b = R.hr_block_put(filt, W, H, pos.shape[0], _p(pos), _p(val), _p(film))
    return film, b
