"""Host-side scene description shared by the XML loader, the synthetic scene
generators and the C-ABI upload path.

A :class:`SceneDesc` is the flattened result of Hikari's XML parse
(src/core/Parser.cpp:9): meshes in XML order with their BSDF and optional
area emitter, one optional environment emitter, the perspective camera, the
reconstruction filter and the pathMIS ``depth``.  Emitter order follows
Scene::AddChild (src/core/Scene.cpp:167): mesh emitters in XML order, the
environment emitter at the position where it is parsed.
"""
from __future__ import annotations

import math
import os
import xml.etree.ElementTree as ET
from dataclasses import dataclass, field
from typing import Dict, List, Optional

import numpy as np

# BSDF kinds, matching hk_bsdf_type in include/hikari_b200.h
BSDF_DIFFUSE, BSDF_ROUGH_CONDUCTOR, BSDF_ROUGH_DIELECTRIC, BSDF_ROUGH_PLASTIC, BSDF_ROUGH_COATING = range(5)
BSDF_MIRROR, BSDF_CONDUCTOR, BSDF_DIELECTRIC, BSDF_PLASTIC, BSDF_TWO_SIDED, BSDF_COATING, BSDF_ROUGH_DIFFUSE = range(5, 12)
# bumpMap / normalMap wrap one nested BSDF; their map texture is textures["kd"] (slot 0)
BSDF_BUMP_MAP, BSDF_NORMAL_MAP = 12, 13
BECKMANN, GGX = 0, 1
BSDF_TYPE_NAMES = {
    "diffuse": BSDF_DIFFUSE,
    "roughConductor": BSDF_ROUGH_CONDUCTOR,
    "roughDielectric": BSDF_ROUGH_DIELECTRIC,
    "roughPlastic": BSDF_ROUGH_PLASTIC,
    "roughCoating": BSDF_ROUGH_COATING,
    "mirror": BSDF_MIRROR,
    "conductor": BSDF_CONDUCTOR,
    "dielectric": BSDF_DIELECTRIC,
    "plastic": BSDF_PLASTIC,
    "twoSided": BSDF_TWO_SIDED,
    "coating": BSDF_COATING,
    "roughDiffuse": BSDF_ROUGH_DIFFUSE,
    "bumpMap": BSDF_BUMP_MAP,
    "normalMap": BSDF_NORMAL_MAP,
}
# BSDFs with a delta (specular) lobe and no microfacet distribution
SMOOTH_BSDFS = (BSDF_MIRROR, BSDF_CONDUCTOR, BSDF_DIELECTRIC, BSDF_PLASTIC, BSDF_COATING)
# BSDFs that nest others: (roughCoating, coating) one, twoSided one or two
LAYER_BSDFS = (BSDF_ROUGH_COATING, BSDF_COATING)
FILTER_KINDS = {"box": 0, "tent": 1, "gaussian": 2, "mitchell": 3}

AIR_IOR = 1.000277  # DEFAULT_*_EXT_IOR, include/core/Common.hpp:333


class SceneError(RuntimeError):
    """Raised for malformed scenes (the reference throws HikariException)."""


# Procedural textures, matching hk_texture_kind in include/hikari_b200.h
TEX_CHECKERBOARD, TEX_GRID, TEX_SCALE, TEX_BITMAP, TEX_WIREFRAME, TEX_CURVATURE = 1, 2, 3, 4, 5, 6
TEX_TYPE_NAMES = {"checkerboard": TEX_CHECKERBOARD, "grid": TEX_GRID, "scale": TEX_SCALE, "bitmap": TEX_BITMAP,
                  "wireframe": TEX_WIREFRAME, "curvature": TEX_CURVATURE}
# bitmap "filterType" and "uWrapMode" / "vWrapMode" (src/texture/BitmapTexture.cpp:15-46)
FILTER_NEAREST, FILTER_BILINEAR, FILTER_TRILINEAR, FILTER_EWA = 0, 1, 2, 3
FILTER_NAMES = {"nearest": FILTER_NEAREST, "bilinear": FILTER_BILINEAR, "trilinear": FILTER_TRILINEAR,
                "ewa": FILTER_EWA}
WRAP_REPEAT, WRAP_CLAMP, WRAP_BLACK = 0, 1, 2
WRAP_NAMES = {"repeat": WRAP_REPEAT, "clamp": WRAP_CLAMP, "black": WRAP_BLACK}
# textured BSDF parameters, in the order of hk_bsdf_desc.tex
TEX_SLOTS = ("kd", "ks", "ks_refract", "sigma_a", "alpha_u", "alpha_v")


@dataclass
class TextureDesc:
    """A procedural texture (src/texture/{Checkerboard,Grid,Scale}Texture.cpp),
    a bitmap (src/texture/BitmapTexture.cpp) or a texture of the hit's geometry
    (src/texture/{Wireframe,Curvature}Texture.cpp); defaults are the reference's
    (include/core/Common.hpp:425-462).  Wireframe: a interiorColor, b edgeColor,
    width edgeWidth (0: a tenth of the mean edge length of the first mesh that
    uses it), scale transitionWidth.  Curvature: a positiveColor, b
    negativeColor, scale, count 1 "gaussian" / 0 "mean"."""
    kind: int
    count: int = 10                    # checkerboard "blocks", grid "lines"
    width: float = 0.01                # grid "lineWidth"
    scale: float = 1.0                 # scale "scale"
    uv_scale: List[float] = field(default_factory=lambda: [1.0, 1.0])
    uv_offset: List[float] = field(default_factory=lambda: [0.0, 0.0])
    a: List[float] = field(default_factory=lambda: [0.4, 0.4, 0.4])   # colorA / lineColor
    b: List[float] = field(default_factory=lambda: [0.2, 0.2, 0.2])   # colorB / backgroundColor
    nested: Optional["TextureDesc"] = None                           # scale: the scaled texture
    # bitmap: 8-bit pixels as stbi_load returns them (height x width x channels, row 0 = top)
    pixels: Optional[np.ndarray] = None
    filter: int = FILTER_EWA
    wrap_u: int = WRAP_REPEAT
    wrap_v: int = WRAP_REPEAT
    channels: int = 3                  # "channel": r (1) or rgb (3)
    gamma: float = 1.0
    max_anisotropy: float = 20.0


@dataclass
class BSDFDesc:
    """Properties of one BSDF; defaults are the reference's
    (include/core/Common.hpp:331-392)."""

    type: int = BSDF_DIFFUSE
    distribution: int = BECKMANN
    anisotropic: bool = False
    nonlinear: bool = False
    alpha_u: float = 0.1
    alpha_v: float = 0.1
    int_ior: float = 1.5046
    ext_ior: float = AIR_IOR
    eta: Optional[List[float]] = None  # per-channel conductor eta; None -> int_ior/ext_ior
    k: List[float] = field(default_factory=lambda: [1.0, 1.0, 1.0])
    ks: List[float] = field(default_factory=lambda: [1.0, 1.0, 1.0])
    ks_refract: List[float] = field(default_factory=lambda: [1.0, 1.0, 1.0])
    kd: List[float] = field(default_factory=lambda: [0.5, 0.5, 0.5])
    sigma_a: List[float] = field(default_factory=lambda: [0.0, 0.0, 0.0])
    thickness: float = 1.0
    nested: Optional["BSDFDesc"] = None    # roughCoating's BSDF, twoSided's front BSDF
    nested2: Optional["BSDFDesc"] = None   # twoSided's back BSDF (None: the front one)
    fast_approx: bool = False              # roughDiffuse "fastApprox"
    textures: Dict[str, "TextureDesc"] = field(default_factory=dict)   # slot (TEX_SLOTS) -> texture

    def conductor_eta(self) -> List[float]:
        if self.eta is not None:
            return list(self.eta)
        e = np.float32(self.int_ior) / np.float32(self.ext_ior)
        return [float(e)] * 3


@dataclass
class MeshDesc:
    positions: np.ndarray  # (nv, 3) float32, world space
    indices: np.ndarray  # (nt, 3) uint32
    bsdf: BSDFDesc
    normals: Optional[np.ndarray] = None  # (nv, 3) float32
    radiance: Optional[List[float]] = None  # area emitter
    bbox: Optional[np.ndarray] = None  # (2,3): includes unreferenced vertices
    uv: Optional[np.ndarray] = None  # (nv, 2) float32 texture coordinates (OBJ "vt")


@dataclass
class EnvDesc:
    rgb: np.ndarray  # (H, W, 3) float32
    to_world: np.ndarray  # (4,4) float32
    scale: float = 1.0


@dataclass
class LightDesc:
    """A point or a directional light (src/emitter/PointLight.cpp:8,
    src/emitter/DirectionalLight.cpp:8)."""
    kind: str                # "point" or "directional"
    color: List[float]       # power (point) or irradiance (directional)
    vector: List[float]      # position (point) or direction of travel (directional)
    emitter_index: int = -1  # position in the emitter list (Scene::AddChild order); -1: after the others


@dataclass
class CameraDesc:
    width: int = 1280
    height: int = 720
    to_world: np.ndarray = field(default_factory=lambda: np.eye(4, dtype=np.float32))
    fov: float = 30.0
    near_clip: float = 1e-4
    far_clip: float = 1e4


@dataclass
class FilterDesc:
    kind: int = 2
    radius: float = 2.0
    p0: float = 0.5  # gaussian stddev / mitchell B
    p1: float = 0.0  # mitchell C


@dataclass
class SceneDesc:
    meshes: List[MeshDesc] = field(default_factory=list)
    env: Optional[EnvDesc] = None
    env_constant: Optional[List[float]] = None  # ConstantLight radiance (instead of an environment map)
    env_emitter_index: int = -1  # position of the env emitter in the emitter list
    lights: List[LightDesc] = field(default_factory=list)
    camera: CameraDesc = field(default_factory=CameraDesc)
    filter: FilterDesc = field(default_factory=FilterDesc)
    depth: int = 32
    spp: int = 1
    background: List[float] = field(default_factory=lambda: [0.0, 0.0, 0.0])
    force_background: bool = False
    integrator: str = "pathMIS"

    @property
    def n_triangles(self) -> int:
        return int(sum(m.indices.shape[0] for m in self.meshes))

    def emitter_order(self) -> List[int]:
        """The emitter list in Scene::AddChild order: a mesh index per area
        emitter, -1 for the environment (map or constant), -2 - k for
        lights[k].  Non-mesh emitters sit at the positions recorded when they
        were parsed."""
        order = [i for i, m in enumerate(self.meshes) if m.radiance is not None]
        extra = []
        if self.env is not None or self.env_constant is not None:
            extra.append((self.env_emitter_index, -1))
        extra += [(l.emitter_index, -2 - k) for k, l in enumerate(self.lights)]
        for pos, code in sorted(extra, key=lambda t: (t[0] < 0, t[0])):
            order.insert(pos if 0 <= pos <= len(order) else len(order), code)
        return order

    def build_steps(self) -> List[tuple]:
        """Scene construction steps that reproduce emitter_order(): ("mesh", i)
        in mesh order, ("env", 0) and ("light", k) each just before the mesh
        emitter it precedes."""
        steps, mi = [], 0
        for code in self.emitter_order():
            if code >= 0:
                while mi <= code:
                    steps.append(("mesh", mi))
                    mi += 1
            else:
                steps.append(("env", 0) if code == -1 else ("light", -2 - code))
        steps += [("mesh", i) for i in range(mi, len(self.meshes))]
        return steps


# ----------------------------------------------------------------- transforms
def _vec3(s: str) -> np.ndarray:
    """ToVector3f  src/core/Common.cpp:108 (exactly 3 comma/space separated values)."""
    toks = [t for t in s.replace(",", " ").split() if t]
    if len(toks) != 3:
        raise SceneError(f"Expected 3 values, got {s!r}")
    return np.array([float(np.float32(t)) for t in toks], dtype=np.float32)


def _angle_axis(angle_rad: float, axis: np.ndarray) -> np.ndarray:
    """Eigen::AngleAxis matrix (the axis is used as given, not re-normalised)."""
    x, y, z = (float(a) for a in axis)
    c, s = math.cos(angle_rad), math.sin(angle_rad)
    C = 1 - c
    R = np.array(
        [
            [x * x * C + c, x * y * C - z * s, x * z * C + y * s],
            [y * x * C + z * s, y * y * C + c, y * z * C - x * s],
            [z * x * C - y * s, z * y * C + x * s, z * z * C + c],
        ],
        dtype=np.float64,
    )
    M = np.eye(4)
    M[:3, :3] = R
    return M


def parse_transform(node: ET.Element) -> np.ndarray:
    """<transform> children composed as Trans = Op * Trans (src/core/Parser.cpp:311-372)."""
    T = np.eye(4, dtype=np.float64)
    for ch in node:
        tag = ch.tag
        if tag == "translate":
            v = _vec3(ch.attrib["value"])
            M = np.eye(4)
            M[:3, 3] = v
        elif tag == "scale":
            v = _vec3(ch.attrib["value"])
            M = np.diag([v[0], v[1], v[2], 1.0])
        elif tag == "rotate":
            ang = math.radians(float(ch.attrib["angle"]))
            M = _angle_axis(ang, _vec3(ch.attrib["axis"]))
        elif tag == "matrix":
            vals = [float(t) for t in ch.attrib["value"].replace(",", " ").split() if t]
            if len(vals) != 16:
                raise SceneError("Expected 16 values")
            M = np.array(vals, dtype=np.float64).reshape(4, 4)
        elif tag == "lookat":
            o = _vec3(ch.attrib["origin"]).astype(np.float64)
            t = _vec3(ch.attrib["target"]).astype(np.float64)
            up = _vec3(ch.attrib["up"]).astype(np.float64)
            d = t - o
            d /= np.linalg.norm(d)
            left = np.cross(up / np.linalg.norm(up), d)
            left /= np.linalg.norm(left)
            nup = np.cross(d, left)
            nup /= np.linalg.norm(nup)
            M = np.eye(4)
            M[:3, 0], M[:3, 1], M[:3, 2], M[:3, 3] = left, nup, d, o
        else:
            raise SceneError(f"Unhandled element {tag!r}")
        T = M @ T
    return T.astype(np.float32)


# ----------------------------------------------------------------------- OBJ
def load_obj(path: str, to_world: Optional[np.ndarray] = None):
    """WavefrontObjMesh ctor (src/mesh/WavefrontObjMesh.cpp:10-152): positions are
    transformed as points, normals by the inverse transpose and normalised,
    vertices are de-duplicated on their (p, uv, n) index triple in first-use
    order, and quads split into (v1,v2,v3), (v4,v1,v3)."""
    M = np.eye(4, dtype=np.float64) if to_world is None else np.asarray(to_world, dtype=np.float64)
    Minv_t = np.linalg.inv(M)[:3, :3].T
    P, N, UV, F = [], [], [], []
    vmap: Dict[tuple, int] = {}
    verts: List[tuple] = []
    with open(path, "r") as fh:
        for line in fh:
            toks = line.split()
            if not toks:
                continue
            pre = toks[0]
            if pre == "v":
                p = np.array([float(toks[1]), float(toks[2]), float(toks[3]), 1.0])
                q = M @ p
                P.append(q[:3] / q[3])
            elif pre == "vt":
                UV.append((float(toks[1]), float(toks[2])))
            elif pre == "vn":
                n = Minv_t @ np.array([float(toks[1]), float(toks[2]), float(toks[3])])
                N.append(n / np.linalg.norm(n))
            elif pre == "f":
                fv = toks[1:5]
                keys = []
                for s in fv:
                    parts = s.split("/")
                    if len(parts) < 1 or len(parts) > 3:
                        raise SceneError(f"Invalid OBJ vertex {s!r}")
                    pi = int(parts[0])
                    ti = int(parts[1]) if len(parts) > 1 and parts[1] else 0
                    ni = int(parts[2]) if len(parts) > 2 and parts[2] else 0
                    keys.append((pi, ti, ni))
                tri = keys[:3] + ([keys[3], keys[0], keys[2]] if len(keys) == 4 else [])
                for k in tri:
                    if k not in vmap:
                        vmap[k] = len(verts)
                        verts.append(k)
                    F.append(vmap[k])
    Parr = np.asarray(P, dtype=np.float32).reshape(-1, 3)
    positions = np.array([Parr[k[0] - 1] for k in verts], dtype=np.float32).reshape(-1, 3)
    normals = None
    if N:
        Narr = np.asarray(N, dtype=np.float32)
        normals = np.array([Narr[k[2] - 1] for k in verts], dtype=np.float32).reshape(-1, 3)
    uvs = None
    if UV:
        UVarr = np.asarray(UV, dtype=np.float32)
        uvs = np.array([UVarr[k[1] - 1] for k in verts], dtype=np.float32).reshape(-1, 2)
    indices = np.asarray(F, dtype=np.uint32).reshape(-1, 3)
    bbox = np.stack([Parr.min(0), Parr.max(0)]) if len(Parr) else None
    return positions, indices, normals, bbox, uvs


# ----------------------------------------------------------------------- XML
def _props(node: ET.Element) -> Dict[str, object]:
    out: Dict[str, object] = {}
    for ch in node:
        name = ch.attrib.get("name")
        if ch.tag == "float":
            out[name] = float(np.float32(ch.attrib["value"]))
        elif ch.tag == "integer":
            out[name] = int(ch.attrib["value"])
        elif ch.tag == "boolean":
            out[name] = ch.attrib["value"].strip().lower() == "true"
        elif ch.tag == "string":
            out[name] = ch.attrib["value"]
        elif ch.tag in ("color", "point", "vector"):
            out[name] = [float(x) for x in _vec3(ch.attrib["value"])]
        elif ch.tag == "transform":
            out[name] = parse_transform(ch)
    return out


def _transmits(d: Optional[BSDFDesc]) -> bool:
    """Whether a BSDF has a transmission lobe; coatings inherit their nested
    BSDF's lobes (src/bsdf/RoughCoatingBSDF.cpp:317)."""
    if d is None:
        return False
    if d.type in (BSDF_DIELECTRIC, BSDF_ROUGH_DIELECTRIC):
        return True
    return _transmits(d.nested) or _transmits(d.nested2)


# XML names of the textured parameters each BSDF accepts (the plugins' AddChild)
_TEX_NAMES = {
    BSDF_DIFFUSE: {"albedo": "kd"},
    BSDF_ROUGH_DIFFUSE: {"albedo": "kd", "alpha": "alpha_u"},
    BSDF_CONDUCTOR: {"ks": "ks"},
    BSDF_DIELECTRIC: {"ksReflect": "ks", "ksRefract": "ks_refract"},
    BSDF_PLASTIC: {"kd": "kd", "ks": "ks"},
    BSDF_ROUGH_CONDUCTOR: {"ks": "ks", "alpha": "alpha_u", "alphaU": "alpha_u", "alphaV": "alpha_v"},
    BSDF_ROUGH_DIELECTRIC: {"ksReflect": "ks", "ksRefract": "ks_refract", "alpha": "alpha_u", "alphaU": "alpha_u",
                            "alphaV": "alpha_v"},
    BSDF_ROUGH_PLASTIC: {"kd": "kd", "ks": "ks", "alpha": "alpha_u"},
    BSDF_ROUGH_COATING: {"ks": "ks", "sigmaA": "sigma_a", "alpha": "alpha_u"},
    BSDF_COATING: {"ks": "ks", "sigmaA": "sigma_a"},
}


_XML_BASE = ["."]   # directory of the scene file being parsed (bitmap file names resolve against it)


def _bitmap_from_xml(d: TextureDesc, p: dict) -> TextureDesc:
    """BitmapTexture ctor (src/texture/BitmapTexture.cpp:7): the image decoded
    by the library like stbi_load (hikari_b200.image_load)."""
    from hikari_b200 import image_load

    d.gamma = float(p.get("gamma", 1.0))

    def wrap(w):
        if w not in WRAP_NAMES:
            raise SceneError(f"Illegal wrap mode [{w}].")
        return WRAP_NAMES[w]

    if p.get("wrapMode", ""):
        d.wrap_u = d.wrap_v = wrap(p["wrapMode"])
    else:
        d.wrap_u, d.wrap_v = wrap(p.get("uWrapMode", "repeat")), wrap(p.get("vWrapMode", "repeat"))
    ft = p.get("filterType", "ewa")
    if ft not in FILTER_NAMES:
        raise SceneError(f"Illegal filter type [{ft}].")
    d.filter = FILTER_NAMES[ft]
    d.max_anisotropy = float(p.get("maxAnisotropy", 20.0))
    ch = p.get("channel", "rgb")
    if ch not in ("r", "rgb"):
        raise SceneError(f"Illegal channel [{ch}].")
    d.channels = 1 if ch == "r" else 3
    d.pixels = image_load(os.path.join(_XML_BASE[-1], p["filename"]), d.channels)
    return d


def _texture_from_xml(node: ET.Element) -> TextureDesc:
    """CheckerboardTexture / GridTexture / ScaleTexture / BitmapTexture ctors (src/texture/*.cpp)."""
    t = node.attrib["type"]
    if t not in TEX_TYPE_NAMES:
        raise SceneError(f"texture type {t!r} is not supported by the CUDA pathMIS core")
    p = _props(node)
    d = TextureDesc(kind=TEX_TYPE_NAMES[t])
    d.uv_scale = [float(p.get("uScale", 1.0)), float(p.get("vScale", 1.0))]
    d.uv_offset = [float(p.get("uOffset", 0.0)), float(p.get("vOffset", 0.0))]
    if d.kind == TEX_BITMAP:
        return _bitmap_from_xml(d, p)
    if d.kind == TEX_WIREFRAME:   # WireframeTexture ctor (src/texture/WireframeTexture.cpp:10)
        d.a = [float(c) for c in p.get("interiorColor", [0.5, 0.5, 0.5])]
        d.b = [float(c) for c in p.get("edgeColor", [0.1, 0.1, 0.1])]
        d.width = float(p.get("edgeWidth", 0.0))
        d.scale = float(p.get("transitionWidth", 0.5))
        return d
    if d.kind == TEX_CURVATURE:   # CurvatureTexture ctor (src/texture/CurvatureTexture.cpp:9)
        d.a = [float(c) for c in p.get("positiveColor", [1.0, 0.0, 0.0])]
        d.b = [float(c) for c in p.get("negativeColor", [0.0, 0.0, 1.0])]
        d.scale = float(p.get("scale", 1.0))
        ct = p.get("curvatureType", "")
        if ct not in ("gaussian", "mean"):
            raise SceneError(f"Unexpected curvature type <{ct}>.")
        d.count = 1 if ct == "gaussian" else 0
        return d
    if d.kind == TEX_CHECKERBOARD:
        d.count = int(p.get("blocks", 10))
        d.a = [float(c) for c in p.get("colorA", [0.4, 0.4, 0.4])]
        d.b = [float(c) for c in p.get("colorB", [0.2, 0.2, 0.2])]
    elif d.kind == TEX_GRID:
        d.count = int(p.get("lines", 10))
        d.a = [float(c) for c in p.get("lineColor", [0.4, 0.4, 0.4])]
        d.b = [float(c) for c in p.get("backgroundColor", [0.2, 0.2, 0.2])]
        d.width = float(p.get("lineWidth", 0.01))
    else:
        if "scale" not in p:
            raise SceneError("Property 'scale' is missing!")
        d.scale = float(p["scale"])
        nested = [c for c in node if c.tag == "texture"]
        if len(nested) != 1:
            raise SceneError("ScaleTexture needs exactly one nested texture")
        d.nested = _texture_from_xml(nested[0])
    if d.kind != TEX_SCALE and d.count <= 0:
        raise SceneError("texture block / line count must be positive")
    return d


def _bsdf_from_xml(node: ET.Element) -> BSDFDesc:
    t = node.attrib["type"]
    if t not in BSDF_TYPE_NAMES:
        raise SceneError(f"BSDF type {t!r} is not supported by the CUDA pathMIS core")
    p = _props(node)
    d = BSDFDesc(type=BSDF_TYPE_NAMES[t])
    dist = p.get("type", "beckmann")
    if dist not in ("beckmann", "ggx"):
        raise SceneError(f"Unexpected distribution type : {dist}")
    d.distribution = GGX if dist == "ggx" else BECKMANN
    if d.type == BSDF_DIFFUSE:
        d.kd = p.get("albedo", [0.5, 0.5, 0.5])
    elif d.type == BSDF_ROUGH_CONDUCTOR:
        d.int_ior = p.get("intIOR", 1.5046)
        d.ext_ior = p.get("extIOR", AIR_IOR)
        d.k = p.get("k", [1.0, 1.0, 1.0])
        d.ks = p.get("ks", [1.0, 1.0, 1.0])
    elif d.type == BSDF_ROUGH_DIELECTRIC:
        d.int_ior = p.get("intIOR", 1.5046)
        d.ext_ior = p.get("extIOR", AIR_IOR)
        d.ks = p.get("ksReflect", [1.0, 1.0, 1.0])
        d.ks_refract = p.get("ksRefract", [1.0, 1.0, 1.0])
    elif d.type == BSDF_ROUGH_PLASTIC:
        d.int_ior = p.get("intIOR", 1.49)
        d.ext_ior = p.get("extIOR", AIR_IOR)
        d.ks = p.get("ks", [1.0, 1.0, 1.0])
        d.kd = p.get("kd", [0.5, 0.5, 0.5])
        d.nonlinear = bool(p.get("nonlinear", False))
    elif d.type == BSDF_CONDUCTOR:   # src/bsdf/ConductorBSDF.cpp:11
        d.int_ior = p.get("intIOR", 1.5046)
        d.ext_ior = p.get("extIOR", AIR_IOR)
        d.k = p.get("k", [1.0, 1.0, 1.0])
        d.ks = p.get("ks", [1.0, 1.0, 1.0])
    elif d.type == BSDF_DIELECTRIC:   # src/bsdf/DielectricBSDF.cpp:9
        d.int_ior = p.get("intIOR", 1.5046)
        d.ext_ior = p.get("extIOR", AIR_IOR)
        d.ks = p.get("ksReflect", [1.0, 1.0, 1.0])
        d.ks_refract = p.get("ksRefract", [1.0, 1.0, 1.0])
    elif d.type == BSDF_PLASTIC:   # src/bsdf/PlasticBSDF.cpp:10
        d.int_ior = p.get("intIOR", 1.5046)
        d.ext_ior = p.get("extIOR", AIR_IOR)
        d.ks = p.get("ks", [1.0, 1.0, 1.0])
        d.kd = p.get("kd", [0.5, 0.5, 0.5])
        d.nonlinear = bool(p.get("nonlinear", False))
    elif d.type == BSDF_TWO_SIDED:   # src/bsdf/TwoSidedBSDF.cpp:86-125
        nested = [c for c in node if c.tag == "bsdf"]
        if not nested:
            raise SceneError("TwoSidedBSDF needs at least one nested BSDF!")
        if len(nested) > 2:
            raise SceneError("TwoSidedBSDF: tried to specify the third nested BSDF")
        d.nested = _bsdf_from_xml(nested[0])
        d.nested2 = _bsdf_from_xml(nested[1]) if len(nested) == 2 else None
        if _transmits(d.nested) or _transmits(d.nested2):
            raise SceneError("Only BSDF without transmission can be nested!")
    elif d.type == BSDF_ROUGH_COATING:
        d.int_ior = p.get("intIOR", 1.49)
        d.ext_ior = p.get("extIOR", AIR_IOR)
        d.ks = p.get("ks", [1.0, 1.0, 1.0])
        d.sigma_a = p.get("sigmaA", [0.0, 0.0, 0.0])
        d.thickness = p.get("thickness", 1.0)
        nested = [c for c in node if c.tag == "bsdf"]
        if len(nested) != 1:
            raise SceneError("RoughCoatingBSDF needs a nested BSDF!")
        d.nested = _bsdf_from_xml(nested[0])
    elif d.type == BSDF_COATING:   # src/bsdf/CoatingBSDF.cpp:9-23, Activate :255
        d.int_ior = p.get("intIOR", 1.49)
        d.ext_ior = p.get("extIOR", AIR_IOR)
        d.ks = p.get("ks", [1.0, 1.0, 1.0])
        d.sigma_a = p.get("sigmaA", [0.0, 0.0, 0.0])
        d.thickness = p.get("thickness", 1.0)
        nested = [c for c in node if c.tag == "bsdf"]
        if not nested:
            raise SceneError("CoatingBSDF needs a nested BSDF!")
        if len(nested) > 1:
            raise SceneError("CoatingBSDF: tried to specify multiple nested BSDF")
        d.nested = _bsdf_from_xml(nested[0])
    elif d.type == BSDF_ROUGH_DIFFUSE:   # src/bsdf/RoughDiffuseBSDF.cpp:10-17
        d.kd = p.get("albedo", [0.5, 0.5, 0.5])
        d.fast_approx = bool(p.get("fastApprox", False))
    elif d.type in (BSDF_BUMP_MAP, BSDF_NORMAL_MAP):   # src/bsdf/{BumpMap,NormalMap}BSDF.cpp AddChild / Activate
        nested = [c for c in node if c.tag == "bsdf"]
        maps = [c for c in node if c.tag == "texture"]
        if len(nested) > 1:
            raise SceneError(f"{t}: tried to specify multiple nested BSDF")
        if len(maps) > 1:
            raise SceneError(f"{t}: tried to specify multiple map textures")
        if not nested or not maps:
            raise SceneError(f"{t} needs a nested BSDF and a map texture")
        d.nested = _bsdf_from_xml(nested[0])
        d.textures["kd"] = _texture_from_xml(maps[0])
        return d
    if d.type in (BSDF_ROUGH_CONDUCTOR, BSDF_ROUGH_DIELECTRIC):
        d.anisotropic = bool(p.get("as", False))
    if d.anisotropic:
        d.alpha_u = p.get("alphaU", 0.1)
        d.alpha_v = p.get("alphaV", 0.1)
    else:
        d.alpha_u = d.alpha_v = p.get("alpha", 0.2 if d.type == BSDF_ROUGH_DIFFUSE else 0.1)
    if d.type == BSDF_ROUGH_DIFFUSE:
        d.alpha_u = d.alpha_v = min(max(d.alpha_u, 5e-4), 1.0)   # Clamp(alpha, MIN_ALPHA, MAX_ALPHA)
    for c in node:
        if c.tag != "texture":
            continue
        name = c.attrib.get("name", "")
        slot = _TEX_NAMES.get(d.type, {}).get(name)
        if slot is None:
            raise SceneError(f"{t}: a texture named {name!r} is not supported")
        if slot in d.textures:
            raise SceneError(f"{t}: tried to specify multiple {name} textures")
        d.textures[slot] = _texture_from_xml(c)
    return d


def parse_scene_node(node: ET.Element, base_dir: str, env_loader=None) -> SceneDesc:
    _XML_BASE.append(base_dir)
    try:
        return _parse_scene_node(node, base_dir, env_loader)
    finally:
        _XML_BASE.pop()


def _parse_scene_node(node: ET.Element, base_dir: str, env_loader=None) -> SceneDesc:
    sd = SceneDesc()
    p = _props(node)
    sd.background = p.get("background", [0.0, 0.0, 0.0])
    sd.force_background = bool(p.get("forceBackground", False))
    n_emit = 0
    for ch in node:
        if ch.tag == "integrator":
            sd.integrator = ch.attrib["type"]
            ip = _props(ch)
            if "depth" not in ip:
                raise SceneError("Property 'depth' is missing")
            sd.depth = int(ip["depth"])
        elif ch.tag == "camera":
            cp = _props(ch)
            cam = CameraDesc()
            cam.width = int(cp.get("width", 1280))
            cam.height = int(cp.get("height", 720))
            cam.fov = float(cp.get("fov", 30.0))
            cam.near_clip = float(cp.get("nearClip", 1e-4))
            cam.far_clip = float(cp.get("farClip", 1e4))
            if "toWorld" in cp:
                cam.to_world = cp["toWorld"]
            for f in ch:
                if f.tag == "rfilter":
                    fp = _props(f)
                    kind = FILTER_KINDS[f.attrib["type"]]
                    if kind == 0:
                        sd.filter = FilterDesc(0, 0.5)
                    elif kind == 1:
                        sd.filter = FilterDesc(1, 1.0)
                    elif kind == 2:
                        sd.filter = FilterDesc(2, fp.get("radius", 2.0), fp.get("stddev", 0.5))
                    else:
                        sd.filter = FilterDesc(3, fp.get("radius", 2.0), fp.get("B", 1 / 3), fp.get("C", 1 / 3))
            sd.camera = cam
        elif ch.tag == "sampler":
            sd.spp = int(_props(ch).get("sampleCount", 1))
        elif ch.tag == "mesh":
            mp = _props(ch)
            fn = os.path.join(base_dir, mp["filename"])
            pos, idx, nrm, bbox, uv = load_obj(fn, mp.get("toWorld"))
            bs = [c for c in ch if c.tag == "bsdf"]
            bsdf = _bsdf_from_xml(bs[0]) if bs else BSDFDesc()
            em = [c for c in ch if c.tag == "emitter"]
            rad = None
            if em:
                if em[0].attrib["type"] != "area":
                    raise SceneError("only area emitters attach to meshes")
                rad = _props(em[0])["radiance"]
                n_emit += 1
            sd.meshes.append(MeshDesc(pos, idx, bsdf, nrm, rad, bbox, uv))
        elif ch.tag == "emitter":
            et = ch.attrib["type"]
            ep = _props(ch)
            if et in ("point", "directional"):   # src/emitter/PointLight.cpp:8, DirectionalLight.cpp:8
                try:
                    color = ep["power" if et == "point" else "irradiance"]
                    vec = ep["position" if et == "point" else "direction"]
                except KeyError as e:
                    raise SceneError(f"Property {e.args[0]!r} is missing!") from None
                sd.lights.append(LightDesc(et, [float(c) for c in color], [float(c) for c in vec], n_emit))
                n_emit += 1
                continue
            if et not in ("env", "constant"):
                raise SceneError(f"emitter type {et!r} is not supported by the CUDA pathMIS core")
            if sd.env is not None or sd.env_constant is not None:
                raise SceneError("Only one environment emiiter is allowed for the entire scene")
            if et == "constant":   # src/emitter/ConstantLight.cpp:8
                if "radiance" not in ep:
                    raise SceneError("Property 'radiance' is missing!")
                sd.env_constant = [float(c) for c in ep["radiance"]]
            else:
                if env_loader is None:
                    raise SceneError("no environment-map loader given")
                rgb = env_loader(os.path.join(base_dir, ep["filename"]))
                sd.env = EnvDesc(rgb, ep.get("toWorld", np.eye(4, dtype=np.float32)), ep.get("scale", 1.0))
            sd.env_emitter_index = n_emit
            n_emit += 1
        elif ch.tag == "accelerator" or ch.tag == "acceleration":
            pass
    return sd


def parse_xml(path: str, env_loader=None) -> List[SceneDesc]:
    """Parse a scene file: one <scene>, or a <test> holding several scenes.
    Returns the list of scenes and, for tests, attaches ``references``."""
    root = ET.parse(path).getroot()
    base = os.path.dirname(os.path.abspath(path))
    if root.tag == "scene":
        return [parse_scene_node(root, base, env_loader)]
    scenes = [parse_scene_node(n, base, env_loader) for n in root if n.tag == "scene"]
    refs = [c for c in root if c.tag == "string" and c.attrib.get("name") == "references"]
    if refs:
        vals = [float(v) for v in refs[0].attrib["value"].replace(",", " ").split() if v]
        for s, r in zip(scenes, vals):
            s.reference = r  # type: ignore[attr-defined]
    return scenes
