"""Write a :class:`SceneDesc` as a Hikari scene: one XML file in the
reference's format (src/core/Parser.cpp), an OBJ file per mesh and an
uncompressed FLOAT OpenEXR file for an environment map, so that the
reference renderer (and this library's own XML loader) read the same scene
the generators describe.

Floats are written with nine significant digits, so every float32 value (OBJ
positions, matrices, colours) reads back bit for bit.  Meshes are written in
world space with an identity ``toWorld``; faces keep their order, so triangle
ids agree with the description's.  Emitters are written in the description's
Scene::AddChild order (:meth:`SceneDesc.build_steps`).

Not expressible in the reference's format, and rejected: per-channel
conductor ``eta`` (the reference's conductors take a scalar intIOR / extIOR),
and textured parameters (bitmaps would need an image file per texture).
"""
from __future__ import annotations

import os
import struct
from typing import List, Optional

import numpy as np

from .scenedesc import (BSDF_BUMP_MAP, BSDF_COATING, BSDF_CONDUCTOR, BSDF_DIELECTRIC, BSDF_DIFFUSE, BSDF_MIRROR,
                        BSDF_NORMAL_MAP, BSDF_PLASTIC, BSDF_ROUGH_COATING, BSDF_ROUGH_CONDUCTOR,
                        BSDF_ROUGH_DIELECTRIC, BSDF_ROUGH_DIFFUSE, BSDF_ROUGH_PLASTIC, BSDF_TWO_SIDED, BSDF_TYPE_NAMES,
                        GGX, BSDFDesc, SceneDesc, SceneError)

_TYPE_NAME = {v: k for k, v in BSDF_TYPE_NAMES.items()}
_FILTER_NAME = {0: "box", 1: "tent", 2: "gaussian", 3: "mitchell"}


def _f(x) -> str:
    return "%.9g" % float(np.float32(x))


def _col(v) -> str:
    return " ".join(_f(c) for c in v)


def write_exr(path: str, rgb: np.ndarray) -> None:
    """Uncompressed scanline OpenEXR with FLOAT B, G, R channels (H x W x 3)."""
    rgb = np.ascontiguousarray(rgb, dtype=np.float32)
    h, w = rgb.shape[:2]

    def attr(name, typ, data):
        return name.encode() + b"\0" + typ.encode() + b"\0" + struct.pack("<I", len(data)) + data

    ch = b"".join(c + b"\0" + struct.pack("<iIii", 2, 0, 1, 1) for c in (b"B", b"G", b"R")) + b"\0"
    box = struct.pack("<iiii", 0, 0, w - 1, h - 1)
    hdr = struct.pack("<II", 20000630, 2)
    hdr += attr("channels", "chlist", ch)
    hdr += attr("compression", "compression", b"\0")
    hdr += attr("dataWindow", "box2i", box)
    hdr += attr("displayWindow", "box2i", box)
    hdr += attr("lineOrder", "lineOrder", b"\0")
    hdr += attr("pixelAspectRatio", "float", struct.pack("<f", 1.0))
    hdr += attr("screenWindowCenter", "v2f", struct.pack("<ff", 0.0, 0.0))
    hdr += attr("screenWindowWidth", "float", struct.pack("<f", 1.0))
    hdr += b"\0"
    line = 8 + w * 12
    first = len(hdr) + 8 * h
    offsets = np.arange(h, dtype=np.uint64) * line + first
    with open(path, "wb") as f:
        f.write(hdr)
        f.write(offsets.tobytes())
        planar = np.stack([rgb[..., 2], rgb[..., 1], rgb[..., 0]], 1)   # h x 3 x w
        for y in range(h):
            f.write(struct.pack("<iI", y, w * 12))
            f.write(planar[y].tobytes())


def write_obj(path: str, positions: np.ndarray, indices: np.ndarray, normals: Optional[np.ndarray] = None,
              uv: Optional[np.ndarray] = None) -> None:
    P = np.asarray(positions, np.float32)
    F = np.asarray(indices, np.int64) + 1
    lines: List[str] = ["v %s %s %s" % tuple(_f(c) for c in p) for p in P]
    if uv is not None:
        lines += ["vt %s %s" % tuple(_f(c) for c in t) for t in np.asarray(uv, np.float32)]
    if normals is not None:
        lines += ["vn %s %s %s" % tuple(_f(c) for c in n) for n in np.asarray(normals, np.float32)]
    if uv is not None and normals is not None:
        lines += ["f %d/%d/%d %d/%d/%d %d/%d/%d" % (a, a, a, b, b, b, c, c, c) for a, b, c in F]
    elif uv is not None:
        lines += ["f %d/%d %d/%d %d/%d" % (a, a, b, b, c, c) for a, b, c in F]
    elif normals is not None:
        lines += ["f %d//%d %d//%d %d//%d" % (a, a, b, b, c, c) for a, b, c in F]
    else:
        lines += ["f %d %d %d" % tuple(t) for t in F]
    with open(path, "w") as f:
        f.write("\n".join(lines) + "\n")


def _bsdf_xml(d: BSDFDesc, ind: str) -> str:
    if d.textures:
        raise SceneError("textured BSDF parameters are not written")
    if d.type in (BSDF_BUMP_MAP, BSDF_NORMAL_MAP):
        raise SceneError("bump and normal maps are not written")
    t = d.type
    out = [f'{ind}<bsdf type="{_TYPE_NAME[t]}">']
    p = ind + "\t"

    def col(name, v):
        out.append(f'{p}<color name="{name}" value="{_col(v)}"/>')

    def flt(name, v):
        out.append(f'{p}<float name="{name}" value="{_f(v)}"/>')

    if t in (BSDF_ROUGH_CONDUCTOR, BSDF_ROUGH_DIELECTRIC, BSDF_ROUGH_PLASTIC, BSDF_ROUGH_COATING):
        out.append(f'{p}<string name="type" value="{"ggx" if d.distribution == GGX else "beckmann"}"/>')
        if d.anisotropic:
            out.append(f'{p}<boolean name="as" value="true"/>')
            flt("alphaU", d.alpha_u)
            flt("alphaV", d.alpha_v)
        else:
            flt("alpha", d.alpha_u)
    if t == BSDF_ROUGH_DIFFUSE:
        flt("alpha", d.alpha_u)
        if d.fast_approx:
            out.append(f'{p}<boolean name="fastApprox" value="true"/>')
    if t in (BSDF_DIFFUSE, BSDF_ROUGH_DIFFUSE):
        col("albedo", d.kd)
    if t in (BSDF_ROUGH_CONDUCTOR, BSDF_CONDUCTOR, BSDF_ROUGH_DIELECTRIC, BSDF_DIELECTRIC, BSDF_ROUGH_PLASTIC,
             BSDF_PLASTIC, BSDF_ROUGH_COATING, BSDF_COATING):
        if d.eta is not None:
            raise SceneError("a per-channel conductor eta has no reference XML form")
        flt("intIOR", d.int_ior)
        flt("extIOR", d.ext_ior)
    if t in (BSDF_ROUGH_CONDUCTOR, BSDF_CONDUCTOR):
        col("k", d.k)
        col("ks", d.ks)
    if t in (BSDF_ROUGH_DIELECTRIC, BSDF_DIELECTRIC):
        col("ksReflect", d.ks)
        col("ksRefract", d.ks_refract)
    if t in (BSDF_ROUGH_PLASTIC, BSDF_PLASTIC):
        col("ks", d.ks)
        col("kd", d.kd)
        if d.nonlinear:
            out.append(f'{p}<boolean name="nonlinear" value="true"/>')
    if t in (BSDF_ROUGH_COATING, BSDF_COATING):
        col("ks", d.ks)
        col("sigmaA", d.sigma_a)
        flt("thickness", d.thickness)
    if d.nested is not None:
        out.append(_bsdf_xml(d.nested, p))
    if t == BSDF_TWO_SIDED and d.nested2 is not None:
        out.append(_bsdf_xml(d.nested2, p))
    if t == BSDF_MIRROR:
        return f'{ind}<bsdf type="mirror"/>'
    out.append(f"{ind}</bsdf>")
    return "\n".join(out)


def _matrix(name: str, M, ind: str) -> str:
    vals = " ".join(_f(x) for x in np.asarray(M, np.float32).reshape(16))
    return f'{ind}<transform name="{name}">\n{ind}\t<matrix value="{vals}"/>\n{ind}</transform>'


def write_scene_xml(sd: SceneDesc, out_dir: str, name: str = "scene", spp: Optional[int] = None,
                    accel: str = "hlbvh", leaf_size: int = 10) -> str:
    """Write sd (meshes, emitters, camera, filter, sampler, pathMIS depth) to
    out_dir/name.xml with its OBJ / EXR files beside it; returns the XML path."""
    os.makedirs(out_dir, exist_ok=True)
    lines = ["<scene>", '\t<integrator type="%s">' % sd.integrator,
             f'\t\t<integer name="depth" value="{int(sd.depth)}"/>', "\t</integrator>"]
    if sd.force_background or any(float(c) != 0.0 for c in sd.background):
        lines.append(f'\t<color name="background" value="{_col(sd.background)}"/>')
        if sd.force_background:
            lines.append('\t<boolean name="forceBackground" value="true"/>')
    cam = sd.camera
    f = sd.filter
    lines += ['\t<camera type="perspective">', f'\t\t<float name="fov" value="{_f(cam.fov)}"/>',
              f'\t\t<integer name="width" value="{cam.width}"/>', f'\t\t<integer name="height" value="{cam.height}"/>',
              f'\t\t<float name="nearClip" value="{_f(cam.near_clip)}"/>',
              f'\t\t<float name="farClip" value="{_f(cam.far_clip)}"/>', _matrix("toWorld", cam.to_world, "\t\t")]
    if f.kind == 2:
        lines += ['\t\t<rfilter type="gaussian">', f'\t\t\t<float name="radius" value="{_f(f.radius)}"/>',
                  f'\t\t\t<float name="stddev" value="{_f(f.p0)}"/>', "\t\t</rfilter>"]
    elif f.kind == 3:
        lines += ['\t\t<rfilter type="mitchell">', f'\t\t\t<float name="radius" value="{_f(f.radius)}"/>',
                  f'\t\t\t<float name="B" value="{_f(f.p0)}"/>', f'\t\t\t<float name="C" value="{_f(f.p1)}"/>',
                  "\t\t</rfilter>"]
    else:
        lines.append(f'\t\t<rfilter type="{_FILTER_NAME[f.kind]}"/>')
    lines.append("\t</camera>")
    lines += ['\t<sampler type="independent">',
              f'\t\t<integer name="sampleCount" value="{int(spp if spp is not None else sd.spp)}"/>', "\t</sampler>"]
    if accel == "bruto":
        lines.append('\t<acceleration type="bruto"/>')
    else:
        lines += [f'\t<acceleration type="{accel}">', f'\t\t<integer name="leafSize" value="{int(leaf_size)}"/>',
                  "\t</acceleration>"]
    for kind, i in sd.build_steps():
        if kind == "mesh":
            m = sd.meshes[i]
            fn = f"{name}_mesh{i}.obj"
            write_obj(os.path.join(out_dir, fn), m.positions, m.indices, m.normals, m.uv)
            lines += ['\t<mesh type="obj">', f'\t\t<string name="filename" value="{fn}"/>', _bsdf_xml(m.bsdf, "\t\t")]
            if m.radiance is not None:
                lines += ['\t\t<emitter type="area">', f'\t\t\t<color name="radiance" value="{_col(m.radiance)}"/>',
                          "\t\t</emitter>"]
            lines.append("\t</mesh>")
        elif kind == "env":
            if sd.env_constant is not None:
                lines += ['\t<emitter type="constant">',
                          f'\t\t<color name="radiance" value="{_col(sd.env_constant)}"/>', "\t</emitter>"]
            else:
                fn = f"{name}_env.exr"
                write_exr(os.path.join(out_dir, fn), sd.env.rgb)
                lines += ['\t<emitter type="env">', f'\t\t<string name="filename" value="{fn}"/>',
                          f'\t\t<float name="scale" value="{_f(sd.env.scale)}"/>',
                          _matrix("toWorld", sd.env.to_world, "\t\t"), "\t</emitter>"]
        else:
            l = sd.lights[i]
            if l.kind == "point":
                lines += ['\t<emitter type="point">', f'\t\t<color name="power" value="{_col(l.color)}"/>',
                          f'\t\t<point name="position" value="{_col(l.vector)}"/>', "\t</emitter>"]
            else:
                lines += ['\t<emitter type="directional">', f'\t\t<color name="irradiance" value="{_col(l.color)}"/>',
                          f'\t\t<vector name="direction" value="{_col(l.vector)}"/>', "\t</emitter>"]
    lines.append("</scene>")
    path = os.path.join(out_dir, name + ".xml")
    with open(path, "w") as fh:
        fh.write("\n".join(lines) + "\n")
    return path
