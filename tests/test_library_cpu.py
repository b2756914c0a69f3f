"""The C-ABI library on a machine without a GPU: it builds for sm_100a, loads,
exports every function include/hikari_b200.h declares, and its host-only
parts (the XML plugin layer, EXR I/O, argument checks) work without a device."""
import ctypes as C
import os
import re

import numpy as np
import pytest

import hikari_b200 as hk
from hikari_b200 import build as hkbuild
from hikari_b200.scenedesc import parse_xml

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "hikari_b200.h")


@pytest.fixture(scope="module")
def L():
    hkbuild.build()
    return hk.lib()


def declared_functions():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"^\s*(?:const\s+)?\w+\s*\*?\s*(hk_\w+)\s*\(", src, flags=re.M)))


def test_header_declares_the_boundary():
    names = declared_functions()
    for must in ["hk_scene_create", "hk_scene_build", "hk_render", "hk_render_batch", "hk_render_image_static",
                 "hk_trace", "hk_bsdf_batch", "hk_server_create", "hk_job_submit", "hk_job_poll", "hk_job_cancel",
                 "hk_wavefront_autotune", "hk_scene_load_xml", "hk_exr_read"]:
        assert must in names
    assert len(names) >= 35


def test_library_exports_every_declared_function(L):
    so = C.CDLL(hkbuild.LIB)
    missing = [n for n in declared_functions() if not hasattr(so, n)]
    assert not missing, f"not exported: {missing}"


def test_build_targets_sm100a():
    assert "arch=compute_100a,code=sm_100a" in " ".join(hkbuild.ARCH)
    assert "-fmad=false" in hkbuild.NVCC_FLAGS


SCENE_XML = """<?xml version="1.0"?>
<scene>
  <integrator type="pathMIS"><integer name="depth" value="12"/></integrator>
  <sampler type="independent"><integer name="sampleCount" value="9"/></sampler>
  <camera type="perspective">
    <transform name="toWorld"><lookat origin="0, 1, 4" target="0, 0.5, 0" up="0, 1, 0"/></transform>
    <float name="fov" value="35"/>
    <integer name="width" value="40"/><integer name="height" value="30"/>
  </camera>
  <mesh type="obj">
    <string name="filename" value="quad.obj"/>
    <bsdf type="roughPlastic"><float name="alpha" value="0.2"/><color name="kd" value="0.4, 0.5, 0.6"/></bsdf>
  </mesh>
  <mesh type="obj">
    <string name="filename" value="quad.obj"/>
    <transform name="toWorld"><translate value="0, 3, 0"/></transform>
    <bsdf type="diffuse"/>
    <emitter type="area"><color name="radiance" value="5, 5, 5"/></emitter>
  </mesh>
  <mesh type="obj">
    <string name="filename" value="quad.obj"/>
    <transform name="toWorld"><translate value="0, -1, 0"/></transform>
    <bsdf type="roughCoating">
      <float name="alpha" value="0.2"/>
      <bsdf type="roughConductor"><float name="alpha" value="0.3"/></bsdf>
    </bsdf>
  </mesh>
</scene>
"""
QUAD_OBJ = "v -1 0 -1\nv 1 0 -1\nv 1 0 1\nv -1 0 1\nf 1 4 3 2\n"


def test_xml_plugin_layer_matches_python_parser(L, tmp_path):
    (tmp_path / "quad.obj").write_text(QUAD_OBJ)
    path = str(tmp_path / "scene.xml")
    open(path, "w").write(SCENE_XML)
    info, depth, spp = hk.parse_xml_info(path)
    sd = parse_xml(path)[0]
    assert (depth, spp) == (12, 9) == (sd.depth, sd.spp)
    assert info.n_meshes == len(sd.meshes) == 3
    assert info.n_triangles == sum(len(m.indices) for m in sd.meshes) == 6
    assert info.n_emitters == 1
    assert info.n_bsdfs == 4          # plastic, diffuse, coating + its nested conductor


def test_xml_errors_are_reported(L, tmp_path):
    bad = tmp_path / "bad.xml"
    bad.write_text('<scene><bsdf type="noSuchBSDF"/></scene>')
    with pytest.raises(hk.HikariError):
        hk.parse_xml_info(str(bad))
    with pytest.raises(hk.HikariError):
        hk.parse_xml_info(str(tmp_path / "missing.xml"))


def test_exr_roundtrip(L, tmp_path):
    rng = np.random.default_rng(0)
    img = rng.uniform(0, 100, (7, 13, 3)).astype(np.float32)
    img[0, 0] = [0.0, 1e-30, 3.4e38]
    p = str(tmp_path / "x.exr")
    hk.exr_write(p, img)
    back = hk.exr_read(p)
    assert back.shape == img.shape
    assert np.array_equal(back, img)


def test_argument_checks_without_device(L):
    h = C.c_void_p()
    assert L.hk_scene_create(C.byref(h)) == 0
    try:
        assert L.hk_scene_build(h) == -1                       # no meshes
        assert b"no meshes" in L.hk_last_error()
        d = hk.BsdfDesc()
        d.type = 14
        assert L.hk_scene_add_bsdf(h, C.byref(d), None) == -1  # unknown BSDF type (13 = normalMap is the last)
        d.type = 4
        d.nested = 3
        assert L.hk_scene_add_bsdf(h, C.byref(d), None) == -1  # coating without a nested BSDF
        assert b"nested" in L.hk_last_error()
        d.type = 9
        d.nested = -1
        assert L.hk_scene_add_bsdf(h, C.byref(d), None) == -1  # twoSided without a nested BSDF
        assert b"TwoSidedBSDF" in L.hk_last_error()
        assert L.hk_render(h, None, None, None, None) == -1    # not built
    finally:
        L.hk_scene_destroy(h)


@pytest.mark.parametrize("case", ["random", "grid", "single", "degenerate", "cornell", "spheres"])
def test_bvh_trees_are_consistent(L, case):
    """Both trees cover every triangle once and the quantised 8-wide child
    boxes contain their triangles (checked in double on the host)."""
    from hikari_b200 import scenes

    rng = np.random.default_rng(1)
    if case == "random":
        c = rng.uniform(-50, 50, (20000, 1, 3))
        tris = c + rng.normal(0, 0.5, (20000, 3, 3))
    elif case == "grid":   # axis-aligned, coplanar, zero-thickness boxes
        g = np.stack(np.meshgrid(np.arange(60), np.arange(60), indexing="ij"), -1).reshape(-1, 2).astype(np.float64)
        z = np.zeros((g.shape[0], 1))
        a = np.concatenate([g, z], 1)
        tris = np.stack([a, a + [1, 0, 0], a + [0, 1, 0]], 1)
    elif case == "single":
        tris = np.array([[[0, 0, 0], [1, 0, 0], [0, 1, 0]]], np.float64)
    elif case == "degenerate":   # many identical triangles and far outliers
        tris = np.repeat(np.array([[[0, 0, 0], [1, 0, 0], [0, 1, 0]]], np.float64), 500, 0)
        tris = np.concatenate([tris, rng.uniform(-1e4, 1e4, (50, 3, 3))])
    elif case == "cornell":
        sd = scenes.cornell_box()
        tris = np.concatenate([m.positions[m.indices] for m in sd.meshes])
    else:
        P, F = scenes.displaced_icosphere(5, 1.0, (0, 0, 0), 0.08, 3)
        tris = P[F]
    n2, n8, d8 = hk.bvh_check(tris)
    print(case, "triangles", len(tris), "binary nodes", n2, "8-wide nodes", n8, "8-wide depth", d8)
    assert n8 >= 1 and n2 >= 1
    assert 2 * d8 + 2 <= 64 or len(tris) > 1e6


SMOOTH_XML = """<?xml version="1.0"?>
<scene>
  <integrator type="pathMIS"><integer name="depth" value="8"/></integrator>
  <camera type="perspective">
    <transform name="toWorld"><lookat origin="0, 1, 4" target="0, 0.5, 0" up="0, 1, 0"/></transform>
    <integer name="width" value="16"/><integer name="height" value="16"/>
  </camera>
  <mesh type="obj"><string name="filename" value="quad.obj"/><bsdf type="mirror"/></mesh>
  <mesh type="obj"><string name="filename" value="quad.obj"/>
    <bsdf type="conductor"><float name="intIOR" value="0.3"/><color name="k" value="3, 2.5, 2"/></bsdf></mesh>
  <mesh type="obj"><string name="filename" value="quad.obj"/><bsdf type="dielectric"/></mesh>
  <mesh type="obj"><string name="filename" value="quad.obj"/>
    <bsdf type="plastic"><color name="kd" value="0.2, 0.4, 0.6"/><boolean name="nonlinear" value="true"/></bsdf></mesh>
  <mesh type="obj"><string name="filename" value="quad.obj"/>
    <bsdf type="twoSided">
      <bsdf type="roughCoating"><bsdf type="plastic"/></bsdf>
      <bsdf type="diffuse"/>
    </bsdf>
    <emitter type="area"><color name="radiance" value="1, 1, 1"/></emitter>
  </mesh>
</scene>
"""


def test_xml_smooth_and_two_sided_plugins(L, tmp_path):
    (tmp_path / "quad.obj").write_text(QUAD_OBJ)
    path = str(tmp_path / "smooth.xml")
    open(path, "w").write(SMOOTH_XML)
    info, depth, spp = hk.parse_xml_info(path)
    sd = parse_xml(path)[0]
    assert info.n_meshes == len(sd.meshes) == 5
    assert info.n_bsdfs == 8          # 4 smooth + twoSided, its coating, the coating's plastic, diffuse
    types = [m.bsdf.type for m in sd.meshes]
    assert types == [5, 6, 7, 8, 9]
    two = sd.meshes[4].bsdf
    assert two.nested.type == 4 and two.nested.nested.type == 8 and two.nested2.type == 0
    assert sd.meshes[3].bsdf.nonlinear and sd.meshes[3].bsdf.int_ior == pytest.approx(1.5046)


@pytest.mark.parametrize("body,needle", [
    ('<bsdf type="twoSided"/>', "at least one nested"),
    ('<bsdf type="twoSided"><bsdf type="dielectric"/></bsdf>', "transmission"),
    ('<bsdf type="twoSided"><bsdf type="roughCoating"><bsdf type="roughDielectric"/></bsdf></bsdf>', "transmission"),
    ('<bsdf type="twoSided"><bsdf type="diffuse"/><bsdf type="diffuse"/><bsdf type="diffuse"/></bsdf>', "third"),
])
def test_xml_two_sided_errors(L, tmp_path, body, needle):
    from hikari_b200.scenedesc import SceneError

    (tmp_path / "quad.obj").write_text(QUAD_OBJ)
    path = str(tmp_path / "bad.xml")
    open(path, "w").write(f'<scene><mesh type="obj"><string name="filename" value="quad.obj"/>{body}</mesh></scene>')
    with pytest.raises(hk.HikariError, match=needle):
        hk.parse_xml_info(path)
    with pytest.raises(SceneError, match=needle):
        parse_xml(path)


LIGHTS_XML = """<?xml version="1.0"?>
<scene>
  <integrator type="pathMIS"><integer name="depth" value="8"/></integrator>
  <camera type="perspective">
    <transform name="toWorld"><lookat origin="0, 1, 4" target="0, 0.5, 0" up="0, 1, 0"/></transform>
    <integer name="width" value="16"/><integer name="height" value="16"/>
  </camera>
  <emitter type="point"><color name="power" value="10, 10, 10"/><point name="position" value="0, 3, 0"/></emitter>
  <mesh type="obj"><string name="filename" value="quad.obj"/>
    <bsdf type="coating"><float name="thickness" value="0.5"/><bsdf type="roughDiffuse"><float name="alpha" value="0.4"/></bsdf></bsdf>
  </mesh>
  <mesh type="obj"><string name="filename" value="quad.obj"/><bsdf type="diffuse"/>
    <emitter type="area"><color name="radiance" value="1, 1, 1"/></emitter></mesh>
  <emitter type="constant"><color name="radiance" value="0.5, 0.6, 0.7"/></emitter>
  <emitter type="directional"><color name="irradiance" value="1, 1, 1"/><vector name="direction" value="0, -1, 0"/></emitter>
</scene>
"""


def test_xml_lights_and_layers(L, tmp_path):
    """Point, area, constant and directional emitters keep the XML order in
    both parsers; coating over roughDiffuse parses in both."""
    (tmp_path / "quad.obj").write_text(QUAD_OBJ)
    path = str(tmp_path / "lights.xml")
    open(path, "w").write(LIGHTS_XML)
    info, depth, spp = hk.parse_xml_info(path)
    sd = parse_xml(path)[0]
    assert info.n_emitters == 4 and info.env_index == 2
    assert sd.emitter_order() == [-2, 1, -1, -3]
    assert [l.kind for l in sd.lights] == ["point", "directional"] and sd.env_constant == pytest.approx([0.5, 0.6, 0.7])
    assert info.n_bsdfs == 3
    c = sd.meshes[0].bsdf
    assert c.type == 10 and c.thickness == 0.5 and c.nested.type == 11 and c.nested.alpha_u == pytest.approx(0.4)


def test_oracle_builds_every_light(tmp_path):
    from oracle.oracle import OracleScene

    (tmp_path / "quad.obj").write_text(QUAD_OBJ)
    path = str(tmp_path / "lights.xml")
    open(path, "w").write(LIGHTS_XML)
    sd = parse_xml(path)[0]
    o = OracleScene(sd)
    from oracle import oracle as O
    assert O.lib().ho_scene_num_emitters(o.h) == 4
    p = o.emitter_sample(0, np.float32([0, 0, 0]), (0.5, 0.5, 0.5))   # point light at (0, 3, 0)
    assert np.allclose(p[:3], [0, 3, 0]) and p[9] == 1.0 and np.allclose(p[11:], 10 / (4 * np.pi * 9), rtol=1e-6)
    d = o.emitter_sample(3, np.float32([0, 0, 0]), (0.5, 0.5, 0.5))   # directional light travelling down
    assert np.allclose(d[6:9], [0, 1, 0]) and np.allclose(d[11:], 1.0)


def _mixed_obj(rng, style, n=3000):
    """style: 0 "p", 1 "p/t", 2 "p//n", 3 "p/t/n" face keys (the reference
    reads normals / texcoords of every vertex when the file has any)."""
    lines = ["# OBJ with comments, quads, CRLF, signs and exponents", "o thing", "g group"]
    P = rng.uniform(-5, 5, (n, 3))
    for i, p in enumerate(P):
        x, y, z = (f"{c:+.7e}" if i % 7 == 0 else f"{c:.6f}" for c in p)
        lines.append(f"v {x} {y} {z}" + ("\r" if i % 5 == 0 else ""))
    if style in (1, 3):
        lines += [f"vt {rng.random():.5f} {rng.random():.5f}" for _ in range(n // 2)]
    if style in (2, 3):
        for _ in range(n // 3):
            v = rng.normal(size=3)
            lines.append(f"vn {v[0]:.6f} {v[1]:.6f} {v[2]:.6f}")
    lines.append("s off")
    for i in range(2 * n):
        ids = rng.integers(1, n + 1, 4 if i % 3 == 0 else 3)
        t = lambda: rng.integers(1, n // 2 + 1)
        m = lambda: rng.integers(1, n // 3 + 1)
        keys = [[f"{a}", f"{a}/{t()}", f"{a}//{m()}", f"{a}/{t()}/{m()}"][style] for a in ids]
        lines.append("f " + " ".join(keys))
    return "\n".join(lines) + "\n"


def test_parallel_obj_reader_matches_reference_rules(L, tmp_path):
    """The library's parallel OBJ reader against the line-by-line restatement
    of WavefrontObjMesh: same vertex order and indices, positions and normals
    to float rounding of the transform."""
    from hikari_b200.scenedesc import load_obj

    rng = np.random.default_rng(12)
    M = np.array([[0.5, 0.1, 0, 1], [0, 2, 0.3, -1], [0.2, 0, 1.5, 3], [0, 0, 0, 1]], np.float32)
    for style in range(4):
        path = str(tmp_path / f"mixed{style}.obj")
        open(path, "w", newline="").write(_mixed_obj(rng, style))
        pos, idx, nrm, uv = hk.obj_load(path, M)
        p2, i2, n2, bbox, uv2 = load_obj(path, M)
        assert idx.shape == i2.shape and np.array_equal(idx, i2)
        assert pos.shape == p2.shape and np.allclose(pos, p2, rtol=1e-6, atol=1e-5)
        assert (nrm is None) == (n2 is None) and (nrm is None or np.allclose(nrm, n2, atol=1e-5))
        assert (uv is not None) == (style in (1, 3)) == (uv2 is not None)
        assert uv is None or np.array_equal(uv, uv2)
    # positions-only fast path, with quads
    path2 = str(tmp_path / "plain.obj")
    open(path2, "w").write(QUAD_OBJ + "v 0 1 0\nf 1 2 5\n")
    pos, idx, nrm, uv = hk.obj_load(path2)
    # "f 1 4 3 2" -> (1,4,3) (2,1,3); ids in first-use order 1,4,3,2 then 5
    assert idx.tolist() == [[0, 1, 2], [3, 0, 2], [0, 3, 4]] and nrm is None and uv is None
    assert pos.tolist()[1] == [-1.0, 0.0, 1.0] and pos.tolist()[4] == [0.0, 1.0, 0.0]


@pytest.mark.parametrize("text,needle", [("v 0 0 0\nf 1 2 3\n", "out of range"), ("v 0 0 0\nf 1 a 1\n", "Invalid vertex"),
                                         ("v 0 0 0\nf 1/1/1/1 1 1\n", "Invalid vertex")])
def test_obj_reader_errors(L, tmp_path, text, needle):
    path = str(tmp_path / "bad.obj")
    open(path, "w").write(text)
    with pytest.raises(hk.HikariError, match=needle):
        hk.obj_load(path)


TEXTURE_XML = """<?xml version="1.0"?>
<scene>
  <integrator type="pathMIS"><integer name="depth" value="8"/></integrator>
  <camera type="perspective"><integer name="width" value="16"/><integer name="height" value="16"/></camera>
  <mesh type="obj"><string name="filename" value="quad.obj"/>
    <bsdf type="diffuse">
      <texture type="checkerboard" name="albedo"><integer name="blocks" value="4"/>
        <color name="colorA" value="0.9, 0.1, 0.1"/><float name="uScale" value="2"/></texture>
    </bsdf>
  </mesh>
  <mesh type="obj"><string name="filename" value="quad.obj"/>
    <bsdf type="roughConductor"><boolean name="as" value="true"/>
      <texture type="grid" name="alphaU"><integer name="lines" value="6"/><float name="lineWidth" value="0.05"/></texture>
      <texture type="scale" name="alphaV"><float name="scale" value="0.5"/><texture type="checkerboard"/></texture>
    </bsdf>
  </mesh>
</scene>
"""


def test_xml_textures(L, tmp_path):
    from hikari_b200.scenedesc import TEX_CHECKERBOARD, TEX_GRID, TEX_SCALE

    (tmp_path / "quad.obj").write_text(QUAD_OBJ)
    path = str(tmp_path / "tex.xml")
    open(path, "w").write(TEXTURE_XML)
    info, depth, spp = hk.parse_xml_info(path)
    sd = parse_xml(path)[0]
    assert info.n_bsdfs == 2
    t = sd.meshes[0].bsdf.textures["kd"]
    assert t.kind == TEX_CHECKERBOARD and t.count == 4 and t.a == pytest.approx([0.9, 0.1, 0.1]) and t.uv_scale == [2.0, 1.0]
    c = sd.meshes[1].bsdf.textures
    assert c["alpha_u"].kind == TEX_GRID and c["alpha_u"].width == pytest.approx(0.05)
    assert c["alpha_v"].kind == TEX_SCALE and c["alpha_v"].nested.kind == TEX_CHECKERBOARD


GEOMETRIC_XML = """<?xml version="1.0"?>
<scene>
  <integrator type="pathMIS"><integer name="depth" value="8"/></integrator>
  <camera type="perspective"><integer name="width" value="16"/><integer name="height" value="16"/></camera>
  <mesh type="obj"><string name="filename" value="quad.obj"/>
    <bsdf type="diffuse">
      <texture type="wireframe" name="albedo"><color name="edgeColor" value="0.9, 0.1, 0.1"/>
        <float name="transitionWidth" value="0.25"/></texture>
    </bsdf>
  </mesh>
  <mesh type="obj"><string name="filename" value="quad.obj"/>
    <bsdf type="roughConductor">
      <texture type="curvature" name="ks"><string name="curvatureType" value="gaussian"/>
        <float name="scale" value="3"/></texture>
    </bsdf>
  </mesh>
</scene>
"""


def test_xml_wireframe_and_curvature_textures(L, tmp_path):
    """The wireframe and curvature plugins (src/texture/{Wireframe,Curvature}Texture.cpp
    ctors) in both parsers, with the reference's defaults."""
    from hikari_b200.scenedesc import TEX_CURVATURE, TEX_WIREFRAME

    (tmp_path / "quad.obj").write_text(QUAD_OBJ)
    path = str(tmp_path / "geo.xml")
    open(path, "w").write(GEOMETRIC_XML)
    info, depth, spp = hk.parse_xml_info(path)
    assert info.n_bsdfs == 2
    sd = parse_xml(path)[0]
    w = sd.meshes[0].bsdf.textures["kd"]
    assert w.kind == TEX_WIREFRAME and w.b == pytest.approx([0.9, 0.1, 0.1]) and w.a == pytest.approx([0.5] * 3)
    assert w.width == 0.0 and w.scale == pytest.approx(0.25)
    c = sd.meshes[1].bsdf.textures["ks"]
    assert c.kind == TEX_CURVATURE and c.count == 1 and c.scale == pytest.approx(3.0)
    assert c.a == pytest.approx([1, 0, 0]) and c.b == pytest.approx([0, 0, 1])
    bad = GEOMETRIC_XML.replace('value="gaussian"', 'value="total"')
    open(path, "w").write(bad)
    with pytest.raises(hk.HikariError, match="curvature type"):
        hk.parse_xml_info(path)


@pytest.mark.parametrize("body,needle", [
    ('<bsdf type="diffuse"><texture type="checkerboard" name="ks"/></bsdf>', "not supported"),
    ('<bsdf type="roughPlastic"><texture type="checkerboard" name="sigmaA"/></bsdf>', "not supported"),
    ('<bsdf type="diffuse"><texture type="scale" name="albedo"><float name="scale" value="2"/></texture></bsdf>',
     "nested texture"),
])
def test_xml_texture_errors(L, tmp_path, body, needle):
    from hikari_b200.scenedesc import SceneError

    (tmp_path / "quad.obj").write_text(QUAD_OBJ)
    path = str(tmp_path / "bad.xml")
    open(path, "w").write(f'<scene><mesh type="obj"><string name="filename" value="quad.obj"/>{body}</mesh></scene>')
    with pytest.raises(hk.HikariError, match=needle):
        hk.parse_xml_info(path)
    with pytest.raises(SceneError, match=needle):
        parse_xml(path)


BITMAP_XML = """<?xml version="1.0"?>
<scene>
  <integrator type="pathMIS"><integer name="depth" value="8"/></integrator>
  <camera type="perspective"><integer name="width" value="16"/><integer name="height" value="16"/></camera>
  <mesh type="obj"><string name="filename" value="quad.obj"/>
    <bsdf type="diffuse"><texture type="bitmap" name="albedo">
      <string name="filename" value="tex/a.png"/><float name="gamma" value="2.2"/>
      <float name="uScale" value="2"/></texture></bsdf>
  </mesh>
  <mesh type="obj"><string name="filename" value="quad.obj"/>
    <bsdf type="roughConductor"><string name="type" value="ggx"/>
      <texture type="bitmap" name="alpha"><string name="filename" value="tex/b.ppm"/>
        <string name="channel" value="r"/><string name="wrapMode" value="clamp"/>
        <string name="filterType" value="trilinear"/><float name="maxAnisotropy" value="8"/></texture>
    </bsdf>
  </mesh>
</scene>
"""


def test_xml_bitmap_textures(L, tmp_path):
    """BitmapTexture in both parsers: file names resolve against the scene's
    directory, the image is decoded like stbi_load, wrap / filter / channel /
    gamma / anisotropy properties as the reference names them."""
    from hikari_b200 import scenes
    from hikari_b200.scenedesc import FILTER_EWA, FILTER_TRILINEAR, TEX_BITMAP, WRAP_CLAMP, WRAP_REPEAT

    PIL = pytest.importorskip("PIL.Image")
    (tmp_path / "quad.obj").write_text(QUAD_OBJ)
    (tmp_path / "tex").mkdir()
    a = scenes.synthetic_image(20, 12, 3, 1)
    PIL.fromarray(a).save(tmp_path / "tex" / "a.png")
    b = scenes.synthetic_image(9, 7, 3, 2)
    (tmp_path / "tex" / "b.ppm").write_bytes(b"P6 9 7 255\n" + b.tobytes())
    path = str(tmp_path / "bitmap.xml")
    open(path, "w").write(BITMAP_XML)
    info, depth, spp = hk.parse_xml_info(path)
    assert info.n_bsdfs == 2 and info.n_meshes == 2
    sd = parse_xml(path)[0]
    ta = sd.meshes[0].bsdf.textures["kd"]
    assert ta.kind == TEX_BITMAP and ta.filter == FILTER_EWA and ta.wrap_u == ta.wrap_v == WRAP_REPEAT
    assert ta.gamma == pytest.approx(2.2) and ta.uv_scale == [2.0, 1.0] and ta.channels == 3
    np.testing.assert_array_equal(ta.pixels, a)
    tb = sd.meshes[1].bsdf.textures["alpha_u"]
    assert tb.channels == 1 and tb.filter == FILTER_TRILINEAR and tb.wrap_u == tb.wrap_v == WRAP_CLAMP
    assert tb.max_anisotropy == 8.0
    luma = (b[..., 0].astype(int) * 77 + b[..., 1].astype(int) * 150 + b[..., 2].astype(int) * 29) >> 8
    np.testing.assert_array_equal(tb.pixels[:, :, 0], luma)


@pytest.mark.parametrize("prop,needle", [
    ('<string name="filterType" value="cubic"/>', "Illegal filter type"),
    ('<string name="wrapMode" value="mirror"/>', "Illegal wrap mode"),
    ('<string name="channel" value="rg"/>', "Illegal channel"),
])
def test_xml_bitmap_errors(L, tmp_path, prop, needle):
    from hikari_b200 import scenes
    from hikari_b200.scenedesc import SceneError

    (tmp_path / "quad.obj").write_text(QUAD_OBJ)
    (tmp_path / "a.ppm").write_bytes(b"P6 4 4 255\n" + scenes.synthetic_image(4, 4, 3, 0).tobytes())
    path = str(tmp_path / "bad.xml")
    open(path, "w").write('<scene><mesh type="obj"><string name="filename" value="quad.obj"/><bsdf type="diffuse">'
                          '<texture type="bitmap" name="albedo"><string name="filename" value="a.ppm"/>'
                          f'{prop}</texture></bsdf></mesh></scene>')
    with pytest.raises(hk.HikariError, match=needle):
        hk.parse_xml_info(path)
    with pytest.raises(SceneError, match=needle):
        parse_xml(path)


def test_image_load_errors(L, tmp_path):
    p = tmp_path / "x.bin"
    p.write_bytes(b"not an image")
    with pytest.raises(hk.HikariError, match="unknown image format"):
        hk.image_load(str(p), 3)
    with pytest.raises(hk.HikariError, match="cannot open"):
        hk.image_load(str(tmp_path / "missing.png"), 3)
    (tmp_path / "p.jpg").write_bytes(b"\xff\xd8\xff\xc2\x00\x0b\x08\x00\x10\x00\x10\x01\x01\x11\x00\xff\xd9")
    with pytest.raises(hk.HikariError, match="progressive"):
        hk.image_load(str(tmp_path / "p.jpg"), 3)


BUMP_XML = """<?xml version="1.0"?>
<scene>
  <integrator type="pathMIS"><integer name="depth" value="8"/></integrator>
  <camera type="perspective"><integer name="width" value="16"/><integer name="height" value="16"/></camera>
  <mesh type="obj"><string name="filename" value="quad.obj"/>
    <bsdf type="bumpMap">
      <texture type="scale"><float name="scale" value="0.1"/>
        <texture type="checkerboard"><integer name="blocks" value="5"/></texture></texture>
      <bsdf type="roughConductor"><string name="type" value="ggx"/></bsdf>
    </bsdf>
  </mesh>
  <mesh type="obj"><string name="filename" value="quad.obj"/>
    <bsdf type="normalMap">
      <bsdf type="diffuse"/>
      <texture type="grid"/>
    </bsdf>
  </mesh>
</scene>
"""


def test_xml_bump_and_normal_maps(L, tmp_path):
    """bumpMap / normalMap in both parsers: one nested BSDF and one map
    texture of any name, in either order."""
    from hikari_b200.scenedesc import (BSDF_BUMP_MAP, BSDF_DIFFUSE, BSDF_NORMAL_MAP, BSDF_ROUGH_CONDUCTOR, TEX_GRID,
                                       TEX_SCALE)

    (tmp_path / "quad.obj").write_text(QUAD_OBJ)
    path = str(tmp_path / "bump.xml")
    open(path, "w").write(BUMP_XML)
    info, depth, spp = hk.parse_xml_info(path)
    assert info.n_bsdfs == 4
    sd = parse_xml(path)[0]
    b, n = sd.meshes[0].bsdf, sd.meshes[1].bsdf
    assert b.type == BSDF_BUMP_MAP and b.nested.type == BSDF_ROUGH_CONDUCTOR and b.textures["kd"].kind == TEX_SCALE
    assert n.type == BSDF_NORMAL_MAP and n.nested.type == BSDF_DIFFUSE and n.textures["kd"].kind == TEX_GRID


def test_bump_map_needs_normals_and_uv(L, tmp_path):
    """The quad has neither vertex normals nor texture coordinates: a
    bump-mapped mesh is rejected when the scene is built."""
    (tmp_path / "quad.obj").write_text(QUAD_OBJ)
    path = str(tmp_path / "bump.xml")
    open(path, "w").write(BUMP_XML)
    sd = parse_xml(path)[0]
    with pytest.raises(hk.HikariError, match="vertex normals and texture coordinates"):
        hk.Scene.from_desc(sd)
