"""Pins of the oracle restatement (oracle/hk_oracle.c) against the reference
renderer compiled from its own sources (oracle/ref_build.py):

* ray queries: the oracle's SAH BVH and brute-force loop against the
  reference's HLBVHAcceleration (src/acceleration/HLBVHAcceleration.cpp:206),
  BVHAcceleration and brute-force Acceleration (src/core/Acceleration.cpp:45)
  with Mesh::RayIntersect (src/core/Mesh.cpp:340-384);
* EnvironmentLight::Sample / Eval / Pdf (src/emitter/EnvironmentLight.cpp:8-110)
  over DiscretePDF2D (src/core/DiscretePDF.cpp:93-133);
* the reconstruction filters (src/filter/*.cpp) tabulated by ImageBlock and
  ImageBlock::Put (src/core/Block.cpp:95-134);
* whole renders: the reference's Render block loop (src/Main.cpp:46-147)
  against the oracle's, on the same per-block sample streams.

Bit-exact equality where both sides do the same float operations; where the
oracle is known to differ by an ulp (its camera ray is within an ulp of
PerspectiveCamera::SampleRay), the tolerance is stated at the assertion.
CPU only: these tests need the reference checkout to build the library and
are skipped without it.
"""
import os

import numpy as np
import pytest

from hikari_b200 import scenes
from hikari_b200.scenedesc import BSDF_DIFFUSE, BSDFDesc, EnvDesc, FilterDesc, MeshDesc, SceneDesc
from hikari_b200.scenexml import write_exr, write_scene_xml
from oracle.oracle import OracleScene

reference = pytest.importorskip("oracle.reference")


@pytest.fixture(scope="module")
def R():
    try:
        return reference.lib()
    except reference.ReferenceUnavailable as e:
        pytest.skip(str(e))


def _displaced_scene(level=5):
    P, F = scenes.displaced_icosphere(level, 1.0, (0.0, 1.0, 0.0), 0.08, 3)
    sd = SceneDesc()
    sd.meshes.append(MeshDesc(P, F, BSDFDesc(type=BSDF_DIFFUSE)))
    gp, gi = scenes.quad((-10, 0, -10), (-10, 0, 10), (10, 0, 10), (10, 0, -10))
    sd.meshes.append(MeshDesc(gp, gi, BSDFDesc(type=BSDF_DIFFUSE)))
    sd.camera = scenes.CameraDesc(64, 64, scenes.look_at((0, 1.6, 4.2), (0, 0.9, 0), (0, 1, 0)), 40.0, 1e-4, 1e4)
    return sd


def _rays(sd, os_, n, seed):
    """Camera rays through random film positions plus rays from random points
    inside the scene box in uniform directions (closest hit, full range)."""
    rng = np.random.default_rng(seed)
    cam = sd.camera
    out = []
    for _ in range(n // 2):
        out.append(os_.camera_ray(rng.uniform(0, cam.width), rng.uniform(0, cam.height)))
    lo = np.min([m.positions.min(0) for m in sd.meshes], 0)
    hi = np.max([m.positions.max(0) for m in sd.meshes], 0)
    o = rng.uniform(lo, hi, (n - n // 2, 3)).astype(np.float32)
    d = rng.normal(size=(n - n // 2, 3))
    d = (d / np.linalg.norm(d, axis=1, keepdims=True)).astype(np.float32)
    r = np.concatenate([o, d, np.full((len(o), 1), 1e-4, np.float32), np.full((len(o), 1), np.inf, np.float32)], 1)
    return np.concatenate([np.array(out, np.float32).reshape(-1, 8), r], 0)


@pytest.mark.parametrize("scene", ["cornell", "displaced"])
@pytest.mark.parametrize("kind", ["hlbvh", "bvh", "bruto"])
def test_trace_vs_reference_accel(R, scene, kind):
    sd = scenes.cornell_box(width=64, height=64) if scene == "cornell" else _displaced_scene()
    os_ = OracleScene(sd)
    rays = _rays(sd, os_, 6000 if kind == "bruto" and scene == "displaced" else 40000, 1)
    acc = reference.RefAccel(sd.meshes, kind)
    rt, rtt, ru, rv = acc.trace(rays)
    for use_bvh in (True, False):
        if not use_bvh and scene == "displaced" and len(rays) > 6000:
            continue   # the brute-force loop over 20k triangles is slow; covered against "bruto"
        ot, ott, ou, ov = os_.trace(rays, use_bvh=use_bvh)
        same = ot == rt
        hit = rt >= 0
        # a different triangle only on an exact tie in t (coplanar or shared
        # edges), where the answer depends on the visit order
        diff = ~same
        assert np.all(ott[diff] == rtt[diff]), f"{np.sum(ott[diff] != rtt[diff])} non-tie mismatches"
        assert diff.mean() < 2e-3, f"tie rate {diff.mean():.4f}"
        # where the triangle agrees, t, u and v are the reference's bit for bit
        m = same & hit
        assert np.array_equal(ott[m], rtt[m]) and np.array_equal(ou[m], ru[m]) and np.array_equal(ov[m], rv[m])
    # any-hit agrees everywhere (shadow segments toward random points)
    sh = rays.copy()
    sh[:, 7] = np.where(rt >= 0, rtt * 0.999, 5.0)
    ra = acc.trace(sh, any_hit=True)[0]
    oa = os_.trace(sh, any_hit=True, use_bvh=True)[0]
    assert np.array_equal(ra, oa)


def _sky(w=128, h=64, nan_texel=False):
    rgb, tw = scenes.sky_envmap(w, h, sun_deg=6.0)
    if nan_texel:
        # an invalid texel: Eval and Sample return zero there; its NaN
        # luminance also spreads through the reference's CDFs
        rgb[h // 3, w // 5] = np.nan
    return rgb, tw


@pytest.mark.parametrize("nan_texel", [False, True])
def test_env_light_vs_reference(R, tmp_path, nan_texel):
    rgb, tw = _sky(nan_texel=nan_texel)
    path = str(tmp_path / "sky.exr")
    write_exr(path, rgb)
    ref = reference.env_light(path, tw, 1.5)
    sd = _displaced_scene(2)
    sd.env = EnvDesc(rgb, tw, 1.5)
    sd.env_emitter_index = 0
    os_ = OracleScene(sd)
    rng = np.random.default_rng(4)
    n = 4000
    refp = rng.uniform(-1, 1, (n, 3)).astype(np.float32)
    u = rng.random((n, 3), dtype=np.float32)
    u[:50, :2] = 0.0          # corner of the CDFs
    u[50:100, :2] = np.nextafter(np.float32(1), np.float32(0))
    o = np.array([os_.emitter_sample(0, refp[i], u[i]) for i in range(n)], np.float32)
    q = np.concatenate([refp, u, o[:, 10:11]], 1)
    r = reference.emitter_sample(ref, q)
    # (p, n, wi, pdf, distance, value) bit for bit (NaN where both are NaN)
    np.testing.assert_array_equal(o[:, :14], r[:, :14])
    # Eval and Pdf at the sampled directions and at random ones
    d = rng.normal(size=(n, 3)).astype(np.float32)
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    wi = np.concatenate([o[:, 6:9], d], 0)
    re = reference.emitter_eval_dir(ref, wi)
    oe = np.array([os_.env_eval(w) for w in wi], np.float32)
    np.testing.assert_array_equal(oe, re[:, :3])
    if not nan_texel:
        op = np.array([os_.emitter_pdf(0, np.zeros(3, np.float32), w, -w) for w in wi], np.float32)
        assert np.isfinite(re[:, 3]).all()
        np.testing.assert_array_equal(op, re[:, 3])
    reference.lib().hr_object_free(ref)


FILTERS = [FilterDesc(0, 0.5), FilterDesc(1, 1.0), FilterDesc(2, 2.0, 0.5), FilterDesc(3, 2.0, 1 / 3, 1 / 3),
           FilterDesc(2, 1.3, 0.35), FilterDesc(3, 2.7, 0.5, 0.25)]


@pytest.mark.parametrize("fi", range(len(FILTERS)))
def test_filters_and_block_put_vs_reference(R, fi):
    f = FILTERS[fi]
    W, H = 37, 23
    sd = scenes.cornell_box(width=W, height=H)
    sd.filter = f
    os_ = OracleScene(sd)
    rf = reference.filter_create(f.kind, f.radius, f.p0, f.p1)
    # the tabulated filter: ImageBlock's 32 entries + 0 and its lookup factor
    tab = np.zeros(33, np.float32)
    import ctypes as C
    from oracle import oracle as O

    lookup = C.c_float()
    O.lib().ho_filter_table(os_.h, tab.ctypes.data, C.byref(lookup))
    r = np.float32(f.radius if f.kind >= 2 else (0.5 if f.kind == 0 else 1.0))
    x = np.array([(r * np.float32(i)) / np.float32(32) for i in range(32)], np.float32)
    ev = np.zeros(32, np.float32)
    reference.lib().hr_filter_eval(rf, 32, x.ctypes.data, ev.ctypes.data)
    np.testing.assert_array_equal(tab[:32], ev)
    assert tab[32] == 0.0 and lookup.value == np.float32(32) / r
    rng = np.random.default_rng(fi)
    n = 3000
    pos = np.stack([rng.uniform(-1, W + 1, n), rng.uniform(-1, H + 1, n)], 1).astype(np.float32)
    pos[:40] = np.floor(pos[:40]) + 0.5   # pixel centres and integer edges
    pos[40:80] = np.floor(pos[40:80])
    val = rng.uniform(0, 4, (n, 3)).astype(np.float32)
    val[80:90, 1] = -1e-3    # negative, NaN and Inf samples are dropped whole
    val[90:95, 0] = np.nan
    val[95:100, 2] = np.inf
    # one sample at a time: every film cell the reference writes, bit for bit
    for i in range(0, n, 97):
        rfilm, b = reference.block_put(rf, W, H, pos[i:i + 1], val[i:i + 1])
        ofilm, dropped = os_.film_put(pos[i:i + 1], val[i:i + 1])
        assert b == O.lib().ho_film_border(os_.h)
        np.testing.assert_array_equal(ofilm.astype(np.float32), rfilm)
    # all samples: float accumulation (reference) against double (oracle)
    rfilm, b = reference.block_put(rf, W, H, pos, val)
    ofilm, dropped = os_.film_put(pos, val)
    assert dropped == 20
    np.testing.assert_allclose(rfilm, ofilm, rtol=2e-6, atol=1e-6)
    reference.lib().hr_object_free(rf)


def _block_pixels(a, b, blocks, W, H, rel):
    """Per block: number of pixels whose values differ beyond rel."""
    out = []
    bx = (W + 31) // 32
    for blk in blocks:
        x0, y0 = (blk % bx) * 32, (blk // bx) * 32
        A, B = a[y0:y0 + 32, x0:x0 + 32], b[y0:y0 + 32, x0:x0 + 32]
        d = np.abs(A - B).max(-1) > rel * np.maximum(np.abs(B).max(-1), 1e-3)
        out.append(int(d.sum()))
    return out


@pytest.mark.parametrize("name", ["cornell", "heterogeneous"])
def test_render_vs_reference_same_streams(R, tmp_path, name):
    """One sample per pixel and a box filter: every pixel is one path of the
    reference's own per-block stream.  With the reference's Next2D order the
    oracle replays the reference path for path: values agree to float
    rounding (the oracle's camera ray is within an ulp of the reference's) and
    a block's stream never shifts (a shift would change every later pixel of
    the block)."""
    if name == "cornell":
        sd = scenes.cornell_box(width=64, height=64, spp=1)
    else:
        sd = scenes.heterogeneous(width=64, height=64, spp=1, n_spheres=12, levels=(3, 4), level_p=(0.5, 0.5),
                                  env_res=(256, 128))
    sd.filter = FilterDesc(0, 0.5)
    xml = write_scene_xml(sd, str(tmp_path), name, spp=1)
    rs = reference.RefScene(xml)
    blocks = list(range(((sd.camera.width + 31) // 32) * ((sd.camera.height + 31) // 32)))
    film, _ = rs.render(nthreads=4)
    os_ = OracleScene(sd)
    os_.set_reference_draw_order(True)
    ofilm, dropped, _ = os_.render(1, nthreads=4)
    a, b = rs.resolve(film), os_.resolve(ofilm)
    W, H = sd.camera.width, sd.camera.height
    bad = _block_pixels(a, b, blocks, W, H, 1e-4)
    assert sum(bad) <= 0.01 * W * H, bad
    # image sums agree closely
    assert abs(a.sum() / b.sum() - 1) < 1e-4


def test_render_gaussian_film_vs_reference(R, tmp_path):
    """The Cornell box at 8 samples per pixel through the Gaussian filter
    (radius 2, stddev 0.5): the reference's film and the oracle's agree cell
    by cell, blocks whose stream stayed aligned to float rounding."""
    sd = scenes.cornell_box(width=64, height=64, spp=8)
    xml = write_scene_xml(sd, str(tmp_path), "cbox", spp=8)
    rs = reference.RefScene(xml)
    film, _ = rs.render(nthreads=4)
    os_ = OracleScene(sd)
    os_.set_reference_draw_order(True)
    ofilm, _, _ = os_.render(8, nthreads=4)
    rel = np.abs(film[..., 3] - ofilm[..., 3]) / np.maximum(ofilm[..., 3], 1e-6)
    # the filter weights depend only on the sample positions: equal unless a
    # block's stream shifted
    assert (rel < 1e-5).mean() > 0.97
    a, b = rs.resolve(film), os_.resolve(ofilm)
    close = np.abs(a - b).max(-1) <= 2e-4 * np.maximum(np.abs(b).max(-1), 1e-3)
    assert close.mean() > 0.95
