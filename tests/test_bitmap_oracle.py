"""Pin of the oracle's bitmap textures against the reference's own classes
compiled from its sources (oracle/ref_build.py): BitmapTexture over MipMap
(Lanczos resampling to powers of two, box pyramid, nearest / bilinear /
trilinear / EWA lookups, wrap modes, r and rgb channels, gamma), the
PerspectiveCamera's differential rays and Intersection::
ComputeScreenSpacePartial.  Images are written as PNG files that the
reference reads through its own stb_image path; the oracle gets the same
8-bit pixels.  Bit-exact equality is required (NaN where the reference makes
NaN)."""
import ctypes as C
import os

import numpy as np
import pytest

from hikari_b200.scenedesc import (BSDF_DIFFUSE, BSDF_ROUGH_CONDUCTOR, BSDF_ROUGH_PLASTIC, FILTER_BILINEAR,
                                   FILTER_EWA, FILTER_NEAREST, FILTER_TRILINEAR, GGX, TEX_BITMAP, TEX_SCALE,
                                   TEX_SLOTS, WRAP_BLACK, WRAP_CLAMP, WRAP_REPEAT, BSDFDesc, CameraDesc, MeshDesc,
                                   SceneDesc, TextureDesc)
from oracle import oracle as O

from test_oracle_vs_reference import _ref_lib, records

PIL = pytest.importorskip("PIL.Image")


def _ref():
    R = _ref_lib()
    R.hr_bitmap_create.restype = C.c_void_p
    R.hr_bitmap_create.argtypes = [C.c_char_p, C.c_char_p, C.c_int, C.c_int, C.c_int, C.c_int, C.c_float, C.c_float,
                                   C.c_void_p, C.c_void_p]
    R.hr_texture_eval.argtypes = [C.c_void_p, C.c_uint64, C.c_void_p, C.c_void_p, C.c_void_p]
    R.hr_texture_average.argtypes = [C.c_void_p, C.c_void_p]
    R.hr_texture_create.restype = C.c_void_p
    R.hr_texture_create.argtypes = [C.c_int, C.c_int, C.c_float, C.c_float] + [C.c_void_p] * 5
    R.hr_bsdf_batch.argtypes = [C.c_void_p, C.c_uint64] + [C.c_void_p] * 12
    R.hr_image_load.restype = C.c_uint64
    R.hr_image_load.argtypes = [C.c_char_p, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p]
    R.hr_camera_create.restype = C.c_void_p
    R.hr_camera_create.argtypes = [C.c_int, C.c_int, C.c_void_p, C.c_float, C.c_float, C.c_float]
    R.hr_camera_ray.argtypes = [C.c_void_p, C.c_float, C.c_float, C.c_void_p]
    R.hr_mesh_create.restype = C.c_void_p
    R.hr_mesh_create.argtypes = [C.c_void_p, C.c_uint32, C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint32]
    R.hr_screen_partials.argtypes = [C.c_void_p, C.c_void_p, C.c_uint32, C.c_float, C.c_float, C.c_float, C.c_float,
                                     C.c_void_p]
    return R


def image(w, h, ch, seed):
    """Smooth gradients plus noise: every MIP level carries detail."""
    rng = np.random.default_rng(seed)
    y, x = np.mgrid[0:h, 0:w]
    base = np.stack([(x * 255 // max(w - 1, 1)), (y * 255 // max(h - 1, 1)), ((x + y) * 7) % 256], -1)
    img = (0.6 * base + 0.4 * rng.integers(0, 256, (h, w, 3))).astype(np.uint8)
    return img[:, :, :ch] if ch == 3 else img[:, :, :1]


def write_png(path, img):
    PIL.fromarray(img[:, :, 0] if img.shape[2] == 1 else img).save(path)


def ref_bitmap(R, tmp_path, name, img, t):
    write_png(os.path.join(tmp_path, name), img)
    f = lambda a: np.ascontiguousarray(a, np.float32)
    us, uo = f(t.uv_scale), f(t.uv_offset)
    h = R.hr_bitmap_create(str(tmp_path).encode(), name.encode(), t.filter, t.wrap_u, t.wrap_v, t.channels, t.gamma,
                           t.max_anisotropy, O._p(us), O._p(uo))
    assert h
    return h


def queries(n, seed, zero_frac=0.1):
    rng = np.random.default_rng(seed)
    uv = rng.uniform(-0.3, 1.3, (n, 2)).astype(np.float32)
    mag = 10.0 ** rng.uniform(-4.5, 0.3, (n, 4))
    duv = (mag * rng.choice([-1, 1], (n, 4))).astype(np.float32)
    duv[: int(n * zero_frac)] = 0.0                       # the partials of a hit without differentials
    duv[int(n * zero_frac): int(n * 2 * zero_frac), 2:] = 0.0   # degenerate ellipse (minor axis 0)
    duv[-50:, 2:] = duv[-50:, :2] * 1e-3                   # eccentric: clamped by maxAnisotropy
    return uv, duv


def eq_nan(a, b):
    return a.shape == b.shape and np.array_equal(np.isnan(a), np.isnan(b)) and np.array_equal(a[~np.isnan(a)],
                                                                                             b[~np.isnan(b)])


CASES = {
    # name: (w, h, channels, filter, wrap_u, wrap_v, gamma, uv_scale, uv_offset, max_anisotropy)
    "pow2_rgb_ewa": (32, 16, 3, FILTER_EWA, WRAP_REPEAT, WRAP_REPEAT, 1.0, [1, 1], [0, 0], 20.0),
    "npot_rgb_ewa": (37, 23, 3, FILTER_EWA, WRAP_REPEAT, WRAP_REPEAT, 1.0, [1, 1], [0, 0], 20.0),
    "npot_rgb_ewa_clamp": (45, 19, 3, FILTER_EWA, WRAP_CLAMP, WRAP_CLAMP, 2.2, [1.5, 0.75], [0.1, -0.2], 8.0),
    "npot_r_ewa": (29, 31, 1, FILTER_EWA, WRAP_REPEAT, WRAP_CLAMP, 1.0, [1, 1], [0, 0], 20.0),
    "npot_rgb_trilinear": (50, 33, 3, FILTER_TRILINEAR, WRAP_REPEAT, WRAP_REPEAT, 1.0, [2, 2], [0, 0], 20.0),
    "pow2_r_trilinear": (64, 64, 1, FILTER_TRILINEAR, WRAP_CLAMP, WRAP_REPEAT, 1.8, [1, 1], [0.3, 0], 20.0),
    "npot_rgb_bilinear": (21, 13, 3, FILTER_BILINEAR, WRAP_REPEAT, WRAP_REPEAT, 1.0, [1, 1], [0, 0], 20.0),
    "npot_rgb_nearest": (21, 13, 3, FILTER_NEAREST, WRAP_REPEAT, WRAP_REPEAT, 2.2, [3, 1], [0, 0.5], 20.0),
    "black_wrap_ewa": (24, 20, 3, FILTER_EWA, WRAP_BLACK, WRAP_REPEAT, 1.0, [1, 1], [0, 0], 20.0),
    "one_pow2_side": (16, 12, 3, FILTER_EWA, WRAP_REPEAT, WRAP_REPEAT, 1.0, [1, 1], [0, 0], 20.0),   # NaN texels
    "thin": (7, 3, 3, FILTER_EWA, WRAP_REPEAT, WRAP_REPEAT, 1.0, [1, 1], [0, 0], 20.0),
}


def bitmap_desc(case, img):
    w, h, ch, flt, wu, wv, gamma, us, uo, ma = CASES[case]
    return TextureDesc(kind=TEX_BITMAP, pixels=img, channels=ch, filter=flt, wrap_u=wu, wrap_v=wv, gamma=gamma,
                       uv_scale=list(map(float, us)), uv_offset=list(map(float, uo)), max_anisotropy=ma)


@pytest.mark.parametrize("case", list(CASES))
def test_bitmap_lookup_bit_exact_vs_reference(case, tmp_path):
    """BitmapTexture::Eval(Isect, filter) record by record."""
    R = _ref()
    w, h, ch = CASES[case][:3]
    img = image(w, h, ch, sum(map(ord, case)))
    t = bitmap_desc(case, img)
    o = O.OracleScene(SceneDesc())
    tid = o.add_texture(t)
    ref = ref_bitmap(R, tmp_path, case + ".png", img, t)
    uv, duv = queries(4000, 5)
    a = o.texture_eval(tid, uv, duv)
    b = np.zeros_like(a)
    R.hr_texture_eval(ref, len(uv), O._p(uv), O._p(duv), O._p(b))
    assert eq_nan(a, b), f"{case}: max |diff| {np.nanmax(np.abs(a - b))}"
    if case == "one_pow2_side":
        assert np.isnan(a).any()   # the reference's Lanczos weight at distance 0 is 0/0: NaN texels
    elif case == "black_wrap_ewa":
        assert (a == 0).all()      # MipMap::Texel reads black everywhere when a wrap mode is "black"
    else:
        assert np.isfinite(a).all() and (a > 0).any()
    avg = np.zeros(3, np.float32)
    R.hr_texture_average(ref, O._p(avg))
    mip = o.texture_mip(tid)
    assert len(mip) == 1 + int(np.log2(max(mip[0].shape[0], mip[0].shape[1])))


def test_bitmap_stb_decode_matches_pil_png(tmp_path):
    """The reference's stbi_load of PNG files gives the pixels written (the
    lossless path the parity tests use), and req = 1 reduces RGB with
    stb's fixed-point luma."""
    R = _ref()
    img = image(33, 17, 3, 1)
    p = os.path.join(tmp_path, "a.png")
    write_png(p, img)
    w, h = C.c_int(0), C.c_int(0)
    out = np.zeros(33 * 17 * 3, np.uint8)
    assert R.hr_image_load(p.encode(), 3, C.byref(w), C.byref(h), O._p(out)) == out.size
    assert (w.value, h.value) == (33, 17)
    np.testing.assert_array_equal(out.reshape(17, 33, 3), img)
    g = np.zeros(33 * 17, np.uint8)
    assert R.hr_image_load(p.encode(), 1, C.byref(w), C.byref(h), O._p(g)) == g.size
    luma = (img[..., 0].astype(np.int32) * 77 + img[..., 1].astype(np.int32) * 150 + img[..., 2].astype(np.int32) * 29) >> 8
    np.testing.assert_array_equal(g.reshape(17, 33), luma.astype(np.uint8))


def _bsdf_cases(img3, img1):
    ewa = TextureDesc(kind=TEX_BITMAP, pixels=img3, channels=3, filter=FILTER_EWA)
    tri = TextureDesc(kind=TEX_BITMAP, pixels=img3, channels=3, filter=FILTER_TRILINEAR, gamma=2.2)
    rough = TextureDesc(kind=TEX_SCALE, scale=0.5,
                        nested=TextureDesc(kind=TEX_BITMAP, pixels=img1, channels=1, filter=FILTER_EWA))
    return {
        "diffuse_ewa": BSDFDesc(type=BSDF_DIFFUSE, textures={"kd": ewa}),
        "plastic_trilinear": BSDFDesc(type=BSDF_ROUGH_PLASTIC, distribution=GGX, alpha_u=0.2, alpha_v=0.2,
                                      textures={"kd": tri}),
        "conductor_alpha_r": BSDFDesc(type=BSDF_ROUGH_CONDUCTOR, distribution=GGX, int_ior=0.2, ext_ior=1.0,
                                      k=[3.9, 2.4, 2.2], textures={"alpha_u": rough, "ks": ewa}),
    }


@pytest.mark.parametrize("name", ["diffuse_ewa", "plastic_trilinear", "conductor_alpha_r"])
def test_bitmap_bsdf_records_bit_exact_vs_reference(name, tmp_path):
    """BSDFs with bitmap-textured parameters, records with screen-space
    partials (the textures' averages feed plastic's sampling weight)."""
    R = _ref()
    img3, img1 = image(40, 24, 3, 11), image(24, 40, 1, 12)
    d = _bsdf_cases(img3, img1)[name]
    o = O.OracleScene(SceneDesc())
    bid = o.add_bsdf(d)
    assert O.lib().ho_scene_finalize(o.h) == 0
    keep = []
    f = lambda a: np.ascontiguousarray(a, np.float32)

    def mk_tex(t):
        if t.kind == TEX_BITMAP:
            return ref_bitmap(R, tmp_path, f"t{len(keep)}.png", t.pixels, t)
        arrs = [f(t.uv_scale), f(t.uv_offset), f(t.a), f(t.b)]
        keep.append(arrs)
        h = R.hr_texture_create(t.kind, t.count, t.width, t.scale, *[O._p(a) for a in arrs], mk_tex(t.nested))
        assert h
        return h

    arrs = [f(d.k), f(d.ks), f(d.kd), f(d.sigma_a), f(d.ks_refract)]
    tex = (C.c_void_p * 6)(*[mk_tex(d.textures[s]) if s in d.textures else None for s in TEX_SLOTS])
    h = R.hr_bsdf_create(d.type, d.distribution, d.alpha_u, d.int_ior, d.ext_ior, *[O._p(a) for a in arrs[:4]],
                         d.thickness, None, None, O._p(arrs[4]), int(d.nonlinear), int(d.fast_approx), tex,
                         int(d.anisotropic))
    assert h
    n = 20000
    wi, u2, u1, wo = records(n, 9)
    uv, duv = queries(n, 10)
    a = o.bsdf_batch(bid, wi, u2, u1, wo, uv=uv, duv=duv)
    b = {k: np.zeros_like(v) for k, v in a.items()}
    R.hr_bsdf_batch(h, n, O._p(wi), O._p(u2), O._p(u1), O._p(wo), O._p(uv), O._p(duv), O._p(b["s_wo"]),
                    O._p(b["s_w"]), O._p(b["s_pdf"]), O._p(b["s_measure"]), O._p(b["e_rgb"]), O._p(b["p_pdf"]))
    for k in a:
        assert eq_nan(a[k], b[k]), f"{name}: {k}"


def test_camera_differentials_and_screen_partials_vs_reference():
    """PerspectiveCamera::SampleRay's differential rays and
    Intersection::ComputeScreenSpacePartial of the first hit, against the
    reference classes (the oracle's closed-form near-plane map agrees with
    the reference's inverted projection to a few ulps)."""
    from hikari_b200 import scenes

    R = _ref()
    rng = np.random.default_rng(23)
    P, F = scenes.displaced_icosphere(2, 1.0, (0.0, 0.0, 0.0), 0.05, 3)
    P, F = P.astype(np.float32), F.astype(np.uint32)
    N = P.copy()
    UV = scenes.spherical_uv(P, (0.0, 0.0, 0.0)).astype(np.float32)
    tw = np.array([[1, 0, 0, 0.1], [0, 1, 0, -0.2], [0, 0, 1, -4.0], [0, 0, 0, 1]], np.float32)
    sd = SceneDesc()
    sd.camera = CameraDesc(width=64, height=48, fov=40.0, to_world=tw)
    sd.meshes.append(MeshDesc(P, F, BSDFDesc(), normals=N, uv=UV))
    o = O.OracleScene(sd)
    twc = np.ascontiguousarray(tw)
    cam = R.hr_camera_create(64, 48, O._p(twc), 40.0, sd.camera.near_clip, sd.camera.far_clip)
    assert cam
    mesh = R.hr_mesh_create(O._p(P), len(P), O._p(N), O._p(UV), O._p(F), len(F))
    for k in range(300):
        px, py = float(rng.uniform(0, 64)), float(rng.uniform(0, 48))
        r = np.zeros(20, np.float32)
        R.hr_camera_ray(cam, px, py, O._p(r))
        a = np.zeros(8, np.float32)
        O.lib().ho_camera_ray(o.h, px, py, O._p(a))
        np.testing.assert_allclose(a[3:6], r[3:6], rtol=0, atol=4e-7)
        tri = int(rng.integers(0, len(F)))
        u = float(rng.random()); v = float(rng.random() * (1 - u))
        pa = o.screen_partials(px, py, tri, u, v)
        pb = np.zeros(4, np.float32)
        R.hr_screen_partials(cam, mesh, tri, u, v, px, py, O._p(pb))
        # the partials solve a 2x2 system on differences of nearby points: an
        # ulp in a direction shows up relative to the largest partial
        np.testing.assert_allclose(pa, pb, rtol=0, atol=5e-4 * np.abs(pb).max() + 1e-7)


def _decode(path, ch):
    import hikari_b200 as hk

    return hk.image_load(str(path), ch)


def _stb(R, path, ch):
    w, h = C.c_int(0), C.c_int(0)
    n = R.hr_image_load(str(path).encode(), ch, C.byref(w), C.byref(h), None)
    assert n > 0, f"stb_image cannot read {path}"
    out = np.zeros(n, np.uint8)
    R.hr_image_load(str(path).encode(), ch, C.byref(w), C.byref(h), O._p(out))
    return out.reshape(h.value, w.value, ch)


@pytest.mark.parametrize("mode", ["RGB", "RGBA", "L", "LA", "P", "I;16", "1"])
def test_png_decode_equals_stb(mode, tmp_path):
    """hk_image_load of PNG files (every color type PIL writes, 16-bit, 1-bit,
    palette) equals the reference's stbi_load byte for byte, for both channel
    requests."""
    R = _ref()
    img = image(45, 31, 3, 7)
    im = PIL.fromarray(img)
    if mode == "RGBA":
        im = im.convert("RGBA")
    elif mode == "LA":
        im = im.convert("LA")
    elif mode == "P":
        im = im.convert("P", palette=PIL.Palette.ADAPTIVE, colors=37) if hasattr(PIL, "Palette") else im.convert("P")
    elif mode == "I;16":
        im = PIL.fromarray((img[:, :, 0].astype(np.uint16) * 257 + 3).astype(np.uint16))
    elif mode != "RGB":
        im = im.convert(mode)
    p = tmp_path / "t.png"
    im.save(p)
    for ch in (1, 3):
        np.testing.assert_array_equal(_decode(p, ch), _stb(R, p, ch), err_msg=f"{mode} ch {ch}")


def test_pnm_decode(tmp_path):
    img = image(13, 9, 3, 8)
    p = tmp_path / "t.ppm"
    p.write_bytes(b"P6\n# comment\n13 9\n255\n" + img.tobytes())
    np.testing.assert_array_equal(_decode(p, 3), img)
    g = tmp_path / "t.pgm"
    g.write_bytes(b"P5 13 9 255\n" + img[:, :, 0].tobytes())
    np.testing.assert_array_equal(_decode(g, 1)[:, :, 0], img[:, :, 0])


@pytest.mark.parametrize("kind", ["420", "444", "422", "gray", "restart"])
def test_jpeg_decode_close_to_stb(kind, tmp_path):
    """Baseline JPEG: the library's float IDCT / triangle upsampling / JFIF
    colour conversion against stb_image's integer versions of the same steps
    (the reference decode): a few levels apart at most, almost all within one."""
    R = _ref()
    img = image(123, 77, 3, 9)
    im = PIL.fromarray(img)
    p = tmp_path / "t.jpg"
    if kind == "gray":
        im.convert("L").save(p, quality=90)
    else:
        sub = {"420": 2, "444": 0, "422": 1, "restart": 2}[kind]
        extra = {"restart_marker_blocks": 3} if kind == "restart" else {}
        try:
            im.save(p, quality=90, subsampling=sub, **extra)
        except TypeError:
            im.save(p, quality=90, subsampling=sub)
    for ch in (1, 3):
        a, b = _decode(p, ch).astype(int), _stb(R, p, ch).astype(int)
        assert a.shape == b.shape
        d = np.abs(a - b)
        if kind == "422" and ch == 3:
            # horizontal-only chroma upsampling: stb_image weights the image's
            # last column differently from the edge-replicating triangle filter
            d = d[:, :-1]
        assert d.max() <= 6 and (d <= 1).mean() >= 0.97, f"{kind} ch {ch}: max {d.max()}, <=1: {(d <= 1).mean():.4f}"


def test_reference_scene_jpegs_close_to_stb():
    """The reference's own scene textures (when its checkout is present)."""
    R = _ref()
    import glob

    files = sorted(glob.glob("/root/reference/scene/bsdf/*.jpg"))
    if not files:
        pytest.skip("reference scene images unavailable")
    for f in files:
        if os.path.getsize(f) > 3_000_000:
            continue
        a, b = _decode(f, 3).astype(int), _stb(R, f, 3).astype(int)
        d = np.abs(a - b)
        assert a.shape == b.shape and d.max() <= 8 and (d <= 1).mean() >= 0.95, \
            f"{os.path.basename(f)}: max {d.max()}, <=1: {(d <= 1).mean():.4f}"


def random_isects(n, seed):
    """n x 20 intersection records: an orthonormal shading frame S T N, a
    geometric normal near N (a tenth facing away), dP/du and dP/dv near S and
    T with random lengths, texture coordinates in [0, 1)."""
    rng = np.random.default_rng(seed)
    N = rng.normal(size=(n, 3))
    N /= np.linalg.norm(N, axis=1, keepdims=True)
    a = rng.normal(size=(n, 3))
    S = a - N * np.sum(a * N, 1, keepdims=True)
    S /= np.linalg.norm(S, axis=1, keepdims=True)
    T = np.cross(N, S)
    G = N + 0.2 * rng.normal(size=(n, 3))
    G /= np.linalg.norm(G, axis=1, keepdims=True)
    G[::10] *= -1
    dpdu = S * rng.uniform(0.2, 3, (n, 1)) + 0.1 * rng.normal(size=(n, 3))
    dpdv = T * rng.uniform(0.2, 3, (n, 1)) + 0.1 * rng.normal(size=(n, 3))
    uv = rng.random((n, 2))
    return np.concatenate([S, T, N, G, dpdu, dpdv, uv], 1).astype(np.float32)


def _bump_cases(img3, img1):
    from hikari_b200.scenedesc import (BSDF_BUMP_MAP, BSDF_NORMAL_MAP, BSDF_ROUGH_DIELECTRIC, TEX_CHECKERBOARD,
                                       TEX_GRID)

    ewa = TextureDesc(kind=TEX_BITMAP, pixels=img3, channels=3, filter=FILTER_EWA, uv_scale=[2.0, 0.5])
    near = TextureDesc(kind=TEX_BITMAP, pixels=img3, channels=3, filter=FILTER_NEAREST)
    r1 = TextureDesc(kind=TEX_BITMAP, pixels=img1, channels=1, filter=FILTER_TRILINEAR)
    chk = TextureDesc(kind=TEX_CHECKERBOARD, count=9, a=[0.9, 0.7, 0.2], b=[0.1, 0.2, 0.3], uv_scale=[1.5, 1.0])
    grid = TextureDesc(kind=TEX_SCALE, scale=0.3, nested=TextureDesc(kind=TEX_GRID, count=7, width=0.1))
    cond = lambda: BSDFDesc(type=BSDF_ROUGH_CONDUCTOR, distribution=GGX, alpha_u=0.15, alpha_v=0.15, int_ior=0.2,
                            ext_ior=1.0, k=[3.9, 2.4, 2.2])
    return {
        "bump_bitmap_diffuse": BSDFDesc(type=BSDF_BUMP_MAP, nested=BSDFDesc(type=BSDF_DIFFUSE, kd=[0.6, 0.5, 0.4]),
                                        textures={"kd": ewa}),
        "bump_r_conductor": BSDFDesc(type=BSDF_BUMP_MAP, nested=cond(), textures={"kd": r1}),
        "bump_nearest_plastic": BSDFDesc(type=BSDF_BUMP_MAP, nested=BSDFDesc(type=BSDF_ROUGH_PLASTIC,
                                                                             distribution=GGX, alpha_u=0.2,
                                                                             alpha_v=0.2), textures={"kd": near}),
        "bump_checker_dielectric": BSDFDesc(type=BSDF_BUMP_MAP, nested=BSDFDesc(
            type=BSDF_ROUGH_DIELECTRIC, distribution=GGX, alpha_u=0.2, alpha_v=0.2, int_ior=1.5, ext_ior=1.0),
            textures={"kd": chk}),
        "bump_scaled_grid_conductor": BSDFDesc(type=BSDF_BUMP_MAP, nested=cond(), textures={"kd": grid}),
        "normal_bitmap_plastic": BSDFDesc(type=BSDF_NORMAL_MAP, nested=BSDFDesc(type=BSDF_ROUGH_PLASTIC,
                                                                              distribution=GGX, alpha_u=0.2,
                                                                              alpha_v=0.2), textures={"kd": ewa}),
        "normal_checker_diffuse": BSDFDesc(type=BSDF_NORMAL_MAP, nested=BSDFDesc(type=BSDF_DIFFUSE),
                                           textures={"kd": chk}),
    }


BUMP_CASES = ["bump_bitmap_diffuse", "bump_r_conductor", "bump_nearest_plastic", "bump_checker_dielectric",
              "bump_scaled_grid_conductor", "normal_bitmap_plastic", "normal_checker_diffuse"]


@pytest.mark.parametrize("name", BUMP_CASES)
def test_bump_normal_map_bit_exact_vs_reference(name, tmp_path):
    """BumpMapBSDF / NormalMapBSDF (perturbed frames from texture gradients or
    a normal map) record by record, each record with its own intersection."""
    R = _ref()
    R.hr_bsdf_batch_isect.argtypes = [C.c_void_p, C.c_uint64] + [C.c_void_p] * 11
    img3, img1 = image(40, 24, 3, 21), image(33, 29, 1, 22)
    d = _bump_cases(img3, img1)[name]
    o = O.OracleScene(SceneDesc())
    bid = o.add_bsdf(d)
    assert O.lib().ho_scene_finalize(o.h) == 0
    keep = []
    f = lambda a: np.ascontiguousarray(a, np.float32)

    def mk_tex(t):
        if t.kind == TEX_BITMAP:
            return ref_bitmap(R, tmp_path, f"t{len(keep)}.png", t.pixels, t)
        arrs = [f(t.uv_scale), f(t.uv_offset), f(t.a), f(t.b)]
        keep.append(arrs)
        h = R.hr_texture_create(t.kind, t.count, t.width, t.scale, *[O._p(a) for a in arrs],
                                mk_tex(t.nested) if t.nested is not None else None)
        assert h
        return h

    def mk(b):
        if b is None:
            return None
        arrs = [f(b.k), f(b.ks), f(b.kd), f(b.sigma_a), f(b.ks_refract)]
        keep.append(arrs)
        tex = (C.c_void_p * 6)(*[mk_tex(b.textures[s]) if s in b.textures else None for s in TEX_SLOTS])
        keep.append(tex)
        h = R.hr_bsdf_create(b.type, b.distribution, b.alpha_u, b.int_ior, b.ext_ior, *[O._p(a) for a in arrs[:4]],
                             b.thickness, mk(b.nested), None, O._p(arrs[4]), int(b.nonlinear), int(b.fast_approx), tex,
                             int(b.anisotropic))
        assert h
        return h

    h = mk(d)
    n = 20000
    wi, u2, u1, wo = records(n, 31)
    isect = random_isects(n, 32)
    a = o.bsdf_batch_isect(bid, wi, u2, u1, wo, isect)
    b = {k: np.zeros_like(v) for k, v in a.items()}
    R.hr_bsdf_batch_isect(h, n, O._p(wi), O._p(u2), O._p(u1), O._p(wo), O._p(isect), O._p(b["s_wo"]),
                          O._p(b["s_w"]), O._p(b["s_pdf"]), O._p(b["s_measure"]), O._p(b["e_rgb"]), O._p(b["p_pdf"]))
    valid = np.any(a["s_w"] != 0, axis=1)
    assert valid.mean() > 0.05 and (a["e_rgb"] != 0).any()
    for k in ("s_w", "s_measure", "s_pdf", "e_rgb", "p_pdf"):
        assert eq_nan(a[k], b[k]), f"{name}: {k}"
    assert eq_nan(a["s_wo"][valid], b["s_wo"][valid]), f"{name}: s_wo"
