"""Bitmap textures on the device against the oracle: MIP lookups (nearest,
bilinear, trilinear, EWA; r and rgb; wrap modes; resampled and NaN-texel
pyramids) through hk_texture_eval, and BSDF records with bitmap-textured
parameters and screen-space partials through hk_bsdf_batch.

Nearest and bilinear lookups are bit-exact.  Trilinear and EWA choose their
level with log2f, whose last place may differ between CUDA and the host libm;
the lerp between two levels then moves by about that much, so those lookups
are held to 2e-6 absolute (+ 1e-5 relative) and most are still bit-exact."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

import hikari_b200 as hk  # noqa: E402
from hikari_b200 import scenes  # noqa: E402
from hikari_b200.scenedesc import (BSDF_DIFFUSE, BSDF_ROUGH_CONDUCTOR, BSDF_ROUGH_PLASTIC, FILTER_BILINEAR,  # noqa: E402
                                   FILTER_EWA, FILTER_NEAREST, FILTER_TRILINEAR, GGX, TEX_BITMAP, TEX_SCALE,
                                   WRAP_BLACK, WRAP_CLAMP, WRAP_REPEAT, BSDFDesc, TextureDesc)
from oracle.oracle import OracleScene  # noqa: E402

DEV = "cuda:0"

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
    "one_pow2_side": (16, 12, 3, FILTER_EWA, WRAP_REPEAT, WRAP_REPEAT, 1.0, [1, 1], [0, 0], 20.0),
    "large_ewa": (1000, 700, 3, FILTER_EWA, WRAP_REPEAT, WRAP_REPEAT, 2.2, [1, 1], [0, 0], 20.0),
}


def queries(n, seed):
    rng = np.random.default_rng(seed)
    uv = rng.uniform(-0.3, 1.3, (n, 2)).astype(np.float32)
    duv = (10.0 ** rng.uniform(-4.5, 0.3, (n, 4)) * rng.choice([-1, 1], (n, 4))).astype(np.float32)
    duv[: n // 10] = 0.0
    duv[n // 10: n // 5, 2:] = 0.0
    duv[-50:, 2:] = duv[-50:, :2] * 1e-3
    return uv, duv


def close(g, o, exact):
    both_nan = np.isnan(g) & np.isnan(o)
    if exact:
        return np.array_equal(np.isnan(g), np.isnan(o)) and np.array_equal(g[~both_nan], o[~both_nan])
    ok = both_nan | (np.abs(g - o) <= 2e-6 + 1e-5 * np.abs(o))
    return bool(ok.all())


@pytest.mark.parametrize("case", list(CASES))
def test_gpu_bitmap_lookups_match_oracle(case):
    w, h, ch, flt, wu, wv, gamma, us, uo, ma = CASES[case]
    t = TextureDesc(kind=TEX_BITMAP, pixels=scenes.synthetic_image(w, h, ch, sum(map(ord, case))), channels=ch,
                    filter=flt, wrap_u=wu, wrap_v=wv, gamma=gamma, uv_scale=list(map(float, us)),
                    uv_offset=list(map(float, uo)), max_anisotropy=ma)
    sd = scenes.bsdf_scene([("d", BSDFDesc(type=BSDF_DIFFUSE, textures={"kd": t}))])
    gs = hk.Scene.from_desc(sd)
    os_ = OracleScene(sd)
    os_.add_texture(t)
    uv, duv = queries(20000, 3)
    g = gs.texture_eval(gs.tex_ids[id(t)], torch.from_numpy(uv).to(DEV), torch.from_numpy(duv).to(DEV)).cpu().numpy()
    o = os_.texture_eval(t, uv, duv)
    exact = flt in (FILTER_NEAREST, FILTER_BILINEAR)
    assert close(g, o, exact), f"{case}: max |diff| {np.nanmax(np.abs(g - o))}"
    same = np.mean(np.all((g == o) | (np.isnan(g) & np.isnan(o)), axis=1))
    print(f"{case}: {same:.4f} of lookups bit-exact")
    assert same >= 0.9


def test_gpu_bitmap_bsdf_records_match_oracle():
    img3, img1 = scenes.synthetic_image(40, 24, 3, 11), scenes.synthetic_image(24, 40, 1, 12)
    ewa = TextureDesc(kind=TEX_BITMAP, pixels=img3, channels=3, filter=FILTER_EWA)
    tri = TextureDesc(kind=TEX_BITMAP, pixels=img3, channels=3, filter=FILTER_TRILINEAR, gamma=2.2)
    rough = TextureDesc(kind=TEX_SCALE, scale=0.5,
                        nested=TextureDesc(kind=TEX_BITMAP, pixels=img1, channels=1, filter=FILTER_EWA))
    mats = [("diffuse_ewa", BSDFDesc(type=BSDF_DIFFUSE, textures={"kd": ewa})),
            ("plastic_trilinear", BSDFDesc(type=BSDF_ROUGH_PLASTIC, distribution=GGX, alpha_u=0.2, alpha_v=0.2,
                                           textures={"kd": tri})),
            ("conductor_alpha_r", BSDFDesc(type=BSDF_ROUGH_CONDUCTOR, distribution=GGX, int_ior=0.2, ext_ior=1.0,
                                           k=[3.9, 2.4, 2.2], textures={"alpha_u": rough, "ks": ewa}))]
    sd = scenes.bsdf_scene(mats)
    gs = hk.Scene.from_desc(sd)
    os_ = OracleScene(sd)
    rng = np.random.default_rng(4)
    n = 20000
    z = rng.uniform(-0.2, 1, n)
    ph = rng.uniform(0, 2 * np.pi, n)
    wi = np.stack([np.sqrt(1 - z * z) * np.cos(ph), np.sqrt(1 - z * z) * np.sin(ph), z], 1).astype(np.float32)
    z2 = rng.uniform(0.05, 1, n)
    ph2 = rng.uniform(0, 2 * np.pi, n)
    wo = np.stack([np.sqrt(1 - z2 * z2) * np.cos(ph2), np.sqrt(1 - z2 * z2) * np.sin(ph2), z2], 1).astype(np.float32)
    u2 = rng.random((n, 2), dtype=np.float32)
    u1 = rng.random(n, dtype=np.float32)
    uv, duv = queries(n, 5)
    T = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(DEV)
    for (name, d), bid in zip(mats, range(len(mats))):
        gid = gs.bsdf_ids[id(d)]
        oid = os_.bsdf_ids[id(d)]
        g = {k: v.cpu().numpy() for k, v in gs.bsdf_batch(gid, T(wi), T(u2), T(u1), T(wo), uv=T(uv), duv=T(duv)).items()}
        o = os_.bsdf_batch(oid, wi, u2, u1, wo, uv=uv, duv=duv)
        np.testing.assert_array_equal(g["s_measure"], o["s_measure"], err_msg=name)
        assert close(g["e_rgb"], o["e_rgb"], False), f"{name} e_rgb: max |diff| {np.nanmax(np.abs(g['e_rgb'] - o['e_rgb']))}"
        # sampled weights also carry the sampled direction's ulps (CUDA's sinf / cosf / expf)
        tight = np.all(np.abs(g["s_w"] - o["s_w"]) <= 2e-6 + 1e-5 * np.abs(o["s_w"]), axis=1)
        assert tight.mean() >= 0.999, f"{name} s_w: {tight.mean():.5f} within 1e-5"
        np.testing.assert_allclose(g["s_w"], o["s_w"], rtol=1e-3, atol=1e-5, err_msg=f"{name} s_w")
        np.testing.assert_allclose(g["p_pdf"], o["p_pdf"], rtol=1e-5, atol=1e-6, err_msg=f"{name} p_pdf")
        # the sampled direction carries CUDA's sinf / cosf (ulps from the host's):
        # its pdf moves by a few 1e-6 near grazing angles, by < 1e-4 relative on sharp lobes
        np.testing.assert_allclose(g["s_pdf"], o["s_pdf"], rtol=5e-4, atol=1e-5, err_msg=f"{name} s_pdf")
