"""Parity of the CUDA core (through the C ABI) with the CPU oracle.

Tolerances (the arithmetic order is the reference's; the only source of
disagreement is the ulp difference between CUDA's sinf/cosf/logf/expf/powf
and the host libm's):
  * integer outputs (sample measure) match exactly;
  * BSDF Eval and Pdf at identical inputs agree within 1e-5 relative on
    >= 99.99% of records and within 1e-3 on all (the Oren-Nayar model takes
    acosf of the cosines and subtracts terms that nearly cancel);
  * sampled directions agree within 1e-5 absolute (unit vectors) on >= 99.99%
    of records and within 1e-3 on all; sampled
    weights and pdfs agree within 1e-5 relative on >= 99.8% of records and
    within 1e-2 on all -- a 1-ulp difference of sin/cos/log of the random
    number is amplified by the conditioning of the sampling map near grazing
    angles, which the chi2 tests below cover distributionally;
  * triangle ids match except on exact t-ties (coplanar triangles) and on
    edges, where the reference's own answer depends on traversal order;
  * rendered images are compared statistically.
"""
import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

import hikari_b200 as hk  # noqa: E402
from hikari_b200 import scenes  # noqa: E402
from hikari_b200.scenedesc import FilterDesc, parse_xml  # noqa: E402
from oracle.oracle import OracleScene, students_t_test  # noqa: E402
from tests.gpu_helpers import bsdf_records, rel_close  # noqa: E402

DEV = "cuda:0"
RTOL = 1e-5


@pytest.fixture(scope="module", params=["rough", "smooth", "textured", "nested"])
def bsdf_pair(request):
    """The BSDF-batch material set (rough BSDFs and a coating), the smooth and
    two-sided set, the set with procedural textures (records carry texture
    coordinates), or layers nested deeper than one coating over a leaf."""
    mats = {"rough": scenes.config2_materials, "smooth": scenes.smooth_materials,
            "textured": scenes.textured_materials, "nested": scenes.nested_materials}[request.param]()
    sd = scenes.bsdf_scene(mats)
    return mats, hk.Scene.from_desc(sd), OracleScene(sd), request.param


def _t(a):
    return torch.from_numpy(np.ascontiguousarray(a)).to(DEV)


def test_bsdf_batch_parity(bsdf_pair):
    mats, gs, os_, kind = bsdf_pair
    n = 1 << 17
    wi, u2, u1, wo = bsdf_records(n, 11)
    if kind != "rough":   # a tenth of the evaluation directions on the mirror direction
        wo[0::10] = wi[0::10] * np.float32([-1, -1, 1])
    uv = (np.random.default_rng(5).random((n, 2)) * 4 - 1).astype(np.float32) if kind == "textured" else None
    tuv = _t(uv) if uv is not None else None
    twi, tu2, tu1, two = _t(wi), _t(u2), _t(u1), _t(wo)
    report = []
    for i, (name, d) in enumerate(mats):
        gid = gs.bsdf_ids[id(d)]
        oid = os_.bsdf_ids[id(d)]
        g = {k: v.cpu().numpy() for k, v in gs.bsdf_batch(gid, twi, tu2, tu1, two, uv=tuv).items()}
        o = os_.bsdf_batch(oid, wi, u2, u1, wo, uv=uv)
        for key in ("e_rgb", "p_pdf"):
            ok = rel_close(g[key], o[key], RTOL).reshape(n, -1).all(1)
            loose = rel_close(g[key], o[key], 1e-3).reshape(n, -1).all(1)
            report.append((name, key, ok.mean()))
            assert ok.mean() >= 0.9999, f"{name} {key}: {ok.mean():.6f} within {RTOL}"
            assert loose.all(), f"{name} {key}: {np.sum(~loose)} records beyond 1e-3"
        # Sampling: a 1-ulp difference can flip a threshold (u1 against the
        # Fresnel term, a direction at the horizon); flips must stay below 1e-4
        # of the records, every other record is held to the tolerances.
        flip = (g["s_measure"] != o["s_measure"]) | (np.all(g["s_w"] == 0, 1) != np.all(o["s_w"] == 0, 1))
        assert flip.mean() <= 1e-4, f"{name}: {flip.sum()} sampling branch flips"
        keep = ~flip
        valid = keep & np.any(o["s_w"] != 0, axis=1)
        dwo = np.abs(g["s_wo"][valid].astype(np.float64) - o["s_wo"][valid]).max(1)
        # z = sqrt(1 - r^2) is ill-conditioned at the horizon: the cosine warp's
        # output, and a coating's refraction out of the layer near the critical
        # angle (dz_out / dz_in ~ eta^2 z_in / z_out); grazing records
        # (|z| < 0.05, where a few-ulp difference of sin/cos can exceed 1e-5)
        # are held to the looser bound only.  A coating's specular probability
        # comes from the rough-transmittance lookup (powf) and divides u: a
        # 1-ulp change there moves samples in the microfacet tail by up to 1e-4
        # (perturbing the oracle's lookup by one ulp moves them as much), so
        # 2e-4 of the records may exceed 1e-5.
        steep = np.abs(o["s_wo"][valid][:, 2]) >= 0.05
        bad = (dwo > 1e-5) & steep
        assert np.mean(~bad) >= 0.9998, f"{name}: sampled directions differ by > 1e-5 on {bad.sum()} steep records"
        assert dwo.max() <= 1e-3, f"{name}: sampled directions differ by {dwo.max()}"
        # weights and pdfs: 1e-2 on every record whose sampled direction is not
        # grazing; at grazing exits the Fresnel transmittance near the critical
        # angle (a square-root edge) and the cosine map turn ulps into percents
        idx = np.nonzero(keep)[0]
        steep_all = np.abs(o["s_wo"][idx][:, 2]) >= 0.05
        for key in ("s_w", "s_pdf"):
            ok = rel_close(g[key][idx], o[key][idx], RTOL).reshape(len(idx), -1).all(1)
            loose = rel_close(g[key][idx], o[key][idx], 1e-2).reshape(len(idx), -1).all(1)
            report.append((name, key, ok.mean()))
            # anisotropic microfacet sampling goes through tanf / atanf of the
            # random number: 0.2% of its weights may differ beyond 1e-5
            assert ok.mean() >= 0.998, f"{name} {key}: {ok.mean():.6f} within {RTOL}"
            far = idx[~loose & steep_all]
            assert len(far) == 0, (f"{name} {key}: {len(far)} steep records beyond 1e-2, first {far[0]}: wi {wi[far[0]]} "
                                   f"u2 {u2[far[0]]} u1 {u1[far[0]]} gpu {g[key][far[0]]} oracle {o[key][far[0]]} "
                                   f"wo {o['s_wo'][far[0]]}")
            assert np.isfinite(g[key][idx]).all() == np.isfinite(o[key][idx]).all()
    worst = min(report, key=lambda r: r[2])
    print("worst BSDF agreement:", worst)


def test_camera_rays_parity():
    sd = scenes.cornell_box(width=64, height=48)
    gs, os_ = hk.Scene.from_desc(sd), OracleScene(sd)
    rng = np.random.default_rng(3)
    pos = np.stack([rng.uniform(0, 64, 4096), rng.uniform(0, 48, 4096)], 1).astype(np.float32)
    g = gs.camera_rays(_t(pos)).cpu().numpy()
    o = np.stack([os_.camera_ray(float(p[0]), float(p[1])) for p in pos])
    assert rel_close(g, o, 1e-6, atol=1e-7).all()


def _camera_rays(sd, os_, n, seed):
    rng = np.random.default_rng(seed)
    W, H = sd.camera.width, sd.camera.height
    return np.stack([os_.camera_ray(float(x), float(y)) for x, y in
                     zip(rng.uniform(0, W, n), rng.uniform(0, H, n))]).astype(np.float32)


@pytest.mark.parametrize("accel", [hk.ACCEL_BVH2, hk.ACCEL_BVH8])
def test_trace_parity_cornell(accel):
    sd = scenes.cornell_box(width=64, height=64)
    gs, os_ = hk.Scene.from_desc(sd), OracleScene(sd)
    gs.set_accel(accel)
    assert gs.info.accel == accel
    rays = _camera_rays(sd, os_, 20000, 5)
    # add random interior rays (origins inside the box, random directions)
    rng = np.random.default_rng(9)
    o = np.stack([rng.uniform(-0.9, 0.9, 20000), rng.uniform(0.1, 1.9, 20000), rng.uniform(-0.9, 0.9, 20000)], 1)
    d = rng.normal(size=(20000, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    extra = np.concatenate([o, d, np.full((20000, 1), 1e-4), np.full((20000, 1), np.inf)], 1).astype(np.float32)
    rays = np.concatenate([rays, extra], 0)
    tri_g, t_g, u_g, v_g, _ = gs.trace(_t(rays))
    tri_g, t_g = tri_g.cpu().numpy(), t_g.cpu().numpy()
    tri_o, t_o, u_o, v_o = os_.trace(rays, use_bvh=False)
    same = tri_g == tri_o
    # every mismatch is a t-tie (coplanar triangles: the box bottoms lie on the
    # floor) or an edge hit; hit/miss decisions agree except on edges
    bad = ~same
    edge = np.minimum(np.minimum(u_o, v_o), 1 - u_o - v_o) < 1e-5
    tie = (tri_g >= 0) & (tri_o >= 0) & rel_close(t_g, t_o, 1e-6)
    assert np.all(tie[bad] | edge[bad]), f"{np.sum(bad & ~tie & ~edge)} non-tie, non-edge mismatches"
    print(f"triangle ids bit-exact on {same.mean():.5f} of rays, {np.sum(bad & tie)} ties, {np.sum(bad & ~tie)} edges")
    both = same & (tri_o >= 0)
    assert rel_close(t_g[both], t_o[both], 1e-6).mean() > 0.999
    # any-hit agrees on the hit/miss decision
    any_g = gs.trace(_t(rays), any_hit=True)[0].cpu().numpy()
    any_o = os_.trace(rays, any_hit=True, use_bvh=False)[0]
    assert (any_g == any_o).mean() > 0.999


@pytest.mark.parametrize("accel", [hk.ACCEL_BVH2, hk.ACCEL_BVH8])
def test_trace_parity_displaced_sphere(accel):
    """Closest and any hit on a 20k-triangle displaced icosphere over a ground
    quad, rays from outside and inside, against the oracle's brute force."""
    sd = scenes.mesh_heavy("conductor", width=16, height=16, level=5, env_res=(64, 32))
    gs, os_ = hk.Scene.from_desc(sd), OracleScene(sd)
    gs.set_accel(accel)
    rng = np.random.default_rng(21)
    n = 30000
    o = np.concatenate([rng.uniform(-3, 3, (n // 2, 3)) + [0, 1.5, 0],
                        rng.normal(0, 0.3, (n - n // 2, 3)) + [0, 1.0, 0]]).astype(np.float32)
    d = rng.normal(size=(n, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    rays = np.concatenate([o, d, np.full((n, 1), 1e-4), np.full((n, 1), np.inf)], 1).astype(np.float32)
    tri_g, t_g, _, _, visits = gs.trace(_t(rays))
    tri_g, t_g = tri_g.cpu().numpy(), t_g.cpu().numpy()
    tri_o, t_o, u_o, v_o = os_.trace(rays, use_bvh=False)
    same = tri_g == tri_o
    bad = ~same
    edge = np.minimum(np.minimum(u_o, v_o), 1 - u_o - v_o) < 1e-5
    tie = (tri_g >= 0) & (tri_o >= 0) & rel_close(t_g, t_o, 1e-6)
    print(f"accel {accel}: ids bit-exact on {same.mean():.6f}, {np.sum(bad & tie)} ties, {np.sum(bad & ~tie)} others; "
          f"node visits per ray {visits[0].item() / n:.1f}, triangle tests per ray {visits[1].item() / n:.1f}")
    assert np.all(tie[bad] | edge[bad]), f"{np.sum(bad & ~tie & ~edge)} non-tie, non-edge mismatches"
    assert same.mean() > 0.999
    both = same & (tri_o >= 0)
    assert rel_close(t_g[both], t_o[both], 1e-6).mean() > 0.999
    any_g = gs.trace(_t(rays), any_hit=True)[0].cpu().numpy()
    any_o = os_.trace(rays, any_hit=True, use_bvh=False)[0]
    assert (any_g == any_o).mean() > 0.999


def test_area_emitter_sample_parity():
    sd = scenes.cornell_box(width=16, height=16)
    gs, os_ = hk.Scene.from_desc(sd), OracleScene(sd)
    rng = np.random.default_rng(4)
    n = 4096
    inp = np.zeros((n, 8), np.float32)
    inp[:, 0] = rng.uniform(-0.9, 0.9, n)
    inp[:, 1] = rng.uniform(0.1, 1.5, n)
    inp[:, 2] = rng.uniform(-0.9, 0.9, n)
    inp[:, 3:6] = rng.random((n, 3))
    g = gs.emitter_sample(0, _t(inp)).cpu().numpy()
    o = np.stack([os_.emitter_sample(0, r[:3], (r[3], r[4], r[5])) for r in inp])
    assert rel_close(g[:, :14], o[:, :14], 1e-5, atol=1e-6).mean() > 0.9999


@pytest.mark.parametrize("emitter", [0, 1, 2, 3])
def test_light_emitter_sample_parity(emitter):
    """Point light, area light, constant environment and directional light
    (the emitter order of the lights scene) sampled on the GPU and by the oracle."""
    sd = scenes.lights_scene(width=16, height=16)
    gs, os_ = hk.Scene.from_desc(sd), OracleScene(sd)
    assert gs.info.n_emitters == 4 and gs.info.env_index == 2
    rng = np.random.default_rng(40 + emitter)
    n = 4096
    inp = np.zeros((n, 8), np.float32)
    inp[:, 0:3] = rng.uniform(-3, 3, (n, 3)) + [0, 2, 0]
    inp[:, 3:6] = rng.random((n, 3))
    g = gs.emitter_sample(emitter, _t(inp)).cpu().numpy()
    o = np.stack([os_.emitter_sample(emitter, r[:3], (r[3], r[4], r[5])) for r in inp])
    ok = rel_close(g[:, :14], o[:, :14], 1e-5, atol=1e-5)
    print("emitter", emitter, "records within 1e-5:", ok.all(1).mean())
    assert ok.all(1).mean() > 0.999
    if emitter == 2:   # the constant environment's Eval and Pdf
        d = rng.normal(size=(n, 3)).astype(np.float32)
        d /= np.linalg.norm(d, axis=1, keepdims=True)
        rgb, pdf = gs.env_eval(_t(d))
        assert np.array_equal(rgb.cpu().numpy(), np.tile(np.float32(sd.env_constant), (n, 1)))
        po = np.array([os_.emitter_pdf(2, np.zeros(3), x, np.zeros(3)) for x in d], np.float32)
        assert rel_close(pdf.cpu().numpy(), po, 1e-5).mean() > 0.999


def test_env_emitter_parity():
    sd = scenes.mesh_heavy("conductor", width=32, height=32, level=2, env_res=(256, 128))
    gs, os_ = hk.Scene.from_desc(sd), OracleScene(sd)
    e = sd.emitter_order().index(-1)
    rng = np.random.default_rng(8)
    n = 4096
    inp = np.zeros((n, 8), np.float32)
    inp[:, 0:3] = rng.uniform(-1, 1, (n, 3))
    inp[:, 3:6] = rng.random((n, 3))
    g = gs.emitter_sample(e, _t(inp)).cpu().numpy()
    o = np.stack([os_.emitter_sample(e, r[:3], (r[3], r[4], r[5])) for r in inp])
    assert rel_close(g[:, :14], o[:, :14], 1e-5, atol=1e-5).mean() > 0.999
    d = rng.normal(size=(n, 3)).astype(np.float32)
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    rgb_g, _ = gs.env_eval(_t(d))
    rgb_o = np.stack([os_.env_eval(x) for x in d])
    assert rel_close(rgb_g.cpu().numpy(), rgb_o, 1e-6).mean() > 0.999


def _render_mean_over_seeds(gs, depth, spp, k, film_shape):
    means = []
    for s in range(k):
        film = torch.zeros(film_shape, dtype=torch.float32, device=DEV)
        gs.render(film, spp=spp, depth=depth, seed=1000 + s)
        rgb = torch.empty((gs.desc.camera.height, gs.desc.camera.width, 3), dtype=torch.float32, device=DEV)
        gs.resolve(film, rgb)
        c = rgb.cpu().numpy().reshape(-1, 3).mean(0)
        means.append(c[0] * 0.212671 + c[1] * 0.715160 + c[2] * 0.072169)
    return np.array(means)


@pytest.mark.parametrize("fname", ["test-direct.xml", "test-furnace.xml"])
def test_render_golden_ttest(golden_dir, fname):
    """The reference's pathMIS known answers, rendered by the CUDA megakernel:
    K independent renders of N spp each; t-test of their mean against the
    reference value (Sidak-corrected like hypothesis::students_t_test)."""
    import os

    all_scenes = parse_xml(os.path.join(golden_dir, "pa5", fname))
    mis = [s for s in all_scenes if s.integrator == "pathMIS"]
    for sd in mis:
        gs = hk.Scene.from_desc(sd)
        shape = gs.film_shape()
        m = _render_mean_over_seeds(gs, sd.depth, 2000, 64, shape)
        ok, p = students_t_test(m.mean(), m.var(ddof=1), sd.reference, len(m), 0.01, len(all_scenes))
        assert ok, f"{fname}: GPU mean {m.mean()} vs reference {sd.reference} (p={p})"


def test_render_cornell_matches_oracle():
    """Per-pixel means of the GPU image (box filter) against the oracle's
    per-pixel means and variances."""
    sd = scenes.cornell_box(width=48, height=48)
    sd.filter = FilterDesc(0, 0.5)
    gs, os_ = hk.Scene.from_desc(sd), OracleScene(sd)
    spp_g, spp_o = 4096, 2048
    img, ctr = gs.render_image(spp_g, sd.depth, seed=7)
    pix = np.stack(np.meshgrid(np.arange(48), np.arange(48), indexing="xy"), -1).reshape(-1, 2)
    mean_o, var_o = os_.pixel_stats(pix, spp_o, seed=3)
    g = img.reshape(-1, 3).astype(np.float64)
    se = np.sqrt(var_o / spp_g + var_o / spp_o) + 1e-6
    z = (g - mean_o) / se
    frac3 = np.mean(np.abs(z) > 3)
    print("z mean", z.mean(), "frac |z|>3", frac3, "max", np.abs(z).max(), "counters", ctr)
    assert abs(g.mean() / mean_o.mean() - 1) < 0.01
    # normal tail P(|z| > 3) = 0.27%; the per-pixel variances are estimates
    assert frac3 < 0.008
    assert ctr[0] >= 48 * 48 * spp_g


def test_layer_nesting_depth_limit():
    """Coatings stack up to four layers over a leaf BSDF on the device; a fifth
    is rejected when the scene is built, with the limit in the message."""
    from hikari_b200.scenedesc import BSDF_COATING, BSDF_DIFFUSE, BSDF_ROUGH_COATING, GGX, BSDFDesc

    def stack(n):
        d = BSDFDesc(type=BSDF_DIFFUSE, kd=[0.5, 0.5, 0.5])
        for k in range(n):
            d = BSDFDesc(type=BSDF_COATING if k % 2 else BSDF_ROUGH_COATING, distribution=GGX, alpha_u=0.2,
                         alpha_v=0.2, nested=d)
        return d

    four = scenes.bsdf_scene([("four", stack(4))])
    gs, os_ = hk.Scene.from_desc(four), OracleScene(four)
    wi, u2, u1, wo = bsdf_records(1 << 12, 3)
    d = four.meshes[0].bsdf
    g = gs.bsdf_batch(gs.bsdf_ids[id(d)], _t(wi), _t(u2), _t(u1), _t(wo))
    o = os_.bsdf_batch(os_.bsdf_ids[id(d)], wi, u2, u1, wo)
    assert rel_close(g["e_rgb"].cpu().numpy(), o["e_rgb"], 1e-4).all(1).mean() >= 0.999
    with pytest.raises(hk.HikariError, match="deeper than 4"):
        hk.Scene.from_desc(scenes.bsdf_scene([("five", stack(5))]))
