"""The wavefront integrator against the megakernel and the reference's known
answers.  Both run the reference estimator; their sample streams differ, so
images are compared statistically."""
import os

import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

import hikari_b200 as hk  # noqa: E402
from hikari_b200 import scenes  # noqa: E402
from hikari_b200.scenedesc import FilterDesc, parse_xml  # noqa: E402
from oracle.oracle import OracleScene, students_t_test  # noqa: E402

DEV = "cuda:0"


def _resolve(gs, film):
    cam = gs.desc.camera
    rgb = torch.empty((cam.height, cam.width, 3), dtype=torch.float32, device=DEV)
    gs.resolve(film, rgb)
    return rgb.cpu().numpy()


@pytest.mark.parametrize("fname", ["test-direct.xml", "test-furnace.xml"])
def test_wavefront_golden_ttest(golden_dir, fname):
    all_scenes = parse_xml(os.path.join(golden_dir, "pa5", fname))
    for sd in [s for s in all_scenes if s.integrator == "pathMIS"]:
        gs = hk.Scene.from_desc(sd)
        k = 64
        films = [torch.zeros(gs.film_shape(), dtype=torch.float32, device=DEV) for _ in range(k)]
        gs.render_batch(films, spp=2000, depth=sd.depth, seeds=list(range(100, 100 + k)), capacity=1 << 16)
        means = []
        for f in films:
            c = _resolve(gs, f).reshape(-1, 3).mean(0)
            means.append(c[0] * 0.212671 + c[1] * 0.715160 + c[2] * 0.072169)
        m = np.array(means)
        ok, p = students_t_test(m.mean(), m.var(ddof=1), sd.reference, len(m), 0.01, len(all_scenes))
        assert ok, f"{fname}: wavefront mean {m.mean()} vs reference {sd.reference} (p={p})"


def test_wavefront_cornell_matches_oracle():
    sd = scenes.cornell_box(width=48, height=48)
    sd.filter = FilterDesc(0, 0.5)
    gs, os_ = hk.Scene.from_desc(sd), OracleScene(sd)
    film = torch.zeros(gs.film_shape(), dtype=torch.float32, device=DEV)
    ctr = torch.zeros(7, dtype=torch.int64, device=DEV)
    gs.render_batch([film], spp=4096, depth=sd.depth, seeds=[7], counters=ctr, capacity=1 << 18)
    g = _resolve(gs, film).reshape(-1, 3).astype(np.float64)
    pix = np.stack(np.meshgrid(np.arange(48), np.arange(48), indexing="xy"), -1).reshape(-1, 2)
    mean_o, var_o = os_.pixel_stats(pix, 2048, seed=3)
    z = (g - mean_o) / (np.sqrt(var_o / 4096 + var_o / 2048) + 1e-6)
    frac3 = np.mean(np.abs(z) > 3)
    c = ctr.cpu().numpy()
    print("z mean", z.mean(), "frac |z|>3", frac3, "max", np.abs(z).max(), "counters", c)
    assert abs(g.mean() / mean_o.mean() - 1) < 0.01
    # normal tail P(|z| > 3) = 0.27%; the per-pixel variances are estimates
    assert frac3 < 0.008
    assert c[0] >= 48 * 48 * 4096


def test_wavefront_matches_megakernel_heterogeneous():
    """Same scene, same views: the two integrators agree on the image mean per
    view and per channel within their statistical error."""
    sd = scenes.heterogeneous(width=96, height=96, spp=64)
    cams = scenes.heterogeneous_cameras(2)
    gs = hk.Scene.from_desc(sd)
    mk, wf = [], []
    for v, cam in enumerate(cams):
        means_m, means_w = [], []
        for rep in range(6):
            f = torch.zeros(gs.film_shape(), dtype=torch.float32, device=DEV)
            gs.render(f, spp=64, depth=sd.depth, seed=10 * rep + v, camera=cam)
            means_m.append(_resolve(gs, f).mean((0, 1)))
            f2 = torch.zeros(gs.film_shape(), dtype=torch.float32, device=DEV)
            gs.render_batch([f2], spp=64, depth=sd.depth, seeds=[1000 + 10 * rep + v], cameras=[cam],
                            capacity=1 << 18)
            means_w.append(_resolve(gs, f2).mean((0, 1)))
        mm, mw = np.array(means_m), np.array(means_w)
        se = np.sqrt(mm.var(0, ddof=1) / len(mm) + mw.var(0, ddof=1) / len(mw)) + 1e-6
        z = (mm.mean(0) - mw.mean(0)) / se
        print("view", v, "megakernel", mm.mean(0), "wavefront", mw.mean(0), "z", z)
        assert np.all(np.abs(z) < 4.5), (v, z)


def test_wavefront_batch_of_images_equals_separate_images():
    """Every image of a batch is the image rendered alone (same seeds): the
    sample streams depend on (seed, sample, pixel) only."""
    sd = scenes.cornell_box(width=40, height=32)
    gs = hk.Scene.from_desc(sd)
    cams = [scenes.look_at((0.3 * i, 1, 3.8), (0, 1, 0), (0, 1, 0)) for i in range(3)]
    batch = [torch.zeros(gs.film_shape(), dtype=torch.float32, device=DEV) for _ in cams]
    gs.render_batch(batch, spp=32, depth=sd.depth, seeds=[5, 6, 7], cameras=cams, capacity=1 << 14)
    for i, cam in enumerate(cams):
        alone = torch.zeros(gs.film_shape(), dtype=torch.float32, device=DEV)
        gs.render_batch([alone], spp=32, depth=sd.depth, seeds=[5 + i], cameras=[cam], image_indices=[i],
                        capacity=1 << 12)
        a, b = _resolve(gs, batch[i]), _resolve(gs, alone)
        assert np.allclose(a, b, rtol=1e-5, atol=1e-6), np.abs(a - b).max()


def test_progressive_passes_equal_one_render(tmp_path):
    """Passes over consecutive sample ranges accumulate to the single render of
    all samples (each sample's stream depends only on seed, sample and pixel);
    the preview written after each pass reads back as that pass's image."""
    sd = scenes.cornell_box(width=48, height=40)
    gs = hk.Scene.from_desc(sd)
    path = str(tmp_path / "progress.exr")
    imgs = [img for _, img in gs.render_progressive(4, 16, sd.depth, seed=5, exr_path=path, capacity=1 << 14)]
    assert np.array_equal(hk.exr_read(path), imgs[-1])
    film = torch.zeros(gs.film_shape(), dtype=torch.float32, device=DEV)
    gs.render_batch([film], spp=64, depth=sd.depth, seeds=[5], image_indices=[0], capacity=1 << 14)
    one = _resolve(gs, film)
    d = np.abs(imgs[-1].astype(np.float64) - one)
    print("progressive vs one render: max abs", d.max(), "mean", one.mean())
    assert np.all(d <= 2e-4 * np.abs(one) + 1e-5)
    # earlier passes are noisier estimates of the same image
    errs = [np.mean((i - one) ** 2) for i in imgs]
    assert errs[0] > errs[-1]


def test_render_image_forms_agree():
    """hk_render_image, the call a pathMISCuda plugin's RenderImage makes,
    renders large images with the wavefront: both forms draw the same
    per-sample streams, so the images agree up to the order of the film's
    float additions, and so do the ray counters."""
    sd = scenes.cornell_box(width=256, height=256)
    gs = hk.Scene.from_desc(sd)
    imgs, ctrs = {}, {}
    for form in (hk.FORM_MEGAKERNEL, hk.FORM_WAVEFRONT, hk.FORM_AUTO):
        gs.set_image_form(form)
        imgs[form], ctrs[form] = gs.render_image(64, sd.depth, seed=31)
    a, b, c = imgs[hk.FORM_MEGAKERNEL], imgs[hk.FORM_WAVEFRONT], imgs[hk.FORM_AUTO]
    scale = float(np.abs(a).max())
    close = np.abs(a.astype(np.float64) - b) <= 1e-4 * np.abs(a) + 1e-6 * scale
    print("megakernel vs wavefront: max abs", np.abs(a - b).max(), "close", close.mean(),
          "sums", a.sum(), b.sum())
    # a pixel mixes ~1600 paths through the filter: one path that an ulp sends
    # elsewhere changes it, so the bar is on nearly all pixels and the image sum
    assert close.mean() > 0.99
    assert abs(a.sum() / b.sum() - 1) < 1e-4
    assert np.allclose(b, c, rtol=1e-5, atol=1e-6 * scale)   # auto picks the wavefront at this size
    m, w = ctrs[hk.FORM_MEGAKERNEL], ctrs[hk.FORM_WAVEFRONT]
    print("counters megakernel", m, "wavefront", w)
    # both end a path by Russian roulette before tracing its continuation ray
    assert abs(int(m[0]) - int(w[0])) <= 1e-3 * m[0] and abs(int(m[1]) - int(w[1])) <= 1e-3 * m[1]
    # an autotuned configuration is kept for render_image
    gs.autotune(4, sd.depth)
    gs.set_image_form(hk.FORM_AUTO)
    d, _ = gs.render_image(64, sd.depth, seed=31)
    assert np.allclose(d, b, rtol=1e-4, atol=1e-6 * scale)


@pytest.mark.parametrize("lean", [0, 2])
def test_shadow_test_modes_agree(lean):
    """The shadow rays' triangle tests -- each lane its own, postponed, or
    shared out over the warp (hk_wavefront_config.shadow_tests 0 / 1 / 2) --
    decide occlusion by the same Moller-Trumbore test on the same triangles,
    and an any-hit decision does not depend on the order of the tests: the
    images agree up to the order of the film's float additions, the ray
    counts exactly."""
    sd = scenes.heterogeneous(width=128, height=128, spp=8, depth=8, n_spheres=12, levels=(3, 4),
                              level_p=(0.5, 0.5), env_res=(256, 128))
    gs = hk.Scene.from_desc(sd)
    gs.set_accel(hk.ACCEL_BVH8)
    imgs, ctrs = [], []
    for mode in (0, 1, 2):
        f = torch.zeros(gs.film_shape(), dtype=torch.float32, device="cuda")
        ctr = torch.zeros(7, dtype=torch.int64, device="cuda")
        gs.render_batch([f], spp=8, depth=8, seeds=[3], counters=ctr, capacity=1 << 16, threads_extend=64,
                        shadow_tests=mode, reg_lean=lean)
        imgs.append(f.cpu().numpy().astype(np.float64))
        ctrs.append(ctr.cpu().numpy())
    scale = float(np.abs(imgs[0]).max())
    for mode in (1, 2):
        print(f"mode {mode}: counters {ctrs[mode]} vs {ctrs[0]}, max abs diff {np.abs(imgs[mode] - imgs[0]).max():.3e}")
        assert ctrs[mode][0] == ctrs[0][0] and ctrs[mode][1] == ctrs[0][1]
        assert np.allclose(imgs[mode], imgs[0], rtol=1e-5, atol=1e-6 * scale)


@pytest.mark.parametrize("lean", [0, 1])
def test_closest_test_modes_agree(lean):
    """The closest-hit rays' triangle tests each lane its own or shared out
    over the warp (hk_wavefront_config.closest_tests 0 / 2) keep the same hit:
    the least t of the triangles a ray reaches, the later test on equal t.
    Paths then follow the same vertices, so the ray counts agree exactly and
    the images up to the order of the film's float additions."""
    sd = scenes.heterogeneous(width=128, height=128, spp=8, depth=8, n_spheres=12, levels=(3, 4),
                              level_p=(0.5, 0.5), env_res=(256, 128))
    gs = hk.Scene.from_desc(sd)
    gs.set_accel(hk.ACCEL_BVH8)
    imgs, ctrs = [], []
    for mode in (0, 2):
        f = torch.zeros(gs.film_shape(), dtype=torch.float32, device="cuda")
        ctr = torch.zeros(7, dtype=torch.int64, device="cuda")
        gs.render_batch([f], spp=8, depth=8, seeds=[3], counters=ctr, capacity=1 << 16, threads_extend=64,
                        closest_tests=mode, reg_lean=lean)
        imgs.append(f.cpu().numpy().astype(np.float64))
        ctrs.append(ctr.cpu().numpy())
    scale = float(np.abs(imgs[0]).max())
    print(f"counters {ctrs[1]} vs {ctrs[0]}, max abs diff {np.abs(imgs[1] - imgs[0]).max():.3e}")
    assert ctrs[1][0] == ctrs[0][0] and ctrs[1][1] == ctrs[0][1]
    assert np.allclose(imgs[1], imgs[0], rtol=1e-5, atol=1e-6 * scale)


def test_sample_major_dispatch_renders_the_same_image():
    """Dealing a job's work sample by sample over the whole image instead of
    tile by tile (hk_wavefront_config.sample_major) changes which paths are in
    flight together, not the paths: each sample's stream depends on (seed,
    sample, pixel, image) only, so ray counts agree exactly and images up to
    the order of the film's float additions."""
    sd = scenes.cornell_box(width=80, height=56)   # 5 x 4 tiles, the last row partial
    gs = hk.Scene.from_desc(sd)
    imgs, ctrs = [], []
    for order in (0, 1):
        f = torch.zeros(gs.film_shape(), dtype=torch.float32, device=DEV)
        ctr = torch.zeros(7, dtype=torch.int64, device=DEV)
        gs.render_batch([f], spp=32, depth=sd.depth, seeds=[9], counters=ctr, capacity=1 << 14, sample_major=order)
        imgs.append(_resolve(gs, f).astype(np.float64))
        ctrs.append(ctr.cpu().numpy())
    print("counters", ctrs, "max abs diff", np.abs(imgs[1] - imgs[0]).max())
    assert ctrs[1][0] == ctrs[0][0] and ctrs[1][1] == ctrs[0][1] and ctrs[1][2] == ctrs[0][2]
    assert np.allclose(imgs[1], imgs[0], rtol=1e-5, atol=1e-6 * float(np.abs(imgs[0]).max()))
