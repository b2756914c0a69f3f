"""GPU images against images rendered by the reference renderer itself
(tests/golden/*_reference.npz, made by tests/golden/make_reference_images.py
with the reference's own sources: its parser, HLBVH, PathMISIntegrator,
Gaussian filter and ImageBlock, and Render's block loop).

* config 1 exactly as the benchmark set states it: the seed-0 Cornell box,
  256 x 256, 64 samples per pixel, Gaussian filter radius 2, pathMIS depth 64:
  every pixel of the GPU estimate lies within 3 sigma of the reference image
  except the expected tail;
* RMSE against the reference falls like 1/sqrt(spp);
* the wavefront and the plain megakernel have equal RMSE at equal spp (the
  Cornell box and a small heterogeneous scene with every rough material, the
  sky and area lights).

The reference images are stored as float16; their rounding (2^-11
relative) is part of each tolerance.
"""
import os

import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

import hikari_b200 as hk  # noqa: E402
from hikari_b200 import scenes  # noqa: E402

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def _reference(name):
    d = np.load(os.path.join(GOLDEN, name + ".npz"))
    return d["rgb"].astype(np.float64), int(d["spp"])


def _config1():
    return scenes.cornell_box(width=256, height=256)


def _hetero_small():
    return scenes.heterogeneous(width=96, height=96, depth=16, n_spheres=12, levels=(3, 4), level_p=(0.5, 0.5),
                                env_res=(256, 128))


def _images(gs, sd, spp, seeds, form):
    out = []
    for s in seeds:
        if form == "mega":
            f = torch.zeros(gs.film_shape(), dtype=torch.float32, device="cuda")
            gs.render(f, spp=spp, depth=sd.depth, seed=s)
        else:
            f = torch.zeros(gs.film_shape(), dtype=torch.float32, device="cuda")
            gs.render_batch([f], spp=spp, depth=sd.depth, seeds=[s], image_indices=[0], capacity=1 << 18)
        rgb = torch.empty((sd.camera.height, sd.camera.width, 3), dtype=torch.float32, device="cuda")
        gs.resolve(f, rgb)
        out.append(rgb.cpu().numpy().astype(np.float64))
    return np.stack(out)


@pytest.mark.parametrize("form", ["mega", "wave"])
def test_config1_within_3_sigma_of_reference_image(form):
    ref, n_ref = _reference("config1_reference")
    sd = _config1()
    assert sd.spp == 64 and sd.filter.kind == 2 and sd.filter.radius == 2.0 and sd.depth == 64
    gs = hk.Scene.from_desc(sd)
    K = 48
    imgs = _images(gs, sd, 64, [1000 + k for k in range(K)], form)
    mean = imgs.mean(0)
    var = imgs.var(0, ddof=1)   # variance of one 64-spp render, per pixel and channel
    se2 = var / K + var * 64.0 / n_ref + (np.abs(ref) * 2.0 ** -11) ** 2
    z = (mean - ref) / np.sqrt(se2 + 1e-30)
    tail = np.mean(np.abs(z) > 3)
    # Student t with K - 1 = 47 degrees of freedom: P(|t| > 3) = 0.43%
    print(f"{form}: |z| > 3 on {tail:.4%} of pixel channels, mean z {z.mean():+.4f}, "
          f"image mean ratio {mean.mean() / ref.mean():.5f}")
    assert tail < 0.0065
    # (the mean of z is not a test: a path-traced pixel is right-skewed -- rare
    # bright paths -- so most K-render means fall below the expectation)
    assert abs(mean.mean() / ref.mean() - 1) < 2e-3


def test_rmse_scales_with_spp_against_reference():
    """MSE against the reference image falls like 1/spp: 4x the samples, 1/4
    of the error (the reference's own noise at 16384 spp is 1/64 of the GPU's
    at 256 spp)."""
    ref, n_ref = _reference("config1_reference")
    sd = _config1()
    gs = hk.Scene.from_desc(sd)
    mse = []
    for spp in (16, 64, 256):
        imgs = _images(gs, sd, spp, [3000 * spp + k for k in range(4)], "mega")
        mse.append(float(np.mean((imgs - ref) ** 2)))
    r1, r2 = mse[0] / mse[1], mse[1] / mse[2]
    print("mse", mse, "ratios", r1, r2)
    assert 3.2 < r1 < 4.8 and 3.2 < r2 < 4.8, mse


@pytest.mark.parametrize("scene", ["config1", "hetero_small"])
def test_equal_rmse_wavefront_and_megakernel_against_reference(scene):
    """At equal spp the wavefront and the megakernel have equal RMSE against
    the reference renderer's image (they run the same estimator), and the
    error is the estimator's variance: no bias against the reference."""
    ref, n_ref = _reference(scene + "_reference")
    sd = _config1() if scene == "config1" else _hetero_small()
    gs = hk.Scene.from_desc(sd)
    spp = 64
    k = 8 if scene == "config1" else 16
    m = _images(gs, sd, spp, [9000 + s for s in range(k)], "mega")
    w = _images(gs, sd, spp, [7000 + s for s in range(k)], "wave")
    mse_m = float(np.mean((m - ref) ** 2))
    mse_w = float(np.mean((w - ref) ** 2))
    var_one = float(np.mean(np.concatenate([m, w]).var(0, ddof=1)))
    noise_ref = var_one * spp / n_ref   # the reference image's own noise
    print(f"{scene}: MSE at {spp} spp megakernel {mse_m:.4e} wavefront {mse_w:.4e}; variance of one render "
          f"{var_one:.4e}, reference noise {noise_ref:.2e}")
    assert 0.8 < mse_w / mse_m < 1.25
    assert mse_m < 1.3 * (var_one + noise_ref) and mse_w < 1.3 * (var_one + noise_ref)
