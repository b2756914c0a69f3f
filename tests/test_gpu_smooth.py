"""The smooth (delta) BSDFs, two-sided compositions and roughDiffuse rendered end to end:
the megakernel and the wavefront against the oracle on a Cornell box with a
smooth-plastic floor, a glass box, a smooth conductor, a mirror and two-sided
panels.  Caustics through the glass are reached by BSDF sampling alone, so
some pixels are heavy-tailed: the GPU side is K independent renders, and each
pixel's z-score uses both sides' variance estimates (the GPU's from the spread
of its K renders); 4 x 4 blocks of pixels are compared as well."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

import hikari_b200 as hk  # noqa: E402
from hikari_b200 import scenes  # noqa: E402
from hikari_b200.scenedesc import FilterDesc  # noqa: E402
from oracle.oracle import OracleScene  # noqa: E402

DEV = "cuda:0"
W = H = 32
K, SPP_K = 16, 512          # GPU: K renders of SPP_K samples per pixel
SPP_O = 2048                # oracle samples per pixel


@pytest.fixture(scope="module")
def smooth_scene():
    sd = scenes.cornell_smooth(width=W, height=H)
    sd.filter = FilterDesc(0, 0.5)   # box filter: pixels are independent estimates
    os_ = OracleScene(sd)
    pix = np.stack(np.meshgrid(np.arange(W), np.arange(H), indexing="xy"), -1).reshape(-1, 2)
    mean_o, var_o = os_.pixel_stats(pix, SPP_O, seed=3)
    return sd, hk.Scene.from_desc(sd), mean_o, var_o


def _compare(imgs, mean_o, var_o, label):
    imgs = np.stack([i.reshape(-1, 3).astype(np.float64) for i in imgs])
    g = imgs.mean(0)
    se2_g = imgs.var(0, ddof=1) / len(imgs)          # variance of the GPU mean
    se2_o = var_o / SPP_O
    z = (g - mean_o) / (np.sqrt(se2_g + se2_o) + 1e-6)
    frac3 = np.mean(np.abs(z) > 3)
    # 4 x 4 blocks: mean of 16 independent pixel estimates
    blk = lambda a: a.reshape(H // 4, 4, W // 4, 4, 3).mean((1, 3))
    gb, ob = blk(g.reshape(H, W, 3)), blk(mean_o.reshape(H, W, 3))
    vb = (blk(se2_g.reshape(H, W, 3)) + blk(se2_o.reshape(H, W, 3))) / 16
    zb = (gb - ob) / (np.sqrt(vb) + 1e-6)
    ratio = g.mean() / mean_o.mean()
    print(label, "mean ratio", ratio, "pixel frac |z|>3", frac3, "max |z|", np.abs(z).max(),
          "block max |z|", np.abs(zb).max())
    assert abs(ratio - 1) < 0.01
    assert frac3 < 0.02
    # heavy tails (caustics through glass and off the coated wall) put about one
    # block of 192 beyond 3 sigma in oracle-against-oracle trials
    assert np.abs(zb).max() < 5.0
    assert np.sum(np.abs(zb) > 3) <= 3


def test_megakernel_smooth_matches_oracle(smooth_scene):
    sd, gs, mean_o, var_o = smooth_scene
    imgs = []
    for k in range(K):
        img, ctr = gs.render_image(SPP_K, sd.depth, seed=100 + k)
        assert ctr[0] >= W * H * SPP_K
        imgs.append(img)
    _compare(imgs, mean_o, var_o, "megakernel")


def test_wavefront_smooth_matches_oracle(smooth_scene):
    sd, gs, mean_o, var_o = smooth_scene
    films = [torch.zeros(gs.film_shape(), dtype=torch.float32, device=DEV) for _ in range(K)]
    ctr = torch.zeros(7, dtype=torch.int64, device=DEV)
    gs.render_batch(films, spp=SPP_K, depth=sd.depth, seeds=list(range(200, 200 + K)), counters=ctr,
                    capacity=1 << 18)
    imgs = []
    for f in films:
        rgb = torch.empty((H, W, 3), dtype=torch.float32, device=DEV)
        gs.resolve(f, rgb)
        imgs.append(rgb.cpu().numpy())
    _compare(imgs, mean_o, var_o, "wavefront")
    assert ctr.cpu().numpy()[0] >= K * W * H * SPP_K
