"""The smooth (delta) BSDFs and two-sided compositions rendered end to end:
the megakernel and the wavefront against the oracle on a Cornell box with a
smooth-plastic floor, a glass box, a smooth conductor, a mirror and two-sided
panels.  Caustics through the glass make single pixels heavy-tailed, so the
comparison is per 4 x 4 block of pixels (z-scores from the oracle's per-pixel
variances) plus the per-pixel fraction of |z| > 3."""
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
SPP_G, SPP_O = 8192, 2048


@pytest.fixture(scope="module")
def smooth_scene():
    sd = scenes.cornell_smooth(width=W, height=H)
    sd.filter = FilterDesc(0, 0.5)   # box filter: pixels are independent estimates
    os_ = OracleScene(sd)
    pix = np.stack(np.meshgrid(np.arange(W), np.arange(H), indexing="xy"), -1).reshape(-1, 2)
    mean_o, var_o = os_.pixel_stats(pix, SPP_O, seed=3)
    return sd, hk.Scene.from_desc(sd), mean_o, var_o


def _compare(g, mean_o, var_o, label):
    g = g.reshape(-1, 3).astype(np.float64)
    z = (g - mean_o) / (np.sqrt(var_o / SPP_G + var_o / SPP_O) + 1e-6)
    frac3 = np.mean(np.abs(z) > 3)
    # 4 x 4 blocks: mean of 16 independent pixel estimates
    blk = lambda a: a.reshape(H // 4, 4, W // 4, 4, 3).mean((1, 3))
    gb, ob = blk(g.reshape(H, W, 3)), blk(mean_o.reshape(H, W, 3))
    vb = blk(var_o.reshape(H, W, 3)) / 16 * (1.0 / SPP_G + 1.0 / SPP_O)
    zb = (gb - ob) / (np.sqrt(vb) + 1e-6)
    ratio = g.mean() / mean_o.mean()
    print(label, "mean ratio", ratio, "pixel frac |z|>3", frac3, "block max |z|", np.abs(zb).max())
    assert abs(ratio - 1) < 0.01
    assert frac3 < 0.02
    assert np.abs(zb).max() < 4.5
    assert np.mean(np.abs(zb) > 3) <= 2 / zb.size


def test_megakernel_smooth_matches_oracle(smooth_scene):
    sd, gs, mean_o, var_o = smooth_scene
    img, ctr = gs.render_image(SPP_G, sd.depth, seed=7)
    _compare(img, mean_o, var_o, "megakernel")
    assert ctr[0] >= W * H * SPP_G


def test_wavefront_smooth_matches_oracle(smooth_scene):
    sd, gs, mean_o, var_o = smooth_scene
    film = torch.zeros(gs.film_shape(), dtype=torch.float32, device=DEV)
    ctr = torch.zeros(7, dtype=torch.int64, device=DEV)
    gs.render_batch([film], spp=SPP_G, depth=sd.depth, seeds=[11], counters=ctr, capacity=1 << 18)
    rgb = torch.empty((H, W, 3), dtype=torch.float32, device=DEV)
    gs.resolve(film, rgb)
    _compare(rgb.cpu().numpy(), mean_o, var_o, "wavefront")
    assert ctr.cpu().numpy()[0] >= W * H * SPP_G
