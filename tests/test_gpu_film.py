"""Film splatting through the reconstruction filters on the GPU against the
oracle, sample for sample.

With one sample per pixel both CUDA renderers draw pixel (x, y)'s film
position and path from pcg32 seeded (splitmix64(seed, 0), pixel), the stream
the oracle's ho_pixel_samples replays.  The oracle puts those samples through
ImageBlock::Put (src/core/Block.cpp:95-134, itself pinned bit for bit against
the reference's ImageBlock) into a bordered film of doubles; the megakernel
splats into a shared-memory tile plus filter margin and flushes it with global
atomics, the wavefront splats with 128-bit vector reductions.  The image is
53 x 37, so tiles are ragged at the right and bottom edges and the border
cells receive splats from several tiles.

The filter weights depend only on the film positions, so the weight channel
must agree in every cell (up to the float order of the atomic sums); the
radiance channels agree wherever the paths agree (all but the rare paths
where an ulp difference of CUDA's transcendental functions flips a
threshold, see tests/test_gpu_replay.py).
"""
import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

import hikari_b200 as hk  # noqa: E402
from hikari_b200 import scenes  # noqa: E402
from hikari_b200.scenedesc import FilterDesc  # noqa: E402
from oracle.oracle import OracleScene  # noqa: E402
from tests.gpu_helpers import rel_close  # noqa: E402
from tests.test_gpu_replay import splitmix64  # noqa: E402

FILTERS = {
    "gaussian_r2": FilterDesc(2, 2.0, 0.5),     # config 1's filter
    "tent": FilterDesc(1, 1.0),
    "mitchell": FilterDesc(3, 2.0, 1 / 3, 1 / 3),
    "gaussian_r3.3": FilterDesc(2, 3.3, 0.9),   # border 3: wider tile margins
    "box": FilterDesc(0, 0.5),
}


@pytest.mark.parametrize("form", ["megakernel", "wavefront"])
@pytest.mark.parametrize("filt", list(FILTERS))
def test_film_splat_replays_oracle(filt, form):
    W, H = 53, 37
    sd = scenes.cornell_box(width=W, height=H)
    sd.filter = FILTERS[filt]
    gs, os_ = hk.Scene.from_desc(sd), OracleScene(sd)
    seed = 4242
    film = torch.zeros(gs.film_shape(), dtype=torch.float32, device="cuda")
    if form == "megakernel":
        gs.render(film, spp=1, depth=sd.depth, seed=seed)
    else:
        gs.render_batch([film], spp=1, depth=sd.depth, seeds=[seed], image_indices=[0], capacity=1 << 14)
    g = film.cpu().numpy().astype(np.float64)
    pix = np.stack(np.meshgrid(np.arange(W), np.arange(H), indexing="xy"), -1).reshape(-1, 2)
    pos, L = os_.pixel_samples(pix, splitmix64(seed, 0))
    o, dropped = os_.film_put(pos, L)
    assert g.shape == o.shape
    # weights: every cell, up to the order of the float additions
    wok = rel_close(g[..., 3], o[..., 3], 2e-6, atol=1e-7)
    assert wok.mean() > 0.995, f"{filt} {form}: weights differ in {np.sum(~wok)} of {wok.size} cells"
    # radiance: cells fed by agreeing paths
    scale = float(np.abs(o[..., :3]).max())
    ok = rel_close(g[..., :3], o[..., :3], 1e-4, atol=1e-6 * scale).all(-1)
    print(f"{filt} {form}: weights equal in {wok.mean():.5f}, radiance in {ok.mean():.5f} of the cells")
    assert ok.mean() > 0.98, f"{filt} {form}: radiance differs in {np.sum(~ok)} of {ok.size} cells"
    assert abs(g[..., :3].sum() / o[..., :3].sum() - 1.0) < 2e-3
    # the resolved image (ImageBlock::ToBitmap on the device) against the oracle's resolve
    rgb = torch.empty((H, W, 3), dtype=torch.float32, device="cuda")
    gs.resolve(film, rgb)
    a, b = rgb.cpu().numpy(), os_.resolve(o)
    assert rel_close(a, b, 1e-4, atol=1e-6 * float(np.abs(b).max())).all(-1).mean() > 0.98
