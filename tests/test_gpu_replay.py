"""Path-level replay: the CUDA renderers and the oracle draw the same random
streams, so each GPU sample can be compared with the oracle's estimate of the
same path.

A sample of pixel (x, y) in the megakernel and in the wavefront seeds pcg32
with (splitmix64(seed, sample), y * width + x + image * width * height); the
oracle's per-pixel estimator seeds (seed', y * width + x) and renders its
samples from that one stream, so one oracle sample with seed' =
splitmix64(seed, sample) is the GPU's sample.  With one sample per pixel and a
box filter of radius 0.5 each pixel holds exactly one path's radiance.

Paths agree exactly up to the ulp differences of CUDA's sinf/cosf/expf/logf/
powf against the host libm, which move directions by ulps (the radiance stays
within 1e-4 relative) and can, rarely, flip a threshold decision (a triangle
edge, u against a Fresnel term), after which the two paths diverge."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

import hikari_b200 as hk  # noqa: E402
from hikari_b200 import scenes  # noqa: E402
from hikari_b200.scenedesc import FilterDesc  # noqa: E402
from oracle.oracle import OracleScene  # noqa: E402

DEV = "cuda:0"
M64 = (1 << 64) - 1


def splitmix64(seed, s):
    """The per-sample stream state of both CUDA renderers (hk_kernels.cu mix_seed)."""
    z = (seed + 0x9E3779B97F4A7C15 * (s + 1)) & M64
    z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & M64
    z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & M64
    return z ^ (z >> 31)


SCENES = {
    "cornell": lambda: scenes.cornell_box(width=32, height=32),
    "smooth": lambda: scenes.cornell_smooth(width=32, height=32),
    "heterogeneous": lambda: scenes.heterogeneous(width=32, height=32, n_spheres=12, levels=(3,), level_p=(1.0,), env_res=(256, 128)),
    "lights": lambda: scenes.lights_scene(width=32, height=32),
    "shading_normals_uv": lambda: scenes.lights_scene(width=32, height=32, shading_normals=True),
    "textured": lambda: scenes.lights_scene(width=32, height=32, shading_normals=True, textured=True),
    "bitmap": lambda: scenes.lights_scene(width=32, height=32, shading_normals=True, textured=True, bitmap=True),
    "bump": lambda: scenes.lights_scene(width=32, height=32, shading_normals=True, textured=True, bitmap=True,
                                        bump=True),
    # wireframe and curvature textures: the edge distance and the curvatures of
    # each hit computed on the device and by the oracle (pinned to the reference)
    "geometric": lambda: scenes.lights_scene(width=32, height=32, shading_normals=True, textured=True,
                                             geometric=True),
    # coatings over coatings and over two-sided BSDFs, two-sided BSDFs inside
    # two-sided ones (the device's bounded-depth layer dispatch)
    "nested": lambda: scenes.cornell_nested(width=32, height=32),
}


@pytest.fixture(scope="module", params=list(SCENES))
def replay_scene(request):
    sd = SCENES[request.param]()
    sd.filter = FilterDesc(0, 0.5)
    return request.param, sd, hk.Scene.from_desc(sd), OracleScene(sd)


def _oracle_samples(sd, os_, seeds):
    W, H = sd.camera.width, sd.camera.height
    pix = np.stack(np.meshgrid(np.arange(W), np.arange(H), indexing="xy"), -1).reshape(-1, 2)
    out = []
    for s in seeds:
        m, _ = os_.pixel_stats(pix, 1, seed=splitmix64(s, 0))
        out.append(np.nan_to_num(m, nan=0.0, posinf=0.0, neginf=0.0))
    return np.concatenate(out)


def _agreement(g, o, label):
    g = g.astype(np.float64)
    rel = np.abs(g - o).max(1) / (np.abs(o).max(1) + 1e-6)
    same = rel <= 1e-4
    print(f"{label}: {same.mean():.5f} of {len(g)} paths within 1e-4; sums gpu {g.sum():.4f} oracle {o.sum():.4f}")
    assert same.mean() >= 0.999, f"{label}: only {same.mean():.5f} of the paths agree"
    return same


def test_megakernel_replays_oracle_paths(replay_scene):
    name, sd, gs, os_ = replay_scene
    seeds = list(range(500, 508))
    g = np.concatenate([gs.render_image(1, sd.depth, seed=s)[0].reshape(-1, 3) for s in seeds])
    _agreement(g, _oracle_samples(sd, os_, seeds), f"megakernel {name}")


def test_wavefront_replays_oracle_paths(replay_scene):
    name, sd, gs, os_ = replay_scene
    W, H = sd.camera.width, sd.camera.height
    seeds = list(range(600, 608))
    films = [torch.zeros(gs.film_shape(), dtype=torch.float32, device=DEV) for _ in seeds]
    gs.render_batch(films, spp=1, depth=sd.depth, seeds=seeds, image_indices=[0] * len(seeds), capacity=1 << 14)
    g = []
    for f in films:
        rgb = torch.empty((H, W, 3), dtype=torch.float32, device=DEV)
        gs.resolve(f, rgb)
        g.append(rgb.cpu().numpy().reshape(-1, 3))
    _agreement(np.concatenate(g), _oracle_samples(sd, os_, seeds), f"wavefront {name}")
