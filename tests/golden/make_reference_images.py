"""Render the reference images the GPU image tests compare against, with the
reference renderer itself (its own sources compiled by oracle/ref_build.py:
LoadFromXML, HLBVH, PathMISIntegrator, ImageBlock, Render's block loop).

  * config1_reference.npz: the plain-method scene of the benchmark set -- the
    seed-0 Cornell box, 256 x 256, Gaussian filter radius 2 (stddev 0.5),
    pathMIS depth 64 -- at 16384 samples per pixel;
  * hetero_small_reference.npz: a small heterogeneous scene (12 displaced
    icospheres of levels 3-4 with the six material types, 4 area lights and a
    256 x 128 sky), 96 x 96, Gaussian filter, depth 16, at 4096 samples per pixel.

Each file holds the resolved image as float16 (`rgb`), the samples per pixel
(`spp`) and the render seconds.  The reference's sampler is seeded by block
offsets only, so a render is deterministic: running this again gives the
same files.

usage: python tests/golden/make_reference_images.py [--threads N] [--only NAME]
"""
import argparse
import os
import sys
import tempfile
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from hikari_b200 import scenes  # noqa: E402
from hikari_b200.scenexml import write_scene_xml  # noqa: E402


def config1():
    return scenes.cornell_box(width=256, height=256), 16384


def hetero_small():
    sd = scenes.heterogeneous(width=96, height=96, depth=16, n_spheres=12, levels=(3, 4), level_p=(0.5, 0.5),
                              env_res=(256, 128))
    return sd, 4096


CASES = {"config1_reference": config1, "hetero_small_reference": hetero_small}


def render(name, threads):
    from oracle import reference

    sd, spp = CASES[name]()
    d = tempfile.mkdtemp(prefix="hk_golden_")
    xml = write_scene_xml(sd, d, name, spp=spp, accel="hlbvh")
    rs = reference.RefScene(xml)
    t0 = time.time()
    film, secs = rs.render(nthreads=threads)
    rgb = rs.resolve(film)
    out = os.path.join(HERE, name + ".npz")
    np.savez_compressed(out, rgb=rgb.astype(np.float16), spp=np.int32(spp), seconds=np.float32(secs))
    print(f"{name}: {sd.camera.width}x{sd.camera.height} x {spp} spp in {time.time() - t0:.0f} s -> {out}")


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--threads", type=int, default=0)
    ap.add_argument("--only", default=None)
    a = ap.parse_args()
    for n in CASES:
        if a.only is None or a.only == n:
            render(n, a.threads)
