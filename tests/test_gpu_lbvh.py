"""The device tree builder (hikari_b200/csrc/hk_lbvh.cu, HK_BUILDER_GPU).

* structure: the 8-wide tree built on the device passes the host build's
  structural check (every triangle in exactly one leaf, every quantised child
  box containing its triangles, every node reachable) on triangle soups,
  meshes, degenerate input (all centroids equal, zero-area triangles) and 1 to
  9 triangles;
* hit parity: a scene built on the device traces like the reference's HLBVH
  (src/acceleration/HLBVHAcceleration.cpp:206) on 50 000 rays, with the same
  tie and edge rules as the host-built tree (tests/test_gpu_reference.py);
* images: a render of a device-built scene equals the render of the
  host-built scene up to the float order of the film and the tie rule;
* speed: the 4.75M-triangle heterogeneous scene builds its tree in a small
  fraction of the host build's time.
"""
import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

import hikari_b200 as hk  # noqa: E402
from hikari_b200 import scenes  # noqa: E402
from oracle.oracle import OracleScene  # noqa: E402


def _tris(sd):
    out = [m.positions[m.indices].reshape(-1, 9) for m in sd.meshes]
    return np.concatenate(out, 0).astype(np.float32)


def _soup(n, seed, spread=10.0):
    rng = np.random.default_rng(seed)
    c = rng.uniform(-spread, spread, (n, 1, 3))
    return (c + rng.normal(0, 0.3, (n, 3, 3))).astype(np.float32).reshape(n, 9)


CASES = {
    "soup_10k": lambda: _soup(10000, 1),
    "soup_wide_range": lambda: _soup(5000, 2, spread=1e4),
    "cornell": lambda: _tris(scenes.cornell_box()),
    "displaced_l5": lambda: _tris(scenes.mesh_heavy("plastic", width=8, height=8, level=5, env_res=(16, 8))),
    "same_centroid": lambda: np.tile(np.array([[0, 0, 0, 1, 0, 0, 0, 1, 0]], np.float32), (300, 1))
                             + np.random.default_rng(3).normal(0, 1e-3, (300, 9)).astype(np.float32),
    "zero_area": lambda: np.repeat(np.random.default_rng(4).uniform(-1, 1, (200, 1, 3)), 3, 1).astype(np.float32).reshape(200, 9),
}
for _n in (1, 2, 3, 4, 5, 9):
    CASES[f"n{_n}"] = (lambda n=_n: _soup(n, 10 + n))


@pytest.mark.parametrize("case", list(CASES))
def test_device_tree_structure(case):
    tris = CASES[case]()
    nw, depth = hk.bvh_check_gpu(tris)
    print(f"{case}: {tris.shape[0]} triangles, {nw} 8-wide nodes, depth {depth}")
    assert nw >= 1 and depth >= 1


def test_device_tree_structure_1m():
    tris = _tris(scenes.mesh_heavy("plastic", width=8, height=8, level=8, env_res=(16, 8)))
    nw, depth = hk.bvh_check_gpu(tris)
    print(f"level-8 sphere: {tris.shape[0]} triangles, {nw} 8-wide nodes, depth {depth}")
    assert depth <= 30


reference = pytest.importorskip("oracle.reference")


@pytest.mark.parametrize("scene", ["cornell", "displaced"])
def test_device_tree_hit_parity_with_reference(scene):
    try:
        reference.lib()
    except reference.ReferenceUnavailable as e:
        pytest.skip(str(e))
    if scene == "cornell":
        sd = scenes.cornell_box(width=64, height=64)
        lo, hi = (-0.9, 0.1, -0.9), (0.9, 1.9, 0.9)
    else:
        sd = scenes.mesh_heavy("conductor", width=64, height=64, level=6, env_res=(64, 32))
        lo, hi = (-2.5, 0.05, -2.5), (2.5, 2.5, 2.5)
    gs = hk.Scene.from_desc(sd, builder=hk.BUILDER_GPU)
    assert gs.info.n_bvh_nodes == 0 and gs.info.n_wide_nodes > 0
    with pytest.raises(hk.HikariError):
        gs.set_accel(hk.ACCEL_BVH2)   # the device build makes the 8-wide tree only
    os_ = OracleScene(sd)
    from tests.test_gpu_reference import _rays

    rays = _rays(sd, os_, 50000, 23, lo, hi)
    tri_r, t_r, u_r, v_r = reference.RefAccel(sd.meshes, "hlbvh").trace(rays)
    tri_g, t_g, u_g, v_g, _ = gs.trace(torch.from_numpy(rays).cuda())
    tri_g, t_g = tri_g.cpu().numpy(), t_g.cpu().numpy()
    bad = tri_g != tri_r
    edge = np.minimum(np.minimum(u_r, v_r), 1 - u_r - v_r) < 1e-5
    tie = (tri_g >= 0) & (tri_r >= 0) & (np.abs(t_g - t_r) <= 1e-6 * np.abs(t_r))
    print(f"{scene}: equal on {1 - bad.mean():.5f}, {np.sum(bad & tie)} ties, {np.sum(bad & ~tie)} edges")
    assert np.all(tie[bad] | edge[bad])
    assert bad.mean() < 0.005
    both = ~bad & (tri_r >= 0)
    assert (t_g[both] == t_r[both]).mean() > 0.999


def test_device_tree_renders_like_host_tree():
    sd = scenes.heterogeneous(width=96, height=96, spp=16, n_spheres=12, levels=(3, 4), level_p=(0.5, 0.5),
                              env_res=(256, 128))
    a = hk.Scene.from_desc(sd)
    b = hk.Scene.from_desc(sd, builder=hk.BUILDER_GPU)
    ia, ca = a.render_image(64, sd.depth, seed=5)
    ib, cb = b.render_image(64, sd.depth, seed=5)
    scale = float(np.abs(ia).max())
    close = np.abs(ia.astype(np.float64) - ib) <= 1e-4 * np.abs(ia) + 1e-6 * scale
    print("host vs device tree: close", close.mean(), "sums", ia.sum(), ib.sum(), "rays", ca[:2], cb[:2])
    assert close.mean() > 0.98
    assert abs(ia.sum() / ib.sum() - 1) < 1e-3
    assert ca[0] == cb[0] or abs(int(ca[0]) - int(cb[0])) < 1e-3 * ca[0]


def test_device_tree_build_time():
    sd = scenes.heterogeneous(width=64, height=64, spp=1)
    g = hk.Scene.from_desc(sd, builder=hk.BUILDER_GPU)   # first build: module load, allocations
    g = hk.Scene.from_desc(sd, builder=hk.BUILDER_GPU)
    t_gpu = g.tree_build_seconds()
    h = hk.Scene.from_desc(sd)
    t_host = h.tree_build_seconds()
    print(f"{sd.n_triangles} triangles: device tree {t_gpu * 1e3:.1f} ms (upload and gather included), "
          f"host trees {t_host * 1e3:.0f} ms; 8-wide nodes {g.info.n_wide_nodes} vs {h.info.n_wide_nodes}, "
          f"depth {g.info.wide_depth} vs {h.info.wide_depth}")
    assert t_gpu < 0.25 * t_host
