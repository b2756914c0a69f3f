"""Seeded synthetic scenes of the benchmark configurations.

* ``cornell_box``      -- plain-method small case: a Cornell box of OBJ quads
* ``cornell_smooth``   -- the Cornell box with smooth (delta) and two-sided materials
* ``lights_scene``     -- an open scene lit by every emitter kind (area, point, directional, constant)
* ``icosphere``        -- subdivided icosahedron, optionally displaced by value noise
* ``sky_envmap``       -- procedural lat-long sky (sun disk of radiance 2e4 + gradient)
* ``mesh_heavy``       -- displaced level-8 icosphere on a ground quad under the sky
* ``heterogeneous``    -- 64 displaced icospheres with random materials, 4 area lights + sky

All geometry is generated in world space with the winding the reference's
one-sided BSDFs need (src/bsdf/DiffuseBSDF.cpp:45): the geometric normal
cross(p1 - p0, p2 - p0) points towards the viewer side.
"""
from __future__ import annotations

import math
from typing import List, Optional

import numpy as np

from .scenedesc import (AIR_IOR, BECKMANN, BSDF_COATING, BSDF_CONDUCTOR, BSDF_DIELECTRIC, BSDF_DIFFUSE, BSDF_MIRROR,
                        BSDF_PLASTIC, BSDF_ROUGH_COATING, BSDF_ROUGH_CONDUCTOR, BSDF_ROUGH_DIELECTRIC,
                        BSDF_ROUGH_DIFFUSE, BSDF_ROUGH_PLASTIC, BSDF_TWO_SIDED, BSDF_BUMP_MAP, BSDF_NORMAL_MAP,
                        FILTER_BILINEAR, FILTER_EWA,
                        FILTER_NEAREST, FILTER_TRILINEAR, GGX, TEX_BITMAP, TEX_CHECKERBOARD, TEX_CURVATURE, TEX_GRID, TEX_SCALE,
                        TEX_WIREFRAME,
                        WRAP_CLAMP, BSDFDesc, CameraDesc, EnvDesc, FilterDesc, LightDesc, MeshDesc, SceneDesc,
                        TextureDesc)

# Per-channel complex IOR (n, k) of copper and gold at R, G, B ~ (650, 550, 450) nm,
# rounded from Johnson & Christy (1972) optical constants.
CU_ETA = [0.27, 0.98, 1.16]
CU_K = [3.41, 2.58, 2.40]
AU_ETA = [0.17, 0.42, 1.37]
AU_K = [3.57, 2.39, 1.79]
# Scalar-IOR versions (the mean eta of the three channels with the per-channel
# k): the reference's conductors take one intIOR / extIOR for every channel
# (src/bsdf/RoughConductorBSDF.cpp:43), so scenes that the reference renderer
# must read use these.
CU_IOR = 0.80
AU_IOR = 0.65


def look_at(origin, target, up) -> np.ndarray:
    """The <lookat> transform of src/core/Parser.cpp:353 (columns left, up, dir, origin)."""
    o, t, u = (np.asarray(v, np.float64) for v in (origin, target, up))
    d = t - o
    d /= np.linalg.norm(d)
    left = np.cross(u / np.linalg.norm(u), d)
    left /= np.linalg.norm(left)
    nup = np.cross(d, left)
    M = np.eye(4)
    M[:3, 0], M[:3, 1], M[:3, 2], M[:3, 3] = left, nup, d, o
    return M.astype(np.float32)


def quad(p0, p1, p2, p3):
    """Quad p0..p3 split like the OBJ loader: (v1,v2,v3), (v4,v1,v3)."""
    pos = np.array([p0, p1, p2, p3], np.float32)
    idx = np.array([[0, 1, 2], [3, 0, 2]], np.uint32)
    return pos, idx


def box_mesh(center, size, angle_deg):
    """Axis box rotated about +y, faces wound outwards (12 triangles)."""
    cx, cy, cz = center
    sx, sy, sz = size
    a = math.radians(angle_deg)
    ca, sa = math.cos(a), math.sin(a)
    corners = []
    for x in (-0.5, 0.5):
        for y in (0.0, 1.0):
            for z in (-0.5, 0.5):
                px, pz = x * sx, z * sz
                corners.append((cx + ca * px + sa * pz, cy + y * sy, cz - sa * px + ca * pz))
    C = np.array(corners, np.float32)
    # corner index = 4*xi + 2*yi + zi
    faces = [
        (0, 1, 3, 2),  # -x
        (4, 6, 7, 5),  # +x
        (0, 4, 5, 1),  # -z... reorder below by normal check
        (2, 3, 7, 6),
        (0, 2, 6, 4),  # bottom
        (1, 5, 7, 3),  # top
    ]
    pos, idx = [], []
    cen = C.mean(0)
    for f in faces:
        q = [C[i] for i in f]
        n = np.cross(q[1] - q[0], q[2] - q[0])
        fc = np.mean(q, 0)
        if np.dot(n, fc - cen) < 0:
            q = q[::-1]
        base = len(pos)
        pos += q
        idx += [[base, base + 1, base + 2], [base + 3, base, base + 2]]
    return np.array(pos, np.float32), np.array(idx, np.uint32)


def cornell_box(seed: int = 0, width: int = 256, height: int = 256, spp: int = 64, depth: int = 64) -> SceneDesc:
    """Five 2x2 diffuse walls (white 0.725, red (0.63,0.065,0.05), green
    (0.14,0.45,0.09)), two 12-triangle boxes rotated about y by U[0,45] deg
    (seeded), a 0.5x0.5 area light of radiance (17,12,4); perspective fov 40,
    independent sampler, Gaussian filter radius 2."""
    rng = np.random.default_rng(seed)
    white = BSDFDesc(type=BSDF_DIFFUSE, kd=[0.725, 0.725, 0.725])
    red = BSDFDesc(type=BSDF_DIFFUSE, kd=[0.63, 0.065, 0.05])
    green = BSDFDesc(type=BSDF_DIFFUSE, kd=[0.14, 0.45, 0.09])
    sd = SceneDesc()
    # interior of [-1,1] x [0,2] x [-1,1]; normals point inwards
    walls = [
        (quad((-1, 0, -1), (-1, 0, 1), (1, 0, 1), (1, 0, -1)), white),   # floor  (+y)
        (quad((-1, 2, -1), (1, 2, -1), (1, 2, 1), (-1, 2, 1)), white),   # ceiling (-y)
        (quad((-1, 0, -1), (1, 0, -1), (1, 2, -1), (-1, 2, -1)), white),  # back (+z)
        (quad((-1, 0, -1), (-1, 2, -1), (-1, 2, 1), (-1, 0, 1)), red),    # left (+x)
        (quad((1, 0, -1), (1, 0, 1), (1, 2, 1), (1, 2, -1)), green),      # right (-x)
    ]
    for (pos, idx), b in walls:
        n = np.cross(pos[1] - pos[0], pos[2] - pos[0])
        sd.meshes.append(MeshDesc(pos, idx, b))
    a1, a2 = rng.uniform(0, 45, 2)
    for (c, s, a) in [((-0.35, 0.0, -0.3), (0.55, 1.2, 0.55), a1), ((0.4, 0.0, 0.35), (0.55, 0.6, 0.55), -a2)]:
        pos, idx = box_mesh(c, s, a)
        sd.meshes.append(MeshDesc(pos, idx, white))
    lp, li = quad((-0.25, 1.98, -0.25), (0.25, 1.98, -0.25), (0.25, 1.98, 0.25), (-0.25, 1.98, 0.25))
    sd.meshes.append(MeshDesc(lp, li, BSDFDesc(type=BSDF_DIFFUSE, kd=[0.0, 0.0, 0.0]), radiance=[17.0, 12.0, 4.0]))
    sd.camera = CameraDesc(width, height, look_at((0, 1, 3.8), (0, 1, 0), (0, 1, 0)), 40.0, 1e-4, 1e4)
    sd.filter = FilterDesc(2, 2.0, 0.5)
    sd.depth = depth
    sd.spp = spp
    return sd


def cornell_smooth(seed: int = 0, width: int = 256, height: int = 256, spp: int = 64, depth: int = 64) -> SceneDesc:
    """The Cornell box with the smooth BSDFs: a smooth-plastic floor, a
    two-sided diffuse back wall, an Oren-Nayar (roughDiffuse, alpha 0.5) red
    left wall, a smooth coating over the green diffuse right wall, a smooth
    gold-like conductor for the tall box,
    a glass box (dielectric 1.5046 in air), a mirror panel on the left wall and
    a two-sided panel (smooth plastic in front, Beckmann rough conductor behind)
    whose back faces the camera, under a 1 x 1 light of radiance (4.25, 3, 1)."""
    sd = cornell_box(seed, width, height, spp, depth)
    floor, ceil, back, left, right, tall, short, light = sd.meshes
    floor.bsdf = BSDFDesc(type=BSDF_PLASTIC, int_ior=1.5046, ext_ior=AIR_IOR, kd=[0.725, 0.725, 0.725])
    back.bsdf = BSDFDesc(type=BSDF_TWO_SIDED, nested=BSDFDesc(type=BSDF_DIFFUSE, kd=[0.725, 0.725, 0.725]))
    left.bsdf = BSDFDesc(type=BSDF_ROUGH_DIFFUSE, kd=[0.63, 0.065, 0.05], alpha_u=0.5, alpha_v=0.5)
    right.bsdf = BSDFDesc(type=BSDF_COATING, int_ior=1.49, ext_ior=AIR_IOR, sigma_a=[0.2, 0.1, 0.3], thickness=0.5,
                          nested=BSDFDesc(type=BSDF_DIFFUSE, kd=[0.14, 0.45, 0.09]))
    tall.bsdf = BSDFDesc(type=BSDF_CONDUCTOR, int_ior=0.4, ext_ior=1.0, k=[3.5, 2.5, 1.5], ks=[1.0, 0.85, 0.6])
    short.bsdf = BSDFDesc(type=BSDF_DIELECTRIC, int_ior=1.5046, ext_ior=AIR_IOR)
    # lift the glass box off the floor: a bottom face coplanar with the floor
    # makes the closest hit a tie between two materials, which the reference
    # resolves by its own traversal order
    short.positions = short.positions + np.float32([0.0, 1e-3, 0.0])
    mp, mi = quad((-0.98, 0.3, -0.7), (-0.98, 1.3, -0.7), (-0.98, 1.3, 0.1), (-0.98, 0.3, 0.1))   # faces +x
    sd.meshes.insert(5, MeshDesc(mp, mi, BSDFDesc(type=BSDF_MIRROR)))
    two = BSDFDesc(type=BSDF_TWO_SIDED, nested=BSDFDesc(type=BSDF_PLASTIC, kd=[0.2, 0.3, 0.7]),
                   nested2=BSDFDesc(type=BSDF_ROUGH_CONDUCTOR, distribution=BECKMANN, alpha_u=0.3, alpha_v=0.3,
                                    int_ior=1.0, ext_ior=1.0, eta=CU_ETA, k=CU_K))
    # front face towards -z (away from the camera at z = 3.8): the camera sees the back side
    pp, pi = quad((0.55, 1.1, 0.0), (0.55, 1.7, 0.0), (0.95, 1.7, -0.3), (0.95, 1.1, -0.3))
    sd.meshes.insert(6, MeshDesc(pp, pi, two))
    # a 1 x 1 light of a quarter of the radiance (same power): caustics reached
    # by BSDF sampling alone are found four times as often
    lp, li = quad((-0.5, 1.98, -0.5), (0.5, 1.98, -0.5), (0.5, 1.98, 0.5), (-0.5, 1.98, 0.5))
    light.positions, light.indices, light.radiance = lp, li, [4.25, 3.0, 1.0]
    return sd


def vertex_normals(P: np.ndarray, F: np.ndarray) -> np.ndarray:
    """Area-weighted vertex normals of a triangle mesh (unit length, float32)."""
    n = np.cross(P[F[:, 1]] - P[F[:, 0]], P[F[:, 2]] - P[F[:, 0]]).astype(np.float64)
    acc = np.zeros((len(P), 3))
    for k in range(3):
        np.add.at(acc, F[:, k], n)
    return (acc / np.linalg.norm(acc, axis=1, keepdims=True)).astype(np.float32)


def spherical_uv(P: np.ndarray, center) -> np.ndarray:
    """Latitude-longitude texture coordinates of points about a center."""
    d = P - np.asarray(center, np.float32)
    d = d / np.linalg.norm(d, axis=1, keepdims=True)
    u = np.arctan2(d[:, 2], d[:, 0]) / (2 * np.pi) + 0.5
    v = np.arccos(np.clip(d[:, 1], -1, 1)) / np.pi
    return np.stack([u, v], 1).astype(np.float32)


def synthetic_image(width: int, height: int, channels: int, seed: int) -> np.ndarray:
    """8-bit test pixels (height x width x channels, row 0 = top): smooth
    gradients, a fine stripe pattern and noise, so that every MIP level and
    filter footprint sees structure."""
    rng = np.random.default_rng(seed)
    y, x = np.mgrid[0:height, 0:width]
    base = np.stack([x * 255 // max(width - 1, 1), y * 255 // max(height - 1, 1), ((x // 3 + y // 3) % 2) * 200 + 30],
                    -1)
    img = (0.7 * base + 0.3 * rng.integers(0, 256, (height, width, 3))).astype(np.uint8)
    return np.ascontiguousarray(img[:, :, :channels])


def lights_scene(width: int = 64, height: int = 64, spp: int = 16, depth: int = 12, seed: int = 0,
                 shading_normals: bool = False, textured: bool = False, bitmap: bool = False,
                 bump: bool = False, geometric: bool = False) -> SceneDesc:
    """A ground quad and five displaced icospheres (diffuse, roughDiffuse,
    smooth plastic, rough conductor, smooth dielectric) lit, in emitter order,
    by a point light, an emissive quad, a constant environment and a
    directional light -- the emitter kinds interleaved as an XML scene lists
    them.  With shading_normals the spheres carry vertex normals and
    latitude-longitude texture coordinates (the shading frame then follows
    dP/du) and the conductor is anisotropic (alpha 0.05 x 0.4).  textured (with
    shading_normals) adds procedural textures: a checkerboard ground, a grid on
    the diffuse sphere, checkerboard roughness on the roughDiffuse sphere, a
    scaled checkerboard on the plastic's kd, textured alphaU / alphaV on the
    conductor and a grid on the glass's refraction colour.  bitmap (with
    textured) swaps in bitmap textures where they differ most: an EWA-filtered
    ground (with vertex normals, so first hits carry screen-space partials), a
    trilinear albedo on the diffuse sphere, a bilinear roughDiffuse albedo, a
    scaled one-channel EWA roughness on the conductor and a nearest, clamped
    refraction colour on the glass.  bump (with bitmap) wraps the ground in a
    bumpMap over an EWA bitmap, the roughDiffuse sphere in a normalMap and the
    conductor in a bumpMap over a checkerboard.  geometric (with textured)
    gives the textures of the hit's geometry: a wireframe albedo with the
    automatic edge width on the diffuse sphere, a wireframe with a fixed edge
    width on the ground, mean curvature on the plastic's kd and scaled
    Gaussian curvature on the conductor's ks."""
    sd = SceneDesc()
    gp, gi = quad((-6, 0, 6), (6, 0, 6), (6, 0, -6), (-6, 0, -6))
    ground = MeshDesc(gp, gi, BSDFDesc(type=BSDF_DIFFUSE, kd=[0.5, 0.5, 0.5]))
    if textured:
        ground.uv = np.float32([[0, 0], [1, 0], [1, 1], [0, 1]])
        ground.bsdf.textures["kd"] = TextureDesc(kind=TEX_CHECKERBOARD, count=12, a=[0.7, 0.7, 0.65],
                                                 b=[0.15, 0.2, 0.3])
        if bitmap:
            ground.normals = np.float32([[0, 1, 0]] * 4)
            ground.bsdf.textures["kd"] = TextureDesc(kind=TEX_BITMAP, pixels=synthetic_image(96, 80, 3, seed + 1),
                                                     filter=FILTER_EWA, gamma=2.2, uv_scale=[3.0, 3.0])
    sd.meshes.append(ground)
    mats = [BSDFDesc(type=BSDF_DIFFUSE, kd=[0.7, 0.3, 0.2]),
            BSDFDesc(type=BSDF_ROUGH_DIFFUSE, kd=[0.3, 0.6, 0.3], alpha_u=0.6, alpha_v=0.6),
            BSDFDesc(type=BSDF_PLASTIC, int_ior=1.5046, ext_ior=AIR_IOR, kd=[0.2, 0.3, 0.7]),
            BSDFDesc(type=BSDF_ROUGH_CONDUCTOR, distribution=GGX, alpha_u=0.2, alpha_v=0.2, int_ior=1.0, ext_ior=1.0,
                     eta=AU_ETA, k=AU_K),
            BSDFDesc(type=BSDF_DIELECTRIC, int_ior=1.5046, ext_ior=AIR_IOR)]
    if shading_normals:
        mats[3] = BSDFDesc(type=BSDF_ROUGH_CONDUCTOR, distribution=GGX, anisotropic=True, alpha_u=0.05, alpha_v=0.4,
                           int_ior=1.0, ext_ior=1.0, eta=AU_ETA, k=AU_K)
    if textured:
        checker = TextureDesc(kind=TEX_CHECKERBOARD, count=8, a=[0.9, 0.85, 0.8], b=[0.1, 0.1, 0.1])
        mats[0].textures["kd"] = TextureDesc(kind=TEX_GRID, count=12, width=0.06, a=[0.05, 0.05, 0.05],
                                             b=[0.8, 0.3, 0.2])
        mats[1].textures["alpha_u"] = TextureDesc(kind=TEX_CHECKERBOARD, count=6, a=[0.05] * 3, b=[0.9] * 3)
        mats[2].textures["kd"] = TextureDesc(kind=TEX_SCALE, scale=0.7, nested=checker)
        mats[3].textures["alpha_u"] = TextureDesc(kind=TEX_GRID, count=8, width=0.1, a=[0.4] * 3, b=[0.02] * 3)
        mats[3].textures["alpha_v"] = TextureDesc(kind=TEX_CHECKERBOARD, count=5, uv_scale=[2, 1], a=[0.3] * 3,
                                                  b=[0.05] * 3)
        mats[4].textures["ks_refract"] = TextureDesc(kind=TEX_GRID, count=6, width=0.05, a=[0.2, 0.2, 0.2],
                                                     b=[1.0, 1.0, 1.0])
    if textured and bitmap:
        mats[0].textures["kd"] = TextureDesc(kind=TEX_BITMAP, pixels=synthetic_image(64, 64, 3, seed + 2),
                                             filter=FILTER_TRILINEAR)
        mats[1].textures["kd"] = TextureDesc(kind=TEX_BITMAP, pixels=synthetic_image(40, 30, 3, seed + 3),
                                             filter=FILTER_BILINEAR)
        mats[3].textures["alpha_u"] = TextureDesc(
            kind=TEX_SCALE, scale=0.5, nested=TextureDesc(kind=TEX_BITMAP, pixels=synthetic_image(50, 70, 1, seed + 4),
                                                          channels=1, filter=FILTER_EWA, max_anisotropy=8.0))
        mats[4].textures["ks_refract"] = TextureDesc(kind=TEX_BITMAP, pixels=synthetic_image(33, 17, 3, seed + 5),
                                                     filter=FILTER_NEAREST, wrap_u=WRAP_CLAMP, wrap_v=WRAP_CLAMP)
    if textured and geometric:
        ground.bsdf.textures["kd"] = TextureDesc(kind=TEX_WIREFRAME, a=[0.6, 0.6, 0.55], b=[0.05, 0.05, 0.2],
                                                 width=0.4, scale=0.5)
        mats[0].textures["kd"] = TextureDesc(kind=TEX_WIREFRAME, a=[0.8, 0.4, 0.2], b=[0.1, 0.1, 0.1], width=0.0,
                                             scale=0.6)
        mats[2].textures["kd"] = TextureDesc(kind=TEX_CURVATURE, a=[0.9, 0.3, 0.1], b=[0.1, 0.4, 0.9], scale=0.8,
                                             count=0)
        mats[3].textures["ks"] = TextureDesc(kind=TEX_SCALE, scale=0.9, nested=TextureDesc(
            kind=TEX_CURVATURE, a=[1.0, 0.8, 0.3], b=[0.3, 0.8, 1.0], scale=2.0, count=1))
    if textured and bitmap and bump:
        ground.bsdf = BSDFDesc(type=BSDF_BUMP_MAP, nested=ground.bsdf, textures={"kd": TextureDesc(
            kind=TEX_SCALE, scale=0.02, nested=TextureDesc(kind=TEX_BITMAP, pixels=synthetic_image(60, 44, 3, seed + 6),
                                                           filter=FILTER_EWA, uv_scale=[4.0, 4.0]))})
        mats[1] = BSDFDesc(type=BSDF_NORMAL_MAP, nested=mats[1], textures={"kd": TextureDesc(
            kind=TEX_BITMAP, pixels=np.clip(synthetic_image(32, 32, 3, seed + 7) // 4 + [96, 96, 190], 0, 255)
            .astype(np.uint8), filter=FILTER_BILINEAR)})
        mats[3] = BSDFDesc(type=BSDF_BUMP_MAP, nested=mats[3], textures={"kd": TextureDesc(
            kind=TEX_CHECKERBOARD, count=6, a=[0.01] * 3, b=[0.0] * 3)})
    for k, b in enumerate(mats):
        c = (-3.2 + 1.6 * k, 0.85, 0.3 * ((k % 2) * 2 - 1))
        P, F = displaced_icosphere(2, 0.8, c, 0.05, seed + k)
        P, F = P.astype(np.float32), F.astype(np.uint32)
        if shading_normals:
            sd.meshes.append(MeshDesc(P, F, b, normals=vertex_normals(P, F), uv=spherical_uv(P, c)))
        else:
            sd.meshes.append(MeshDesc(P, F, b))
    lp, li = quad((-1, 4, -1), (1, 4, -1), (1, 4, 1), (-1, 4, 1))   # faces down
    sd.meshes.append(MeshDesc(lp, li, BSDFDesc(type=BSDF_DIFFUSE, kd=[0.0, 0.0, 0.0]), radiance=[3.0, 3.0, 3.0]))
    sd.lights.append(LightDesc("point", [40.0, 32.0, 24.0], [2.5, 3.0, 2.0], emitter_index=0))
    sd.env_constant = [0.3, 0.35, 0.45]
    sd.env_emitter_index = 2
    sd.lights.append(LightDesc("directional", [1.2, 1.1, 0.9], [-0.4, -1.0, -0.3], emitter_index=3))
    sd.camera = CameraDesc(width, height, look_at((0, 3.5, 8), (0, 0.6, 0), (0, 1, 0)), 45.0, 1e-4, 1e4)
    sd.filter = FilterDesc(2, 2.0, 0.5)
    sd.depth = depth
    sd.spp = spp
    return sd


# ------------------------------------------------------------ icosphere
def icosphere(level: int):
    """Unit icosahedron subdivided `level` times (20 * 4^level triangles), outward winding."""
    t = (1.0 + math.sqrt(5.0)) / 2.0
    V = np.array([(-1, t, 0), (1, t, 0), (-1, -t, 0), (1, -t, 0), (0, -1, t), (0, 1, t), (0, -1, -t), (0, 1, -t),
                  (t, 0, -1), (t, 0, 1), (-t, 0, -1), (-t, 0, 1)], np.float64)
    V /= np.linalg.norm(V, axis=1, keepdims=True)
    F = np.array([(0, 11, 5), (0, 5, 1), (0, 1, 7), (0, 7, 10), (0, 10, 11), (1, 5, 9), (5, 11, 4), (11, 10, 2),
                  (10, 7, 6), (7, 1, 8), (3, 9, 4), (3, 4, 2), (3, 2, 6), (3, 6, 8), (3, 8, 9), (4, 9, 5), (2, 4, 11),
                  (6, 2, 10), (8, 6, 7), (9, 8, 1)], np.int64)
    for _ in range(level):
        e = np.concatenate([F[:, [0, 1]], F[:, [1, 2]], F[:, [2, 0]]], 0)
        e.sort(axis=1)
        key = e[:, 0] * (len(V) + 1) + e[:, 1]
        uk, inv = np.unique(key, return_inverse=True)
        a, b = uk // (len(V) + 1), uk % (len(V) + 1)
        mid = V[a] + V[b]
        mid /= np.linalg.norm(mid, axis=1, keepdims=True)
        m = inv.reshape(3, -1).T + len(V)
        V = np.concatenate([V, mid], 0)
        v0, v1, v2 = F[:, 0], F[:, 1], F[:, 2]
        m01, m12, m20 = m[:, 0], m[:, 1], m[:, 2]
        F = np.concatenate([np.stack([v0, m01, m20], 1), np.stack([v1, m12, m01], 1), np.stack([v2, m20, m12], 1),
                            np.stack([m01, m12, m20], 1)], 0)
    # make the winding outward
    n = np.cross(V[F[:, 1]] - V[F[:, 0]], V[F[:, 2]] - V[F[:, 0]])
    flip = np.einsum("ij,ij->i", n, V[F[:, 0]]) < 0
    F[flip] = F[flip][:, [0, 2, 1]]
    return V, F


def value_noise_3d(p: np.ndarray, seed: int, octaves: int = 4) -> np.ndarray:
    """Seeded fractal value noise in [-1, 1] (trilinear lattice noise, smoothstep
    fade, octave frequency x2, amplitude x0.5)."""
    rng = np.random.default_rng(seed)
    perm = rng.permutation(256)
    vals = rng.uniform(-1.0, 1.0, 256)

    def lattice(ix, iy, iz):
        h = perm[(perm[(perm[ix & 255] + iy) & 255] + iz) & 255]
        return vals[h]

    out = np.zeros(len(p))
    amp, freq, norm = 1.0, 2.0, 0.0
    for _ in range(octaves):
        q = p * freq + 17.0
        i0 = np.floor(q).astype(np.int64)
        f = q - i0
        w = f * f * (3 - 2 * f)
        acc = 0.0
        for dx in (0, 1):
            for dy in (0, 1):
                for dz in (0, 1):
                    wt = (w[:, 0] if dx else 1 - w[:, 0]) * (w[:, 1] if dy else 1 - w[:, 1]) * (w[:, 2] if dz else 1 - w[:, 2])
                    acc = acc + wt * lattice(i0[:, 0] + dx, i0[:, 1] + dy, i0[:, 2] + dz)
        out += amp * acc
        norm += amp
        amp *= 0.5
        freq *= 2.0
    return out / norm


def displaced_icosphere(level: int, radius: float, center, amplitude: float, seed: int):
    V, F = icosphere(level)
    d = value_noise_3d(V, seed) if amplitude != 0.0 else 0.0
    P = V * (radius * (1.0 + amplitude * np.asarray(d))[:, None]) + np.asarray(center, np.float64)
    return P.astype(np.float32), F.astype(np.uint32)


# ------------------------------------------------------------ sky
def sky_envmap(width: int = 2048, height: int = 1024, sun_dir=(0.3, 0.8, 0.5), sun_radiance: float = 2e4,
               sun_deg: float = 0.5):
    """Lat-long sky in the reference's SphericalCoordinates convention
    (theta from +z of the map frame, row 0 at theta = 0): a gradient sky
    brighter at the zenith and a sun disk of angular diameter sun_deg.  The
    map's +z is the world up axis through the returned to_world."""
    # map frame: z = world y (up); x = world x; y = world -z  -> to_world maps map->world
    to_world = np.array([[1, 0, 0, 0], [0, 0, 1, 0], [0, -1, 0, 0], [0, 0, 0, 1]], np.float32)
    th = (np.arange(height) + 0.5) / height * math.pi
    ph = (np.arange(width) + 0.5) / width * 2 * math.pi
    T, Ph = np.meshgrid(th, ph, indexing="ij")
    d_map = np.stack([np.sin(T) * np.cos(Ph), np.sin(T) * np.sin(Ph), np.cos(T)], -1)
    up = np.clip(np.cos(T), -1, 1)
    zen = np.array([0.25, 0.45, 1.0])
    hor = np.array([0.9, 0.95, 1.0])
    gnd = np.array([0.15, 0.13, 0.12])
    s = np.clip(up, 0, 1)[..., None]
    rgb = np.where(up[..., None] >= 0, hor * (1 - s) + zen * s, gnd)
    sd = np.asarray(sun_dir, np.float64)
    sd = sd / np.linalg.norm(sd)
    sd_map = np.linalg.inv(to_world[:3, :3].astype(np.float64)) @ sd
    cosang = np.einsum("ijk,k->ij", d_map, sd_map)
    rgb = rgb.astype(np.float32)
    rgb[cosang >= math.cos(math.radians(sun_deg / 2))] = sun_radiance
    return rgb.astype(np.float32), to_world


def mesh_heavy(material: str = "conductor", width: int = 1024, height: int = 1024, spp: int = 256, depth: int = 16,
               level: int = 8, env_res=(2048, 1024), seed: int = 0) -> SceneDesc:
    """Displaced level-`level` icosphere (20*4^level triangles, 4-octave value
    noise of amplitude 0.08) on a 20x20 diffuse ground quad under the sky.
    material: 'conductor' (GGX alpha 0.2, Cu), 'dielectric' (IOR 1.5, alpha
    0.1), 'plastic' (alpha 0.15)."""
    sd = SceneDesc()
    if material == "conductor":
        b = BSDFDesc(type=BSDF_ROUGH_CONDUCTOR, distribution=GGX, alpha_u=0.2, alpha_v=0.2, int_ior=CU_IOR,
                     ext_ior=1.0, k=CU_K)
    elif material == "dielectric":
        b = BSDFDesc(type=BSDF_ROUGH_DIELECTRIC, distribution=GGX, alpha_u=0.1, alpha_v=0.1, int_ior=1.5, ext_ior=1.0)
    elif material == "plastic":
        b = BSDFDesc(type=BSDF_ROUGH_PLASTIC, distribution=GGX, alpha_u=0.15, alpha_v=0.15, kd=[0.5, 0.5, 0.5])
    else:
        raise ValueError(material)
    P, F = displaced_icosphere(level, 1.0, (0.0, 1.0, 0.0), 0.08, seed)
    sd.meshes.append(MeshDesc(P, F, b))
    gp, gi = quad((-10, 0, -10), (-10, 0, 10), (10, 0, 10), (10, 0, -10))
    sd.meshes.append(MeshDesc(gp, gi, BSDFDesc(type=BSDF_DIFFUSE, kd=[0.5, 0.5, 0.5])))
    rgb, tw = sky_envmap(*env_res)
    sd.env = EnvDesc(rgb, tw, 1.0)
    sd.env_emitter_index = 0
    sd.camera = CameraDesc(width, height, look_at((0, 1.6, 4.2), (0, 0.9, 0), (0, 1, 0)), 40.0, 1e-4, 1e4)
    sd.filter = FilterDesc(2, 2.0, 0.5)
    sd.depth = depth
    sd.spp = spp
    return sd


def random_material(rng, kind: Optional[str] = None) -> BSDFDesc:
    kinds = ["diffuse", "ggx_conductor", "beckmann_conductor", "dielectric", "plastic", "coated"]
    kind = kind or kinds[rng.integers(len(kinds))]
    a = float(rng.uniform(0.05, 0.5))
    col = [float(x) for x in rng.uniform(0.2, 0.9, 3)]
    if kind == "diffuse":
        return BSDFDesc(type=BSDF_DIFFUSE, kd=col)
    if kind in ("ggx_conductor", "beckmann_conductor"):
        cu = rng.random() < 0.5
        return BSDFDesc(type=BSDF_ROUGH_CONDUCTOR, distribution=GGX if kind == "ggx_conductor" else BECKMANN,
                        alpha_u=a, alpha_v=a, int_ior=CU_IOR if cu else AU_IOR, ext_ior=1.0, k=CU_K if cu else AU_K)
    if kind == "dielectric":
        return BSDFDesc(type=BSDF_ROUGH_DIELECTRIC, distribution=GGX, alpha_u=a, alpha_v=a, int_ior=1.5, ext_ior=1.0)
    if kind == "plastic":
        return BSDFDesc(type=BSDF_ROUGH_PLASTIC, distribution=GGX, alpha_u=a, alpha_v=a, kd=col)
    nested = BSDFDesc(type=BSDF_ROUGH_CONDUCTOR, distribution=GGX, alpha_u=a, alpha_v=a, int_ior=AU_IOR, ext_ior=1.0,
                      k=AU_K)
    return BSDFDesc(type=BSDF_ROUGH_COATING, distribution=GGX, alpha_u=0.2, alpha_v=0.2, nested=nested)


def heterogeneous(width: int = 1024, height: int = 1024, spp: int = 128, depth: int = 16, n_spheres: int = 64,
                  levels=(5, 6, 7), level_p=(0.55, 0.30, 0.15), env_res=(2048, 1024), seed: int = 0) -> SceneDesc:
    """64 displaced icospheres (levels 5-7) at seeded positions in a 40x40x10
    box, each with a material drawn uniformly from {diffuse, GGX conductor,
    Beckmann conductor, rough dielectric, rough plastic, coated}, roughness
    U[0.05, 0.5]; a ground plane, 4 area lights and the sky."""
    rng = np.random.default_rng(seed)
    sd = SceneDesc()
    for i in range(n_spheres):
        lvl = int(rng.choice(levels, p=level_p))
        c = (float(rng.uniform(-20, 20)), float(rng.uniform(1.0, 10.0)), float(rng.uniform(-20, 20)))
        r = float(rng.uniform(0.8, 2.0))
        P, F = displaced_icosphere(lvl, r, c, 0.08, seed * 1000 + i)
        sd.meshes.append(MeshDesc(P, F, random_material(rng)))
    gp, gi = quad((-40, 0, -40), (-40, 0, 40), (40, 0, 40), (40, 0, -40))
    sd.meshes.append(MeshDesc(gp, gi, BSDFDesc(type=BSDF_DIFFUSE, kd=[0.5, 0.5, 0.5])))
    for k in range(4):
        cx, cz = (-10 if k % 2 else 10), (-10 if k // 2 else 10)
        lp, li = quad((cx - 2, 14, cz - 2), (cx + 2, 14, cz - 2), (cx + 2, 14, cz + 2), (cx - 2, 14, cz + 2))
        sd.meshes.append(MeshDesc(lp, li, BSDFDesc(type=BSDF_DIFFUSE, kd=[0.0, 0.0, 0.0]),
                                  radiance=[float(x) for x in rng.uniform(20, 40, 3)]))
    rgb, tw = sky_envmap(*env_res)
    sd.env = EnvDesc(rgb, tw, 1.0)
    sd.env_emitter_index = 4
    sd.camera = CameraDesc(width, height, look_at((0, 18, 42), (0, 3, 0), (0, 1, 0)), 45.0, 1e-4, 1e4)
    sd.filter = FilterDesc(2, 2.0, 0.5)
    sd.depth = depth
    sd.spp = spp
    return sd


def heterogeneous_cameras(n: int = 8) -> List[np.ndarray]:
    """Camera-to-world transforms of the 8 views of the heterogeneous scene."""
    out = []
    for k in range(n):
        a = 2 * math.pi * k / n
        out.append(look_at((42 * math.sin(a), 18, 42 * math.cos(a)), (0, 3, 0), (0, 1, 0)))
    return out


def config2_materials():
    """The BSDF-batch material set: Beckmann and GGX rough conductors (alpha in
    {0.05, 0.1, 0.2, 0.3, 0.5}, Cu and Au), rough dielectric IOR 1.5 on the
    same alpha grid, rough plastic alpha 0.15 / 0.3 with kd 0.5, and a rough
    coating (alpha 0.2) over a GGX rough conductor."""
    out = []
    alphas = [0.05, 0.1, 0.2, 0.3, 0.5]
    for dist, dn in ((BECKMANN, "beckmann"), (GGX, "ggx")):
        for metal, eta, k in (("cu", CU_ETA, CU_K), ("au", AU_ETA, AU_K)):
            for a in alphas:
                out.append((f"conductor_{dn}_{metal}_a{a}",
                            BSDFDesc(type=BSDF_ROUGH_CONDUCTOR, distribution=dist, alpha_u=a, alpha_v=a, int_ior=1.0,
                                     ext_ior=1.0, eta=eta, k=k)))
    for dist, dn in ((BECKMANN, "beckmann"), (GGX, "ggx")):
        for a in alphas:
            out.append((f"dielectric_{dn}_a{a}", BSDFDesc(type=BSDF_ROUGH_DIELECTRIC, distribution=dist, alpha_u=a,
                                                          alpha_v=a, int_ior=1.5, ext_ior=1.0)))
    for a in (0.15, 0.3):
        out.append((f"plastic_a{a}", BSDFDesc(type=BSDF_ROUGH_PLASTIC, distribution=GGX, alpha_u=a, alpha_v=a,
                                             kd=[0.5, 0.5, 0.5])))
    nested = BSDFDesc(type=BSDF_ROUGH_CONDUCTOR, distribution=GGX, alpha_u=0.2, alpha_v=0.2, int_ior=1.0, ext_ior=1.0,
                      eta=CU_ETA, k=CU_K)
    out.append(("coated_a0.2", BSDFDesc(type=BSDF_ROUGH_COATING, distribution=GGX, alpha_u=0.2, alpha_v=0.2,
                                        nested=nested)))
    return out


def smooth_materials():
    """The smooth (delta) BSDFs, two-sided compositions and Oren-Nayar: mirror,
    smooth conductors (Cu-like k), dielectrics entering and leaving denser
    media, smooth plastics (linear, nonlinear, IOR below 1), two-sided diffuse,
    plastic / rough conductor and coating / mirror pairs, rough coatings over a
    smooth dielectric and a smooth plastic, smooth coatings over a rough
    conductor, an absorbing layer over diffuse and a rough dielectric, and
    roughDiffuse (full model at two roughnesses, fast approximation)."""
    rc = BSDFDesc(type=BSDF_ROUGH_CONDUCTOR, distribution=GGX, alpha_u=0.2, alpha_v=0.2, int_ior=1.0, ext_ior=1.0,
                  eta=CU_ETA, k=CU_K)
    return [
        ("mirror", BSDFDesc(type=BSDF_MIRROR)),
        ("conductor_cu", BSDFDesc(type=BSDF_CONDUCTOR, int_ior=0.27, ext_ior=1.0, k=CU_K)),
        ("conductor_tinted", BSDFDesc(type=BSDF_CONDUCTOR, int_ior=1.5046, ext_ior=AIR_IOR, k=[1, 1, 1],
                                      ks=[0.9, 0.7, 0.4])),
        ("dielectric_glass", BSDFDesc(type=BSDF_DIELECTRIC, int_ior=1.5046, ext_ior=AIR_IOR)),
        ("dielectric_tinted", BSDFDesc(type=BSDF_DIELECTRIC, int_ior=1.33, ext_ior=1.0, ks=[0.9, 0.95, 1.0],
                                       ks_refract=[1.0, 0.8, 0.6])),
        ("dielectric_bubble", BSDFDesc(type=BSDF_DIELECTRIC, int_ior=1.0, ext_ior=1.33)),
        ("plastic", BSDFDesc(type=BSDF_PLASTIC, int_ior=1.5046, ext_ior=AIR_IOR, kd=[0.6, 0.3, 0.1])),
        ("plastic_nonlinear", BSDFDesc(type=BSDF_PLASTIC, int_ior=1.9, ext_ior=1.0, kd=[0.9, 0.5, 0.2],
                                       nonlinear=True)),
        ("plastic_low_ior", BSDFDesc(type=BSDF_PLASTIC, int_ior=1.0, ext_ior=1.4, kd=[0.5, 0.5, 0.5])),
        ("twosided_diffuse", BSDFDesc(type=BSDF_TWO_SIDED, nested=BSDFDesc(type=BSDF_DIFFUSE, kd=[0.7, 0.2, 0.3]))),
        ("twosided_plastic_conductor", BSDFDesc(type=BSDF_TWO_SIDED, nested=BSDFDesc(type=BSDF_PLASTIC),
                                                nested2=rc)),
        ("twosided_coating_mirror", BSDFDesc(type=BSDF_TWO_SIDED,
                                             nested=BSDFDesc(type=BSDF_ROUGH_COATING, distribution=GGX, alpha_u=0.2,
                                                             alpha_v=0.2, nested=rc),
                                             nested2=BSDFDesc(type=BSDF_MIRROR))),
        ("coated_dielectric", BSDFDesc(type=BSDF_ROUGH_COATING, distribution=BECKMANN, alpha_u=0.3, alpha_v=0.3,
                                       nested=BSDFDesc(type=BSDF_DIELECTRIC, int_ior=1.3, ext_ior=1.0))),
        ("coated_plastic", BSDFDesc(type=BSDF_ROUGH_COATING, distribution=GGX, alpha_u=0.1, alpha_v=0.1,
                                    nested=BSDFDesc(type=BSDF_PLASTIC, kd=[0.3, 0.6, 0.2]))),
        ("smooth_coated_conductor", BSDFDesc(type=BSDF_COATING, nested=rc)),
        ("smooth_coated_absorbing", BSDFDesc(type=BSDF_COATING, int_ior=1.7, ext_ior=1.0, ks=[0.9, 0.9, 0.8],
                                             sigma_a=[0.5, 1.0, 2.0], thickness=0.5,
                                             nested=BSDFDesc(type=BSDF_DIFFUSE, kd=[0.8, 0.6, 0.2]))),
        ("smooth_coated_rough_dielectric", BSDFDesc(type=BSDF_COATING, int_ior=1.3, ext_ior=1.0,
                                                    nested=BSDFDesc(type=BSDF_ROUGH_DIELECTRIC, distribution=GGX,
                                                                    alpha_u=0.2, alpha_v=0.2, int_ior=1.5,
                                                                    ext_ior=1.0))),
        ("twosided_smooth_coating", BSDFDesc(type=BSDF_TWO_SIDED, nested=BSDFDesc(type=BSDF_COATING, nested=rc))),
        ("rough_diffuse", BSDFDesc(type=BSDF_ROUGH_DIFFUSE, kd=[0.7, 0.5, 0.3], alpha_u=0.2, alpha_v=0.2)),
        ("rough_diffuse_rough", BSDFDesc(type=BSDF_ROUGH_DIFFUSE, kd=[0.9, 0.9, 0.9], alpha_u=0.8, alpha_v=0.8)),
        ("rough_diffuse_fast", BSDFDesc(type=BSDF_ROUGH_DIFFUSE, kd=[0.7, 0.5, 0.3], alpha_u=0.4, alpha_v=0.4,
                                        fast_approx=True)),
    ]


def nested_materials():
    """Layered BSDFs nested deeper than one coating over a leaf: a rough
    coating over a smooth coating over a rough conductor, a smooth coating
    over a rough coating over diffuse, three layers (rough over smooth over
    rough) over a plastic, a coating over a two-sided BSDF, a two-sided BSDF
    inside a two-sided one, a two-sided BSDF over a doubly coated conductor,
    and a coating stack over a rough dielectric (the innermost layer still
    transmits)."""
    rc = BSDFDesc(type=BSDF_ROUGH_CONDUCTOR, distribution=GGX, alpha_u=0.2, alpha_v=0.2, int_ior=0.27, ext_ior=1.0,
                  k=CU_K)
    dif = BSDFDesc(type=BSDF_DIFFUSE, kd=[0.7, 0.5, 0.3])
    return [
        ("rough_over_smooth_conductor", BSDFDesc(type=BSDF_ROUGH_COATING, distribution=GGX, alpha_u=0.15,
                                                 alpha_v=0.15, int_ior=1.4, ext_ior=1.0,
                                                 nested=BSDFDesc(type=BSDF_COATING, int_ior=1.6, ext_ior=1.0,
                                                                 sigma_a=[0.3, 0.2, 0.1], thickness=0.4,
                                                                 nested=rc))),
        ("smooth_over_rough_diffuse", BSDFDesc(type=BSDF_COATING, int_ior=1.5, ext_ior=1.0, ks=[0.9, 0.9, 0.8],
                                               nested=BSDFDesc(type=BSDF_ROUGH_COATING, distribution=BECKMANN,
                                                               alpha_u=0.3, alpha_v=0.3, thickness=0.5,
                                                               sigma_a=[0.4, 0.8, 1.2], nested=dif))),
        ("three_layers_plastic", BSDFDesc(type=BSDF_ROUGH_COATING, distribution=BECKMANN, alpha_u=0.25, alpha_v=0.25,
                                          nested=BSDFDesc(type=BSDF_COATING, int_ior=1.3, ext_ior=1.0,
                                                          nested=BSDFDesc(type=BSDF_ROUGH_COATING, distribution=GGX,
                                                                          alpha_u=0.1, alpha_v=0.1, int_ior=1.7,
                                                                          ext_ior=1.0,
                                                                          nested=BSDFDesc(type=BSDF_PLASTIC,
                                                                                          kd=[0.2, 0.5, 0.7]))))),
        ("coating_over_twosided", BSDFDesc(type=BSDF_ROUGH_COATING, distribution=GGX, alpha_u=0.2, alpha_v=0.2,
                                           nested=BSDFDesc(type=BSDF_TWO_SIDED, nested=dif, nested2=rc))),
        ("twosided_in_twosided", BSDFDesc(type=BSDF_TWO_SIDED,
                                          nested=BSDFDesc(type=BSDF_TWO_SIDED, nested=rc, nested2=dif),
                                          nested2=BSDFDesc(type=BSDF_MIRROR))),
        ("twosided_double_coated", BSDFDesc(type=BSDF_TWO_SIDED,
                                            nested=BSDFDesc(type=BSDF_COATING, int_ior=1.5, ext_ior=1.0,
                                                            nested=BSDFDesc(type=BSDF_ROUGH_COATING,
                                                                            distribution=GGX, alpha_u=0.3,
                                                                            alpha_v=0.3, nested=rc)),
                                            nested2=dif)),
        ("coatings_over_rough_dielectric", BSDFDesc(type=BSDF_ROUGH_COATING, distribution=GGX, alpha_u=0.1,
                                                    alpha_v=0.1, int_ior=1.3, ext_ior=1.0,
                                                    nested=BSDFDesc(type=BSDF_COATING, int_ior=1.4, ext_ior=1.0,
                                                                    nested=BSDFDesc(type=BSDF_ROUGH_DIELECTRIC,
                                                                                    distribution=GGX, alpha_u=0.2,
                                                                                    alpha_v=0.2, int_ior=1.5,
                                                                                    ext_ior=1.0)))),
    ]


def cornell_nested(seed: int = 0, width: int = 256, height: int = 256, spp: int = 64, depth: int = 64) -> SceneDesc:
    """The Cornell box with deeply nested layered BSDFs on its walls and boxes
    (the set of nested_materials: coatings over coatings, coatings over
    two-sided BSDFs, two-sided BSDFs inside two-sided ones; the coating stack
    over a rough dielectric is left out, so that no path draws the random
    number of a transmission lobe it may not reach)."""
    sd = cornell_box(seed, width, height, spp, depth)
    mats = dict(nested_materials())
    floor, ceil, back, left, right, tall, short, light = sd.meshes
    floor.bsdf = mats["three_layers_plastic"]
    back.bsdf = mats["twosided_in_twosided"]
    left.bsdf = mats["smooth_over_rough_diffuse"]
    right.bsdf = mats["coating_over_twosided"]
    ceil.bsdf = mats["twosided_double_coated"]
    tall.bsdf = mats["rough_over_smooth_conductor"]
    short.bsdf = BSDFDesc(type=BSDF_COATING, int_ior=1.45, ext_ior=1.0, nested=mats["twosided_in_twosided"])
    return sd


def textured_materials():
    """BSDFs with procedural textures on every textured parameter: diffuse and
    roughDiffuse albedo / roughness, smooth and rough conductors (ks, alphaU /
    alphaV), dielectrics (ksReflect / ksRefract / alpha), plastics (kd, ks,
    roughPlastic alpha), and coatings (ks, sigmaA, roughCoating alpha) over
    diffuse."""
    chk = TextureDesc(kind=TEX_CHECKERBOARD, count=7, a=[0.9, 0.2, 0.1], b=[0.1, 0.3, 0.8], uv_scale=[1.5, 0.7],
                      uv_offset=[0.25, -0.1])
    grid = TextureDesc(kind=TEX_GRID, count=5, width=0.08, a=[0.05, 0.05, 0.05], b=[0.7, 0.6, 0.5])
    scaled = TextureDesc(kind=TEX_SCALE, scale=0.6, nested=TextureDesc(kind=TEX_CHECKERBOARD, count=3))
    a_chk = TextureDesc(kind=TEX_CHECKERBOARD, count=4, a=[0.05] * 3, b=[0.4] * 3)
    a_grid = TextureDesc(kind=TEX_GRID, count=6, width=0.1, a=[0.6] * 3, b=[0.15] * 3)
    return [
        ("tex_diffuse", BSDFDesc(type=BSDF_DIFFUSE, textures={"kd": chk})),
        ("tex_rough_diffuse", BSDFDesc(type=BSDF_ROUGH_DIFFUSE, textures={"kd": grid, "alpha_u": a_chk})),
        ("tex_conductor", BSDFDesc(type=BSDF_CONDUCTOR, int_ior=0.27, ext_ior=1.0, k=CU_K, textures={"ks": chk})),
        ("tex_rough_conductor", BSDFDesc(type=BSDF_ROUGH_CONDUCTOR, distribution=GGX, alpha_u=0.2, alpha_v=0.2,
                                         int_ior=1.0, ext_ior=1.0, eta=CU_ETA, k=CU_K,
                                         textures={"alpha_u": a_chk, "ks": chk})),
        ("tex_rough_conductor_aniso", BSDFDesc(type=BSDF_ROUGH_CONDUCTOR, distribution=BECKMANN, anisotropic=True,
                                               alpha_u=0.1, alpha_v=0.3, int_ior=1.0, ext_ior=1.0, eta=AU_ETA, k=AU_K,
                                               textures={"alpha_u": a_chk, "alpha_v": a_grid})),
        ("tex_dielectric", BSDFDesc(type=BSDF_DIELECTRIC, textures={"ks": grid, "ks_refract": scaled})),
        ("tex_rough_dielectric", BSDFDesc(type=BSDF_ROUGH_DIELECTRIC, distribution=GGX, alpha_u=0.1, alpha_v=0.1,
                                          int_ior=1.5, ext_ior=1.0, textures={"alpha_u": a_grid, "ks_refract": chk})),
        ("tex_plastic", BSDFDesc(type=BSDF_PLASTIC, kd=[0.3, 0.3, 0.3], textures={"kd": grid, "ks": scaled})),
        ("tex_rough_plastic", BSDFDesc(type=BSDF_ROUGH_PLASTIC, distribution=GGX, alpha_u=0.15, alpha_v=0.15,
                                       textures={"kd": chk, "ks": grid})),
        ("tex_rough_coating", BSDFDesc(type=BSDF_ROUGH_COATING, distribution=GGX, alpha_u=0.2, alpha_v=0.2,
                                       thickness=0.5, nested=BSDFDesc(type=BSDF_DIFFUSE, textures={"kd": grid}),
                                       textures={"sigma_a": scaled, "ks": chk})),
        ("tex_coating", BSDFDesc(type=BSDF_COATING, nested=BSDFDesc(type=BSDF_DIFFUSE, textures={"kd": chk}),
                                 textures={"sigma_a": scaled})),
        # textured roughness of the transmittance-table BSDFs (2D table per query)
        ("tex_rough_plastic_alpha", BSDFDesc(type=BSDF_ROUGH_PLASTIC, distribution=GGX, alpha_u=0.15,
                                             alpha_v=0.15, textures={"alpha_u": a_grid, "kd": chk})),
        ("tex_rough_coating_alpha", BSDFDesc(type=BSDF_ROUGH_COATING, distribution=BECKMANN, alpha_u=0.2,
                                             alpha_v=0.2, thickness=0.3, sigma_a=[0.2, 0.4, 0.8],
                                             nested=BSDFDesc(type=BSDF_DIFFUSE, kd=[0.6, 0.5, 0.4]),
                                             textures={"alpha_u": a_chk})),
    ]


def bsdf_scene(materials) -> SceneDesc:
    """A minimal scene holding the given BSDFs (one tiny mesh each) so the BSDF
    batch entry point can address them by id."""
    sd = SceneDesc()
    for i, (_, b) in enumerate(materials):
        p, idx = quad((i, 0, 0), (i + 0.5, 0, 0), (i + 0.5, 0, 0.5), (i, 0, 0.5))
        sd.meshes.append(MeshDesc(p, idx, b))
    sd.camera = CameraDesc(8, 8, np.eye(4, dtype=np.float32), 40.0, 1e-4, 1e4)
    return sd
