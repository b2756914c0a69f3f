"""Record-wise pin of the oracle BSDFs against the reference's own BSDF classes
compiled from its sources (oracle/ref_build.py -> oracle/_ref).  Bit-exact
equality is required: the oracle follows the reference's float evaluation
order, including Eigen's x + (y + z) reduction of 3-vectors."""
import ctypes as C
import os

import numpy as np
import pytest

from hikari_b200.scenedesc import (BECKMANN, BSDF_COATING, BSDF_CONDUCTOR, BSDF_DIELECTRIC, BSDF_DIFFUSE,
                                   BSDF_MIRROR, BSDF_PLASTIC, BSDF_ROUGH_COATING, BSDF_ROUGH_CONDUCTOR,
                                   BSDF_ROUGH_DIELECTRIC, BSDF_ROUGH_DIFFUSE, BSDF_ROUGH_PLASTIC, BSDF_TWO_SIDED, GGX,
                                   SMOOTH_BSDFS, TEX_CHECKERBOARD, TEX_GRID, TEX_SCALE, TEX_SLOTS, BSDFDesc,
                                   SceneDesc, TextureDesc)
from hikari_b200 import scenes
from oracle import oracle as O

from oracle import ref_build  # noqa: E402

REF_LIB = ref_build.LIB


def _ref_lib():
    try:
        ref_build.build()   # incremental; needs the reference checkout
    except FileNotFoundError:
        pass
    if not os.path.exists(REF_LIB):   # no checkout and nothing prebuilt
        pytest.skip("reference library unavailable")
    R = C.CDLL(REF_LIB)
    R.hr_init.argtypes = [C.c_char_p]
    R.hr_bsdf_create.restype = C.c_void_p
    R.hr_bsdf_create.argtypes = [C.c_int, C.c_int, C.c_float, C.c_float, C.c_float] + [C.c_void_p] * 4 + [
        C.c_float, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_void_p, C.c_int]
    R.hr_texture_create.restype = C.c_void_p
    R.hr_texture_create.argtypes = [C.c_int, C.c_int, C.c_float, C.c_float] + [C.c_void_p] * 5
    R.hr_bsdf_eval.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_void_p]
    R.hr_bsdf_pdf.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int]
    R.hr_bsdf_pdf.restype = C.c_float
    R.hr_bsdf_batch.argtypes = [C.c_void_p, C.c_uint64] + [C.c_void_p] * 12
    R.hr_init(os.path.dirname(REF_LIB).encode())
    return R


CU_K = [3.9, 2.4, 2.2]
CHECKER = TextureDesc(kind=TEX_CHECKERBOARD, count=7, a=[0.9, 0.2, 0.1], b=[0.1, 0.3, 0.8], uv_scale=[1.5, 0.7],
                      uv_offset=[0.25, -0.1])
GRID = TextureDesc(kind=TEX_GRID, count=5, width=0.08, a=[0.05, 0.05, 0.05], b=[0.7, 0.6, 0.5])
SCALED = TextureDesc(kind=TEX_SCALE, scale=0.6, nested=TextureDesc(kind=TEX_CHECKERBOARD, count=3))
ALPHA_CHECKER = TextureDesc(kind=TEX_CHECKERBOARD, count=4, a=[0.05, 0.05, 0.05], b=[0.4, 0.4, 0.4])
ALPHA_GRID = TextureDesc(kind=TEX_GRID, count=6, width=0.1, a=[0.6, 0.6, 0.6], b=[0.15, 0.15, 0.15])


def _cases():
    nested = BSDFDesc(type=BSDF_ROUGH_CONDUCTOR, distribution=GGX, alpha_u=0.2, alpha_v=0.2, int_ior=0.2,
                      ext_ior=1.0, k=CU_K)
    return {
        "diffuse": BSDFDesc(type=BSDF_DIFFUSE, kd=[0.3, 0.5, 0.7]),
        "conductor_beckmann": BSDFDesc(type=BSDF_ROUGH_CONDUCTOR, distribution=BECKMANN, alpha_u=0.2,
                                       alpha_v=0.2, int_ior=0.2, ext_ior=1.0, k=CU_K),
        "conductor_ggx": BSDFDesc(type=BSDF_ROUGH_CONDUCTOR, distribution=GGX, alpha_u=0.05, alpha_v=0.05,
                                  int_ior=0.2, ext_ior=1.0, k=CU_K),
        "dielectric_ggx": BSDFDesc(type=BSDF_ROUGH_DIELECTRIC, distribution=GGX, alpha_u=0.1, alpha_v=0.1,
                                   int_ior=1.5, ext_ior=1.0),
        "dielectric_beckmann": BSDFDesc(type=BSDF_ROUGH_DIELECTRIC, distribution=BECKMANN, alpha_u=0.3,
                                        alpha_v=0.3, int_ior=1.5),
        "plastic_ggx": BSDFDesc(type=BSDF_ROUGH_PLASTIC, distribution=GGX, alpha_u=0.15, alpha_v=0.15),
        "plastic_beckmann": BSDFDesc(type=BSDF_ROUGH_PLASTIC, distribution=BECKMANN, alpha_u=0.3, alpha_v=0.3),
        "coating": BSDFDesc(type=BSDF_ROUGH_COATING, distribution=GGX, alpha_u=0.2, alpha_v=0.2, nested=nested),
        "plastic_nonlinear": BSDFDesc(type=BSDF_ROUGH_PLASTIC, distribution=GGX, alpha_u=0.15, alpha_v=0.15,
                                      kd=[0.8, 0.4, 0.1], nonlinear=True),
        "smooth_mirror": BSDFDesc(type=BSDF_MIRROR),
        "smooth_conductor": BSDFDesc(type=BSDF_CONDUCTOR, int_ior=0.2, ext_ior=1.0, k=CU_K, ks=[0.9, 0.8, 0.7]),
        "smooth_dielectric": BSDFDesc(type=BSDF_DIELECTRIC, int_ior=1.5046, ext_ior=1.000277, ks=[0.9, 0.95, 1.0],
                                      ks_refract=[1.0, 0.9, 0.8]),
        "smooth_dielectric_inv": BSDFDesc(type=BSDF_DIELECTRIC, int_ior=1.0, ext_ior=1.33),
        "smooth_plastic": BSDFDesc(type=BSDF_PLASTIC, int_ior=1.5046, ext_ior=1.000277, kd=[0.6, 0.3, 0.1]),
        "smooth_plastic_nonlinear": BSDFDesc(type=BSDF_PLASTIC, int_ior=1.9, ext_ior=1.0, kd=[0.9, 0.5, 0.2],
                                             nonlinear=True),
        "smooth_plastic_low_ior": BSDFDesc(type=BSDF_PLASTIC, int_ior=1.0, ext_ior=1.4, kd=[0.5, 0.5, 0.5]),
        "twosided_one": BSDFDesc(type=BSDF_TWO_SIDED, nested=BSDFDesc(type=BSDF_DIFFUSE, kd=[0.7, 0.2, 0.3])),
        "twosided_two": BSDFDesc(type=BSDF_TWO_SIDED, nested=BSDFDesc(type=BSDF_PLASTIC, kd=[0.2, 0.6, 0.3]),
                                 nested2=BSDFDesc(type=BSDF_ROUGH_CONDUCTOR, distribution=BECKMANN, alpha_u=0.3,
                                                  alpha_v=0.3, int_ior=0.2, ext_ior=1.0, k=CU_K)),
        "twosided_coating": BSDFDesc(type=BSDF_TWO_SIDED, nested=BSDFDesc(type=BSDF_ROUGH_COATING, distribution=GGX,
                                                                           alpha_u=0.2, alpha_v=0.2, nested=nested),
                                     nested2=BSDFDesc(type=BSDF_MIRROR)),
        "coating_over_smooth": BSDFDesc(type=BSDF_ROUGH_COATING, distribution=BECKMANN, alpha_u=0.3, alpha_v=0.3,
                                        nested=BSDFDesc(type=BSDF_DIELECTRIC, int_ior=1.3, ext_ior=1.0)),
        "smooth_coating_conductor": BSDFDesc(type=BSDF_COATING, nested=nested),
        "smooth_coating_absorbing": BSDFDesc(type=BSDF_COATING, int_ior=1.7, ext_ior=1.0, ks=[0.9, 0.9, 0.8],
                                             sigma_a=[0.5, 1.0, 2.0], thickness=0.5,
                                             nested=BSDFDesc(type=BSDF_DIFFUSE, kd=[0.8, 0.6, 0.2])),
        "smooth_coating_dielectric": BSDFDesc(type=BSDF_COATING, int_ior=1.3, ext_ior=1.0,
                                              nested=BSDFDesc(type=BSDF_ROUGH_DIELECTRIC, distribution=GGX,
                                                              alpha_u=0.2, alpha_v=0.2, int_ior=1.5, ext_ior=1.0)),
        "rough_diffuse": BSDFDesc(type=BSDF_ROUGH_DIFFUSE, kd=[0.7, 0.5, 0.3], alpha_u=0.2, alpha_v=0.2),
        "rough_diffuse_rough": BSDFDesc(type=BSDF_ROUGH_DIFFUSE, kd=[0.9, 0.9, 0.9], alpha_u=0.8, alpha_v=0.8),
        "rough_diffuse_fast": BSDFDesc(type=BSDF_ROUGH_DIFFUSE, kd=[0.7, 0.5, 0.3], alpha_u=0.4, alpha_v=0.4,
                                       fast_approx=True),
        # textured parameters (Record.Isect.UV drives Texture2D::Eval)
        "tex_diffuse_checker": BSDFDesc(type=BSDF_DIFFUSE, textures={"kd": CHECKER}),
        "tex_plastic_grid": BSDFDesc(type=BSDF_PLASTIC, kd=[0.3, 0.3, 0.3], textures={"kd": GRID, "ks": SCALED}),
        "tex_rough_conductor_alpha": BSDFDesc(type=BSDF_ROUGH_CONDUCTOR, distribution=GGX, alpha_u=0.2, alpha_v=0.2,
                                              int_ior=0.2, ext_ior=1.0, k=CU_K,
                                              textures={"alpha_u": ALPHA_CHECKER, "ks": CHECKER}),
        "tex_rough_conductor_aniso": BSDFDesc(type=BSDF_ROUGH_CONDUCTOR, distribution=BECKMANN, anisotropic=True,
                                              alpha_u=0.1, alpha_v=0.3, int_ior=0.2, ext_ior=1.0, k=CU_K,
                                              textures={"alpha_u": ALPHA_CHECKER, "alpha_v": ALPHA_GRID}),
        "tex_rough_dielectric": BSDFDesc(type=BSDF_ROUGH_DIELECTRIC, distribution=GGX, alpha_u=0.1, alpha_v=0.1,
                                         int_ior=1.5, ext_ior=1.0,
                                         textures={"alpha_u": ALPHA_GRID, "ks_refract": CHECKER}),
        "tex_rough_plastic": BSDFDesc(type=BSDF_ROUGH_PLASTIC, distribution=GGX, alpha_u=0.15, alpha_v=0.15,
                                      textures={"kd": CHECKER, "ks": GRID}),
        "tex_coating_sigma": BSDFDesc(type=BSDF_ROUGH_COATING, distribution=GGX, alpha_u=0.2, alpha_v=0.2,
                                      thickness=0.5, nested=BSDFDesc(type=BSDF_DIFFUSE, textures={"kd": GRID}),
                                      textures={"sigma_a": SCALED, "ks": CHECKER}),
        "tex_smooth_coating": BSDFDesc(type=BSDF_COATING, nested=BSDFDesc(type=BSDF_DIFFUSE, textures={"kd": CHECKER}),
                                       textures={"sigma_a": SCALED}),
        "tex_rough_diffuse": BSDFDesc(type=BSDF_ROUGH_DIFFUSE, textures={"kd": GRID, "alpha_u": ALPHA_CHECKER}),
        "tex_dielectric": BSDFDesc(type=BSDF_DIELECTRIC, textures={"ks": GRID, "ks_refract": SCALED}),
        "tex_conductor": BSDFDesc(type=BSDF_CONDUCTOR, int_ior=0.27, ext_ior=1.0, k=CU_K, textures={"ks": CHECKER}),
        # textured roughness of the transmittance-table BSDFs: RoughTransmittance::Eval
        # in 2D per query, EvalDiffuse over alpha (src/core/RoughTransmitance.cpp:71-132)
        "tex_rough_plastic_alpha": BSDFDesc(type=BSDF_ROUGH_PLASTIC, distribution=GGX, alpha_u=0.15, alpha_v=0.15,
                                            textures={"alpha_u": ALPHA_GRID, "kd": CHECKER}),
        "tex_rough_plastic_alpha_nonlinear": BSDFDesc(type=BSDF_ROUGH_PLASTIC, distribution=BECKMANN, alpha_u=0.3,
                                                      alpha_v=0.3, kd=[0.8, 0.4, 0.1], nonlinear=True,
                                                      textures={"alpha_u": ALPHA_CHECKER}),
        "tex_coating_alpha": BSDFDesc(type=BSDF_ROUGH_COATING, distribution=GGX, alpha_u=0.2, alpha_v=0.2,
                                      nested=nested, textures={"alpha_u": ALPHA_CHECKER}),
        "tex_coating_alpha_beckmann": BSDFDesc(type=BSDF_ROUGH_COATING, distribution=BECKMANN, alpha_u=0.2,
                                               alpha_v=0.2, thickness=0.3, sigma_a=[0.2, 0.4, 0.8],
                                               nested=BSDFDesc(type=BSDF_DIFFUSE, kd=[0.6, 0.5, 0.4]),
                                               textures={"alpha_u": ALPHA_GRID}),
        # layered BSDFs nested deeper than one coating over a leaf
        **{"nested_" + k: v for k, v in scenes.nested_materials()},
    }


def records(n, seed):
    rng = np.random.default_rng(seed)
    z = rng.uniform(-0.2, 1, n)
    ph = rng.uniform(0, 2 * np.pi, n)
    s = np.sqrt(1 - z * z)
    wi = np.stack([s * np.cos(ph), s * np.sin(ph), z], 1).astype(np.float32)
    u2 = rng.random((n, 2), dtype=np.float32)
    u1 = rng.random(n, dtype=np.float32)
    z2 = np.sqrt(rng.random(n))
    ph2 = rng.uniform(0, 2 * np.pi, n)
    s2 = np.sqrt(1 - z2 * z2)
    sign = np.where(rng.random(n) < 0.8, 1, -1)
    wo = np.stack([s2 * np.cos(ph2), s2 * np.sin(ph2), z2 * sign], 1).astype(np.float32)
    return wi, u2, u1, wo


@pytest.mark.parametrize("name", list(_cases()))
def test_oracle_bsdf_bit_exact_vs_reference(name):
    R = _ref_lib()
    d = _cases()[name]
    n = 50000
    wi, u2, u1, wo = records(n, 7)
    sd = SceneDesc()
    o = O.OracleScene(sd)
    bid = o.add_bsdf(d)
    assert O.lib().ho_scene_finalize(o.h) == 0

    f = lambda a: np.ascontiguousarray(a, np.float32)

    def mk_tex(t):
        arrs = [f(t.uv_scale), f(t.uv_offset), f(t.a), f(t.b)]
        keep.append(arrs)
        nested = mk_tex(t.nested) if t.nested is not None else None
        h = R.hr_texture_create(t.kind, t.count, t.width, t.scale, *[O._p(a) for a in arrs], nested)
        assert h
        return h

    def mk(b):
        if b is None:
            return None
        arrs = [f(b.k), f(b.ks), f(b.kd), f(b.sigma_a), f(b.ks_refract)]
        keep.append(arrs)
        k, ks, kd, sa, kr = arrs
        tex = (C.c_void_p * 6)(*[mk_tex(b.textures[s]) if s in b.textures else None for s in TEX_SLOTS])
        keep.append(tex)
        h = R.hr_bsdf_create(b.type, b.distribution, b.alpha_u, b.int_ior, b.ext_ior, O._p(k), O._p(ks), O._p(kd),
                             O._p(sa), b.thickness, mk(b.nested), mk(b.nested2), O._p(kr), int(b.nonlinear),
                             int(b.fast_approx), tex, int(b.anisotropic))
        assert h
        return h

    keep = []
    h = mk(d)
    if _has_delta(d):
        # a tenth of the evaluation directions on the mirror direction, a tenth on the refracted one
        wo[0::10] = wi[0::10] * [-1, -1, 1]
        t = wi[5::10] * [-0.6, -0.6, 1]
        t[:, 2] = -np.sign(t[:, 2]) * np.sqrt(np.maximum(0, 1 - t[:, 0] ** 2 - t[:, 1] ** 2))
        wo[5::10] = t.astype(np.float32)
    uv = (np.random.default_rng(3).random((n, 2)) * 4 - 1).astype(np.float32)   # texture coordinates
    a = o.bsdf_batch(bid, wi, u2, u1, wo, uv=uv)
    b = {k: np.zeros_like(v) for k, v in a.items()}
    R.hr_bsdf_batch(h, n, O._p(wi), O._p(u2), O._p(u1), O._p(wo), O._p(uv), None, O._p(b["s_wo"]), O._p(b["s_w"]),
                    O._p(b["s_pdf"]), O._p(b["s_measure"]), O._p(b["e_rgb"]), O._p(b["p_pdf"]))
    valid = np.any(a["s_w"] != 0, axis=1)
    np.testing.assert_array_equal(a["s_w"], b["s_w"])
    np.testing.assert_array_equal(a["s_wo"][valid], b["s_wo"][valid])
    np.testing.assert_array_equal(a["s_measure"], b["s_measure"])
    np.testing.assert_array_equal(a["s_pdf"], b["s_pdf"])
    np.testing.assert_array_equal(a["e_rgb"], b["e_rgb"])
    np.testing.assert_array_equal(a["p_pdf"], b["p_pdf"])
    if _has_delta(d):
        # Eval / Pdf on the sampled direction with the sampled measure (the delta lobes),
        # at texture coordinates (0, 0) like the oracle's single-record queries
        R.hr_set_uv(C.c_float(0.0), C.c_float(0.0))
        for i in range(0, 3000):
            m = int(a["s_measure"][i])
            wi_i, wo_i = np.ascontiguousarray(wi[i]), np.ascontiguousarray(a["s_wo"][i])
            er = np.zeros(3, np.float32)
            R.hr_bsdf_eval(h, O._p(wi_i), O._p(wo_i), m, O._p(er))
            np.testing.assert_array_equal(o.bsdf_eval(bid, wi_i, wo_i, m), er)
            assert o.bsdf_pdf(bid, wi_i, wo_i, m) == R.hr_bsdf_pdf(h, O._p(wi_i), O._p(wo_i), m)


def _has_delta(d):
    return d is not None and (d.type in SMOOTH_BSDFS or _has_delta(d.nested) or _has_delta(d.nested2))


LIGHTS = {   # kind (0 point, 1 directional, 2 constant), power / irradiance / radiance, position / direction
    "point": (0, [10.0, 8.0, 6.0], [0.3, 1.5, -0.2]),
    "directional": (1, [2.0, 1.5, 1.0], [0.3, -1.0, 0.2]),
    "constant": (2, [1.28, 1.27, 1.25], [0.0, 0.0, 0.0]),
}


@pytest.mark.parametrize("name", list(LIGHTS))
def test_oracle_lights_bit_exact_vs_reference(name):
    """PointLight / DirectionalLight / ConstantLight::Sample (and the constant
    light's Eval / Pdf) record by record against the reference classes."""
    from hikari_b200.scenedesc import LightDesc, MeshDesc

    R = _ref_lib()
    R.hr_emitter_create.restype = C.c_void_p
    R.hr_emitter_create.argtypes = [C.c_int, C.c_void_p, C.c_void_p]
    R.hr_emitter_sample.argtypes = [C.c_void_p, C.c_uint64, C.c_void_p, C.c_void_p]
    R.hr_emitter_eval_dir.argtypes = [C.c_void_p, C.c_uint64, C.c_void_p, C.c_void_p]
    kind, col, vec = LIGHTS[name]
    sd = SceneDesc()
    quad = np.array([[-1, 0, -1], [1, 0, -1], [1, 0, 1], [-1, 0, 1]], np.float32)
    sd.meshes.append(MeshDesc(quad, np.array([[0, 1, 2], [3, 0, 2]], np.uint32), BSDFDesc()))
    if kind == 2:
        sd.env_constant = col
    else:
        sd.lights.append(LightDesc("point" if kind == 0 else "directional", col, vec))
    o = O.OracleScene(sd)
    bb = o.bbox()
    ext = (bb[3:] - bb[:3]).astype(np.float32)
    radius = np.float32(0.5) * np.sqrt(ext[0] * ext[0] + (ext[1] * ext[1] + ext[2] * ext[2]), dtype=np.float32)
    rng = np.random.default_rng(5)
    n = 4000
    inp = np.concatenate([rng.uniform(-2, 2, (n, 3)), rng.random((n, 3)), np.full((n, 1), radius)], 1).astype(np.float32)
    inp[:8, 4] = [0.0, 1.0, 0.5, 0.25, 1e-8, 1 - 1e-7, 0.0, 1.0]   # theta at the poles for the constant light
    h = R.hr_emitter_create(kind, O._p(np.float32(col)), O._p(np.float32(vec)))
    assert h
    ref = np.zeros((n, 14), np.float32)
    R.hr_emitter_sample(h, n, O._p(inp), O._p(ref))
    got = np.stack([o.emitter_sample(0, inp[i, :3], inp[i, 3:6]) for i in range(n)])
    valid = np.any(ref[:, 11:] != 0, 1)
    np.testing.assert_array_equal(got[:, 11:], ref[:, 11:])          # value
    np.testing.assert_array_equal(got[valid], ref[valid])             # p, n, wi, pdf, distance
    if kind == 2:
        d = rng.normal(size=(n, 3))
        d = (d / np.linalg.norm(d, axis=1, keepdims=True)).astype(np.float32)
        d[:2] = [[0, 0, 1], [0, 0, -1]]
        ev = np.zeros((n, 4), np.float32)
        R.hr_emitter_eval_dir(h, n, O._p(d), O._p(ev))
        for i in range(n):
            np.testing.assert_array_equal(o.env_eval(d[i]), ev[i, :3])
            assert o.emitter_pdf(0, np.zeros(3, np.float32), d[i], np.zeros(3, np.float32)) == ev[i, 3]


def test_oracle_post_intersect_bit_exact_vs_reference():
    """Triangle::PostIntersect (src/core/Mesh.cpp:67-172) on a mesh with vertex
    normals and texture coordinates: the shading frame follows dP/du, with the
    degenerate-UV and zero-area fallbacks."""
    from hikari_b200 import scenes
    from hikari_b200.scenedesc import MeshDesc

    R = _ref_lib()
    R.hr_mesh_create.restype = C.c_void_p
    R.hr_mesh_create.argtypes = [C.c_void_p, C.c_uint32, C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint32]
    R.hr_post_intersect.argtypes = [C.c_void_p, C.c_uint32, C.c_float, C.c_float, C.c_void_p]
    rng = np.random.default_rng(17)
    P, F = scenes.displaced_icosphere(2, 1.0, (0.3, -0.2, 0.1), 0.08, 4)
    P = P.astype(np.float32)
    F = F.astype(np.uint32)
    N = (P + rng.normal(0, 0.05, P.shape)).astype(np.float32)   # unnormalised on purpose
    UV = rng.random((len(P), 2)).astype(np.float32)
    UV[F[0]] = UV[F[0][0]]                                # triangle 0: degenerate UVs (det == 0)
    P[F[1][1]] = P[F[1][0]]                                 # triangle 1: zero area
    cases = {"normals+uv": (N, UV), "normals": (N, None), "uv": (None, UV), "plain": (None, None)}
    for name, (n, uv) in cases.items():
        sd = SceneDesc()
        sd.meshes.append(MeshDesc(P, F, BSDFDesc(), normals=n, uv=uv))
        o = O.OracleScene(sd)
        h = R.hr_mesh_create(O._p(P), len(P), O._p(n), O._p(uv), O._p(F), len(F))
        tri = np.concatenate([[0, 0, 1, 1], rng.integers(0, len(F), 4000)]).astype(np.uint32)
        u = rng.random(len(tri)).astype(np.float32)
        v = (rng.random(len(tri)) * (1 - u)).astype(np.float32)
        for k in range(len(tri)):
            a = np.zeros(14, np.float32)
            b = np.zeros(14, np.float32)
            O.lib().ho_post_intersect(o.h, int(tri[k]), float(u[k]), float(v[k]), O._p(a))
            R.hr_post_intersect(h, int(tri[k]), float(u[k]), float(v[k]), O._p(b))
            assert np.array_equal(a, b) or (np.isnan(a) == np.isnan(b)).all() and np.array_equal(a[~np.isnan(a)], b[~np.isnan(b)]), \
                f"{name}: triangle {tri[k]} ({u[k]}, {v[k]}): oracle {a} reference {b}"


def _config2_complex_ior():
    """The config-2 materials with a per-channel complex IOR (Cu, Au) and the
    coated conductor, whose nested conductor has one too."""
    from hikari_b200 import scenes

    return [(name, d) for name, d in scenes.config2_materials()
            if d.eta is not None or (d.nested is not None and d.nested.eta is not None)]


@pytest.mark.parametrize("case", range(len(_config2_complex_ior())))
def test_per_channel_ior_pinned_channel_by_channel(case):
    """The reference's conductors take one IOR for every channel
    (m_Eta = Color3f(intIOR / extIOR), src/bsdf/RoughConductorBSDF.cpp:43), so a
    per-channel eta is pinned one channel at a time: the reference built with
    intIOR = eta_c (extIOR 1) gives channel c of the oracle's per-channel
    material bit for bit.  D and G do not depend on eta and the conductor
    Fresnel term is channel-wise (src/core/Common.cpp:529), so the sampled
    directions, measures and pdfs agree on every channel too."""
    import copy

    R = _ref_lib()
    name, d = _config2_complex_ior()[case]
    n = 20000
    wi, u2, u1, wo = records(n, 11)
    o = O.OracleScene(SceneDesc())
    bid = o.add_bsdf(d)
    assert O.lib().ho_scene_finalize(o.h) == 0
    a = o.bsdf_batch(bid, wi, u2, u1, wo)
    f = lambda x: np.ascontiguousarray(x, np.float32)
    keep = []

    def mk(b):
        if b is None:
            return None
        arrs = [f(b.k), f(b.ks), f(b.kd), f(b.sigma_a), f(b.ks_refract)]
        keep.append(arrs)
        k, ks, kd, sa, kr = arrs
        tex = (C.c_void_p * 6)()
        keep.append(tex)
        h = R.hr_bsdf_create(b.type, b.distribution, b.alpha_u, b.int_ior, b.ext_ior, O._p(k), O._p(ks), O._p(kd),
                             O._p(sa), b.thickness, mk(b.nested), mk(b.nested2), O._p(kr), int(b.nonlinear),
                             int(b.fast_approx), tex, int(b.anisotropic))
        assert h
        return h

    for c in range(3):
        dc = copy.deepcopy(d)
        target = dc if dc.eta is not None else dc.nested
        target.int_ior, target.ext_ior, target.eta = float(np.float32(d.eta[c] if d.eta is not None
                                                                       else d.nested.eta[c])), 1.0, None
        h = mk(dc)
        b = {k: np.zeros_like(v) for k, v in a.items()}
        R.hr_bsdf_batch(h, n, O._p(wi), O._p(u2), O._p(u1), O._p(wo), None, None, O._p(b["s_wo"]), O._p(b["s_w"]),
                        O._p(b["s_pdf"]), O._p(b["s_measure"]), O._p(b["e_rgb"]), O._p(b["p_pdf"]))
        np.testing.assert_array_equal(a["s_w"][:, c], b["s_w"][:, c], err_msg=f"{name} channel {c}")
        np.testing.assert_array_equal(a["e_rgb"][:, c], b["e_rgb"][:, c], err_msg=f"{name} channel {c}")
        valid = np.any(a["s_w"] != 0, axis=1)
        np.testing.assert_array_equal(a["s_wo"][valid], b["s_wo"][valid])
        np.testing.assert_array_equal(a["s_pdf"], b["s_pdf"])
        np.testing.assert_array_equal(a["p_pdf"], b["p_pdf"])


_GEO_TEX = {}


def _geo_textures(R):
    """The reference's wireframe and curvature textures for the pin, made once
    per process and kept: CurvatureTexture::Eval (src/texture/CurvatureTexture.cpp:39)
    keeps its colour lookup in a function-local static lambda that captures the
    first evaluated instance, so every curvature texture of a process colours
    with that instance's scale and colours -- the pin gives both of its
    curvature textures the same ones."""
    from hikari_b200.scenedesc import TEX_CURVATURE, TEX_WIREFRAME

    if not _GEO_TEX:
        descs = {
            "wire_auto": TextureDesc(kind=TEX_WIREFRAME, a=[0.8, 0.7, 0.6], b=[0.05, 0.1, 0.2], width=0.0, scale=0.5),
            "wire_fixed": TextureDesc(kind=TEX_WIREFRAME, a=[0.9, 0.9, 0.9], b=[0.3, 0.0, 0.0], width=0.02,
                                      scale=0.25),
            "curv_mean": TextureDesc(kind=TEX_CURVATURE, a=[1.0, 0.2, 0.0], b=[0.0, 0.3, 1.0], scale=0.7, count=0),
            "curv_gauss": TextureDesc(kind=TEX_CURVATURE, a=[1.0, 0.2, 0.0], b=[0.0, 0.3, 1.0], scale=0.7, count=1),
        }
        for name, t in descs.items():
            arrs = [np.array(x, np.float32) for x in (t.uv_scale, t.uv_offset, t.a, t.b)]
            h = R.hr_texture_create(t.kind, t.count, t.width, t.scale, *[O._p(a) for a in arrs], None)
            assert h, name
            _GEO_TEX[name] = (t, h, arrs)
    return _GEO_TEX


def test_oracle_wireframe_and_curvature_bit_exact_vs_reference():
    """WireframeTexture::Eval (src/texture/WireframeTexture.cpp:22: distance to
    the nearest edge line, the automatic edge width of a tenth of the mean edge
    length) and CurvatureTexture::Eval over Shape::ComputeCurvature
    (src/core/Shape.cpp:30, from the dP/du, dN/du partials of
    Triangle::PostIntersect) at hits of a displaced icosphere with vertex
    normals and texture coordinates, bit for bit."""
    from hikari_b200 import scenes
    from hikari_b200.scenedesc import MeshDesc

    R = _ref_lib()
    R.hr_mesh_create.restype = C.c_void_p
    R.hr_mesh_create.argtypes = [C.c_void_p, C.c_uint32, C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint32]
    R.hr_texture_eval_hit.argtypes = [C.c_void_p, C.c_void_p, C.c_uint64, C.c_void_p, C.c_void_p, C.c_void_p]
    R.hr_object_free.argtypes = [C.c_void_p]
    tex = _geo_textures(R)
    rng = np.random.default_rng(23)
    P, F = scenes.displaced_icosphere(2, 1.0, (0.1, 0.2, -0.3), 0.1, 4)
    P = P.astype(np.float32)
    F = F.astype(np.uint32)
    N = (P + rng.normal(0, 0.05, P.shape)).astype(np.float32)
    # texture coordinates from the sphere's longitude and latitude, so the UV
    # partials (and the curvatures) are smooth over most triangles
    c = P - P.mean(0)
    UV = np.stack([np.arctan2(c[:, 1], c[:, 0]) / (2 * np.pi) + 0.5,
                   np.arccos(np.clip(c[:, 2] / np.linalg.norm(c, axis=1), -1, 1)) / np.pi], 1).astype(np.float32)
    UV[F[0]] = UV[F[0][0]]                                # triangle 0: degenerate UVs (det == 0)
    bsdf = BSDFDesc(type=BSDF_ROUGH_DIELECTRIC, distribution=GGX, alpha_u=0.3, alpha_v=0.3)
    bsdf.textures = {"ks": tex["wire_auto"][0], "ks_refract": tex["wire_fixed"][0],
                     "alpha_u": tex["curv_mean"][0], "alpha_v": tex["curv_gauss"][0]}
    for name, (n_, uv_) in {"normals+uv": (N, UV), "plain": (None, None)}.items():
        sd = SceneDesc()
        sd.meshes.append(MeshDesc(P, F, bsdf, normals=n_, uv=uv_))
        o = O.OracleScene(sd)
        h = R.hr_mesh_create(O._p(P), len(P), O._p(n_), O._p(uv_), O._p(F), len(F))
        tri = np.concatenate([[0, 0], rng.integers(0, len(F), 3000)]).astype(np.uint32)
        u = rng.random(len(tri)).astype(np.float32)
        v = (rng.random(len(tri)) * (1 - u)).astype(np.float32)
        # barycentrics on and near the edges, where the wireframe's transition lies
        u[2:200:3] = 0.0
        v[3:200:3] = (1.0 - u[3:200:3]).astype(np.float32)
        buv = np.stack([u, v], 1).astype(np.float32)
        nz = 0
        for key, (t, ht, _) in tex.items():
            got = o.texture_eval_hit(t, tri, u, v)
            ref = np.zeros((len(tri), 3), np.float32)
            R.hr_texture_eval_hit(ht, h, len(tri), O._p(tri), O._p(buv), O._p(ref))
            same = (got == ref) | (np.isnan(got) & np.isnan(ref))
            assert same.all(), f"{name} {key}: {np.sum(~same.all(1))} hits differ, e.g. {got[~same.all(1)][:2]} vs " \
                               f"{ref[~same.all(1)][:2]}"
            nz += int(np.any(got != got[0], axis=1).sum())
        assert nz > 0   # the textures vary over the hits
        R.hr_object_free(h)
