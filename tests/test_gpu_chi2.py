"""Chi-square goodness-of-fit of the CUDA BSDF sampling against the BSDF's own
Pdf, following the reference's Chi2Test (src/core/Chi2Test.cpp:71-200):
samples histogrammed on a cos(theta) x phi grid (20 x 40), expected
frequencies from integrating Pdf over each cell, cells with expected
frequency below 5 pooled, Sidak-corrected significance 0.01.  Unlike the
reference test harness (which passes a null sampler, freezing the rough
dielectric's reflect/refract choice), the dielectric's Next1D draw is a real
uniform, so both lobes are tested."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

import hikari_b200 as hk  # noqa: E402
from hikari_b200 import scenes  # noqa: E402
from oracle.oracle import chi2_test  # noqa: E402

RES_T, RES_P = 20, 40
SUB = 24                      # Simpson intervals per cell and axis (even)
N_SAMPLES = 10_000_000


def simpson_weights(n_cells, sub):
    n = n_cells * sub
    w = np.ones(n + 1)
    w[1:-1:2] = 4
    w[2:-1:2] = 2
    return w / 3.0


@pytest.fixture(scope="module")
def bsdf_scene():
    mats = scenes.config2_materials()
    return mats, hk.Scene.from_desc(scenes.bsdf_scene(mats))


def expected_frequencies(gs, bid, wi):
    nt, npd = RES_T * SUB, RES_P * SUB
    ct = np.linspace(-1.0, 1.0, nt + 1)
    ph = np.linspace(0.0, 2 * np.pi, npd + 1)
    C, P = np.meshgrid(ct, ph, indexing="ij")
    S = np.sqrt(np.maximum(0.0, 1.0 - C * C))
    wo = np.stack([S * np.cos(P), S * np.sin(P), C], -1).reshape(-1, 3).astype(np.float32)
    n = wo.shape[0]
    dev = "cuda"
    twi = torch.from_numpy(np.repeat(wi[None, :], n, 0)).to(dev)
    zeros2 = torch.zeros((n, 2), dtype=torch.float32, device=dev)
    out = gs.bsdf_batch(bid, twi, zeros2, None, torch.from_numpy(wo).to(dev))
    pdf = out["p_pdf"].cpu().numpy().astype(np.float64).reshape(nt + 1, npd + 1)
    wt = simpson_weights(RES_T, SUB) * (2.0 / nt)
    wp = simpson_weights(RES_P, SUB) * (2 * np.pi / npd)
    exp = np.zeros((RES_T, RES_P))
    for i in range(RES_T):
        for j in range(RES_P):
            blk = pdf[i * SUB:(i + 1) * SUB + 1, j * SUB:(j + 1) * SUB + 1]
            exp[i, j] = wt[: SUB + 1] @ blk @ wp[: SUB + 1]
    return exp * N_SAMPLES


def observed_frequencies(gs, bid, wi, seed):
    dev = "cuda"
    g = torch.Generator(device=dev)
    g.manual_seed(seed)
    u2 = torch.rand((N_SAMPLES, 2), generator=g, device=dev)
    u1 = torch.rand((N_SAMPLES,), generator=g, device=dev)
    twi = torch.from_numpy(np.ascontiguousarray(np.repeat(wi[None, :], N_SAMPLES, 0))).to(dev)
    out = gs.bsdf_batch(bid, twi, u2, u1, twi)
    w, wo = out["s_w"], out["s_wo"]
    ok = (w != 0).any(1)
    wo = wo[ok]
    tb = torch.clamp(torch.floor((wo[:, 2] * 0.5 + 0.5) * RES_T).long(), 0, RES_T - 1)
    sp = torch.atan2(wo[:, 1], wo[:, 0]) * (1.0 / (2 * np.pi))
    sp = torch.where(sp < 0, sp + 1, sp)
    pb = torch.clamp(torch.floor(sp * RES_P).long(), 0, RES_P - 1)
    hist = torch.bincount(tb * RES_P + pb, minlength=RES_T * RES_P)
    return hist.cpu().numpy().astype(np.float64).reshape(RES_T, RES_P)


def test_bsdf_sampling_chi2(bsdf_scene):
    mats, gs = bsdf_scene
    rng = np.random.default_rng(2024)
    failures = []
    for k, (name, d) in enumerate(mats):
        ct = rng.random()
        phi = 2 * np.pi * rng.random()
        st = np.sqrt(max(0.0, 1 - ct * ct))
        wi = np.array([np.cos(phi) * st, np.sin(phi) * st, ct], np.float32)
        bid = gs.bsdf_ids[id(d)]
        obs = observed_frequencies(gs, bid, wi, seed=k)
        exp = expected_frequencies(gs, bid, wi)
        ok, p, msg = chi2_test(obs, exp, N_SAMPLES, 5.0, 0.01, len(mats))
        print(f"{name:30s} p={p:.4f} {msg}")
        if not ok:
            failures.append((name, p, msg))
    assert not failures, failures
