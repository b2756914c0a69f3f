"""Serving loop: continuous batching over resident scenes.

A job's image must be the same whether it renders alone or among other jobs
(each path's random stream depends only on seed, sample, pixel and image
index, so only the order of the film's float additions differs), and the same
as the offline wavefront batch of the same request.  Admission must respect
the device-memory budget, cancellation must end jobs, and the statistics must
add up."""
import time

import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

import hikari_b200 as hk  # noqa: E402
from hikari_b200 import scenes, serving  # noqa: E402
from hikari_b200.scenedesc import FilterDesc  # noqa: E402

DEV = "cuda:0"
RTOL = 2e-4   # float-addition order of the film accumulation (up to a few hundred terms per pixel)


def _scenes():
    a = scenes.cornell_box(width=96, height=96)
    b = scenes.cornell_box(width=128, height=96)
    b.filter = FilterDesc(0, 0.5)                       # box filter: another film border
    c = scenes.mesh_heavy(level=4, material="plastic", width=128, height=128, env_res=(512, 256))
    return [a, b, c]


def _close(a, b):
    d = np.abs(a.astype(np.float64) - b.astype(np.float64))
    tol = RTOL * np.abs(b.astype(np.float64)) + 1e-5
    return bool(np.all(d <= tol)), float((d / (np.abs(b) + 1e-5)).max())


@pytest.fixture(scope="module")
def resident():
    sds = _scenes()
    gss = [hk.Scene.from_desc(sd) for sd in sds]
    return sds, gss


def _requests(sds):
    # (scene, width, height, spp, seed)
    return [(0, 96, 96, 64, 11), (1, 64, 48, 32, 12), (2, 128, 128, 16, 13), (0, 40, 72, 128, 14),
            (2, 80, 80, 48, 15), (1, 128, 96, 16, 16)]


@pytest.mark.parametrize("policy", [serving.SRPT, serving.SRPT_ACROSS, serving.SRPT_SMALL])
def test_same_alone_and_in_mix(resident, policy):
    sds, gss = resident
    reqs = _requests(sds)
    with serving.Server(capacity=1 << 16, iterations_per_poll=4, policy=policy) as srv:
        ids = [srv.add_scene(g) for g in gss]
        assert ids == [0, 1, 2]
        alone = []
        for (s, w, h, spp, seed) in reqs:
            jid, out = srv.submit(s, spp, sds[s].depth, seed, w, h)
            st = srv.wait(jid, timeout_s=120)
            assert st["state"] == serving.DONE
            alone.append(out.copy())
        # the same requests all at once, interleaved with unrelated jobs
        mixed = []
        for k, (s, w, h, spp, seed) in enumerate(reqs):
            srv.submit((s + 1) % 3, 24, sds[(s + 1) % 3].depth, 900 + k, 64, 64)
            mixed.append(srv.submit(s, spp, sds[s].depth, seed, w, h))
        for (jid, out), ref, r in zip(mixed, alone, reqs):
            st = srv.wait(jid, timeout_s=120)
            assert st["state"] == serving.DONE and (st["width"], st["height"]) == (r[1], r[2])
            ok, worst = _close(out, ref)
            print("request", r, "max rel diff alone vs mix", worst, "mean", ref.mean())
            assert ok, f"request {r}: image differs alone vs in the mix (max rel {worst})"
            assert ref.mean() > 0 and np.isfinite(ref).all()
        st = srv.stats()
        assert st["jobs_done"] == 3 * len(reqs) and st["jobs_running"] == 0 and st["jobs_queued"] == 0
        assert st["paths_done"] == sum(2 * w * h * spp for (_, w, h, spp, _) in reqs) + len(reqs) * 64 * 64 * 24
        assert st["rays"] > 0 and st["bytes_in_use"] > 0   # the scenes' pools stay resident


def test_serving_matches_offline_batch(resident):
    """A served job equals hk_render_batch of the same request (same streams)."""
    sds, gss = resident
    s, w, h, spp, seed = 2, 80, 80, 48, 15
    film = torch.zeros(gss[s].film_shape(w, h), dtype=torch.float32, device=DEV)
    gss[s].render_batch([film], spp=spp, depth=sds[s].depth, seeds=[seed], image_indices=[0], sizes=[(w, h)],
                        capacity=1 << 16)
    # resolve on the host: RGB / W of the film interior
    B = gss[s].info.film_border
    f = film.cpu().numpy().astype(np.float64)[B:B + h, B:B + w]
    ref = (f[..., :3] / np.where(f[..., 3:] != 0, f[..., 3:], 1.0)).astype(np.float32)
    with serving.Server(capacity=1 << 16) as srv:
        for g in gss:
            srv.add_scene(g)
        jid, out = srv.submit(s, spp, sds[s].depth, seed, w, h)
        srv.wait(jid, timeout_s=120)
    ok, worst = _close(out, ref)
    print("served vs offline batch: max rel diff", worst)
    assert ok


def test_admission_by_budget_and_cancel(resident):
    sds, gss = resident
    pool = None
    with serving.Server(capacity=1 << 14) as probe:
        probe.add_scene(gss[0])
        jid, _ = probe.submit(0, 4, sds[0].depth, 1, 256, 256)
        probe.wait(jid, timeout_s=60)
        pool = probe.stats()["bytes_in_use"]   # the scene's pool, charged at its first job
    B = gss[0].info.film_border
    job_bytes = (256 + 2 * B) * (256 + 2 * B) * 16 + 256 * 256 * 12
    budget = pool + job_bytes + job_bytes // 2    # room for one 256 x 256 job at a time
    with serving.Server(capacity=1 << 14, hbm_budget=budget) as srv:
        srv.add_scene(gss[0])
        with pytest.raises(hk.HikariError):
            srv.submit(0, 4, sds[0].depth, 1, 2048, 2048)   # film alone exceeds the budget
        ids = [srv.submit(0, 64, sds[0].depth, 30 + k, 256, 256)[0] for k in range(4)]
        victim = srv.submit(0, 64, sds[0].depth, 99, 256, 256)[0]
        srv.cancel(victim)
        peak = 0
        t_end = time.time() + 120
        while time.time() < t_end:
            st = srv.stats()
            peak = max(peak, st["bytes_in_use"])
            if st["jobs_done"] + st["jobs_cancelled"] == 5:
                break
            time.sleep(0.001)
        sts = [srv.wait(i, timeout_s=60) for i in ids]
        assert srv.poll(victim)["state"] == serving.CANCELLED
        assert peak <= budget
        # one job at a time: each admission follows the previous job's end
        for a, b in zip(sts, sts[1:]):
            assert b["admit_s"] >= a["done_s"] - 1e-6
        assert srv.stats()["bytes_in_use"] == pool


def test_cancel_running_job(resident):
    sds, gss = resident
    with serving.Server(capacity=1 << 14) as srv:
        srv.add_scene(gss[2])
        big, _ = srv.submit(0, 4096, sds[2].depth, 5, 256, 256)
        small, out = srv.submit(0, 16, sds[2].depth, 6, 64, 64)
        time.sleep(0.05)
        srv.cancel(big)
        st = srv.wait(big, timeout_s=120)
        assert st["state"] == serving.CANCELLED
        assert srv.wait(small, timeout_s=120)["state"] == serving.DONE
        assert out.mean() > 0
        s = srv.stats()
        assert s["jobs_cancelled"] == 1 and s["jobs_done"] == 1


def test_poisson_driver_reports_percentiles(resident):
    sds, gss = resident
    rng = np.random.default_rng(3)
    with serving.Server(capacity=1 << 16) as srv:
        for g in gss:
            srv.add_scene(g)
        jobs = serving.job_mix(24, 3, rng, [sd.depth for sd in sds], sizes=(64, 128), spps=(4, 16))
        iso = serving.isolated_latencies(srv, jobs)
        res = serving.run_poisson(srv, jobs, rate_hz=200.0, seed=1, isolated=iso)
        summ = res.summary()
        print(summ)
        assert summ["jobs"] == 24 and summ["p50_s"] <= summ["p95_s"] <= summ["p99_s"]
        assert summ["mpaths_per_s"] > 0 and np.all(res.latencies > 0)


def test_progressive_preview(resident):
    """The preview of a running job is its film so far: finite, its finished
    fraction grows, it converges to the final image, and a finished job's
    preview is the final image."""
    sds, gss = resident
    with serving.Server(capacity=1 << 14, iterations_per_poll=2) as srv:
        srv.add_scene(gss[0])
        jid, out = srv.submit(0, 2048, sds[0].depth, 21, 96, 96)
        fracs, imgs = [], []
        t_end = time.time() + 60
        while time.time() < t_end:
            img, frac = srv.preview(jid)
            assert np.isfinite(img).all() and (img >= 0).all()
            fracs.append(frac)
            imgs.append(img)
            if frac >= 1.0 or srv.poll(jid)["state"] == serving.DONE:
                break
            time.sleep(0.02)
        st = srv.wait(jid, timeout_s=120)
        assert st["state"] == serving.DONE
        final, ff = srv.preview(jid)
        assert ff == 1.0 and np.array_equal(final, out)
        print("preview fractions", [round(f, 3) for f in fracs[:10]], "... of", len(fracs))
        assert all(b >= a for a, b in zip(fracs, fracs[1:]))
        mid = [i for i, f in enumerate(fracs) if 0.05 < f < 0.95]
        assert mid, "no preview taken mid-render"
        # work is dispatched tile by tile (all samples of a 16 x 16 tile, then
        # the next): a partial image has finished tiles and empty ones
        m = imgs[mid[len(mid) // 2]]
        cov = m.sum(-1) > 0
        assert 0 < cov.mean() < 1
        assert abs(m[cov].mean() / out[cov].mean() - 1) < 0.1
        victim, _ = srv.submit(0, 4096, sds[0].depth, 22, 96, 96)
        srv.cancel(victim)
        srv.wait(victim, timeout_s=120)
        z, fz = srv.preview(victim)
        assert fz == 0.0 and not z.any()
