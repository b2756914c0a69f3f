"""Serving loop: continuous batching of render jobs (hk_server_* of the C ABI).

A Server keeps scenes resident on the device and renders jobs (scene, image
size, spp, camera) as they arrive; jobs of one scene share that scene's
wavefront path pool, so a job that arrives while others render starts in the
next iteration instead of waiting for them.  The loop itself is native (one
host thread inside the library); this module is the Python face of it plus a
Poisson-arrival load driver that reports p50/p95/p99 job latency.

The reference renders one scene file per process (src/Main.cpp:150-190) and
has no serving loop; the jobs here are its Render() call (src/Main.cpp:46)
with the image size, sample count and camera pose as parameters.
"""
from __future__ import annotations

import ctypes as C
import time
from dataclasses import dataclass, field
from typing import Dict, List, Optional, Sequence

import numpy as np

from . import HikariError, JobStatus, Scene, ServerConfig, ServerStats, check, lib, render_desc

SRPT, FIFO, SRPT_ACROSS, SRPT_SMALL = 0, 1, 2, 3
QUEUED, RUNNING, DONE, CANCELLED, FAILED = 0, 1, 2, 3, 4
HK_ERR_TIMEOUT = -5


def _status_dict(st: JobStatus) -> dict:
    return dict(state=st.state, scene=st.scene, width=st.width, height=st.height, paths=st.paths,
                device_bytes=st.device_bytes, submit_s=st.submit_s, admit_s=st.admit_s, done_s=st.done_s,
                latency_s=st.latency_s)


class Server:
    """hk_server handle.  Output images are host float32 arrays (H x W x 3);
    pass pinned ones (torch.empty(..., pin_memory=True).numpy()) to skip the
    staging copy."""

    def __init__(self, capacity: int = 0, threads_extend: int = 0, threads_shade: int = 0,
                 iterations_per_poll: int = 0, policy: int = SRPT, max_jobs: int = 0, hbm_budget: int = 0,
                 small_work: int = 0):
        cfg = ServerConfig(capacity, threads_extend, threads_shade, iterations_per_poll, policy, max_jobs, hbm_budget,
                           small_work)
        h = C.c_void_p()
        check(lib().hk_server_create(C.byref(cfg), C.byref(h)))
        self.h = h
        self._scenes: List[Scene] = []
        self._outs: Dict[int, np.ndarray] = {}

    def close(self) -> None:
        if self.h:
            check(lib().hk_server_destroy(self.h))
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def add_scene(self, scene: Scene) -> int:
        sid = C.c_int32()
        check(lib().hk_server_add_scene(self.h, scene.h, C.byref(sid)))
        self._scenes.append(scene)
        return sid.value

    def submit(self, scene_id: int, spp: int, depth: int, seed: int = 0, width: int = 0, height: int = 0,
               camera=None, image_index: int = 0, rr_start: int = 0, out: Optional[np.ndarray] = None):
        """Queue a job; returns (job id, output array that receives the image)."""
        sc = self._scenes[scene_id].desc.camera
        w, h = (width or sc.width), (height or sc.height)
        if out is None:
            out = np.empty((h, w, 3), np.float32)
        if out.shape != (h, w, 3) or out.dtype != np.float32 or not out.flags.c_contiguous:
            raise HikariError("output must be a contiguous float32 array of shape (height, width, 3)")
        d = render_desc(spp, depth, seed, 0, rr_start, image_index, 0, camera, width, height)
        jid = C.c_uint64()
        check(lib().hk_job_submit(self.h, scene_id, C.byref(d), out.ctypes.data, C.byref(jid)))
        self._outs[jid.value] = out
        return jid.value, out

    def poll(self, job_id: int) -> dict:
        st = JobStatus()
        check(lib().hk_job_poll(self.h, job_id, C.byref(st)))
        return _status_dict(st)

    def wait(self, job_id: int, timeout_s: float = -1.0) -> dict:
        st = JobStatus()
        rc = lib().hk_job_wait(self.h, job_id, float(timeout_s), C.byref(st))
        if rc == HK_ERR_TIMEOUT:
            raise TimeoutError(f"job {job_id} not finished within {timeout_s} s")
        check(rc)
        self._outs.pop(job_id, None)
        return _status_dict(st)

    def cancel(self, job_id: int) -> None:
        check(lib().hk_job_cancel(self.h, job_id))

    def preview(self, job_id: int, timeout_s: float = 10.0):
        """Progressive preview: (the image accumulated so far, H x W x 3, and
        the fraction of the job's paths finished)."""
        st = self.poll(job_id)
        img = np.empty((st["height"], st["width"], 3), np.float32)
        frac = C.c_double()
        check(lib().hk_job_preview(self.h, job_id, img.ctypes.data, timeout_s, C.byref(frac)))
        return img, frac.value

    def stats(self) -> dict:
        s = ServerStats()
        check(lib().hk_server_get_stats(self.h, C.byref(s)))
        return {k: getattr(s, k) for k, _ in ServerStats._fields_}


# ---------------------------------------------------------------- load driver
@dataclass
class JobSpec:
    scene: int
    width: int
    height: int
    spp: int
    depth: int
    seed: int
    camera: Optional[np.ndarray] = None

    @property
    def paths(self) -> int:
        return self.width * self.height * self.spp


@dataclass
class LoadResult:
    rate_hz: float
    latencies: np.ndarray            # seconds, per job in submission order
    slowdowns: Optional[np.ndarray]  # latency / isolated latency of the same job
    paths: int
    wall_s: float
    stats: dict = field(default_factory=dict)

    def summary(self) -> dict:
        lat = self.latencies
        out = dict(rate_hz=self.rate_hz, jobs=int(lat.size), mpaths_per_s=self.paths / self.wall_s / 1e6,
                   p50_s=float(np.percentile(lat, 50)), p95_s=float(np.percentile(lat, 95)),
                   p99_s=float(np.percentile(lat, 99)), wall_s=self.wall_s)
        if self.slowdowns is not None:
            sd = self.slowdowns
            out.update(slowdown_p50=float(np.percentile(sd, 50)), slowdown_p95=float(np.percentile(sd, 95)),
                       slowdown_p99=float(np.percentile(sd, 99)))
        return out


def job_mix(n: int, n_scenes: int, rng: np.random.Generator, depths: Sequence[int],
            sizes=(256, 512, 1024), spps=(16, 64, 256)) -> List[JobSpec]:
    """n jobs over n_scenes scenes, each with a size from `sizes` (square) and an spp from `spps`."""
    jobs = []
    for k in range(n):
        s = int(rng.integers(n_scenes))
        r = int(sizes[rng.integers(len(sizes))])
        jobs.append(JobSpec(s, r, r, int(spps[rng.integers(len(spps))]), int(depths[s]), 1000 + k))
    return jobs


def isolated_latencies(server: Server, jobs: Sequence[JobSpec]) -> np.ndarray:
    """Latency of each job submitted alone to an idle server."""
    out = np.empty(len(jobs))
    for k, j in enumerate(jobs):
        jid, _ = server.submit(j.scene, j.spp, j.depth, j.seed, j.width, j.height, j.camera)
        out[k] = server.wait(jid)["latency_s"]
    return out


def run_poisson(server: Server, jobs: Sequence[JobSpec], rate_hz: float, seed: int = 0,
                isolated: Optional[np.ndarray] = None, keep=None) -> LoadResult:
    """Submit `jobs` with exponential inter-arrival gaps of mean 1/rate_hz and
    wait for all; the latency of a job runs from its submission to its image
    being in host memory.  keep(job) -> bool selects the jobs whose images are
    returned (LoadResult.images: job index -> image)."""
    rng = np.random.default_rng(seed)
    gaps = rng.exponential(1.0 / rate_hz, len(jobs))
    ids, imgs = [], {}
    t0 = time.perf_counter()
    t_next = t0
    for k, (j, g) in enumerate(zip(jobs, gaps)):
        t_next += g
        while True:
            dt = t_next - time.perf_counter()
            if dt <= 0:
                break
            time.sleep(min(dt, 0.002))
        jid, img = server.submit(j.scene, j.spp, j.depth, j.seed, j.width, j.height, j.camera)
        ids.append(jid)
        if keep is not None and keep(j):
            imgs[k] = img
    lat = np.array([server.wait(i)["latency_s"] for i in ids])
    wall = time.perf_counter() - t0
    paths = sum(j.paths for j in jobs)
    sd = lat / isolated if isolated is not None else None
    res = LoadResult(rate_hz, lat, sd, paths, wall, server.stats())
    res.images = imgs
    return res
