"""Benchmark of the pathMIS core on one B200 node.

A step renders, with the wavefront integrator (--form megakernel: the plain
one-thread-per-path kernel), the heterogeneous scene (64 displaced icospheres with six
material types, 4 area lights and a procedural 2048x1024 sky) from 8 views at
1024x1024 and 128 spp with the reference integrator rule (pathMIS, depth 16,
Russian roulette from depth 0).  Scene and BVH are resident in HBM before the
timed region, as the reference's render timer excludes scene load
(src/Main.cpp:72-123).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                  [--workload heterogeneous|mesh_heavy|cornell|textured] [--spp S] [--views V]

N > 1 runs under torch.distributed (one process per GPU, replicas: every
rank renders its own 8 views, "scaling": "weak").  Rank 0 prints one JSON
line.  --impl reference times the reference renderer itself on the host cores:
its own sources compiled by oracle/ref_build.py (the prebuilt
oracle/_ref/libhikari_ref.so), the scene written as reference XML and read by
its parser, its Render block loop on all host threads, on a bounded block
sample of the same workload.  Where that library is missing, the CPU oracle
(a C restatement) stands in and the line says "kind": "port".
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

FALLBACK_HBM_GBS = 6650.0
# Per-ray figures of the 8-wide traversal kernels from ncu captures of launches
# 2-4 of each kernel (the steady state, a full pool of 2^22 slots) in
# `python -m hikari_b200.profiling render --views 1 --spp 16 --accel bvh8
# --config-json <the tuned configuration>` (the heterogeneous scene), divided by
# the rays those launches traced (hk_wavefront_launch_log): DRAM bytes
# (dram__bytes_read.sum + dram__bytes_write.sum), L2 bytes (lts__t_bytes.sum)
# and warp instructions issued (smsp__inst_executed.sum).  The bench scales them
# by the rays of its own launches.
TRAVERSAL_PER_RAY = {"bvh8": {"extend": {"dram": 231.40, "l2": 964.0, "inst": 343.9},
                              "shadow": {"dram": 114.43, "l2": 798.4, "inst": 241.9}}}
SMS, SCHEDULERS_PER_SM = 148, 4
MEASURED_SM_MAX_MHZ = 1965.0


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="heterogeneous",
                    choices=["heterogeneous", "mesh_heavy", "cornell", "textured", "serving", "bsdf"])
    ap.add_argument("--records", type=int, default=1 << 26, help="bsdf: records per material")
    ap.add_argument("--small-work", type=int, default=0,
                    help="serving, srpt_small: paths left below which a job gates the other scenes (0 = 2^22)")
    ap.add_argument("--material", default="conductor", choices=["conductor", "dielectric", "plastic"],
                    help="mesh_heavy: the icosphere's material (the three runs of the mesh-heavy workload)")
    ap.add_argument("--accel", default="bvh8", choices=["bvh8", "bvh2"],
                    help="tree the kernels traverse: compressed 8-wide (80-byte nodes) or binary (64-byte nodes)")
    ap.add_argument("--jobs", type=int, default=400, help="serving: jobs of the Poisson run")
    ap.add_argument("--load", type=float, default=0.8, help="serving: arrival rate as a fraction of the peak")
    ap.add_argument("--capacity", type=int, default=1 << 19, help="serving: path slots of each scene's pool")
    ap.add_argument("--policy", default="srpt", choices=["srpt", "fifo", "srpt_across", "srpt_small"],
                    help="serving: dispatch policy (SRPT within a scene; srpt_across also gates scenes; srpt_small "
                         "gates them only while a small job renders)")
    ap.add_argument("--spp", type=int, default=0)
    ap.add_argument("--views", type=int, default=0)
    ap.add_argument("--res", type=int, default=0)
    ap.add_argument("--cpu-seconds", type=float, default=15.0)
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline (profiling runs)")
    ap.add_argument("--no-e2e", action="store_true", help="skip the end-to-end pass (profiling runs)")
    ap.add_argument("--no-plain", action="store_true", help="skip the plain-megakernel comparison sample")
    ap.add_argument("--set", action="append", default=[], metavar="KEY=VALUE",
                    help="override one entry of the autotuned wavefront configuration (e.g. sample_major=1)")
    ap.add_argument("--form", default="wavefront", choices=["wavefront", "megakernel"],
                    help="wavefront (the batched form) or the plain one-thread-per-path megakernel")
    return ap.parse_args()


def make_workload(name, spp=0, views=0, res=0, material="conductor"):
    from hikari_b200 import scenes

    if name == "heterogeneous":
        r = res or 1024
        sd = scenes.heterogeneous(width=r, height=r, spp=spp or 128, depth=16)
        cams = scenes.heterogeneous_cameras(views or 8)
        desc = (f"heterogeneous: 64 displaced icospheres (levels 5-7), 6 material types, 4 area lights + "
                f"2048x1024 sky; {len(cams)} views x {r}x{r} x {sd.spp} spp, pathMIS depth 16")
    elif name == "mesh_heavy":
        r = res or 1024
        sd = scenes.mesh_heavy(material, width=r, height=r, spp=spp or 256, depth=16)
        cams = [None] * (views or 1)
        mat = {"conductor": "GGX rough conductor alpha 0.2", "dielectric": "rough dielectric IOR 1.5 alpha 0.1",
               "plastic": "rough plastic alpha 0.15"}[material]
        desc = f"mesh_heavy: displaced level-8 icosphere (1.31M tris), {mat}, sky; {r}x{r} x {sd.spp} spp"
    elif name == "textured":
        r = res or 1024
        sd = scenes.lights_scene(width=r, height=r, spp=spp or 64, depth=12, shading_normals=True, textured=True,
                                 bitmap=True, bump=True)
        cams = [None] * (views or 4)
        desc = (f"textured: ground and five spheres under point, area, constant and directional lights; bitmap "
                f"textures under every filter (EWA with first-hit ray differentials, trilinear, bilinear, nearest), "
                f"procedural textures, a bump-mapped ground, a normal-mapped and a bump-mapped sphere; "
                f"{len(cams)} views x {r}x{r} x {sd.spp} spp, pathMIS depth 12")
    else:
        r = res or 256
        sd = scenes.cornell_box(width=r, height=r, spp=spp or 64)
        cams = [None] * (views or 1)
        desc = f"cornell: Cornell box {r}x{r} x {sd.spp} spp, pathMIS depth {sd.depth}"
    return sd, cams, desc


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms."""

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.lines = []

    def __enter__(self):
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": mx, "reasons": ["unsampled"]}
        load = [x for x in sm if x > 0.5 * max(sm)] or sm
        return {"sm_mhz": float(np.median(load)), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


def slowest_rank_seconds(seconds, device="cuda"):
    """The longest time of any rank (all ranks call this; max all-reduce when
    torch.distributed runs with more than one rank).  Whole-job throughput of
    independent replicas is the units all ranks processed over this time."""
    import torch
    import torch.distributed as dist

    t = torch.tensor([float(seconds)], dtype=torch.float64, device=device)
    if dist.is_available() and dist.is_initialized() and dist.get_world_size() > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def l2_copy_gbs():
    """L2 bandwidth as a plain copy sees it: a 16 MiB float buffer copied into
    another (both L2-resident after the first pass), read + write bytes over
    the best of 20 timed copies."""
    import torch

    a = torch.ones(4 << 20, device="cuda")
    b = torch.empty_like(a)
    for _ in range(5):
        b.copy_(a)
    best = float("inf")
    for _ in range(20):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        b.copy_(a)
        e1.record()
        e1.synchronize()
        best = min(best, e0.elapsed_time(e1) / 1e3)
    return 2 * a.numel() * 4 / best / 1e9


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return FALLBACK_HBM_GBS, "fallback"


class CpuBaseline:
    """The CPU oracle (the reference algorithm restated in C, OpenMP over 32x32
    blocks like src/Main.cpp:121) on the host cores, timed on bounded block
    samples of view 0 of the workload.  The scene and its BVH are built once."""

    def __init__(self, sd, cams, depth):
        from oracle.oracle import OracleScene

        self.nthreads = os.cpu_count() or 1
        if cams and cams[0] is not None:
            sd.camera.to_world = cams[0]
        self.sd, self.depth = sd, depth
        self.o = OracleScene(sd)
        W, H = sd.camera.width, sd.camera.height
        self.nbx = (W + 31) // 32
        self.order = np.random.default_rng(0).permutation(self.nbx * ((H + 31) // 32)).astype(np.int32)
        self.pos = 0
        self.block_s = None

    def _blocks(self, n):
        n = min(n, len(self.order))
        if self.pos + n > len(self.order):
            self.pos = 0
        b = self.order[self.pos:self.pos + n]
        self.pos += n
        return b

    def _render(self, blocks):
        W, H, spp = self.sd.camera.width, self.sd.camera.height, self.sd.spp
        t0 = time.perf_counter()
        _, _, ctr = self.o.render(spp, depth=self.depth, blocks=blocks, nthreads=self.nthreads)
        dt = time.perf_counter() - t0
        paths = sum(min(32, W - 32 * (b % self.nbx)) * min(32, H - 32 * (b // self.nbx)) * spp for b in blocks)
        return paths, dt, ctr

    def sample(self, seconds):
        if self.block_s is None:   # calibrate: one block per thread
            nb = max(1, self.nthreads)
            _, dt, _ = self._render(self._blocks(nb))
            self.block_s = max(dt, 1e-3) / nb
        nb = int(max(4 * self.nthreads, seconds / self.block_s))   # >= 4 blocks per thread: balanced threads
        blocks = self._blocks(nb)
        paths, dt, ctr = self._render(blocks)
        return {"value": paths / dt / 1e6, "unit": "Mpaths/s", "cores": self.nthreads, "kind": "port",
                "sample": f"{len(blocks)} blocks of 32x32 px x {self.sd.spp} spp of view 0 ({paths} paths, {dt:.1f} s)",
                "mrays_per_s": float(ctr[1] + ctr[2]) / dt / 1e6}


class RefBaseline(CpuBaseline):
    """The reference renderer compiled from its own sources
    (oracle/_ref/libhikari_ref.so): the workload's view 0 written as reference
    XML (hlbvh accelerator, leafSize 10) and loaded by its LoadFromXML, then
    its Render block loop (src/Main.cpp:46-147, driven headless by
    oracle/ref_shim/ref_render.cpp) on all host threads over bounded block
    samples.  Only the block loop is timed, as the reference's own render
    timer does; the scene export and load are reported beside it."""

    def __init__(self, sd, cams, depth):
        import tempfile

        from hikari_b200.scenexml import write_scene_xml
        from oracle import reference

        self.nthreads = os.cpu_count() or 1
        if cams and cams[0] is not None:
            sd.camera.to_world = cams[0]
        sd.depth = depth
        self.sd, self.depth = sd, depth
        t0 = time.perf_counter()
        xml = write_scene_xml(sd, tempfile.mkdtemp(prefix="hk_ref_scene_"), "scene", spp=sd.spp, accel="hlbvh")
        t1 = time.perf_counter()
        self.rs = reference.RefScene(xml)
        self.setup = {"xml_write_s": round(t1 - t0, 2), "parse_and_hlbvh_build_s": round(time.perf_counter() - t1, 2)}
        W, H = sd.camera.width, sd.camera.height
        self.nbx = (W + 31) // 32
        self.order = np.random.default_rng(0).permutation(self.nbx * ((H + 31) // 32)).astype(np.int32)
        self.pos = 0
        self.block_s = None

    def _render(self, blocks):
        W, H, spp = self.sd.camera.width, self.sd.camera.height, self.sd.spp
        _, dt = self.rs.render(nthreads=self.nthreads, blocks=blocks)
        paths = sum(min(32, W - 32 * (b % self.nbx)) * min(32, H - 32 * (b // self.nbx)) * spp for b in blocks)
        return paths, dt, None

    def sample(self, seconds):
        if self.block_s is None:   # calibrate: one block per thread
            nb = max(1, self.nthreads)
            _, dt, _ = self._render(self._blocks(nb))
            self.block_s = max(dt, 1e-3) / nb
        nb = int(max(2 * self.nthreads, seconds / self.block_s))
        blocks = self._blocks(nb)
        paths, dt, _ = self._render(blocks)
        return {"value": paths / dt / 1e6, "unit": "Mpaths/s", "cores": self.nthreads, "kind": "reference",
                "sample": (f"{len(blocks)} blocks of 32x32 px x {self.sd.spp} spp of view 0 ({paths} paths, "
                           f"{dt:.1f} s): the reference's Render block loop built from its sources, hlbvh"),
                "setup": self.setup}


def cpu_baseline(sd, cams, depth):
    """The reference renderer where its prebuilt library is present, else the
    CPU oracle (kind "port")."""
    try:
        return RefBaseline(sd, cams, depth)
    except Exception as e:   # library missing: the restatement stands in
        print(f"reference renderer unavailable ({e}); timing the C port", file=sys.stderr)
        return CpuBaseline(sd, cams, depth)


def run_reference(args, rank, world):
    if rank != 0:
        return
    sd, cams, desc = make_workload(args.workload, args.spp, args.views, args.res, args.material)
    cb = cpu_baseline(sd, cams, sd.depth)
    vals = [cb.sample(max(3.0, args.cpu_seconds / 3)) for _ in range(args.warmup + args.steps)]
    v = vals[args.warmup:]
    value = float(np.mean([x["value"] for x in v]))
    kind = v[0]["kind"]
    line = {"metric": "Mpaths/s", "value": value, "unit": "Mpaths/s", "impl": "reference", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded procedural scene)",
            "config": {"workload": desc,
                       "parallelism": ("host threads over 32x32 blocks (the reference's Render loop)"
                                       if kind == "reference" else "host threads (OpenMP over 32x32 blocks)")},
            "cpu_baseline": {"value": value, "unit": "Mpaths/s", "cores": v[0]["cores"], "kind": kind,
                             "sample": v[0]["sample"]},
            "e2e": {"value": value, "unit": "Mpaths/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    if "setup" in v[0]:
        line["config"]["reference_setup"] = v[0]["setup"]
    print(json.dumps(line), flush=True)


def serving_scenes():
    """The serving set of config 5: the Cornell box (config 1), the mesh-heavy
    icosphere (config 3, 1.31M triangles), the heterogeneous scene (config 4,
    4.75M) and five seeded variants of it spanning about 10k to 3M triangles."""
    from hikari_b200 import scenes

    sds = [scenes.cornell_box(width=256, height=256, spp=64),
           scenes.mesh_heavy("conductor", width=1024, height=1024, spp=256, depth=16),
           scenes.heterogeneous(width=1024, height=1024, spp=128, depth=16)]
    variants = [(2, (4,), (1.0,)), (4, (5,), (1.0,)), (12, (5, 6), (0.5, 0.5)), (24, (6, 7), (0.5, 0.5)),
                (40, (5, 6, 7), (0.55, 0.30, 0.15))]
    for k, (n, lv, lp) in enumerate(variants):
        sds.append(scenes.heterogeneous(width=1024, height=1024, spp=128, depth=16, n_spheres=n, levels=lv,
                                        level_p=lp, seed=k + 1))
    return sds


def run_serving(args):
    """Serving: a Poisson stream of jobs over 8 resident scenes, each job a
    square image of 256, 512 or 1024 pixels at 16, 64 or 256 spp.  Measures
    the peak sustainable throughput (all jobs submitted at once), each job's
    latency alone on the idle server, and the latencies of a Poisson run at
    --load x the peak arrival rate."""
    import torch

    import hikari_b200 as hk
    from hikari_b200 import serving

    torch.cuda.set_device(0)
    t0 = time.perf_counter()
    sds = serving_scenes()
    gss = [hk.Scene.from_desc(sd) for sd in sds]
    build_s = time.perf_counter() - t0
    # each scene's traversal settings, which the server's engines take (untimed)
    t1 = time.perf_counter()
    for g, sd in zip(gss, sds):
        g.autotune(4, sd.depth)
    tune_s = time.perf_counter() - t1
    tris = [int(g.info.n_triangles) for g in gss]
    rng = np.random.default_rng(7)
    depths = [sd.depth for sd in sds]
    policy = {"srpt": serving.SRPT, "fifo": serving.FIFO, "srpt_across": serving.SRPT_ACROSS,
              "srpt_small": serving.SRPT_SMALL}[args.policy]
    with serving.Server(capacity=args.capacity, iterations_per_poll=4, policy=policy, small_work=args.small_work) as srv:
        for g in gss:
            srv.add_scene(g)
        for k in range(len(gss)):   # engines and graphs of every scene (untimed)
            srv.wait(srv.submit(k, 4, depths[k], 1, 64, 64)[0])
        # peak: a burst of jobs submitted at once
        burst = serving.job_mix(max(16, args.jobs // 2), len(gss), rng, depths)
        t = time.perf_counter()
        ids = [srv.submit(j.scene, j.spp, j.depth, j.seed, j.width, j.height)[0] for j in burst]
        for i in ids:
            srv.wait(i)
        makespan = time.perf_counter() - t
        peak_mpaths = sum(j.paths for j in burst) / makespan / 1e6
        jobs = serving.job_mix(args.jobs, len(gss), rng, depths)
        mean_paths = float(np.mean([j.paths for j in jobs]))
        peak_rate = peak_mpaths * 1e6 / mean_paths
        iso = serving.isolated_latencies(srv, jobs)
        rate = args.load * peak_rate
        res = serving.run_poisson(srv, jobs, rate, seed=11, isolated=iso, keep=lambda j: j.width == 256)
        summ = res.summary()
        st = srv.stats()
    # RMSE of the 256 x 256 jobs rendered in the mix against each scene's
    # reference image (the same scene and view at 256 x 256, 4096 spp)
    rmse = {}
    refs = {}
    for k, img in res.images.items():
        j = jobs[k]
        if j.scene not in refs:
            f = torch.zeros(gss[j.scene].film_shape(256, 256), dtype=torch.float32, device="cuda")
            gss[j.scene].render_batch([f], spp=4096, depth=j.depth, seeds=[424242], image_indices=[0],
                                      sizes=[(256, 256)])
            B = int(gss[j.scene].info.film_border)
            c = f.cpu().numpy().astype(np.float64)[B:B + 256, B:B + 256]
            refs[j.scene] = np.where(c[..., 3:] != 0, c[..., :3] / np.where(c[..., 3:] != 0, c[..., 3:], 1), 0)
        ref = refs[j.scene]
        rel = float(np.sqrt(np.mean((img.astype(np.float64) - ref) ** 2)) / max(np.mean(np.abs(ref)), 1e-12))
        rmse.setdefault(j.spp, []).append(rel)
    rmse_summary = {str(sp): {"jobs": len(v), "relative_rmse_mean": float(np.mean(v))} for sp, v in sorted(rmse.items())}
    line = {
        "metric": "Mpaths/s", "value": summ["mpaths_per_s"], "unit": "Mpaths/s", "n_gpus": 1, "steps": 1,
        "warmup": 1, "ms_per_step": summ["wall_s"] * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded procedural scenes)",
        "config": {"workload": "serving: Poisson arrivals over 8 resident scenes (Cornell box, mesh-heavy 1.31M tris, "
                               "heterogeneous 4.75M tris, 5 heterogeneous variants); jobs of 256/512/1024 px "
                               "square at 16/64/256 spp",
                   "form": f"wavefront serving loop (continuous batching, {args.policy} dispatch)", "triangles": tris,
                   "scene_build_s": round(build_s, 2), "autotune_s": round(tune_s, 2),
                   "traversal": "each scene's autotuned fetch intervals, register budgets and triangle-test modes",
                   "capacity": args.capacity, "jobs": args.jobs, "small_work": args.small_work or (1 << 22),
                   "load": args.load},
        "serving": {
            "peak_mpaths_per_s": peak_mpaths, "peak_rate_hz": peak_rate, "arrival_rate_hz": rate,
            "mean_job_paths": mean_paths,
            "latency_s": {"p50": summ["p50_s"], "p95": summ["p95_s"], "p99": summ["p99_s"]},
            "isolated_latency_s": {"p50": float(np.percentile(iso, 50)), "p95": float(np.percentile(iso, 95)),
                                   "p99": float(np.percentile(iso, 99))},
            "p99_over_isolated_p99": summ["p99_s"] / float(np.percentile(iso, 99)),
            "slowdown": {"p50": summ["slowdown_p50"], "p95": summ["slowdown_p95"], "p99": summ["slowdown_p99"]},
            "rmse_256px_jobs_vs_4096spp_reference": rmse_summary,
            "rays": int(st["rays"]), "shadow_rays": int(st["shadow_rays"]),
        },
    }
    print(json.dumps(line), flush=True)


BSDF_RECORD_BYTES = 84   # in: wi 12 + u2 8 + u1 4 + wo 12; out: sample wo 12 + weight 12 + pdf 4 + measure 4,
                         # eval 12, pdf 4


def bsdf_records_dev(n, seed, device="cuda"):
    """BSDF-batch records (SURVEY config 2): wi uniform on the upper
    hemisphere, u2 and u1 uniform in [0,1), wo cosine-distributed."""
    import torch

    g = torch.Generator(device=device)
    g.manual_seed(seed)
    z = torch.rand(n, generator=g, device=device)
    ph = torch.rand(n, generator=g, device=device) * (2 * np.pi)
    s = torch.sqrt(torch.clamp(1 - z * z, min=0))
    wi = torch.stack([s * torch.cos(ph), s * torch.sin(ph), z], 1).contiguous()
    u2 = torch.rand((n, 2), generator=g, device=device)
    u1 = torch.rand(n, generator=g, device=device)
    z2 = torch.sqrt(torch.rand(n, generator=g, device=device))
    ph2 = torch.rand(n, generator=g, device=device) * (2 * np.pi)
    s2 = torch.sqrt(torch.clamp(1 - z2 * z2, min=0))
    wo = torch.stack([s2 * torch.cos(ph2), s2 * torch.sin(ph2), z2], 1).contiguous()
    return wi, u2, u1, wo


def run_bsdf(args):
    """BSDF batch (SURVEY config 2): Sample, Eval and Pdf of every record for
    each of the 33 materials (Beckmann/GGX rough conductors in Cu and Au and
    rough dielectrics over the alpha grid, rough plastics, a coated
    conductor).  A step is one pass over every material; records stay resident
    in HBM (5.6 GB per material pass at 2^26, far above L2)."""
    import torch

    import hikari_b200 as hk
    from hikari_b200 import scenes

    torch.cuda.set_device(0)
    mats = scenes.config2_materials()
    sd = scenes.bsdf_scene(mats)
    gs = hk.Scene.from_desc(sd)
    n = args.records
    wi, u2, u1, wo = bsdf_records_dev(n, 7)
    out = dict(s_wo=torch.empty((n, 3), device="cuda"), s_w=torch.empty((n, 3), device="cuda"),
               s_pdf=torch.empty(n, device="cuda"), s_m=torch.empty(n, dtype=torch.int32, device="cuda"),
               e_rgb=torch.empty((n, 3), device="cuda"), p_pdf=torch.empty(n, device="cuda"))
    ids = [gs.bsdf_ids[id(d)] for _, d in mats]
    L = hk.lib()
    stream = torch.cuda.current_stream()
    P = hk._p

    def batch(bid):
        # uv, duv: no texture coordinates (the config-2 materials are untextured)
        hk.check(L.hk_bsdf_batch(gs.h, bid, n, P(wi), P(u2), P(u1), P(wo), None, None, P(out["s_wo"]), P(out["s_w"]),
                                 P(out["s_pdf"]), P(out["s_m"]), P(out["e_rgb"]), P(out["p_pdf"]), stream.cuda_stream))

    for _ in range(args.warmup):
        for b in ids:
            batch(b)
    torch.cuda.synchronize()
    per_mat = np.zeros(len(ids))
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in ids]
    with ClockSampler(0) as clk:
        for _ in range(args.steps):
            for k, b in enumerate(ids):
                evs[k][0].record(stream)
                batch(b)
                evs[k][1].record(stream)
            torch.cuda.synchronize()
            per_mat += [a.elapsed_time(e) for a, e in evs]
    total_s = per_mat.sum() / 1e3
    recs = float(n) * len(ids) * args.steps
    hbm, peak_kind = measured_peaks()
    achieved = recs * BSDF_RECORD_BYTES / total_s / 1e9
    slowest = int(np.argmax(per_mat))
    # CPU baseline: the oracle's batch (OpenMP, all host threads) on 2^20 records of every material
    cpu = None
    if not args.no_cpu:
        from oracle.oracle import OracleScene

        os_ = OracleScene(sd)
        m = 1 << 20
        wic, u2c, u1c, woc = (t[:m].cpu().numpy() for t in (wi, u2, u1, wo))
        t0 = time.perf_counter()
        for _, d in mats:
            os_.bsdf_batch(os_.bsdf_ids[id(d)], wic, u2c, u1c, woc)
        dt = time.perf_counter() - t0
        cpu = {"value": m * len(mats) / dt / 1e6, "unit": "Mrecords/s", "cores": os.cpu_count(), "kind": "port",
               "sample": f"2^20 records of each of the {len(mats)} materials ({dt:.1f} s)"}
    line = {
        "metric": "Mrecords/s", "value": recs / total_s / 1e6, "unit": "Mrecords/s", "n_gpus": 1,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": per_mat.sum() / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded records)",
        "config": {"workload": f"bsdf batch: {n} records x {len(ids)} materials, Sample + Eval + Pdf per record",
                   "l2": "records (5.6 GB per material at 2^26) far larger than L2"},
        "per_material_mrecords_s": {name: n * args.steps / (ms / 1e3) / 1e6 for (name, _), ms in zip(mats, per_mat)},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s", "frac": achieved / hbm,
                     "traffic": None, "peak_kind": peak_kind,
                     "basis": f"{BSDF_RECORD_BYTES} B of records in and out per record over the batch kernel time; "
                              f"slowest material {mats[slowest][0]}"},
        "cpu_baseline": cpu,
        "e2e": {"value": None, "unit": "Mrecords/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "gpu_launches": len(ids) * args.steps,
        "clocks": clk.summary(),
    }
    print(json.dumps(line), flush=True)


def main():
    args = parse()
    if args.workload == "bsdf":
        if args.impl == "reference":
            print(json.dumps({"impl": "reference", "unavailable": "the BSDF batch has no separate reference arm; "
                                                                    "its CPU baseline is in the line"}), flush=True)
        elif int(os.environ.get("RANK", "0")) == 0:
            run_bsdf(args)
        return
    if args.workload == "serving":
        if args.impl == "reference":
            print(json.dumps({"impl": "reference", "unavailable": "the reference has no serving loop"}), flush=True)
        elif int(os.environ.get("RANK", "0")) == 0:
            run_serving(args)
        return
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference(args, rank, world)
        return
    import torch
    import torch.distributed as dist

    import hikari_b200 as hk

    torch.cuda.set_device(local)
    if world > 1:
        os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
        from datetime import timedelta

        dist.init_process_group("nccl", timeout=timedelta(seconds=300))

    def barrier():
        if world > 1:
            dist.barrier()

    sd, cams, desc = make_workload(args.workload, args.spp, args.views, args.res, args.material)
    t0 = time.perf_counter()
    gs = hk.Scene.from_desc(sd)
    build_s = time.perf_counter() - t0
    tree_s = {"host": round(gs.tree_build_seconds(), 4)}
    if rank == 0:   # the device builder on the same scene (untimed set-up; the second build is reported)
        for _ in range(2):
            g2 = hk.Scene.from_desc(sd, builder=hk.BUILDER_GPU)
            tree_s["device"] = round(g2.tree_build_seconds(), 4)
            tree_s["device_wide_nodes"] = int(g2.info.n_wide_nodes)
            del g2
        torch.cuda.synchronize()
    gs.set_accel(hk.ACCEL_BVH8 if args.accel == "bvh8" else hk.ACCEL_BVH2)
    accel_name = args.accel
    node_b = 80.0 if args.accel == "bvh8" else 64.0
    W, H, spp, depth = sd.camera.width, sd.camera.height, sd.spp, sd.depth
    V = len(cams)
    shape = gs.film_shape()
    films = [torch.zeros(shape, dtype=torch.float32, device="cuda") for _ in range(V)]
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device="cuda")   # 256 MiB > 126 MB L2
    stream = torch.cuda.current_stream()
    wave = args.form == "wavefront"
    n_ctr = 7 if wave else 5
    counters = torch.zeros(n_ctr, dtype=torch.int64, device="cuda")
    cam_list = [c for c in cams] if cams[0] is not None else None
    tuned, tune_ms = {}, None
    if wave:
        tuned, tune_ms = gs.autotune(min(32, spp), depth, camera=cams[0])   # untimed set-up
        for kv in args.set:
            k, v = kv.split("=", 1)
            if k not in tuned:
                raise SystemExit(f"--set: unknown configuration key {k}")
            tuned[k] = int(v)

    def step(it, ctr=None, **extra):
        for f in films:
            f.zero_()
        if wave:
            gs.render_batch(films, spp=spp, depth=depth, seeds=[77 + 1000 * it + v for v in range(V)], cameras=cam_list,
                            image_indices=[rank * V + v for v in range(V)], counters=ctr, **tuned, **extra)
        else:
            for v, cam in enumerate(cams):
                gs.render(films[v], spp=spp, depth=depth, seed=77 + 1000 * it + v, image_index=rank * V + v,
                          counters=ctr, camera=cam)

    for w in range(args.warmup):
        step(10_000 + w)
    torch.cuda.synchronize()
    barrier()
    counters.zero_()
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    with ClockSampler(local) as clk:
        barrier()
        torch.cuda.synchronize()
        for k in range(args.steps):
            flush.fill_(float(k))   # write 256 MiB: evict L2 between steps (outside the step events)
            evs[k][0].record(stream)
            step(k, counters)
            evs[k][1].record(stream)
        torch.cuda.synchronize()
        barrier()
    step_ms = [a.elapsed_time(b) for a, b in evs]
    total_s = sum(step_ms) / 1e3
    total_max = slowest_rank_seconds(total_s)
    ctr = counters.cpu().numpy().astype(np.float64)
    paths_rank = float(W * H * spp * V * args.steps)
    value = world * paths_rank / total_max / 1e6
    rays = ctr[0] + ctr[1]
    mrays = world * rays / total_max / 1e6
    hbm, peak_kind = measured_peaks()

    # roofline of the dominant kernel, timed live with CUDA events on the launching stream
    if wave:
        kms = np.zeros(4, np.float32)
        kl = np.zeros(4, np.int32)
        pc = torch.zeros(7, dtype=torch.int64, device="cuda")
        step(99_999, pc, kernel_ms=kms, kernel_launches=kl)
        torch.cuda.synchronize()
        pcn = pc.cpu().numpy().astype(np.float64)
        phases = ["regen", "extend", "shade", "shadow"]
        dom = int(np.argmax(kms))
        trav_bytes = {1: pcn[3] * node_b + pcn[4] * 48.0, 3: pcn[5] * node_b + pcn[6] * 48.0}
        traffic = None
        per_ray = TRAVERSAL_PER_RAY.get(args.accel, {}).get({1: "extend", 3: "shadow"}.get(dom, ""), {})
        dom_rays = pcn[0] if dom == 1 else pcn[1]
        if per_ray.get("dram") is not None:
            traffic = per_ray["dram"] * dom_rays / max(1, kl[dom])
        if dom in trav_bytes:
            bytes_per_launch = trav_bytes[dom] / max(1, kl[dom])
            avg_s = float(kms[dom]) / max(1, kl[dom]) / 1e3
            basis = (f"{phases[dom]} kernel: BVH fetch bytes ({int(node_b)} B per {accel_name} node visit + 48 B per "
                     f"triangle test, counted in the kernel) per launch / mean launch time over {int(kl[dom])} launches "
                     f"of a profiled step")
        else:
            # shading: path-state bytes read + written per path vertex (~144 B) as the algorithmic unit
            bytes_per_launch = (pcn[0] * 144.0) / max(1, kl[dom])
            avg_s = float(kms[dom]) / max(1, kl[dom]) / 1e3
            basis = f"{phases[dom]} kernels: path-state bytes (144 B per shaded vertex) per launch"
        achieved = bytes_per_launch / max(avg_s, 1e-12) / 1e9
        # the traversal kernels are bound by instruction issue and SIMT
        # divergence, not by DRAM: their issue rate against one warp
        # instruction per scheduler per cycle, and their L2 bytes against an
        # L2-resident copy measured here
        l2_peak = l2_copy_gbs()
        limiter = {"bound": "hbm"}
        if per_ray.get("inst") is not None:
            dom_s = float(kms[dom]) / 1e3
            issue_rate = per_ray["inst"] * dom_rays / max(dom_s, 1e-12)
            limiter = {"bound": "issue", "issue": {"achieved_ginst_per_s": issue_rate / 1e9,
                                                   "inst_per_ray": per_ray["inst"], "sms": SMS,
                                                   "schedulers_per_sm": SCHEDULERS_PER_SM}}
        if per_ray.get("l2") is not None:
            l2_ach = per_ray["l2"] * dom_rays / max(float(kms[dom]) / 1e3, 1e-12) / 1e9
            limiter["l2"] = {"achieved": l2_ach, "peak": l2_peak, "unit": "GB/s", "frac": l2_ach / l2_peak,
                             "peak_kind": "measured here: L2-resident copy, 2 x 16 MiB, read + write bytes"}
        sm_mhz = clk.summary().get("sm_mhz") or MEASURED_SM_MAX_MHZ
        if "issue" in limiter:
            peak_ginst = SMS * SCHEDULERS_PER_SM * sm_mhz * 1e6 / 1e9
            limiter["issue"].update({"peak_ginst_per_s": peak_ginst, "sm_mhz": sm_mhz,
                                     "frac": limiter["issue"]["achieved_ginst_per_s"] / peak_ginst})
        launches_per_step = int(kl.sum()) + 1
        rays_c, rays_s = max(pcn[0], 1.0), max(pcn[1], 1.0)
        traversal = {"closest": {"node_visits_per_ray": pcn[3] / rays_c, "tri_tests_per_ray": pcn[4] / rays_c,
                                 "ns_per_ray": float(kms[1]) * 1e6 / rays_c},
                     "shadow": {"node_visits_per_ray": pcn[5] / rays_s, "tri_tests_per_ray": pcn[6] / rays_s,
                                "ns_per_ray": float(kms[3]) * 1e6 / rays_s},
                     "node_bytes": node_b, "tri_bytes": 48}
        phase_share = {p: round(float(kms[i] / kms.sum()), 4) for i, p in enumerate(phases)}
    else:
        n_launch = args.steps * V
        bytes_per_launch = (ctr[3] * node_b + ctr[4] * 48.0) / n_launch
        achieved = bytes_per_launch / (total_max / n_launch) / 1e9
        basis = (f"render megakernel: BVH fetch bytes ({int(node_b)} B per {accel_name} node visit + 48 B per triangle "
                 f"test) / mean kernel time")
        launches_per_step = V
        phase_share = None
        traversal = None
        traffic = None
        limiter = {"bound": "hbm"}

    # end to end through the C ABI: host images out, per-view camera pose in
    e2e_value = None
    if not args.no_e2e:
        outs = [np.empty((H, W, 3), np.float32) for _ in range(V)]
        def e2e_call():
            if wave:
                gs.render_batch_host(outs, spp, depth, seeds=[5000 + v for v in range(V)], cameras=cam_list,
                                     image_indices=[rank * V + v for v in range(V)], **tuned)
            else:
                for v, cam in enumerate(cams):
                    gs.render_image(spp, depth, seed=5000 + v, out=outs[v], camera=cam, image_index=rank * V + v)

        e2e_call()   # untimed: the first call allocates the library's host-output films
        torch.cuda.synchronize()
        barrier()
        # device time on the calling stream: the host-to-device pose/desc
        # upload, the render, the resolve and the device-to-host image copies
        # of every view are all ordered on it
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        e2e_call()
        e1.record(stream)
        torch.cuda.synchronize()
        e2e_s = e0.elapsed_time(e1) / 1e3
        e2e_value = world * W * H * spp * V / slowest_rank_seconds(e2e_s) / 1e6

    # the plain megakernel on a short sample of the same scene, for comparison
    plain = None
    if wave and not args.no_plain and rank == 0:
        ps = max(1, min(16, spp))
        f = films[0]
        f.zero_()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        gs.render(f, spp=ps, depth=depth, seed=3, camera=cams[0])
        torch.cuda.synchronize()
        e0.record(stream)
        gs.render(f, spp=ps, depth=depth, seed=4, camera=cams[0])
        e1.record(stream)
        torch.cuda.synchronize()
        plain = {"mpaths_per_s": W * H * ps / (e0.elapsed_time(e1) / 1e3) / 1e6,
                 "sample": f"view 0, {W}x{H} x {ps} spp, render_pathmis_kernel"}
    # the drop-in call a pathMISCuda plugin's RenderImage makes (hk_render_image:
    # host image out, the wavefront at this size with the autotuned configuration)
    drop_in = None
    if wave and rank == 0:
        gs.set_wavefront_config(tuned)
        img = np.empty((H, W, 3), np.float32)
        gs.render_image(spp, depth, seed=6, out=img, camera=cams[0])   # untimed: first call allocates the film
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        gs.render_image(spp, depth, seed=7, out=img, camera=cams[0])
        dt = time.perf_counter() - t0
        drop_in = {"mpaths_per_s": W * H * spp / dt / 1e6,
                   "sample": f"hk_render_image, view 0, {W}x{H} x {spp} spp, host image out, wall clock"}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        try:
            cpu = cpu_baseline(sd, cams, depth).sample(args.cpu_seconds)
            if cpu["kind"] == "reference":   # the C restatement's number beside the reference's
                port = CpuBaseline(sd, cams, depth).sample(args.cpu_seconds / 2)
                cpu["port"] = {k: port[k] for k in ("value", "unit", "cores", "sample")}
        except Exception as e:  # the baseline is reported, never the target
            cpu = {"value": None, "unit": "Mpaths/s", "cores": os.cpu_count(), "kind": "reference",
                   "sample": f"failed: {e}"}
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return
    line = {
        "metric": "Mpaths/s",
        "value": value,
        "unit": "Mpaths/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": total_max * 1e3 / args.steps,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f32",
        "data": "synthetic (seeded procedural scene)",
        "config": {"workload": desc, "form": args.form, "parallelism": f"replicas x{world}",
                   "triangles": int(gs.info.n_triangles), "accel": args.accel,
                   "bvh_nodes": int(gs.info.n_bvh_nodes), "wide_nodes": int(gs.info.n_wide_nodes),
                   "wide_depth": int(gs.info.wide_depth),
                   "scene_build_s": round(build_s, 2), "tree_build_s": tree_s, "wavefront": tuned or None,
                   "autotune_probe_ms": tune_ms,
                   "l2": "256 MiB buffer written between timed steps (outside the step events)",
                   "rr": "reference rule: p=0.95 at every bounce"},
        "mrays_per_s": mrays,
        "rays_per_path": rays / paths_rank,
        "phase_share": phase_share,
        "traversal": traversal,
        "plain_megakernel": plain,
        "drop_in_render_image": drop_in,
        "roofline": {"bound": limiter["bound"], "achieved": achieved, "peak": hbm, "unit": "GB/s",
                     "frac": achieved / hbm, "traffic": traffic, "peak_kind": peak_kind, "basis": basis,
                     "traffic_basis": ("DRAM bytes per ray from an ncu capture of three steady-state launches of the "
                                       "1-view 16-spp case, scaled by the rays per launch"
                                       if traffic is not None else None),
                     **{k: v for k, v in limiter.items() if k != "bound"}},
        "cpu_baseline": cpu,
        "e2e": {"value": e2e_value, "unit": "Mpaths/s", "h2d_bytes_per_step": V * int(hk.C.sizeof(hk.RenderDesc)),
                "d2h_bytes_per_step": V * W * H * 3 * 4},
        "gpu_launches": launches_per_step * args.steps,
        "clocks": clk.summary(),
    }
    print(json.dumps(line), flush=True)


if __name__ == "__main__":
    main()
