"""Summarise ncu output for profiles/: a launch list (`--metrics
gpu__time_duration.sum --csv`) into per-kernel launches / total / share, and
selected raw metrics of a `--set full` report (`ncu -i X --page raw --csv`).

usage: python -m hikari_b200.profiling launches <launches.csv>
       python -m hikari_b200.profiling raw <report.ncu-rep> [regex]
       python -m hikari_b200.profiling render [--workload heterogeneous|textured] [--views V] [--spp S] [--accel bvh2|bvh8] [--out F]
                                              [--threads-extend T] [--threads-shade T] [--fetch-steps K]
                                              [--fetch-min-idle K] [--shadow-tests M] [--closest-tests M]
       python -m hikari_b200.profiling traffic <metrics.csv> <render.json> [skip]

`render` renders the heterogeneous scene once with the wavefront integrator
(no autotuning, no other launches of the traversal kernels; the launch
configuration is given on the command line, e.g. the one bench.py's
autotuner picked) and writes its counters and the rays of every traversal
launch as JSON; run under `ncu --metrics dram__bytes_read.sum,
dram__bytes_write.sum,lts__t_bytes.sum,smsp__inst_executed.sum,
smsp__thread_inst_executed.sum,gpu__time_duration.sum -k regex:wf_shadow
-s <skip> -c 3 --cache-control none`, `traffic` turns the captured launches'
sums into DRAM bytes, L2 bytes and warp instructions per ray of that kernel.
"""
import csv
import io
import re
import subprocess
import sys

UNIT_MS = {"ns": 1e-6, "nsecond": 1e-6, "us": 1e-3, "usecond": 1e-3, "ms": 1.0, "msecond": 1.0, "s": 1e3, "second": 1e3}

RAW = ["gpu__time_duration.sum", "dram__bytes_read.sum", "dram__bytes_write.sum",
       "gpu__dram_throughput.avg.pct_of_peak_sustained_elapsed", "sm__throughput.avg.pct_of_peak_sustained_elapsed",
       "sm__warps_active.avg.pct_of_peak_sustained_active", "launch__registers_per_thread",
       "smsp__thread_inst_executed_per_inst_executed.ratio", "smsp__issue_active.avg.pct_of_peak_sustained_active",
       "l1tex__t_sector_hit_rate.pct", "lts__t_sector_hit_rate.pct",
       "l1tex__t_sectors_pipe_lsu_mem_global_op_ld.sum", "l1tex__t_sectors_pipe_lsu_mem_local_op_ld.sum",
       "smsp__average_warps_issue_stalled_long_scoreboard_per_issue_active.ratio",
       "smsp__average_warps_issue_stalled_barrier_per_issue_active.ratio",
       "smsp__average_warps_issue_stalled_no_instruction_per_issue_active.ratio",
       "smsp__average_warps_issue_stalled_wait_per_issue_active.ratio",
       "smsp__average_warps_issue_stalled_short_scoreboard_per_issue_active.ratio",
       "sm__pipe_tensor_cycles_active.avg.pct_of_peak_sustained_active"]


def launches(path):
    text = open(path).read()
    lines = [ln for ln in text.splitlines() if ln.startswith('"')]
    rows = list(csv.reader(io.StringIO("\n".join(lines))))
    hdr, data = rows[0], rows[1:]
    ki, vi, ui = hdr.index("Kernel Name"), hdr.index("Metric Value"), hdr.index("Metric Unit")
    agg = {}
    for r in data:
        name = r[ki].split("(")[0]
        ms = float(r[vi].replace(",", "")) * UNIT_MS[r[ui]]
        a = agg.setdefault(name, [0, 0.0])
        a[0] += 1
        a[1] += ms
    tot = sum(a[1] for a in agg.values())
    out = ["| kernel | launches | total ms | share |", "|---|---|---|---|"]
    for k, (n, ms) in sorted(agg.items(), key=lambda x: -x[1][1]):
        out.append(f"| {k} | {n} | {ms:.3f} | {100 * ms / tot:.2f}% |")
    return "\n".join(out)


def raw(report, regex=None):
    txt = subprocess.run(["ncu", "-i", report, "--page", "raw", "--csv"], capture_output=True, text=True).stdout
    rows = list(csv.reader(io.StringIO(txt)))
    hdr, units, data = rows[0], rows[1], rows[2:]
    ki = hdr.index("Kernel Name")
    out = []
    for r in data:
        if regex and not re.search(regex, r[ki]):
            continue
        out.append(f"### {r[ki].split('(')[0]}")
        out.append("| metric | unit | value |")
        out.append("|---|---|---|")
        for m in RAW:
            if m in hdr:
                i = hdr.index(m)
                out.append(f"| {m} | {units[i]} | {r[i]} |")
    return "\n".join(out)


def _metric_rows(path):
    text = open(path).read()
    lines = [ln for ln in text.splitlines() if ln.startswith('"')]
    rows = list(csv.reader(io.StringIO("\n".join(lines))))
    hdr, data = rows[0], rows[1:]
    ki, ni, vi, ui = hdr.index("Kernel Name"), hdr.index("Metric Name"), hdr.index("Metric Value"), hdr.index("Metric Unit")
    ii = hdr.index("ID")
    return [(r[ii], r[ki].split("(")[0], r[ni], float(r[vi].replace(",", "")), r[ui]) for r in data]


BYTE_UNIT = {"byte": 1.0, "Kbyte": 1e3, "Mbyte": 1e6, "Gbyte": 1e9, "Tbyte": 1e12}
INST_UNIT = {"inst": 1.0, "Kinst": 1e3, "Minst": 1e6, "Ginst": 1e9}


def traffic(csv_path, render_json, skip=0):
    """Per-ray figures of a traversal kernel from a capture of its launches
    skip, skip + 1, ... (`ncu -k regex:<kernel> -s <skip> -c <n>`, one kernel
    per capture): DRAM bytes (dram__bytes_read.sum + dram__bytes_write.sum),
    L2 bytes (lts__t_bytes.sum), warp instructions issued
    (smsp__inst_executed.sum) and active lanes per warp instruction
    (smsp__thread_inst_executed.sum / smsp__inst_executed.sum), each divided
    by the rays those launches traced (the render's per-launch log; closest-
    hit rays for extend, shadow rays for shadow)."""
    import json

    log = json.load(open(render_json))["launch_rays"]
    agg = {}
    for lid, kern, metric, val, unit in _metric_rows(csv_path):
        a = agg.setdefault(kern, {"launches": set(), "dram": 0.0, "l2": 0.0, "inst": 0.0, "thread_inst": 0.0,
                                  "ms": 0.0})
        a["launches"].add(int(lid))
        if metric.startswith("dram__bytes"):
            a["dram"] += val * BYTE_UNIT[unit]
        elif metric == "lts__t_bytes.sum":
            a["l2"] += val * BYTE_UNIT[unit]
        elif metric == "smsp__inst_executed.sum":
            a["inst"] += val * INST_UNIT.get(unit, 1.0)
        elif metric == "smsp__thread_inst_executed.sum":
            a["thread_inst"] += val * INST_UNIT.get(unit, 1.0)
        elif metric == "gpu__time_duration.sum":
            a["ms"] += val * UNIT_MS[unit]
    rows = ["| kernel | launches | rays | DRAM bytes per ray | L2 bytes per ray | warp instructions per ray "
            "| lanes per instruction | device ms (ncu) |", "|---|---|---|---|---|---|---|---|"]
    for kern, a in sorted(agg.items()):
        kind = "shadow" if "shadow" in kern else "extend"
        n = len(a["launches"])
        rays = max(sum(log[kind][skip + k] for k in range(n) if skip + k < len(log[kind])), 1)
        lanes = a["thread_inst"] / a["inst"] if a["inst"] else float("nan")
        rows.append(f"| {kern} | {skip}..{skip + n - 1} | {rays} | {a['dram'] / rays:.2f} | {a['l2'] / rays:.1f} "
                    f"| {a['inst'] / rays:.1f} | {lanes:.2f} | {a['ms']:.3f} |")
    return "\n".join(rows)


def render(argv):
    import argparse
    import json

    import torch

    import hikari_b200 as hk
    from hikari_b200 import scenes

    ap = argparse.ArgumentParser()
    ap.add_argument("--workload", default="heterogeneous", choices=["heterogeneous", "textured"],
                    help="heterogeneous: 64 displaced icospheres (bench's default workload); textured: the "
                         "bitmap / bump / normal-mapped light scene of bench.py --workload textured")
    ap.add_argument("--views", type=int, default=1)
    ap.add_argument("--spp", type=int, default=16)
    ap.add_argument("--accel", default="bvh2", choices=["bvh2", "bvh8"])
    ap.add_argument("--capacity", type=int, default=1 << 22)
    ap.add_argument("--out", default=None)
    ap.add_argument("--threads-extend", type=int, default=0)
    ap.add_argument("--threads-shade", type=int, default=0)
    ap.add_argument("--fetch-steps", type=int, default=0)
    ap.add_argument("--fetch-min-idle", type=int, default=0)
    ap.add_argument("--iterations-per-check", type=int, default=0)
    ap.add_argument("--fetch-steps-shadow", type=int, default=0)
    ap.add_argument("--fetch-min-idle-shadow", type=int, default=0)
    ap.add_argument("--reg-lean", type=int, default=0)
    ap.add_argument("--shadow-tests", type=int, default=0)
    ap.add_argument("--closest-tests", type=int, default=0)
    ap.add_argument("--sample-major", type=int, default=0)
    ap.add_argument("--config-json", default=None,
                    help="a JSON file with a wavefront configuration (bench.py's config.wavefront); its keys set "
                         "the options above")
    a = ap.parse_args(argv)
    if a.config_json:
        for k, v in json.load(open(a.config_json)).items():
            if hasattr(a, k) and v is not None:
                setattr(a, k, int(v))
    if a.workload == "textured":
        sd = scenes.lights_scene(width=1024, height=1024, spp=a.spp, depth=12, shading_normals=True, textured=True,
                                 bitmap=True, bump=True)
        cams = None
    else:
        sd = scenes.heterogeneous(width=1024, height=1024, spp=a.spp, depth=16)
        cams = scenes.heterogeneous_cameras(a.views)
    gs = hk.Scene.from_desc(sd)
    gs.set_accel(hk.ACCEL_BVH8 if a.accel == "bvh8" else hk.ACCEL_BVH2)
    films = [torch.zeros(gs.film_shape(), device="cuda") for _ in range(a.views)]
    ctr = torch.zeros(7, dtype=torch.int64, device="cuda")
    gs.render_batch(films, spp=a.spp, depth=sd.depth, cameras=cams, counters=ctr, capacity=a.capacity,
                    threads_extend=a.threads_extend, threads_shade=a.threads_shade, fetch_steps=a.fetch_steps,
                    fetch_min_idle=a.fetch_min_idle, iterations_per_check=a.iterations_per_check,
                    fetch_steps_shadow=a.fetch_steps_shadow, fetch_min_idle_shadow=a.fetch_min_idle_shadow,
                    reg_lean=a.reg_lean, shadow_tests=a.shadow_tests, closest_tests=a.closest_tests,
                    sample_major=a.sample_major)
    torch.cuda.synchronize()
    c = [int(x) for x in ctr.cpu().tolist()]
    names = ["rays", "shadow_rays", "dropped", "node_visits", "tri_tests", "node_visits_shadow", "tri_tests_shadow"]
    out = {"workload": f"{a.workload} {a.views} x 1024^2 x {a.spp} spp", "accel": a.accel,
           "launch": {"capacity": a.capacity, "threads_extend": a.threads_extend, "threads_shade": a.threads_shade,
                      "fetch_steps": a.fetch_steps, "fetch_min_idle": a.fetch_min_idle,
                      "fetch_steps_shadow": a.fetch_steps_shadow, "fetch_min_idle_shadow": a.fetch_min_idle_shadow,
                      "reg_lean": a.reg_lean, "shadow_tests": a.shadow_tests, "closest_tests": a.closest_tests,
                      "sample_major": a.sample_major},
           "counters": dict(zip(names, c)),
           # rays of each traversal launch, in launch order (ncu -k <kernel> -s i -c k captures launches i..i+k-1)
           "launch_rays": {"extend": [int(x) for x in gs.wavefront_launch_log(0)],
                           "shadow": [int(x) for x in gs.wavefront_launch_log(1)]}}
    text = json.dumps(out)
    if a.out:
        open(a.out, "w").write(text + "\n")
    print(text)


if __name__ == "__main__":
    if sys.argv[1] == "launches":
        print(launches(sys.argv[2]))
    elif sys.argv[1] == "render":
        render(sys.argv[2:])
    elif sys.argv[1] == "traffic":
        print(traffic(sys.argv[2], sys.argv[3], int(sys.argv[4]) if len(sys.argv) > 4 else 0))
    else:
        print(raw(sys.argv[2], sys.argv[3] if len(sys.argv) > 3 else None))
