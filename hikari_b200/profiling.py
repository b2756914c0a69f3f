"""Summarise ncu output for profiles/: a launch list (`--metrics
gpu__time_duration.sum --csv`) into per-kernel launches / total / share, and
selected raw metrics of a `--set full` report (`ncu -i X --page raw --csv`).

usage: python -m hikari_b200.profiling launches <launches.csv>
       python -m hikari_b200.profiling raw <report.ncu-rep> [regex]
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


if __name__ == "__main__":
    if sys.argv[1] == "launches":
        print(launches(sys.argv[2]))
    else:
        print(raw(sys.argv[2], sys.argv[3] if len(sys.argv) > 3 else None))
