"""Compile the sm_100a CUDA library in-tree (hikari_b200/_build/libhikari_b200.so).

nvcc -gencode arch=compute_100a,code=sm_100a -O3 -lineinfo -fmad=false:
-fmad=false keeps products and sums rounded like the reference's x86 build
(no FMA contraction); box tests use explicit __fmaf_rn where rounding cannot
change a result.
"""
from __future__ import annotations

import concurrent.futures
import os
import re
import subprocess
import sys
import threading

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OUT_DIR = os.path.join(HERE, "_build")
LIB = os.path.join(OUT_DIR, "libhikari_b200.so")
SOURCES = ["hk_render_b8.cu", "hk_render_b8t.cu", "hk_render_b2.cu", "hk_render_b2t.cu", "hk_wf_shade_3.cu",
           "hk_wf_shade_2.cu", "hk_wf_shade_1.cu", "hk_wf_shade_0.cu", "hk_wf_shade_4.cu", "hk_wf_shade_5.cu", "hk_wf_shade_6.cu", "hk_wf_shade_7.cu", "hk_wf_trace_8.cu", "hk_wf_trace_2.cu",
           "hk_batch_0.cu", "hk_batch_1.cu", "hk_batch_2.cu", "hk_batch_3.cu", "hk_batch_4.cu",
           "hk_kernels.cu", "hk_wavefront.cu", "hk_lbvh.cu", "hk_host.cpp", "hk_engine.cpp", "hk_server.cpp", "hk_bvh.cpp", "hk_xml.cpp",
           "hk_obj.cpp", "hk_mipmap.cpp", "hk_image.cpp"]
HEADERS = ["hk_megakernel.cuh", "hk_batch.cuh", "hk_wf_kernels.cuh", "hk_device.h", "hk_math.cuh", "hk_bsdf.cuh", "hk_traverse.cuh", "hk_shading.cuh", "hk_kernels.h",
           "hk_bvh.h", "hk_xml.h", "hk_wavefront.h", "hk_engine.h", "hk_hostutil.h", "hk_internal.h", "hk_obj.h", "hk_mipmap.h"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ARCH + ["-O3", "-lineinfo", "-fmad=false", "-std=c++17", "-Xcompiler", "-fPIC,-O2,-pthread",
                     "--expt-relaxed-constexpr"]


def _nvcc() -> str:
    for p in ("/usr/local/cuda/bin/nvcc",):
        if os.path.exists(p):
            return p
    return "nvcc"


_INC = re.compile(r'^\s*#\s*include\s+"([^"]+)"', re.M)


def _deps(path: str, seen: set | None = None) -> set:
    """The file and every quoted include it reaches (resolved in csrc/ or include/)."""
    seen = set() if seen is None else seen
    if path in seen or not os.path.exists(path):
        return seen
    seen.add(path)
    with open(path, errors="replace") as f:
        for name in _INC.findall(f.read()):
            for d in (os.path.dirname(path), CSRC, os.path.join(os.path.dirname(HERE), "include")):
                cand = os.path.join(d, name)
                if os.path.exists(cand):
                    _deps(cand, seen)
                    break
    return seen


def _stale(src: str, obj: str) -> bool:
    if not os.path.exists(obj):
        return True
    t = os.path.getmtime(obj)
    return any(os.path.getmtime(d) > t for d in _deps(os.path.join(CSRC, src)))


def needs_build() -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    return any(_stale(s, os.path.join(OUT_DIR, s + ".o")) or os.path.getmtime(os.path.join(OUT_DIR, s + ".o")) > t
               for s in SOURCES)


def _host_gb() -> float:
    try:
        return os.sysconf("SC_PAGE_SIZE") * os.sysconf("SC_PHYS_PAGES") / 1e9
    except (ValueError, OSError):
        return 64.0


def _unit_gb(cmd) -> float:
    """Peak host memory (GB) the unit's compile is expected to take."""
    name = next((os.path.basename(a) for a in cmd if a.endswith((".cu", ".cpp"))), "")
    if name in ("hk_render_b8t.cu", "hk_render_b2t.cu", "hk_wf_shade_3.cu"):
        return 22.0
    if name.startswith("hk_render_"):
        return 10.0
    return 3.0


def build(force: bool = False, verbose: bool = False) -> str:
    if not force and not needs_build():
        return LIB
    os.makedirs(OUT_DIR, exist_ok=True)
    cmds, objs = [], []
    for src in SOURCES:
        path = os.path.join(CSRC, src)
        obj = os.path.join(OUT_DIR, src + ".o")
        objs.append(obj)
        if not force and not _stale(src, obj):
            continue
        cmd = [_nvcc()] + NVCC_FLAGS + ["-c", path, "-o", obj]
        if src.endswith(".cpp"):
            cmd = [_nvcc()] + NVCC_FLAGS + ["-x", "cu", "-c", path, "-o", obj]
        if verbose:
            print(" ".join(cmd))
        cmds.append(cmd)
    # translation units compile in parallel (SOURCES lists the slowest first)
    # within a host-memory budget: ptxas takes about 20 GB for the textured
    # megakernels and the run-time-dispatched shade kernel, 9 GB for the other
    # megakernels and a few GB for the rest
    total = max(16.0, _host_gb() * 0.8)
    budget = [total]
    cv = threading.Condition()

    def run(cmd):
        need = min(total, _unit_gb(cmd))
        with cv:
            cv.wait_for(lambda: budget[0] >= need)
            budget[0] -= need
        try:
            return subprocess.check_call(cmd)
        finally:
            with cv:
                budget[0] += need
                cv.notify_all()

    if cmds:
        with concurrent.futures.ThreadPoolExecutor(max_workers=min(len(cmds), os.cpu_count() or 1)) as ex:
            for f in [ex.submit(run, c) for c in cmds]:
                f.result()
    tmp = LIB + ".tmp"
    subprocess.check_call([_nvcc()] + ARCH + ["-shared", "-o", tmp] + objs + ["-lpthread", "-lz"])
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
