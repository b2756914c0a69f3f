"""Build oracle/_ref/libhikari_ref.so: the reference renderer's own sources
compiled where they lie, for the parity tests of the oracle restatement and
as the timed CPU baseline (the reference's own pathMIS renderer).

Every file of src/ is compiled except three:
  * src/Main.cpp and src/core/Screen.cpp (the OpenGL preview window and the
    program's main): oracle/ref_shim/ref_render.cpp is the headless driver
    that runs Render's block loop (src/Main.cpp:46-147) without the window;
  * src/core/Bitmap.cpp (OpenEXR I/O through the OpenEXR library, which needs
    its own CMake build): oracle/ref_shim/ref_bitmap.cpp implements the same
    Bitmap members over a small uncompressed-EXR codec.
ext/pugixml/src/pugixml.cpp (the parser's XML library) is compiled from its
source too.

Recipe (no reference build system is run):
  * a shim include tree (oracle/_ref/shim) of forwarding headers named like
    the reference's backslash include paths ("core\\Common.hpp" -> include/core/
    Common.hpp, "Eigen\\Lu" -> ext/eigen/Eigen/LU), plus oracle/ref_shim/ for
    glog, <windows.h> and a stand-in for the TBB pieces used (blocked_range,
    parallel_for on the calling thread, mutex);
  * -DWIN32 selects the reference's Windows branches (its non-Windows branch
    of Signum has a bare #elif that GCC rejects); oracle/ref_shim/prelude.h
    supplies the MSVC CRT helpers they use;
  * src/core/Common.cpp is the one file that needs a token fix
    (`unsigned int(x)` at :89 is an MSVC-only functional cast): it is piped
    through sed to g++ on stdin, the file itself is not copied;
  * the RFT tables are found through the reference's own file resolver under
    their literal name "data\\GGXRFTData.bin", a symlink in oracle/_ref.

usage: python oracle/ref_build.py [reference-root]   (needs the reference checkout)
"""
import concurrent.futures
import glob
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "_ref")
LIB = os.path.join(OUT, "libhikari_ref.so")
SHIM_SOURCES = ["ref_bridge.cpp", "ref_bitmap.cpp", "ref_render.cpp"]
SKIP = {"Main.cpp", "Screen.cpp", "Bitmap.cpp"}


def _link(src, dst):
    if os.path.lexists(dst):
        os.remove(dst)
    os.symlink(src, dst)


def _forward(src, dst):
    """One-line forwarding header, so that quoted includes inside src resolve
    relative to its real directory."""
    text = f'#include "{src}"\n'
    if os.path.exists(dst) and not os.path.islink(dst):
        with open(dst) as f:
            if f.read() == text:
                return
    if os.path.lexists(dst):
        os.remove(dst)
    with open(dst, "w") as f:
        f.write(text)


def _newer(obj, *deps):
    return not os.path.exists(obj) or any(os.path.getmtime(d) > os.path.getmtime(obj) for d in deps)


def build(ref: str = "/root/reference", jobs: int = 0) -> str:
    if not os.path.isdir(ref):
        raise FileNotFoundError(f"reference checkout not found at {ref}")
    shim = os.path.join(OUT, "shim")
    objd = os.path.join(OUT, "obj")
    os.makedirs(shim, exist_ok=True)
    os.makedirs(objd, exist_ok=True)
    for hdr in glob.glob(os.path.join(ref, "include", "*", "*.hpp")):
        sub = os.path.basename(os.path.dirname(hdr))
        _forward(hdr, os.path.join(shim, f"{sub}\\{os.path.basename(hdr)}"))
    # TwoSidedBSDF.cpp includes its header by the relative Windows path "..\\..\\include\\bsdf\\..."
    _forward(os.path.join(ref, "include", "bsdf", "TwoSidedBSDF.hpp"),
             os.path.join(shim, "..\\..\\include\\bsdf\\TwoSidedBSDF.hpp"))
    for name, real in [("Core", "Core"), ("Geometry", "Geometry"), ("Lu", "LU")]:
        _forward(os.path.join(ref, "ext", "eigen", "Eigen", real), os.path.join(shim, f"Eigen\\{name}"))
    _forward(os.path.join(HERE, "ref_shim", "glog_logging.h"), os.path.join(shim, "glog\\logging.h"))
    _forward(os.path.join(HERE, "ref_shim", "tbb_serial.h"), os.path.join(shim, "tbb\\tbb.h"))
    _forward(os.path.join(HERE, "ref_shim", "tbb_serial.h"), os.path.join(shim, "tbb\\mutex.h"))
    _forward(os.path.join(ref, "ext", "filesystem", "filesystem", "resolver.h"), os.path.join(shim, "filesystem\\resolver.h"))
    data = os.path.join(os.path.dirname(HERE), "hikari_b200", "data")   # identical copies of ref data/
    for f in ("BeckmannRFTData.bin", "GGXRFTData.bin"):
        _link(os.path.join(data, f), os.path.join(OUT, f"data\\{f}"))
    flags = ["g++", "-std=c++14", "-O2", "-ffp-contract=off", "-fPIC", "-w", "-DWIN32", "-DNDEBUG",
             "-include", os.path.join(HERE, "ref_shim", "prelude.h"),
             "-I", shim, "-I", os.path.join(HERE, "ref_shim"), "-I", os.path.join(ref, "include"),
             "-I", os.path.join(ref, "ext", "eigen"), "-I", os.path.join(ref, "ext", "tinyformat"),
             "-I", os.path.join(ref, "ext", "pcg32"), "-I", os.path.join(ref, "ext", "filesystem"),
             "-I", os.path.join(ref, "ext", "stb"), "-I", os.path.join(ref, "ext", "openexr", "IlmBase", "Imath"),
             "-I", os.path.join(ref, "ext", "hypothesis"), "-I", os.path.join(ref, "ext", "pugixml", "src")]
    shim_hdrs = [os.path.join(HERE, "ref_shim", h) for h in ("prelude.h", "tbb_serial.h", "glog_logging.h")]
    srcs = sorted(p for p in glob.glob(os.path.join(ref, "src", "**", "*.cpp"), recursive=True)
                  if os.path.basename(p) not in SKIP)
    srcs += [os.path.join(ref, "ext", "pugixml", "src", "pugixml.cpp")]
    srcs += [os.path.join(HERE, "ref_shim", s) for s in SHIM_SOURCES]
    common = os.path.join(ref, "src", "core", "Common.cpp")
    tasks, objs = [], []
    for s in srcs:
        o = os.path.join(objd, os.path.relpath(s, ref if s.startswith(ref) else HERE).replace(os.sep, "_") + ".o")
        objs.append(o)
        if not _newer(o, s, *shim_hdrs):
            continue
        if s == common:
            sed = subprocess.run(["sed", "s/unsigned int(strtoul/(unsigned int)(strtoul/", common], check=True,
                                 capture_output=True)
            tasks.append((flags + ["-x", "c++", "-c", "-", "-o", o], sed.stdout))
        else:
            tasks.append((flags + ["-c", s, "-o", o], None))

    def run(t):
        subprocess.run(t[0], input=t[1], check=True)

    with concurrent.futures.ThreadPoolExecutor(max_workers=jobs or os.cpu_count() or 4) as ex:
        for f in [ex.submit(run, t) for t in tasks]:
            f.result()
    if tasks or not os.path.exists(LIB):
        tmp = LIB + ".tmp"
        subprocess.check_call(["g++", "-shared", "-o", tmp] + objs + ["-lpthread"])
        os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    print(build(sys.argv[1] if len(sys.argv) > 1 else "/root/reference"))
