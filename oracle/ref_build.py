"""Build oracle/_ref/libhikari_ref_bsdf.so: the reference's own BSDF and
point / directional / constant emitter classes compiled from the reference
sources where they lie, for record-wise parity tests of the oracle
restatement.

Recipe (no reference build system is run):
  * a shim include tree (oracle/_ref/shim) of symlinks named like the
    reference's backslash include paths ("core\\Common.hpp" -> include/core/
    Common.hpp, "Eigen\\Lu" -> ext/eigen/Eigen/LU), plus oracle/ref_shim/ for
    glog, <windows.h> and a serial stand-in for the TBB loops of MipMap;
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
import glob
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "_ref")
LIB = os.path.join(OUT, "libhikari_ref_bsdf.so")

CORE = ["Object", "PropertyList", "BSDF", "Texture", "MicrofacetDistribution", "RoughTransmitance", "Frame",
        "Sampling", "Color", "Vector", "Transform", "Sampler", "Intersection", "Timer", "MemoryArena", "Shape",
        "Mesh", "Emitter", "DiscretePDF", "BoundingBox", "Ray", "MipMap", "Camera", "ReconstructionFilter"]
BSDFS = ["DiffuseBSDF", "RoughConductorBSDF", "RoughDielectricBSDF", "RoughPlasticBSDF", "RoughCoatingBSDF",
         "MirrorBSDF", "ConductorBSDF", "DielectricBSDF", "PlasticBSDF", "TwoSidedBSDF", "CoatingBSDF",
         "RoughDiffuseBSDF", "BumpMapBSDF", "NormalMapBSDF"]
EMITTERS = ["PointLight", "DirectionalLight", "ConstantLight"]
TEXTURES = ["CheckerboardTexture", "GridTexture", "ScaleTexture", "BitmapTexture"]
OTHERS = [("camera", "PerspectiveCamera"), ("filter", "GaussianFilter")]


def _link(src, dst):
    if os.path.lexists(dst):
        os.remove(dst)
    os.symlink(src, dst)


def _forward(src, dst):
    """One-line forwarding header, so that quoted includes inside src resolve
    relative to its real directory."""
    if os.path.lexists(dst):
        os.remove(dst)
    with open(dst, "w") as f:
        f.write(f'#include "{src}"\n')


def build(ref: str = "/root/reference") -> str:
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
             "-I", os.path.join(ref, "ext", "hypothesis")]
    objs = []
    srcs = [os.path.join(ref, "src", "core", c + ".cpp") for c in CORE] + \
           [os.path.join(ref, "src", "bsdf", b + ".cpp") for b in BSDFS] + \
           [os.path.join(ref, "src", "emitter", e + ".cpp") for e in EMITTERS] + \
           [os.path.join(ref, "src", "texture", t + ".cpp") for t in TEXTURES] + \
           [os.path.join(ref, "src", d, f + ".cpp") for d, f in OTHERS] + \
           [os.path.join(HERE, "ref_shim", "ref_bridge.cpp")]
    for s in srcs:
        o = os.path.join(objd, os.path.basename(s) + ".o")
        subprocess.check_call(flags + ["-c", s, "-o", o])
        objs.append(o)
    common = os.path.join(ref, "src", "core", "Common.cpp")
    o = os.path.join(objd, "Common.cpp.o")
    sed = subprocess.run(["sed", "s/unsigned int(strtoul/(unsigned int)(strtoul/", common], check=True,
                         capture_output=True)
    subprocess.run(flags + ["-x", "c++", "-c", "-", "-o", o], input=sed.stdout, check=True)
    objs.append(o)
    subprocess.check_call(["g++", "-shared", "-o", LIB] + objs + ["-lpthread"])
    return LIB


if __name__ == "__main__":
    print(build(sys.argv[1] if len(sys.argv) > 1 else "/root/reference"))
