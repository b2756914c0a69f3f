"""Malformed image files against the library's decoders (hikari_b200/csrc/
hk_image.cpp) under AddressSanitizer and UBSan.

Bitmap textures name files that the library decodes itself, so a texture file
is untrusted input: a damaged or hostile file must fail with an error status
or decode, and never read or write outside the decoder's buffers.  The
decoder is compiled here with -fsanitize=address,undefined into a small driver
that loads every file of a generated corpus (oversubscribed and undefined
Huffman tables, undefined quantisation tables, truncations at every segment,
seeded byte corruptions of JPEG and PNG files) with one and three channels.
"""
import os
import shutil
import subprocess

import numpy as np
import pytest

PIL = pytest.importorskip("PIL.Image")

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CSRC = os.path.join(ROOT, "hikari_b200", "csrc")

DRIVER = r"""
#include <cstdio>
#include <cstdint>
#include <string>
#include "hk_hostutil.h"
extern "C" int hk_image_load(const char *, int32_t, int32_t *, int32_t *, uint8_t **);
extern "C" void hk_image_free(uint8_t *);
namespace hk {
thread_local std::string g_err;
int set_error(int code, const std::string &msg) { g_err = msg; return code; }
}
int main(int argc, char **argv) {
    int ok = 0, failed = 0;
    for (int i = 1; i < argc; ++i)
        for (int ch : {1, 3}) {
            int32_t w = 0, h = 0;
            uint8_t *px = nullptr;
            if (hk_image_load(argv[i], ch, &w, &h, &px) == 0) {
                unsigned sum = 0;   // touch every byte the decoder says it wrote
                for (int64_t k = 0; k < (int64_t)w * h * ch; ++k) sum += px[k];
                if (sum == 0xffffffffu) std::printf("-");
                hk_image_free(px);
                ++ok;
            } else {
                ++failed;
            }
        }
    std::printf("decoded %d failed %d\n", ok, failed);
    return 0;
}
"""


def _segments(jpg: bytes):
    """(marker, start, length-including-marker) of the segments before the scan data."""
    out, p = [], 2
    while p + 4 <= len(jpg):
        assert jpg[p] == 0xFF
        m = jpg[p + 1]
        ln = (jpg[p + 2] << 8) | jpg[p + 3]
        out.append((m, p, ln + 2))
        if m == 0xDA:
            break
        p += ln + 2
    return out


def _corpus(tmp):
    rng = np.random.default_rng(7)
    img = (rng.random((37, 53, 3)) * 255).astype(np.uint8)
    files = []

    def put(name, data):
        p = os.path.join(tmp, name)
        with open(p, "wb") as f:
            f.write(data)
        files.append(p)

    import io

    buf = io.BytesIO()
    PIL.fromarray(img).save(buf, "JPEG", quality=85, subsampling=2)
    jpg = buf.getvalue()
    put("good.jpg", jpg)
    segs = _segments(jpg)
    dht = [s for s in segs if s[0] == 0xC4]
    assert dht
    # oversubscribed code-length tables: 3 (or 255) codes of length 1, 5 of length 2
    for k, counts in enumerate([{1: 3}, {1: 255}, {2: 5}, {1: 2, 2: 1}, {2: 4, 3: 1}]):
        b = bytearray(jpg)
        _, start, _ = dht[0]
        tab = start + 4   # Tc/Th byte
        for l in range(1, 17):
            b[tab + l] = 0
        total = 0
        for l, c in counts.items():
            b[tab + l] = c
            total += c
        # keep the segment length consistent where the table still fits
        old = sum(jpg[tab + 1:tab + 17])
        if total <= old:
            put(f"oversub{k}.jpg", bytes(b))
        else:
            seg_len = (jpg[start + 2] << 8) | jpg[start + 3]
            new = bytes(b[:tab + 17]) + bytes(total) + bytes(b[tab + 17 + old:])
            ln = seg_len + total - old
            new = new[:start + 2] + bytes([ln >> 8, ln & 255]) + new[start + 4:]
            put(f"oversub{k}.jpg", new)
    # scans naming tables no DHT / DQT defined
    sos = [s for s in segs if s[0] == 0xDA][0]
    for k, sel in enumerate([0x33, 0x30, 0x03]):   # DC and / or AC table 3 (PIL defines 0 and 1)
        b = bytearray(jpg)
        ns = b[sos[1] + 4]
        for c in range(ns):
            b[sos[1] + 6 + 2 * c] = sel
        put(f"undef_huff{k}.jpg", bytes(b))
    sof = [s for s in segs if s[0] in (0xC0, 0xC1)][0]
    b = bytearray(jpg)
    for c in range(b[sof[1] + 9]):
        b[sof[1] + 12 + 3 * c] = 3   # quantisation table 3: never defined
    put("undef_qt.jpg", bytes(b))
    # drop each segment in turn; truncate at each segment boundary and inside the scan
    for k, (_, start, ln) in enumerate(segs):
        put(f"drop{k}.jpg", jpg[:start] + jpg[start + ln:])
        put(f"trunc{k}.jpg", jpg[:start + ln // 2])
    for cut in np.linspace(sos[1] + sos[2], len(jpg) - 1, 12).astype(int):
        put(f"scan_cut{cut}.jpg", jpg[:cut])
    buf = io.BytesIO()
    PIL.fromarray(img).save(buf, "PNG")
    png = buf.getvalue()
    put("good.png", png)
    for cut in np.linspace(8, len(png) - 1, 12).astype(int):
        put(f"png_cut{cut}.png", png[:cut])
    # seeded random corruptions: 1-16 bytes overwritten anywhere after the signature
    for k in range(120):
        src = jpg if k % 3 else png
        b = bytearray(src)
        for _ in range(int(rng.integers(1, 17))):
            b[int(rng.integers(4, len(b)))] = int(rng.integers(0, 256))
        put(f"rand{k}.{'jpg' if k % 3 else 'png'}", bytes(b))
    return files


def test_corrupt_images_under_asan(tmp_path):
    if shutil.which("g++") is None:
        pytest.skip("g++ not available")
    drv = tmp_path / "drv.cpp"
    drv.write_text(DRIVER)
    exe = tmp_path / "drv"
    cuda_inc = "/usr/local/cuda/include"
    cmd = ["g++", "-std=c++17", "-O1", "-g", "-fsanitize=address,undefined", "-fno-sanitize-recover=all",
           "-I", CSRC, "-I", cuda_inc, str(drv), os.path.join(CSRC, "hk_image.cpp"), "-o", str(exe),
           "-L/usr/local/cuda/lib64", "-lcudart_static", "-lz", "-lpthread", "-ldl", "-lrt"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0 and "cannot find -lcudart_static" in r.stderr:
        pytest.skip("cudart_static not available")
    assert r.returncode == 0, r.stderr[-2000:]
    files = _corpus(str(tmp_path))
    env = dict(os.environ, ASAN_OPTIONS="detect_leaks=0:abort_on_error=0", UBSAN_OPTIONS="print_stacktrace=1")
    r = subprocess.run([str(exe)] + files, capture_output=True, text=True, env=env, timeout=600)
    assert r.returncode == 0 and "Sanitizer" not in r.stderr, r.stderr[-3000:]
    dec, fail = map(int, r.stdout.strip().split()[-3::2])
    # the intact files decode; the oversubscribed and undefined-table files are rejected
    assert dec >= 4 and fail >= 2 * 9, r.stdout


def test_oversubscribed_huffman_rejected(tmp_path):
    """Through the built library: every oversubscribed or undefined-table file
    fails with an error status naming the table."""
    import hikari_b200 as hk

    files = [f for f in _corpus(str(tmp_path)) if os.path.basename(f).startswith(("oversub", "undef"))]
    assert len(files) == 9
    for f in files:
        with pytest.raises(Exception, match="table"):
            hk.image_load(f, 3)
