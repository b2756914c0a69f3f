// 8-bit image decoding for bitmap textures: the host step that precedes
// LoadImageFromFileR / RGB (src/core/Texture.cpp:12, :74), where the reference
// calls stbi_load (ext/stb/stb_image.h, a third-party header library).  The
// formats the reference's scenes use are read here:
//   * PNG (ISO/IEC 15948): 8- and 16-bit gray / gray+alpha / RGB / RGBA,
//     1-8-bit palette and low-depth gray, non-interlaced; zlib inflates the
//     IDAT stream.  Lossless: the pixels equal stb_image's.
//   * binary PGM / PPM (P5 / P6, maxval 255).
//   * baseline JPEG (ITU-T T.81 sequential Huffman, 8-bit, gray or YCbCr with
//     any sampling factors, restart intervals): a float inverse DCT, triangle
//     ("fancy") chroma upsampling and the JFIF YCbCr -> RGB matrix.  stb_image
//     uses integer approximations of the same steps, so pixels may differ from
//     its decode by a few levels.
// Channel requests follow stbi_load: gray from RGB is the fixed-point luma
// (77 R + 150 G + 29 B) >> 8; a 3-component JPEG asked for one channel gives
// its Y plane; alpha is dropped.
#include <zlib.h>

#include <algorithm>
#include <cctype>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <stdexcept>
#include <string>
#include <thread>
#include <vector>

#include "hk_hostutil.h"

namespace {

// rows [0, n) spread over the host's threads (each row written by one thread)
template <class F>
void parallel_rows(int n, F f) {
    const int nt = std::max(1, std::min<int>((int)std::thread::hardware_concurrency(), n / 16));
    if (nt <= 1) {
        for (int i = 0; i < n; ++i) f(i);
        return;
    }
    std::vector<std::thread> th;
    for (int t = 0; t < nt; ++t)
        th.emplace_back([&, t] {
            for (int i = t; i < n; i += nt) f(i);
        });
    for (auto &x : th) x.join();
}

struct Image {
    int w = 0, h = 0, ch = 0;   // ch: 1 gray, 2 gray+alpha, 3 rgb, 4 rgba
    std::vector<uint8_t> px;
};

[[noreturn]] void bad(const std::string &m) { throw std::runtime_error(m); }

std::vector<uint8_t> read_file(const char *path) {
    FILE *f = std::fopen(path, "rb");
    if (!f) bad(std::string("cannot open ") + path);
    std::vector<uint8_t> b;
    uint8_t buf[1 << 16];
    size_t n;
    while ((n = std::fread(buf, 1, sizeof buf, f)) > 0) b.insert(b.end(), buf, buf + n);
    std::fclose(f);
    return b;
}

uint32_t be32(const uint8_t *p) { return (uint32_t)p[0] << 24 | (uint32_t)p[1] << 16 | (uint32_t)p[2] << 8 | p[3]; }

// ------------------------------------------------------------ PNG
int paeth(int a, int b, int c) {
    const int p = a + b - c, pa = std::abs(p - a), pb = std::abs(p - b), pc = std::abs(p - c);
    if (pa <= pb && pa <= pc) return a;
    return pb <= pc ? b : c;
}

Image decode_png(const std::vector<uint8_t> &f) {
    size_t pos = 8;
    int w = 0, h = 0, depth = 0, ctype = -1, interlace = 0;
    std::vector<uint8_t> idat, plte;
    while (pos + 8 <= f.size()) {
        const uint32_t len = be32(&f[pos]);
        const std::string type(reinterpret_cast<const char *>(&f[pos + 4]), 4);
        if (pos + 12 + (size_t)len > f.size()) bad("truncated PNG chunk");
        const uint8_t *d = &f[pos + 8];
        if (type == "IHDR") {
            if (len < 13) bad("bad IHDR");
            w = (int)be32(d);
            h = (int)be32(d + 4);
            depth = d[8];
            ctype = d[9];
            interlace = d[12];
        } else if (type == "PLTE") {
            plte.assign(d, d + len);
        } else if (type == "IDAT") {
            idat.insert(idat.end(), d, d + len);
        } else if (type == "IEND") {
            break;
        }
        pos += 12 + len;
    }
    if (w <= 0 || h <= 0 || w > 32768 || h > 32768) bad("bad PNG size");
    if (interlace) bad("interlaced PNG is not supported");
    int spp;   // samples per pixel
    switch (ctype) {
    case 0: spp = 1; break;
    case 2: spp = 3; break;
    case 3: spp = 1; break;
    case 4: spp = 2; break;
    case 6: spp = 4; break;
    default: bad("bad PNG color type");
    }
    if (!(depth == 8 || depth == 16 || ((ctype == 0 || ctype == 3) && (depth == 1 || depth == 2 || depth == 4))))
        bad("unsupported PNG bit depth");
    if (ctype == 3 && plte.empty()) bad("PNG palette missing");
    const size_t stride = ((size_t)w * spp * depth + 7) / 8;
    const size_t bpp = std::max<size_t>(1, (size_t)spp * depth / 8);
    std::vector<uint8_t> raw((stride + 1) * (size_t)h);
    z_stream z;
    std::memset(&z, 0, sizeof z);
    if (inflateInit(&z) != Z_OK) bad("zlib init failed");
    z.next_in = idat.data();
    z.avail_in = (uInt)idat.size();
    z.next_out = raw.data();
    z.avail_out = (uInt)raw.size();
    const int zr = inflate(&z, Z_FINISH);
    inflateEnd(&z);
    if (zr != Z_STREAM_END && z.avail_out != 0) bad("corrupt PNG data");
    // unfilter in place, row by row (filter types 0-4)
    std::vector<uint8_t> rows(stride * (size_t)h);
    for (int y = 0; y < h; ++y) {
        const uint8_t ft = raw[(size_t)y * (stride + 1)];
        const uint8_t *in = &raw[(size_t)y * (stride + 1) + 1];
        uint8_t *out = &rows[(size_t)y * stride];
        const uint8_t *up = y ? &rows[(size_t)(y - 1) * stride] : nullptr;
        for (size_t i = 0; i < stride; ++i) {
            const int a = i >= bpp ? out[i - bpp] : 0, b = up ? up[i] : 0, c = (up && i >= bpp) ? up[i - bpp] : 0;
            int v = in[i];
            switch (ft) {
            case 0: break;
            case 1: v += a; break;
            case 2: v += b; break;
            case 3: v += (a + b) >> 1; break;
            case 4: v += paeth(a, b, c); break;
            default: bad("bad PNG filter type");
            }
            out[i] = (uint8_t)v;
        }
    }
    Image im;
    im.w = w;
    im.h = h;
    im.ch = ctype == 3 ? 3 : spp;
    im.px.resize((size_t)w * h * im.ch);
    for (int y = 0; y < h; ++y) {
        const uint8_t *r = &rows[(size_t)y * stride];
        for (int x = 0; x < w; ++x) {
            uint8_t *o = &im.px[((size_t)y * w + x) * im.ch];
            if (depth == 16) {
                for (int c = 0; c < spp; ++c) o[c] = r[((size_t)x * spp + c) * 2];   // high byte (16 -> 8 bits)
            } else if (depth == 8) {
                if (ctype == 3) {
                    const size_t k = (size_t)r[x] * 3;
                    if (k + 3 > plte.size()) bad("PNG palette index out of range");
                    o[0] = plte[k]; o[1] = plte[k + 1]; o[2] = plte[k + 2];
                } else {
                    for (int c = 0; c < spp; ++c) o[c] = r[(size_t)x * spp + c];
                }
            } else {   // 1, 2, 4 bits: gray scaled to 8 bits, or a palette index
                const int per = 8 / depth, shift = (per - 1 - x % per) * depth;
                const int v = (r[x / per] >> shift) & ((1 << depth) - 1);
                if (ctype == 3) {
                    const size_t k = (size_t)v * 3;
                    if (k + 3 > plte.size()) bad("PNG palette index out of range");
                    o[0] = plte[k]; o[1] = plte[k + 1]; o[2] = plte[k + 2];
                } else {
                    o[0] = (uint8_t)(v * (depth == 1 ? 0xff : depth == 2 ? 0x55 : 0x11));
                }
            }
        }
    }
    return im;
}

// ------------------------------------------------------------ PGM / PPM
Image decode_pnm(const std::vector<uint8_t> &f) {
    size_t p = 2;
    auto token = [&]() {
        for (;;) {
            while (p < f.size() && std::isspace(f[p])) ++p;
            if (p < f.size() && f[p] == '#') {
                while (p < f.size() && f[p] != '\n') ++p;
                continue;
            }
            break;
        }
        long v = 0;
        if (p >= f.size() || !std::isdigit(f[p])) bad("bad PNM header");
        while (p < f.size() && std::isdigit(f[p])) v = v * 10 + (f[p++] - '0');
        return v;
    };
    Image im;
    im.ch = f[1] == '5' ? 1 : 3;
    im.w = (int)token();
    im.h = (int)token();
    const long maxval = token();
    ++p;   // one whitespace byte before the raster
    if (im.w <= 0 || im.h <= 0 || im.w > 32768 || im.h > 32768 || maxval != 255) bad("unsupported PNM");
    const size_t n = (size_t)im.w * im.h * im.ch;
    if (p + n > f.size()) bad("truncated PNM");
    im.px.assign(f.begin() + (long)p, f.begin() + (long)(p + n));
    return im;
}

// ------------------------------------------------------------ JPEG (baseline)
struct Huff {
    uint8_t bits[17] = {};
    uint8_t vals[256] = {};
    int mincode[17] = {}, maxcode[18] = {}, valptr[17] = {};
    uint16_t fast[512] = {};   // 9-bit lookahead: (length << 8) | value, 0 = slow path
    bool defined = false;      // set by a DHT segment
    void build() {
        int code = 0, k = 0;
        for (int l = 1; l <= 16; ++l) {
            valptr[l] = k;
            mincode[l] = code;
            code += bits[l];
            // a prefix code has at most 2^l codes of length <= l: more would
            // run the fast table below past its 512 entries
            if (code > (1 << l)) bad("bad JPEG Huffman table");
            k += bits[l];
            maxcode[l] = bits[l] ? code - 1 : -1;
            code <<= 1;
        }
        maxcode[17] = 0x7fffffff;
        std::memset(fast, 0, sizeof fast);
        code = 0;
        k = 0;
        for (int l = 1; l <= 9; ++l) {
            for (int i = 0; i < bits[l]; ++i, ++k, ++code) {
                const int shift = 9 - l;
                for (int j = 0; j < (1 << shift); ++j) fast[(code << shift) | j] = (uint16_t)(l << 8 | vals[k]);
            }
            code <<= 1;
        }
        defined = true;
    }
};

struct JComp {
    int id, hs, vs, tq, td = 0, ta = 0;
    int bw, bh;                 // blocks across / down (whole MCUs)
    std::vector<int16_t> coef;  // dequantised coefficients, 64 per block in natural order
    std::vector<uint8_t> plane; // bw*8 x bh*8 samples
    int dc = 0;
};

const int kZigzag[64] = {0,  1,  8,  16, 9,  2,  3,  10, 17, 24, 32, 25, 18, 11, 4,  5,  12, 19, 26, 33, 40, 48,
                         41, 34, 27, 20, 13, 6,  7,  14, 21, 28, 35, 42, 49, 56, 57, 50, 43, 36, 29, 22, 15, 23,
                         30, 37, 44, 51, 58, 59, 52, 45, 38, 31, 39, 46, 53, 60, 61, 54, 47, 55, 62, 63};

struct BitReader {
    const std::vector<uint8_t> &f;
    size_t p;
    uint32_t acc = 0;
    int n = 0;
    bool marker = false;   // a marker was reached: zeros are fed from here on
    BitReader(const std::vector<uint8_t> &f_, size_t p_) : f(f_), p(p_) {}
    void fill() {
        while (n <= 24) {
            uint32_t b = 0;
            if (!marker && p < f.size()) {
                b = f[p];
                if (b == 0xff) {
                    const uint8_t nx = p + 1 < f.size() ? f[p + 1] : 0;
                    if (nx == 0x00) p += 2;      // stuffed byte
                    else { marker = true; b = 0; }
                } else {
                    ++p;
                }
            }
            acc |= b << (24 - n);
            n += 8;
        }
    }
    int bits(int k) {
        if (k == 0) return 0;
        fill();
        const int v = (int)(acc >> (32 - k));
        acc <<= k;
        n -= k;
        return v;
    }
    int decode(const Huff &hf) {
        fill();
        const uint16_t e = hf.fast[acc >> 23];
        if (e) {
            const int l = e >> 8;
            acc <<= l;
            n -= l;
            return e & 0xff;
        }
        int code = 0;
        for (int l = 1; l <= 16; ++l) {
            code = (code << 1) | (int)(acc >> 31);
            acc <<= 1;
            --n;
            if (code <= hf.maxcode[l]) return hf.vals[hf.valptr[l] + code - hf.mincode[l]];
        }
        bad("corrupt JPEG Huffman code");
    }
    // skip to the byte after the next RSTn marker
    void restart() {
        acc = 0;
        n = 0;
        marker = false;
        while (p + 1 < f.size() && !(f[p] == 0xff && f[p + 1] >= 0xd0 && f[p + 1] <= 0xd7)) ++p;
        if (p + 1 < f.size()) p += 2;
    }
};

int extend(int v, int s) { return v < (1 << (s - 1)) ? v - (1 << s) + 1 : v; }

// Separable float inverse DCT of one block (T.81 A.3.3), level shift, round, clamp.
void idct8x8(const int16_t *in, uint8_t *out, int stride, const float *cosk) {
    float tmp[64];
    for (int x = 0; x < 8; ++x)          // columns: v -> y
        for (int y = 0; y < 8; ++y) {
            float s = 0.0f;
            for (int v = 0; v < 8; ++v) s += cosk[y * 8 + v] * (float)in[v * 8 + x];
            tmp[y * 8 + x] = s;
        }
    for (int y = 0; y < 8; ++y)          // rows: u -> x
        for (int x = 0; x < 8; ++x) {
            float s = 0.0f;
            for (int u = 0; u < 8; ++u) s += cosk[x * 8 + u] * tmp[y * 8 + u];
            const int v = (int)std::lround(s * 0.25f + 128.0f);
            out[y * stride + x] = (uint8_t)std::min(255, std::max(0, v));
        }
}

Image decode_jpeg(const std::vector<uint8_t> &f, int req) {
    uint16_t qt[4][64] = {};
    bool qt_defined[4] = {};
    Huff hdc[4], hac[4];
    std::vector<JComp> comps;
    int w = 0, h = 0, hmax = 1, vmax = 1, restart_interval = 0;
    bool frame = false, adobe_rgb = false;
    size_t p = 2;
    for (;;) {
        while (p < f.size() && f[p] != 0xff) ++p;
        while (p < f.size() && f[p] == 0xff) ++p;
        if (p >= f.size()) bad("truncated JPEG");
        const uint8_t m = f[p++];
        if (m == 0xd9) bad("JPEG without scan");
        if (m == 0xd8 || (m >= 0xd0 && m <= 0xd7) || m == 0x01) continue;
        if (p + 2 > f.size()) bad("truncated JPEG");
        const size_t len = (size_t)f[p] << 8 | f[p + 1];
        if (len < 2 || p + len > f.size()) bad("truncated JPEG segment");
        const uint8_t *d = &f[p + 2];
        const size_t n = len - 2;
        // every read below stays inside the segment
        auto need = [&](size_t k) {
            if (k > n) bad("truncated JPEG segment");
        };
        if (m == 0xdb) {   // DQT
            for (size_t i = 0; i < n;) {
                const int pq = d[i] >> 4, tq = d[i] & 15;
                if (tq > 3 || pq > 1) bad("bad JPEG quantisation table");
                need(i + 1 + 64 * (pq ? 2 : 1));
                ++i;
                for (int k = 0; k < 64; ++k) {
                    qt[tq][kZigzag[k]] = pq ? (uint16_t)(d[i] << 8 | d[i + 1]) : d[i];
                    i += pq ? 2 : 1;
                }
                qt_defined[tq] = true;
            }
        } else if (m == 0xc4) {   // DHT
            for (size_t i = 0; i < n;) {
                const int tc = d[i] >> 4, th = d[i] & 15;
                if (th > 3 || tc > 1) bad("bad JPEG Huffman table");
                need(i + 17);
                Huff &hf = tc ? hac[th] : hdc[th];
                int total = 0;
                for (int l = 1; l <= 16; ++l) total += (hf.bits[l] = d[i + l]);
                if (total > 256) bad("bad JPEG Huffman table");
                need(i + 17 + (size_t)total);
                std::memcpy(hf.vals, d + i + 17, (size_t)total);
                hf.build();
                i += 17 + (size_t)total;
            }
        } else if (m == 0xc0 || m == 0xc1) {   // SOF0 / SOF1
            need(6);
            if (d[0] != 8) bad("only 8-bit JPEG is supported");
            h = d[1] << 8 | d[2];
            w = d[3] << 8 | d[4];
            const int nc = d[5];
            if (w <= 0 || h <= 0 || w > 32768 || h > 32768 || (nc != 1 && nc != 3)) bad("unsupported JPEG frame");
            need(6 + 3 * (size_t)nc);
            if (frame) bad("JPEG with two frames");
            for (int c = 0; c < nc; ++c) {
                JComp jc;
                jc.id = d[6 + 3 * c];
                jc.hs = d[7 + 3 * c] >> 4;
                jc.vs = d[7 + 3 * c] & 15;
                jc.tq = d[8 + 3 * c] & 3;
                if (jc.hs < 1 || jc.hs > 4 || jc.vs < 1 || jc.vs > 4) bad("bad JPEG sampling factors");
                hmax = std::max(hmax, jc.hs);
                vmax = std::max(vmax, jc.vs);
                comps.push_back(jc);
            }
            frame = true;
        } else if (m >= 0xc2 && m <= 0xcf && m != 0xc4 && m != 0xc8 && m != 0xcc) {
            bad("progressive / lossless / arithmetic JPEG is not supported");
        } else if (m == 0xdd) {   // DRI
            need(2);
            restart_interval = d[0] << 8 | d[1];
        } else if (m == 0xee && n >= 12 && std::memcmp(d, "Adobe", 5) == 0) {
            adobe_rgb = d[11] == 0 && comps.size() == 3;
        } else if (m == 0xda) {   // SOS: baseline has one scan holding every component
            if (!frame) bad("JPEG scan before frame");
            need(1);
            const int ns = d[0];
            need(1 + 2 * (size_t)ns);
            if (ns != (int)comps.size()) bad("multi-scan JPEG is not supported");
            for (int s = 0; s < ns; ++s) {
                const int cid = d[1 + 2 * s];
                for (auto &c : comps)
                    if (c.id == cid) { c.td = (d[2 + 2 * s] >> 4) & 3; c.ta = d[2 + 2 * s] & 3; }
            }
            // every table the scan decodes with must have been defined
            for (const auto &c : comps)
                if (!hdc[c.td].defined || !hac[c.ta].defined || !qt_defined[c.tq])
                    bad("JPEG scan names an undefined table");
            p += len;
            break;
        }
        p += len;
    }
    const int mcux = (w + 8 * hmax - 1) / (8 * hmax), mcuy = (h + 8 * vmax - 1) / (8 * vmax);
    for (auto &c : comps) {
        c.bw = mcux * c.hs;
        c.bh = mcuy * c.vs;
        c.coef.assign((size_t)c.bw * c.bh * 64, 0);
    }
    BitReader br(f, p);
    const bool single = comps.size() == 1;
    // a single-component scan is not interleaved: its MCU is one block over ceil(w/8) x ceil(h/8)
    const int sbw = single ? (w * comps[0].hs / hmax + 7) / 8 : 0, sbh = single ? (h * comps[0].vs / vmax + 7) / 8 : 0;
    const long total = single ? (long)sbw * sbh : (long)mcux * mcuy;
    auto block = [&](JComp &c, int bx, int by) {
        int16_t *blk = &c.coef[((size_t)by * c.bw + bx) * 64];
        const int t = br.decode(hdc[c.td]);
        if (t > 11) bad("corrupt JPEG DC");
        c.dc += t ? extend(br.bits(t), t) : 0;
        blk[0] = (int16_t)(c.dc * qt[c.tq][0]);
        for (int k = 1; k < 64;) {
            const int rs = br.decode(hac[c.ta]);
            const int r = rs >> 4, s = rs & 15;
            if (s == 0) {
                if (r != 15) break;   // EOB
                k += 16;
                continue;
            }
            k += r;
            if (k > 63) bad("corrupt JPEG AC");
            blk[kZigzag[k]] = (int16_t)(extend(br.bits(s), s) * qt[c.tq][kZigzag[k]]);
            ++k;
        }
    };
    for (long mcu = 0; mcu < total; ++mcu) {
        if (restart_interval && mcu > 0 && mcu % restart_interval == 0) {
            br.restart();
            for (auto &c : comps) c.dc = 0;
        }
        if (single) {
            block(comps[0], (int)(mcu % sbw), (int)(mcu / sbw));
        } else {
            const int mx = (int)(mcu % mcux), my = (int)(mcu / mcux);
            for (auto &c : comps)
                for (int v = 0; v < c.vs; ++v)
                    for (int u = 0; u < c.hs; ++u) block(c, mx * c.hs + u, my * c.vs + v);
        }
    }
    // inverse DCT: cos table C(u) cos((2x+1) u pi / 16)
    float cosk[64];
    for (int x = 0; x < 8; ++x)
        for (int u = 0; u < 8; ++u)
            cosk[x * 8 + u] = (float)((u == 0 ? std::sqrt(0.5) : 1.0) * std::cos((2 * x + 1) * u * M_PI / 16.0));
    for (auto &c : comps) {
        const int pw = c.bw * 8;
        c.plane.assign((size_t)pw * c.bh * 8, 0);
        parallel_rows(c.bh, [&](int by) {
            for (int bx = 0; bx < c.bw; ++bx)
                idct8x8(&c.coef[((size_t)by * c.bw + bx) * 64], &c.plane[(size_t)by * 8 * pw + bx * 8], pw, cosk);
        });
    }
    // upsample each plane to full resolution: triangle filter for 2x factors
    // (3/4 nearer sample, 1/4 farther), replication otherwise
    auto sample = [&](const JComp &c, std::vector<uint8_t> &full) {
        const int pw = c.bw * 8, ph = c.bh * 8;
        const int fx = hmax / c.hs, fy = vmax / c.vs;
        full.resize((size_t)w * h);
        auto at = [&](int x, int y) {
            x = std::min(std::max(x, 0), pw - 1);
            y = std::min(std::max(y, 0), ph - 1);
            return (int)c.plane[(size_t)y * pw + x];
        };
        const int cw = (w * c.hs + hmax - 1) / hmax, chh = (h * c.vs + vmax - 1) / vmax;   // meaningful samples
        auto atc = [&](int x, int y) { return at(std::min(x, cw - 1), std::min(y, chh - 1)); };
        parallel_rows(h, [&](int y) {
            for (int x = 0; x < w; ++x) {
                int v;
                if (fx == 1 && fy == 1) {
                    v = at(x, y);
                } else if (fx == 2 && fy == 2) {
                    const int sx = x >> 1, sy = y >> 1;
                    const int nx = (x & 1) ? sx + 1 : sx - 1, ny = (y & 1) ? sy + 1 : sy - 1;
                    const int r0 = 3 * atc(sx, sy) + atc(sx, ny), r1 = 3 * atc(nx, sy) + atc(nx, ny);
                    v = (3 * r0 + r1 + 8) >> 4;
                } else if (fx == 2 && fy == 1) {
                    const int sx = x >> 1, nx = (x & 1) ? sx + 1 : sx - 1;
                    v = (3 * atc(sx, y) + atc(nx, y) + 2) >> 2;
                } else {
                    v = atc(x / fx, y / fy);
                }
                full[(size_t)y * w + x] = (uint8_t)v;
            }
        });
    };
    Image im;
    im.w = w;
    im.h = h;
    if (comps.size() == 1) {
        im.ch = 1;
        sample(comps[0], im.px);
        return im;
    }
    std::vector<uint8_t> Y, Cb, Cr;
    sample(comps[0], Y);
    if (req == 1 && !adobe_rgb) {   // stbi_load with one channel keeps the luma plane
        im.ch = 1;
        im.px = std::move(Y);
        return im;
    }
    sample(comps[1], Cb);
    sample(comps[2], Cr);
    im.ch = 3;
    im.px.resize((size_t)w * h * 3);
    parallel_rows(h, [&](int row) {
      for (size_t i = (size_t)row * w; i < (size_t)(row + 1) * w; ++i) {
        int r, g, b;
        if (adobe_rgb) {
            r = Y[i]; g = Cb[i]; b = Cr[i];
        } else {
            const float y = Y[i], cb = (float)Cb[i] - 128.0f, cr = (float)Cr[i] - 128.0f;
            r = (int)std::lround(y + 1.402f * cr);
            g = (int)std::lround(y - 0.344136f * cb - 0.714136f * cr);
            b = (int)std::lround(y + 1.772f * cb);
        }
        im.px[3 * i] = (uint8_t)std::min(255, std::max(0, r));
        im.px[3 * i + 1] = (uint8_t)std::min(255, std::max(0, g));
        im.px[3 * i + 2] = (uint8_t)std::min(255, std::max(0, b));
      }
    });
    return im;
}

// stbi_load's channel conversion of 8-bit pixels: gray from RGB by the
// fixed-point luma, gray replicated to RGB, alpha dropped
std::vector<uint8_t> convert(const Image &im, int req) {
    const size_t n = (size_t)im.w * im.h;
    std::vector<uint8_t> o(n * (size_t)req);
    for (size_t i = 0; i < n; ++i) {
        const uint8_t *s = &im.px[i * im.ch];
        if (req == 3) {
            if (im.ch >= 3) { o[3 * i] = s[0]; o[3 * i + 1] = s[1]; o[3 * i + 2] = s[2]; }
            else o[3 * i] = o[3 * i + 1] = o[3 * i + 2] = s[0];
        } else {
            o[i] = im.ch >= 3 ? (uint8_t)((s[0] * 77 + s[1] * 150 + s[2] * 29) >> 8) : s[0];
        }
    }
    return o;
}

}  // namespace

extern "C" int hk_image_load(const char *path, int32_t channels, int32_t *width, int32_t *height, uint8_t **out) {
    return hk::guarded([&] {
        if (!path || !width || !height || !out || (channels != 1 && channels != 3))
            throw hk::HkError{HK_ERR_INVALID, "bad arguments"};
        Image im;
        try {
            const std::vector<uint8_t> f = read_file(path);
            static const uint8_t png_sig[8] = {0x89, 'P', 'N', 'G', 0x0d, 0x0a, 0x1a, 0x0a};
            if (f.size() >= 8 && std::memcmp(f.data(), png_sig, 8) == 0) im = decode_png(f);
            else if (f.size() >= 3 && f[0] == 0xff && f[1] == 0xd8) im = decode_jpeg(f, channels);
            else if (f.size() >= 3 && f[0] == 'P' && (f[1] == '5' || f[1] == '6')) im = decode_pnm(f);
            else bad("unknown image format");
        } catch (const std::runtime_error &e) {
            throw hk::HkError{HK_ERR_INVALID, std::string(path) + ": " + e.what()};
        }
        std::vector<uint8_t> px = convert(im, channels);
        uint8_t *buf = static_cast<uint8_t *>(std::malloc(px.size()));
        if (!buf) throw hk::HkError{HK_ERR_NOMEM, "out of host memory"};
        std::memcpy(buf, px.data(), px.size());
        *width = im.w;
        *height = im.h;
        *out = buf;
        return HK_OK;
    });
}

extern "C" void hk_image_free(uint8_t *p) { std::free(p); }
