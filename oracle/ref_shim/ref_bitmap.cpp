/* The reference's Bitmap class (include/core/Bitmap.hpp) for the oracle's
 * build of the reference: src/core/Bitmap.cpp reads and writes OpenEXR files
 * through the OpenEXR library, which needs its own CMake build, so this file
 * supplies the same three members over a small scanline EXR codec written for
 * the oracle.  Bitmap(filename) reads RGB(A) scanline files without
 * compression, with HALF or FLOAT channels (what the library's own EXR writer
 * and the scene generators write); Save writes an uncompressed FLOAT RGB file.
 * Test infrastructure only. */
#include <core\Bitmap.hpp>

#include <cstdio>
#include <cstring>
#include <fstream>
#include <map>
#include <vector>

NAMESPACE_BEGIN

namespace {
float half_to_float(uint16_t h) {
    const uint32_t s = (uint32_t)(h >> 15) << 31, e = (h >> 10) & 31, m = h & 1023;
    uint32_t bits;
    if (e == 0) {
        if (m == 0) {
            bits = s;
        } else {   // subnormal half: normalise
            int k = -1;
            uint32_t mm = m;
            do { mm <<= 1; ++k; } while (!(mm & 1024));
            bits = s | ((uint32_t)(127 - 15 - k) << 23) | ((mm & 1023) << 13);
        }
    } else if (e == 31) {
        bits = s | 0x7f800000u | (m << 13);
    } else {
        bits = s | ((e + 127 - 15) << 23) | (m << 13);
    }
    float f;
    std::memcpy(&f, &bits, 4);
    return f;
}

template <class T>
T rd(const std::vector<char> &b, size_t &p) {
    if (p + sizeof(T) > b.size()) throw HikariException("truncated EXR file");
    T v;
    std::memcpy(&v, &b[p], sizeof(T));
    p += sizeof(T);
    return v;
}
std::string rd_str(const std::vector<char> &b, size_t &p) {
    std::string s;
    while (p < b.size() && b[p]) s += b[p++];
    if (p >= b.size()) throw HikariException("truncated EXR file");
    ++p;
    return s;
}
template <class T>
void wr(std::ofstream &o, T v) { o.write(reinterpret_cast<const char *>(&v), sizeof(T)); }
void wr_str(std::ofstream &o, const std::string &s) { o.write(s.c_str(), (std::streamsize)s.size() + 1); }
}  // namespace

Bitmap::Bitmap(const Vector2i &Size) : Base(Size.y(), Size.x()) {}

Bitmap::Bitmap(const std::string &Filename) {
    std::ifstream f(Filename, std::ios::binary);
    if (!f) throw HikariException("Cannot open EXR file \"%s\"", Filename);
    std::vector<char> b((std::istreambuf_iterator<char>(f)), std::istreambuf_iterator<char>());
    size_t p = 0;
    if (rd<uint32_t>(b, p) != 20000630u) throw HikariException("\"%s\" is not an OpenEXR file", Filename);
    const uint32_t version = rd<uint32_t>(b, p);
    if (version & 0x200) throw HikariException("tiled EXR files are not supported");
    struct Ch { int type; };
    std::map<std::string, int> chans;   // name -> pixel type (1 HALF, 2 FLOAT)
    int compression = -1;
    int32_t xmin = 0, ymin = 0, xmax = -1, ymax = -1;
    for (;;) {
        const std::string name = rd_str(b, p);
        if (name.empty()) break;
        const std::string type = rd_str(b, p);
        const uint32_t size = rd<uint32_t>(b, p);
        const size_t end = p + size;
        if (end > b.size()) throw HikariException("truncated EXR header");
        if (name == "channels") {
            while (p < end && b[p]) {
                const std::string cn = rd_str(b, p);
                const int32_t pt = rd<int32_t>(b, p);
                p += 4;                     // pLinear + reserved
                const int32_t xs = rd<int32_t>(b, p), ys = rd<int32_t>(b, p);
                if (xs != 1 || ys != 1) throw HikariException("subsampled EXR channels are not supported");
                chans[cn] = pt;
            }
        } else if (name == "compression") {
            compression = (unsigned char)b[p];
        } else if (name == "dataWindow") {
            size_t q = p;
            xmin = rd<int32_t>(b, q); ymin = rd<int32_t>(b, q); xmax = rd<int32_t>(b, q); ymax = rd<int32_t>(b, q);
        }
        p = end;
    }
    if (compression != 0) throw HikariException("only uncompressed EXR files are read here");
    if (!chans.count("R") || !chans.count("G") || !chans.count("B"))
        throw HikariException("This is not a standard RGB OpenEXR file!");
    const int w = xmax - xmin + 1, h = ymax - ymin + 1;
    if (w <= 0 || h <= 0) throw HikariException("empty EXR data window");
    resize(h, w);
    p += (size_t)h * 8;   // line offset table: lines are stored in order
    std::vector<float> row(w);
    for (int y = 0; y < h; ++y) {
        const int32_t ly = rd<int32_t>(b, p);
        const uint32_t nbytes = rd<uint32_t>(b, p);
        const size_t end = p + nbytes;
        const int yy = ly - ymin;
        if (yy < 0 || yy >= h || end > b.size()) throw HikariException("bad EXR scanline");
        for (const auto &c : chans) {   // channels are stored in name order
            const int bytes = c.second == 1 ? 2 : 4;
            for (int x = 0; x < w; ++x) {
                if (c.second == 1) row[x] = half_to_float(rd<uint16_t>(b, p));
                else if (c.second == 2) row[x] = rd<float>(b, p);
                else throw HikariException("UINT EXR channels are not supported");
            }
            (void)bytes;
            const int k = c.first == "R" ? 0 : c.first == "G" ? 1 : c.first == "B" ? 2 : -1;
            if (k >= 0)
                for (int x = 0; x < w; ++x) coeffRef(yy, x)[k] = row[x];
        }
        p = end;
    }
}

void Bitmap::Save(const std::string &Filename) {
    std::ofstream o(Filename, std::ios::binary);
    if (!o) throw HikariException("Cannot write \"%s\"", Filename);
    const int w = (int)cols(), h = (int)rows();
    wr<uint32_t>(o, 20000630u);
    wr<uint32_t>(o, 2u);
    wr_str(o, "channels"); wr_str(o, "chlist"); wr<uint32_t>(o, 3 * (2 + 16) + 1);
    for (const char *c : {"B", "G", "R"}) {
        wr_str(o, c); wr<int32_t>(o, 2); wr<uint32_t>(o, 0); wr<int32_t>(o, 1); wr<int32_t>(o, 1);
    }
    wr<char>(o, 0);
    wr_str(o, "compression"); wr_str(o, "compression"); wr<uint32_t>(o, 1); wr<unsigned char>(o, 0);
    for (const char *n : {"dataWindow", "displayWindow"}) {
        wr_str(o, n); wr_str(o, "box2i"); wr<uint32_t>(o, 16);
        wr<int32_t>(o, 0); wr<int32_t>(o, 0); wr<int32_t>(o, w - 1); wr<int32_t>(o, h - 1);
    }
    wr_str(o, "lineOrder"); wr_str(o, "lineOrder"); wr<uint32_t>(o, 1); wr<unsigned char>(o, 0);
    wr_str(o, "pixelAspectRatio"); wr_str(o, "float"); wr<uint32_t>(o, 4); wr<float>(o, 1.0f);
    wr_str(o, "screenWindowCenter"); wr_str(o, "v2f"); wr<uint32_t>(o, 8); wr<float>(o, 0.0f); wr<float>(o, 0.0f);
    wr_str(o, "screenWindowWidth"); wr_str(o, "float"); wr<uint32_t>(o, 4); wr<float>(o, 1.0f);
    wr<char>(o, 0);
    const uint64_t line = 8 + (uint64_t)w * 12;
    const uint64_t first = (uint64_t)o.tellp() + (uint64_t)h * 8;
    for (int y = 0; y < h; ++y) wr<uint64_t>(o, first + (uint64_t)y * line);
    for (int y = 0; y < h; ++y) {
        wr<int32_t>(o, y);
        wr<uint32_t>(o, (uint32_t)(w * 12));
        for (int k : {2, 1, 0})
            for (int x = 0; x < w; ++x) wr<float>(o, coeff(y, x)[k]);
    }
}

NAMESPACE_END
