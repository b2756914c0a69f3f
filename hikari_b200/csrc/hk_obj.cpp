// Parallel OBJ reader; see hk_obj.h.
#include "hk_obj.h"

#include <algorithm>
#include <charconv>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <stdexcept>
#include <thread>

namespace hikari {
namespace {

struct Chunk {
    std::vector<float> P, N, T;     // transformed positions, normals, texcoords (file order)
    std::vector<int32_t> keys;      // (p, t, n) per triangle corner, 1-based, 0 = absent
    std::string error;
};

inline bool is_space(char c) { return c == ' ' || c == '\t' || c == '\r' || c == '\f' || c == '\v'; }

// One whitespace-separated token of [b, e) starting at b; returns its end.
inline const char *token_end(const char *b, const char *e) {
    while (b < e && !is_space(*b)) ++b;
    return b;
}
inline const char *skip_space(const char *b, const char *e) {
    while (b < e && is_space(*b)) ++b;
    return b;
}

// operator>>(float&) of the reference's stringstream: the correctly rounded
// value of the decimal token (a leading '+' allowed); a missing or malformed
// token leaves 0.
inline float parse_float(const char *&b, const char *e) {
    b = skip_space(b, e);
    const char *t = token_end(b, e);
    const char *s = b;
    if (s < t && *s == '+') ++s;
    float v = 0.0f;
    std::from_chars(s, t, v, std::chars_format::general);
    b = t;
    return v;
}

// ObjVertex (include/mesh/WavefrontObjMesh.hpp): "p", "p/t", "p//n", "p/t/n"
inline bool parse_key(const char *b, const char *e, int32_t *k) {
    k[0] = k[1] = k[2] = 0;
    int part = 0;
    while (true) {
        const char *s = b;
        while (b < e && *b != '/') ++b;
        if (part > 2) return false;
        if (b > s) {
            auto r = std::from_chars(s, b, k[part]);
            if (r.ec != std::errc() || r.ptr != b) return false;
        } else if (part == 0) {
            return false;
        }
        if (b == e) break;
        ++b;   // '/'
        ++part;
    }
    return true;
}

void parse_chunk(const char *b, const char *e, const float *M, const float *Mi, Chunk &c) {
    while (b < e) {
        const char *le = static_cast<const char *>(std::memchr(b, '\n', (size_t)(e - b)));
        if (!le) le = e;
        const char *p = skip_space(b, le);
        const char *pe = token_end(p, le);
        const size_t n = (size_t)(pe - p);
        if (n == 1 && p[0] == 'v') {
            const char *q = pe;
            float x = parse_float(q, le), y = parse_float(q, le), z = parse_float(q, le);
            float h[4];
            for (int r = 0; r < 4; r++) h[r] = M[4 * r] * x + M[4 * r + 1] * y + M[4 * r + 2] * z + M[4 * r + 3];
            c.P.push_back(h[0] / h[3]);
            c.P.push_back(h[1] / h[3]);
            c.P.push_back(h[2] / h[3]);
        } else if (n == 2 && p[0] == 'v' && p[1] == 'n') {
            const char *q = pe;
            float x = parse_float(q, le), y = parse_float(q, le), z = parse_float(q, le);
            float v[3] = {Mi[0] * x + Mi[4] * y + Mi[8] * z, Mi[1] * x + Mi[5] * y + Mi[9] * z,
                          Mi[2] * x + Mi[6] * y + Mi[10] * z};
            float l2 = v[0] * v[0] + (v[1] * v[1] + v[2] * v[2]);
            float s = l2 > 0.0f ? std::sqrt(l2) : 1.0f;
            for (int i = 0; i < 3; i++) c.N.push_back(l2 > 0.0f ? v[i] / s : v[i]);
        } else if (n == 2 && p[0] == 'v' && p[1] == 't') {
            const char *q = pe;
            float u = parse_float(q, le), v = parse_float(q, le);
            c.T.push_back(u);
            c.T.push_back(v);
        } else if (n == 1 && p[0] == 'f') {
            int32_t k[4][3];
            int nv = 0;
            const char *q = pe;
            while (nv < 4) {
                q = skip_space(q, le);
                if (q >= le) break;
                const char *te = token_end(q, le);
                if (!parse_key(q, te, k[nv])) {
                    c.error = "Invalid vertex data: \"" + std::string(q, te) + "\"";
                    return;
                }
                ++nv;
                q = te;
            }
            if (nv < 3) {
                c.error = "OBJ face with fewer than three vertices";
                return;
            }
            static const int tri[6] = {0, 1, 2, 3, 0, 2};
            for (int i = 0; i < (nv == 4 ? 6 : 3); i++)
                for (int j = 0; j < 3; j++) c.keys.push_back(k[tri[i]][j]);
        }
        b = le + 1;
    }
}

// First-use order of the (p, t, n) triples: open addressing over 64-bit hashes.
struct KeyTable {
    std::vector<int32_t> slot;   // vertex id + 1, 0 empty
    std::vector<int32_t> k;      // 3 per vertex id
    size_t mask = 0;
    explicit KeyTable(size_t n) {
        size_t cap = 16;
        while (cap < 2 * n) cap <<= 1;
        slot.assign(cap, 0);
        mask = cap - 1;
    }
    static uint64_t hash(const int32_t *a) {
        uint64_t h = (uint64_t)(uint32_t)a[0] * 0x9E3779B97F4A7C15ull;
        h ^= (uint64_t)(uint32_t)a[1] * 0xC2B2AE3D27D4EB4Full + (h >> 29);
        h ^= (uint64_t)(uint32_t)a[2] * 0x165667B19E3779F9ull + (h >> 31);
        return h ^ (h >> 33);
    }
    int32_t find_or_add(const int32_t *a) {
        for (size_t i = hash(a) & mask;; i = (i + 1) & mask) {
            int32_t s = slot[i];
            if (s == 0) {
                int32_t id = (int32_t)(k.size() / 3);
                k.insert(k.end(), a, a + 3);
                slot[i] = id + 1;
                return id;
            }
            const int32_t *b = &k[3 * (size_t)(s - 1)];
            if (b[0] == a[0] && b[1] == a[1] && b[2] == a[2]) return s - 1;
        }
    }
};

}  // namespace

ObjMesh load_obj(const std::string &path, const float *M, const float *Minv, int threads) {
    FILE *f = std::fopen(path.c_str(), "rb");
    if (!f) throw std::runtime_error("Unable to open OBJ file \"" + path + "\"!");
    std::fseek(f, 0, SEEK_END);
    long sz = std::ftell(f);
    std::fseek(f, 0, SEEK_SET);
    std::string text((size_t)std::max(sz, 0L), '\0');
    size_t got = sz > 0 ? std::fread(&text[0], 1, (size_t)sz, f) : 0;
    std::fclose(f);
    if ((long)got != sz) throw std::runtime_error("Unable to read OBJ file \"" + path + "\"!");

    // line-aligned chunks of about 2 MB, at most one per thread and pass
    int T = threads > 0 ? threads : (int)std::min(16u, std::max(1u, std::thread::hardware_concurrency()));
    const size_t want = std::max<size_t>(1, std::min<size_t>((size_t)T * 4, text.size() / (2u << 20) + 1));
    std::vector<std::pair<size_t, size_t>> ranges;
    size_t start = 0;
    for (size_t i = 1; i <= want && start < text.size(); i++) {
        size_t end = i == want ? text.size() : std::max(start, text.size() * i / want);
        while (end < text.size() && text[end] != '\n') ++end;
        if (end < text.size()) ++end;
        ranges.push_back({start, end});
        start = end;
    }
    std::vector<Chunk> chunks(ranges.size());
    auto work = [&](size_t w) {
        for (size_t i = w; i < ranges.size(); i += (size_t)T)
            parse_chunk(text.data() + ranges[i].first, text.data() + ranges[i].second, M, Minv, chunks[i]);
    };
    std::vector<std::thread> pool;
    for (int w = 1; w < T && (size_t)w < ranges.size(); w++) pool.emplace_back(work, (size_t)w);
    work(0);
    for (auto &t : pool) t.join();
    for (auto &c : chunks)
        if (!c.error.empty()) throw std::runtime_error(c.error);

    size_t nP = 0, nN = 0, nT = 0, nK = 0;
    for (auto &c : chunks) { nP += c.P.size(); nN += c.N.size(); nT += c.T.size(); nK += c.keys.size(); }
    std::vector<float> P, N, Tc;
    P.reserve(nP); N.reserve(nN); Tc.reserve(nT);
    for (auto &c : chunks) {
        P.insert(P.end(), c.P.begin(), c.P.end());
        N.insert(N.end(), c.N.begin(), c.N.end());
        Tc.insert(Tc.end(), c.T.begin(), c.T.end());
    }
    const int64_t np = (int64_t)(nP / 3), nn = (int64_t)(nN / 3), nt = (int64_t)(nT / 2);

    ObjMesh out;
    out.idx.resize(nK / 3);
    std::vector<int32_t> verts;   // (p, t, n) per output vertex
    bool positions_only = true;
    for (auto &c : chunks)
        for (size_t i = 0; i < c.keys.size() && positions_only; i += 3)
            positions_only = c.keys[i + 1] == 0 && c.keys[i + 2] == 0;
    size_t o = 0;
    if (positions_only) {   // first use of each position index
        std::vector<int32_t> first((size_t)np + 1, -1);
        int32_t next = 0;
        for (auto &c : chunks)
            for (size_t i = 0; i < c.keys.size(); i += 3) {
                int32_t p = c.keys[i];
                if (p < 1 || p > np) throw std::runtime_error("OBJ position index out of range");
                if (first[p] < 0) {
                    first[p] = next++;
                    verts.insert(verts.end(), {p, 0, 0});
                }
                out.idx[o++] = (uint32_t)first[p];
            }
    } else {
        KeyTable tab(nK / 3);
        for (auto &c : chunks)
            for (size_t i = 0; i < c.keys.size(); i += 3) out.idx[o++] = (uint32_t)tab.find_or_add(&c.keys[i]);
        verts.swap(tab.k);
    }
    const size_t nv = verts.size() / 3;
    out.pos.resize(3 * nv);
    for (size_t v = 0; v < nv; v++) {
        int32_t p = verts[3 * v];
        if (p < 1 || p > np) throw std::runtime_error("OBJ position index out of range");
        std::memcpy(&out.pos[3 * v], &P[3 * (size_t)(p - 1)], 12);
    }
    if (nn > 0) {
        out.nrm.resize(3 * nv);
        for (size_t v = 0; v < nv; v++) {
            int32_t n = verts[3 * v + 2];
            if (n < 1 || n > nn) throw std::runtime_error("OBJ normal index out of range");
            std::memcpy(&out.nrm[3 * v], &N[3 * (size_t)(n - 1)], 12);
        }
    }
    if (nt > 0) {
        out.uv.resize(2 * nv);
        for (size_t v = 0; v < nv; v++) {
            int32_t t = verts[3 * v + 1];
            if (t < 1 || t > nt) throw std::runtime_error("OBJ texture coordinate index out of range");
            std::memcpy(&out.uv[2 * v], &Tc[2 * (size_t)(t - 1)], 8);
        }
    }
    return out;
}

}  // namespace hikari

// ------------------------------------------------------------ C ABI
#include "hk_hostutil.h"

extern "C" int hk_obj_load(const char *path, const float *to_world16, uint32_t *nv, uint32_t *nt, float *positions,
                           float *normals, float *uv, uint32_t *indices, int32_t *attrs) {
    return hk::guarded([&] {
        if (!path || !nv || !nt) throw hk::HkError{HK_ERR_INVALID, "bad arguments"};
        float I[16] = {1, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1};
        const float *M = to_world16 ? to_world16 : I;
        float Minv[16];
        if (!hikari::invert4(M, Minv)) throw hk::HkError{HK_ERR_INVALID, "mesh toWorld is singular"};
        hikari::ObjMesh m = hikari::load_obj(path, M, Minv);
        const size_t v = m.pos.size() / 3, t = m.idx.size() / 3;
        if (v > 0xffffffffull || t > 0xffffffffull) throw hk::HkError{HK_ERR_INVALID, "mesh too large"};
        if (positions) {
            if (*nv < v || *nt < t) throw hk::HkError{HK_ERR_INVALID, "output arrays too small"};
            std::memcpy(positions, m.pos.data(), m.pos.size() * sizeof(float));
            std::memcpy(indices, m.idx.data(), m.idx.size() * sizeof(uint32_t));
            if (normals && !m.nrm.empty()) std::memcpy(normals, m.nrm.data(), m.nrm.size() * sizeof(float));
            if (uv && !m.uv.empty()) std::memcpy(uv, m.uv.data(), m.uv.size() * sizeof(float));
        }
        *nv = (uint32_t)v;
        *nt = (uint32_t)t;
        if (attrs) *attrs = (m.nrm.empty() ? 0 : 1) | (m.uv.empty() ? 0 : 2);
        return HK_OK;
    });
}
