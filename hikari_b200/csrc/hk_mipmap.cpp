// Bitmap texture construction on the host (see hk_mipmap.h).  Every float
// operation follows the reference's order, so the pyramid is bit-identical to
// the reference's for the same 8-bit pixels; rows and columns are spread over
// host threads (each output texel is computed by one thread in a fixed order,
// as in the reference's TBB loops).
#include "hk_mipmap.h"

#include <algorithm>
#include <cfloat>
#include <cmath>
#include <stdexcept>
#include <thread>

namespace hk {
namespace {

template <class F>
void parallel_rows(int n, F f) {
    const int nt = std::max(1, std::min<int>((int)std::thread::hardware_concurrency(), (n + 63) / 64));
    if (nt == 1) {
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

bool is_pow2(int v) { return v && !(v & (v - 1)); }
int round_up_pow2(int v) {
    v--;
    v |= v >> 1; v |= v >> 2; v |= v >> 4; v |= v >> 8; v |= v >> 16;
    return v + 1;
}
int log2_int(uint32_t v) {
    int r = 0;
    while (v >>= 1) ++r;
    return r;
}
int mod_int(int a, int b) {
    const int r = a % b;
    return r < 0 ? r + b : r;
}
// Lanczos (src/core/MipMap.cpp:5) as the reference writes it: sin(x tau)/(x tau) * sin(x)/x
float lanczos(float x, float tau) {
    x = std::fabs(x);
    const float sa = std::sin(x * tau) / (x * tau);
    const float lz = std::sin(x) / x;
    return sa * lz;
}
struct Weight {
    int first;
    float w[4];
};
// MipMap::GetResampleWeights :386
std::vector<Weight> resample_weights(int old_n, int new_n) {
    std::vector<Weight> W((size_t)new_n);
    const float fw = 2.0f;
    for (int i = 0; i < new_n; ++i) {
        const float center = ((float)i + 0.5f) * (float)old_n / (float)new_n;
        W[i].first = (int)std::floor((center - fw) + 0.5f);
        for (int j = 0; j < 4; ++j) W[i].w[j] = lanczos(((float)(W[i].first + j) + 0.5f - center) / fw, 2.0f);
        const float inv = 1.0f / (((W[i].w[0] + W[i].w[1]) + W[i].w[2]) + W[i].w[3]);
        for (int j = 0; j < 4; ++j) W[i].w[j] *= inv;
    }
    return W;
}
int wrap_index(int x, int n, int wrap) {
    if (wrap == HK_WRAP_REPEAT) return mod_int(x, n);
    if (wrap == HK_WRAP_CLAMP) return std::min(std::max(x, 0), n - 1);
    return x;
}
float clamp_nonneg(float v) { return v < 0.0f ? 0.0f : (v > FLT_MAX ? FLT_MAX : v); }

}  // namespace

void ewa_weight_lut(float out[128]) {
    for (int i = 0; i < 128; ++i) {
        const float alpha = 2.0f, r2 = (float)i / (float)(128 - 1);
        out[i] = std::exp(-alpha * r2) - std::exp(-alpha);
    }
}

MipPyramid build_bitmap(const hk_texture_desc &d, const uint8_t *pix, int w, int h) {
    if (d.channels != 1 && d.channels != 3) throw std::invalid_argument("bitmap channel must be r (1) or rgb (3)");
    if (!pix || w <= 0 || h <= 0 || w > 32768 || h > 32768) throw std::invalid_argument("invalid bitmap size");
    if (d.filter < HK_FILTER_NEAREST || d.filter > HK_FILTER_EWA) throw std::invalid_argument("invalid filter type");
    if (d.wrap_u < HK_WRAP_REPEAT || d.wrap_u > HK_WRAP_BLACK || d.wrap_v < HK_WRAP_REPEAT || d.wrap_v > HK_WRAP_BLACK)
        throw std::invalid_argument("invalid wrap mode");
    const int ch = d.channels;
    MipPyramid m;
    m.channels = ch;
    // LoadImageFromFile*: 8-bit -> float, GammaCorrect (include/core/Common.hpp:982),
    // rows flipped; the average runs x-major like the reference's loop
    const float inv255 = 1.0f / 255.0f, inv_gamma = 1.0f / d.gamma;
    std::vector<float> t((size_t)w * h * ch);
    parallel_rows(h, [&](int y) {
        for (int x = 0; x < w; ++x)
            for (int c = 0; c < ch; ++c) {
                float v = (float)pix[((size_t)y * w + x) * ch + c] * inv255;
                v = inv_gamma == 1.0f ? v : std::pow(v, inv_gamma);
                t[((size_t)(h - 1 - y) * w + x) * ch + c] = v;
            }
    });
    float avg[3] = {0, 0, 0};
    for (int x = 0; x < w; ++x)
        for (int y = 0; y < h; ++y)
            for (int c = 0; c < ch; ++c) avg[c] += t[((size_t)(h - 1 - y) * w + x) * ch + c];
    for (int c = 0; c < 3; ++c) m.avg[c] = (ch == 1 ? avg[0] : avg[c]) / (float)(w * h);

    int W = w, H = h;
    std::vector<float> l0;
    if (!is_pow2(w) || !is_pow2(h)) {
        W = round_up_pow2(w);
        H = round_up_pow2(h);
        const std::vector<Weight> uw = resample_weights(w, W), vw = resample_weights(h, H);
        l0.assign((size_t)W * H * ch, 0.0f);
        parallel_rows(h, [&](int v) {
            for (int u = 0; u < W; ++u)
                for (int c = 0; c < ch; ++c) {
                    float acc = 0.0f;
                    for (int j = 0; j < 4; ++j) {
                        const int ou = wrap_index(uw[u].first + j, w, d.wrap_u);
                        if (ou >= 0 && ou < w) acc += uw[u].w[j] * t[((size_t)v * w + ou) * ch + c];
                    }
                    l0[((size_t)v * W + u) * ch + c] = acc;
                }
        });
        parallel_rows(W, [&](int u) {
            std::vector<float> col((size_t)H * ch);
            for (int v = 0; v < H; ++v)
                for (int c = 0; c < ch; ++c) {
                    float acc = 0.0f;
                    for (int j = 0; j < 4; ++j) {
                        const int ov = wrap_index(vw[v].first + j, h, d.wrap_v);
                        if (ov >= 0 && ov < h) acc += vw[v].w[j] * l0[((size_t)ov * W + u) * ch + c];
                    }
                    col[(size_t)v * ch + c] = acc;
                }
            for (int v = 0; v < H; ++v)
                for (int c = 0; c < ch; ++c) l0[((size_t)v * W + u) * ch + c] = clamp_nonneg(col[(size_t)v * ch + c]);
        });
    } else {
        l0 = std::move(t);
    }
    m.lw = log2_int((uint32_t)W);
    m.lh = log2_int((uint32_t)H);
    m.levels = 1 + log2_int((uint32_t)std::max(W, H));
    m.lv.resize((size_t)m.levels);
    m.lv[0] = std::move(l0);
    const bool black = d.wrap_u == HK_WRAP_BLACK || d.wrap_v == HK_WRAP_BLACK;
    for (int i = 1; i < m.levels; ++i) {
        const int pw = std::max(1, W >> (i - 1)), ph = std::max(1, H >> (i - 1));
        const int ur = std::max(1, pw / 2), vr = std::max(1, ph / 2);
        const std::vector<float> &P = m.lv[(size_t)i - 1];
        std::vector<float> &L = m.lv[(size_t)i];
        L.assign((size_t)ur * vr * ch, 0.0f);
        // MipMap::Texel :244 -- black outside the level and everywhere with a "black" wrap mode
        auto texel = [&](int x, int y, int c) {
            if (black || x < 0 || x >= pw || y < 0 || y >= ph) return 0.0f;
            return P[((size_t)y * pw + x) * ch + c];
        };
        parallel_rows(vr, [&](int v) {
            for (int u = 0; u < ur; ++u)
                for (int c = 0; c < ch; ++c)
                    L[((size_t)v * ur + u) * ch + c] =
                        0.25f * (((texel(2 * u, 2 * v, c) + texel(2 * u + 1, 2 * v, c)) + texel(2 * u, 2 * v + 1, c)) +
                                 texel(2 * u + 1, 2 * v + 1, c));
        });
    }
    return m;
}

}  // namespace hk
