// Host-side construction of bitmap textures: LoadImageFromFileR / RGB
// (src/core/Texture.cpp:12, :74) after the decode, and the MipMap<T>
// constructor (include/core/MipMap.hpp:67) -- Lanczos resampling to
// power-of-two sizes, then the 2x2 box pyramid.  The device reads the levels
// (hk_bsdf.cuh, mip_*); this file builds them once per texture.
#pragma once
#include <cstdint>
#include <vector>

#include "../../include/hikari_b200.h"

namespace hk {

struct MipPyramid {
    int channels = 3;                      // 1 (r) or 3 (rgb)
    int levels = 0, lw = 0, lh = 0;        // level 0 is 2^lw x 2^lh
    float avg[3] = {0, 0, 0};              // BitmapTexture::GetAverage
    std::vector<std::vector<float>> lv;    // per level, `channels` floats per texel, row-major from v = 0
};

// Throws std::invalid_argument on a bad description or size.
MipPyramid build_bitmap(const hk_texture_desc &d, const uint8_t *pixels, int width, int height);

// MipMap::s_WeightLut (include/core/MipMap.hpp:229): exp(-2 r2) - exp(-2) at r2 = i / 127.
void ewa_weight_lut(float out[128]);

}  // namespace hk
