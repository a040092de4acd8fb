// dxt.h - S3TC block compression of bricks: DXT5 colour (RGBA) and DXT1
// gradient (RGB) brick pools, host and device.
//
// The reference pages compressed bricks into GL_COMPRESSED_RGBA_S3TC_DXT5
// colour and GL_COMPRESSED_RGB_S3TC_DXT1 gradient textures
// (GigaVoxelsRenderer.cpp:235-258, BrickPool::initSpecial
// GigaVoxelsBrickPool.cpp:153-250): 4x4 texel blocks in every z slice of the
// 3D texture.  A brick-pool slot here holds a brick's 10 z slices of 10x10
// texels padded to 12x12, i.e. 3x3 blocks per slice: 90 blocks per slot
// (1440 bytes DXT5, 720 bytes DXT1, against 4000 for RGBA8).  Texel (x,y,z)
// of slot s is texel (x&3, y&3) of block s*90 + z*9 + (y>>2)*3 + (x>>2); the
// padding texels are never sampled.
//
// Block layout (EXT_texture_compression_s3tc): DXT1 = colour0, colour1
// (RGB565, little endian) and 32 bits of 2-bit codes, texel t = 4*y + x at
// bits 2t; DXT5 = alpha0, alpha1 (bytes) and 48 bits of 3-bit codes (texel t
// at bits 3t), then a DXT1 colour block decoded in four-colour mode.  The
// extension leaves the expansion to 8 bits and the interpolation rounding to
// the implementation; this library fixes them (the kernels and the checks
// use exactly this decode):
//   5 -> 8 bits: (c << 3) | (c >> 2); 6 -> 8 bits: (c << 2) | (c >> 4)
//   colour codes 2, 3: (2 c0 + c1 + 1) / 3, (c0 + 2 c1 + 1) / 3 per channel
//     (DXT1 with colour0 <= colour1: code 2 = (c0 + c1 + 1) / 2, code 3 = 0)
//   alpha, alpha0 > alpha1: code k in 2..7 = ((8-k) a0 + (k-1) a1 + 3) / 7
//   alpha, alpha0 <= alpha1: code k in 2..5 = ((6-k) a0 + (k-1) a1 + 2) / 5,
//     code 6 = 0, code 7 = 255
// The encoder (a range fit): colour endpoints are the per-channel maxima and
// minima of the block's brick texels rounded to 565, alpha endpoints the
// largest and smallest alpha, and each texel takes the code whose decoded
// value is nearest (squared RGB distance; absolute alpha difference; the
// lowest code on ties).  A texel of (0,0,0,0) always decodes to (0,0,0,0).
#pragma once

#include <cstdint>

#if defined(__CUDACC__)
#define VV_HD __host__ __device__ __forceinline__
#else
#define VV_HD inline
#endif

namespace vv {
namespace dxt {

constexpr int kBlocksPerSlot = 90;       // 10 slices x 3 x 3 blocks
constexpr int kDxt5SlotBytes = 90 * 16;  // 1440
constexpr int kDxt1SlotBytes = 90 * 8;   // 720

// Block index within its slot and texel within its block of brick texel
// (x,y,z), each in 0..9.
VV_HD int block_of(int x, int y, int z) { return z * 9 + (y >> 2) * 3 + (x >> 2); }
VV_HD int texel_of(int x, int y) { return ((y & 3) << 2) | (x & 3); }

VV_HD uint32_t expand5(uint32_t c) { return (c << 3) | (c >> 2); }
VV_HD uint32_t expand6(uint32_t c) { return (c << 2) | (c >> 4); }

// The four colours of a colour block, RGB888 (r | g << 8 | b << 16).
VV_HD void colour_palette(uint32_t c0, uint32_t c1, bool four, uint32_t pal[4]) {
    const uint32_t r0 = expand5(c0 >> 11), g0 = expand6((c0 >> 5) & 63u), b0 = expand5(c0 & 31u);
    const uint32_t r1 = expand5(c1 >> 11), g1 = expand6((c1 >> 5) & 63u), b1 = expand5(c1 & 31u);
    pal[0] = r0 | (g0 << 8) | (b0 << 16);
    pal[1] = r1 | (g1 << 8) | (b1 << 16);
    if (four) {
        pal[2] = ((2 * r0 + r1 + 1) / 3) | (((2 * g0 + g1 + 1) / 3) << 8) | (((2 * b0 + b1 + 1) / 3) << 16);
        pal[3] = ((r0 + 2 * r1 + 1) / 3) | (((g0 + 2 * g1 + 1) / 3) << 8) | (((b0 + 2 * b1 + 1) / 3) << 16);
    } else {
        pal[2] = ((r0 + r1 + 1) / 2) | (((g0 + g1 + 1) / 2) << 8) | (((b0 + b1 + 1) / 2) << 16);
        pal[3] = 0u;
    }
}

// Alpha code k of an alpha block.
VV_HD uint32_t alpha_value(uint32_t a0, uint32_t a1, uint32_t k) {
    if (k == 0) return a0;
    if (k == 1) return a1;
    if (a0 > a1) return ((8 - k) * a0 + (k - 1) * a1 + 3) / 7;
    if (k == 6) return 0u;
    if (k == 7) return 255u;
    return ((6 - k) * a0 + (k - 1) * a1 + 2) / 5;
}

// Texel t of a DXT5 block (words w[0..3], little endian) as RGBA8.
VV_HD uint32_t decode_dxt5(const uint32_t w[4], int t) {
    const uint32_t a0 = w[0] & 255u, a1 = (w[0] >> 8) & 255u;
    const uint64_t abits = ((uint64_t)(w[0] >> 16)) | ((uint64_t)w[1] << 16);
    const uint32_t ak = (uint32_t)(abits >> (3 * t)) & 7u;
    const uint32_t c0 = w[2] & 0xFFFFu, c1 = w[2] >> 16;
    const uint32_t ck = (w[3] >> (2 * t)) & 3u;
    uint32_t pal[4];
    colour_palette(c0, c1, true, pal);
    return pal[ck] | (alpha_value(a0, a1, ak) << 24);
}

// Texel t of a DXT1 block (words w[0..1]) as RGB888 (alpha 0).
VV_HD uint32_t decode_dxt1(const uint32_t w[2], int t) {
    const uint32_t c0 = w[0] & 0xFFFFu, c1 = w[0] >> 16;
    const uint32_t ck = (w[1] >> (2 * t)) & 3u;
    uint32_t pal[4];
    colour_palette(c0, c1, c0 > c1, pal);
    return pal[ck];
}

VV_HD uint32_t to565(uint32_t r, uint32_t g, uint32_t b) {
    return (((r * 31u + 127u) / 255u) << 11) | (((g * 63u + 127u) / 255u) << 5) | ((b * 31u + 127u) / 255u);
}

VV_HD uint32_t rgb_dist(uint32_t a, uint32_t b) {
    const int dr = (int)(a & 255u) - (int)(b & 255u), dg = (int)((a >> 8) & 255u) - (int)((b >> 8) & 255u),
              db = (int)((a >> 16) & 255u) - (int)((b >> 16) & 255u);
    return (uint32_t)(dr * dr + dg * dg + db * db);
}

// Colour endpoints and codes of the texels of `px` marked in `valid`
// (RGBA8 values, 16 texels).  four: DXT5's four-colour decode; otherwise
// DXT1's (endpoints ordered colour0 >= colour1, equal ones use code 0).
VV_HD void encode_colour(const uint32_t px[16], uint32_t valid, bool four, uint32_t& ends, uint32_t& codes) {
    uint32_t lo[3] = {255u, 255u, 255u}, hi[3] = {0u, 0u, 0u};
    for (int t = 0; t < 16; ++t) {
        if (!((valid >> t) & 1u)) continue;
        for (int c = 0; c < 3; ++c) {
            const uint32_t v = (px[t] >> (8 * c)) & 255u;
            lo[c] = v < lo[c] ? v : lo[c];
            hi[c] = v > hi[c] ? v : hi[c];
        }
    }
    if (!valid) lo[0] = lo[1] = lo[2] = 0u;
    uint32_t c0 = to565(hi[0], hi[1], hi[2]), c1 = to565(lo[0], lo[1], lo[2]);
    if (!four && c0 < c1) {  // DXT1: keep the four-colour mode
        const uint32_t t = c0;
        c0 = c1;
        c1 = t;
    }
    uint32_t pal[4];
    colour_palette(c0, c1, four || c0 > c1, pal);
    codes = 0u;
    for (int t = 0; t < 16; ++t) {
        if (!((valid >> t) & 1u)) continue;
        uint32_t best = 0u, bd = rgb_dist(px[t], pal[0]);
        for (uint32_t k = 1; k < 4; ++k) {
            const uint32_t d = rgb_dist(px[t], pal[k]);
            if (d < bd) {
                bd = d;
                best = k;
            }
        }
        codes |= best << (2 * t);
    }
    ends = c0 | (c1 << 16);
}

// One DXT5 block of 16 RGBA8 texels (`valid`: the brick texels among them).
VV_HD void encode_dxt5(const uint32_t px[16], uint32_t valid, uint32_t out[4]) {
    uint32_t lo = 255u, hi = 0u;
    for (int t = 0; t < 16; ++t) {
        if (!((valid >> t) & 1u)) continue;
        const uint32_t a = px[t] >> 24;
        lo = a < lo ? a : lo;
        hi = a > hi ? a : hi;
    }
    if (!valid) lo = hi = 0u;
    uint64_t abits = 0;
    for (int t = 0; t < 16; ++t) {
        if (!((valid >> t) & 1u)) continue;
        const uint32_t a = px[t] >> 24;
        uint32_t best = 0u, bd = a > hi ? a - hi : hi - a;
        for (uint32_t k = 1; k < 8; ++k) {
            const uint32_t v = alpha_value(hi, lo, k);
            const uint32_t d = a > v ? a - v : v - a;
            if (d < bd) {
                bd = d;
                best = k;
            }
        }
        abits |= (uint64_t)best << (3 * t);
    }
    out[0] = hi | (lo << 8) | ((uint32_t)abits << 16);
    out[1] = (uint32_t)(abits >> 16);
    encode_colour(px, valid, true, out[2], out[3]);
}

// One DXT1 block of 16 RGB texels.
VV_HD void encode_dxt1(const uint32_t px[16], uint32_t valid, uint32_t out[2]) {
    encode_colour(px, valid, false, out[0], out[1]);
}

// The texels of block b of a 10^3 RGBA8 brick (x fastest) and which of them
// lie in the brick.
VV_HD void gather_block(const uint32_t* brick, int b, uint32_t px[16], uint32_t& valid) {
    const int z = b / 9, by = (b / 3) % 3, bx = b % 3;
    valid = 0u;
    for (int t = 0; t < 16; ++t) {
        const int x = bx * 4 + (t & 3), y = by * 4 + (t >> 2);
        if (x < 10 && y < 10) {
            px[t] = brick[(z * 10 + y) * 10 + x];
            valid |= 1u << t;
        } else {
            px[t] = 0u;
        }
    }
}

}  // namespace dxt
}  // namespace vv
