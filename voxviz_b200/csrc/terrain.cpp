// terrain.cpp - fBm heightfield and the column-run mip pyramid.
#include "terrain.h"

#include <algorithm>
#include <cmath>
#include <stdexcept>

#ifdef _OPENMP
#include <omp.h>
#endif

namespace vv {

// 32-bit integer mixer for lattice values (xorshift-multiply finaliser).
uint32_t lattice_hash(uint32_t x, uint32_t y, uint32_t seed) {
    uint32_t h = seed * 0x9E3779B9u;
    h ^= x * 0x85EBCA6Bu;
    h = (h << 13) | (h >> 19);
    h ^= y * 0xC2B2AE35u;
    h ^= h >> 16;
    h *= 0x7FEB352Du;
    h ^= h >> 15;
    h *= 0x846CA68Bu;
    h ^= h >> 16;
    return h;
}

static inline float lattice_value(int32_t x, int32_t y, uint32_t seed) {
    return (float)(lattice_hash((uint32_t)x, (uint32_t)y, seed) >> 8) * (1.0f / 16777216.0f);
}

static inline float smoothstep01(float t) { return (t * t) * (3.0f - 2.0f * t); }

static float value_noise(float x, float y, uint32_t seed) {
    float fx = std::floor(x), fy = std::floor(y);
    int32_t ix = (int32_t)fx, iy = (int32_t)fy;
    float sx = smoothstep01(x - fx), sy = smoothstep01(y - fy);
    float v00 = lattice_value(ix, iy, seed);
    float v10 = lattice_value(ix + 1, iy, seed);
    float v01 = lattice_value(ix, iy + 1, seed);
    float v11 = lattice_value(ix + 1, iy + 1, seed);
    float a = v00 + (v10 - v00) * sx;
    float b = v01 + (v11 - v01) * sx;
    return a + (b - a) * sy;
}

float fbm_height(const TerrainParams& p, float u, float v) {
    float sum = 0.0f, amp = 1.0f, norm = 0.0f, freq = (float)p.base_cells;
    for (int o = 0; o < p.octaves; ++o) {
        uint32_t s = p.seed + (uint32_t)o * 0x632BE5ABu;
        sum = sum + amp * value_noise(u * freq, v * freq, s);
        norm = norm + amp;
        amp = amp * p.gain;
        freq = freq * p.lacunarity;
    }
    return sum / norm;
}

uint32_t band_colour(int band) {
    // soil, clay, sand, grass, forest, rock, scree, snow
    static const uint8_t k[8][3] = {{72, 58, 46},   {112, 84, 56},  {150, 122, 80},
                                    {92, 136, 62},  {54, 104, 48},  {118, 116, 108},
                                    {168, 166, 160}, {242, 242, 248}};
    const uint8_t* c = k[band & 7];
    return (uint32_t)c[0] | ((uint32_t)c[1] << 8) | ((uint32_t)c[2] << 16) | (255u << 24);
}

TerrainVolume::TerrainVolume(const TerrainParams& p) : p_(p) {
    if (p.depth < 0 || p.depth > 10) throw std::invalid_argument("terrain depth must be in [0,10]");
    if (p.octaves < 1 || p.octaves > 16) throw std::invalid_argument("octaves must be in [1,16]");
    dim_ = 8 << p.depth;
#ifdef _OPENMP
    if (p_.threads > 0) omp_set_num_threads(p_.threads);
#endif
    build_heights();
    mips_.resize((size_t)p.depth + 1);
    MipLevel& l0 = mips_[0];
    l0.dim = dim_;
    l0.s.resize((size_t)dim_ * dim_);
    l0.r.assign((size_t)dim_ * dim_, 0);
    l0.off.assign((size_t)dim_ * dim_, 0);
    for (size_t i = 0; i < l0.s.size(); ++i) l0.s[i] = (uint16_t)heights_[i];
    for (int m = 1; m <= p.depth; ++m) build_level(m);
}

TerrainVolume::TerrainVolume(const TerrainParams& p, std::vector<int32_t>&& heights, std::vector<MipLevel>&& mips)
    : p_(p), heights_(std::move(heights)), mips_(std::move(mips)) {
    if (p.depth < 0 || p.depth > 10) throw std::invalid_argument("terrain depth must be in [0,10]");
    dim_ = 8 << p.depth;
    if (heights_.size() != (size_t)dim_ * dim_ || mips_.size() != (size_t)p.depth + 1)
        throw std::invalid_argument("prebuilt terrain of the wrong size");
}

void TerrainVolume::build_heights() {
    const int n = dim_;
    heights_.resize((size_t)n * n);
    const float inv = 1.0f / (float)n;  // exact: n is a power of two
#pragma omp parallel for schedule(static)
    for (int y = 0; y < n; ++y) {
        for (int x = 0; x < n; ++x) {
            float h = fbm_height(p_, (float)x * inv, (float)y * inv);
            float t = h * (float)n;
            int H = (int)std::ceil(t);
            if (H < 0) H = 0;
            if (H > n) H = n;
            heights_[(size_t)y * n + x] = H;
        }
    }
}

void TerrainVolume::build_level(int m) {
    const MipLevel& P = mips_[m - 1];
    MipLevel& L = mips_[m];
    const int dp = P.dim;
    const int d = dp >> 1;
    L.dim = d;
    L.s.assign((size_t)d * d, 0);
    L.r.assign((size_t)d * d, 0);
    L.off.assign((size_t)d * d, 0);
    std::vector<std::vector<uint32_t>> rows((size_t)d);

#pragma omp parallel for schedule(dynamic, 8)
    for (int Y = 0; Y < d; ++Y) {
        std::vector<uint32_t>& out = rows[(size_t)Y];
        std::vector<uint32_t> vals;
        for (int X = 0; X < d; ++X) {
            int lo = 1 << 30, hi = 0;
            for (int j = 0; j < 2; ++j)
                for (int i = 0; i < 2; ++i) {
                    size_t c = (size_t)(2 * Y + j) * dp + (2 * X + i);
                    int s = P.s[c], e = s + P.r[c];
                    lo = std::min(lo, s);
                    hi = std::max(hi, e);
                }
            int zlo = lo >> 1, zhi = (hi + 1) >> 1;
            vals.clear();
            for (int Z = zlo; Z < zhi; ++Z) {
                uint32_t sr = 0, sg = 0, sb = 0, sa = 0;
                for (int k = 0; k < 2; ++k)
                    for (int j = 0; j < 2; ++j)
                        for (int i = 0; i < 2; ++i) {
                            uint32_t v = voxel(m - 1, 2 * X + i, 2 * Y + j, 2 * Z + k);
                            sr += v & 255u;
                            sg += (v >> 8) & 255u;
                            sb += (v >> 16) & 255u;
                            sa += v >> 24;
                        }
                // GetBoxFilterAverage: floor(sum * (1/8) + 0.5) == (sum + 4) >> 3
                uint32_t v = ((sr + 4) >> 3) | (((sg + 4) >> 3) << 8) | (((sb + 4) >> 3) << 16) |
                             (((sa + 4) >> 3) << 24);
                vals.push_back(v);
            }
            // Trim voxels whose value equals the implicit one.
            size_t b = 0, e = vals.size();
            while (b < e && vals[b] == band_colour(band(m, zlo + (int)b))) ++b;
            while (e > b && vals[e - 1] == 0u) --e;
            size_t c = (size_t)Y * d + X;
            L.s[c] = (uint16_t)(zlo + (int)b);
            L.r[c] = (uint16_t)(e - b);
            L.off[c] = out.size();  // row-local for now
            out.insert(out.end(), vals.begin() + (long)b, vals.begin() + (long)e);
        }
    }
    size_t total = 0;
    std::vector<size_t> rowoff((size_t)d);
    for (int Y = 0; Y < d; ++Y) {
        rowoff[(size_t)Y] = total;
        total += rows[(size_t)Y].size();
    }
    L.data.resize(total);
#pragma omp parallel for schedule(static)
    for (int Y = 0; Y < d; ++Y) {
        std::copy(rows[(size_t)Y].begin(), rows[(size_t)Y].end(), L.data.begin() + (long)rowoff[(size_t)Y]);
        for (int X = 0; X < d; ++X) L.off[(size_t)Y * d + X] += rowoff[(size_t)Y];
    }
}

}  // namespace vv
