// terrain.h - synthetic fBm terrain and its sparse mip pyramid.
//
// The reference builds a dense RGBA8 mip pyramid of the whole volume
// (GenerateMipMaps / GenerateMipMap / GetBoxFilterAverage,
// VoxViz/GigaVoxels/GigaVoxelsOctTree.cpp:809-1194).  A 8192^3 volume does
// not fit that way, so every level here is stored as columns: for column
// (x,y) of mip level m the voxels below `s` are solid with the colour of
// their height band, the next `r` voxels are stored explicitly and
// everything above is transparent black.  The values are exactly those of
// the reference cascade: level m+1 is the 2x2x2 box average of level m with
// the reference's round-half-up (floor(sum * (1/8) + 0.5)).
#pragma once

#include <cstddef>
#include <cstdint>
#include <vector>

namespace vv {

struct TerrainParams {
    uint32_t seed = 1;
    int depth = 5;          // leaf level L; volume dim = 8 << L
    int octaves = 4;
    float lacunarity = 2.0f;
    float gain = 0.5f;
    int base_cells = 4;
    int threads = 0;
};

// 2D fBm value noise in [0,1] at (u,v) in [0,1]^2 (float32 arithmetic,
// no contraction, so any IEEE implementation reproduces it bit for bit).
float fbm_height(const TerrainParams& p, float u, float v);
uint32_t lattice_hash(uint32_t x, uint32_t y, uint32_t seed);

// RGBA8 (r | g<<8 | b<<16 | a<<24) of height band b in [0,8).
uint32_t band_colour(int band);

struct MipLevel {
    int dim = 0;                  // voxels per axis at this level
    std::vector<uint16_t> s;      // per column: count of pure solid voxels
    std::vector<uint16_t> r;      // per column: explicit run length
    std::vector<uint64_t> off;    // per column: offset of the run in data
    std::vector<uint32_t> data;   // explicit RGBA8 voxels
};

class TerrainVolume {
public:
    explicit TerrainVolume(const TerrainParams& p);
    // A volume whose heights and mip pyramid were built elsewhere (the GPU
    // builder): the same values the constructor above computes.
    TerrainVolume(const TerrainParams& p, std::vector<int32_t>&& heights, std::vector<MipLevel>&& mips);

    const TerrainParams& params() const { return p_; }
    int depth() const { return p_.depth; }
    int dim() const { return dim_; }
    int levels() const { return (int)mips_.size(); }
    const MipLevel& mip(int m) const { return mips_[m]; }
    const std::vector<int32_t>& heights() const { return heights_; }

    // RGBA8 voxel of mip level m (0 = leaf resolution).
    inline uint32_t voxel(int m, int x, int y, int z) const {
        const MipLevel& L = mips_[m];
        size_t c = (size_t)y * L.dim + x;
        int s = L.s[c];
        if (z < s) return band_colour(((z << m) >> p_.depth) & 7);
        int r = L.r[c];
        if (z < s + r) return L.data[L.off[c] + (size_t)(z - s)];
        return 0u;
    }
    // Band of voxel z at mip level m.
    inline int band(int m, int z) const { return ((z << m) >> p_.depth) & 7; }

private:
    void build_heights();
    void build_level(int m);  // level m from level m-1

    TerrainParams p_;
    int dim_;
    std::vector<int32_t> heights_;   // dim*dim solid column counts
    std::vector<MipLevel> mips_;
};

}  // namespace vv
