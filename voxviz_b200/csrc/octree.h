// octree.h - host data model of one GigaVoxels octree (N^3-tree, N = 2).
//
// Mirrors gv::GigaVoxelsOctTree + gv::OctTreeNodePool
// (VoxViz/GigaVoxels/GigaVoxelsOctTree.h:34-516, GigaVoxelsOctTreeNodePool.h:28-44):
// nodes are allocated in blocks of 8 children in depth-first pre-order
// (BuildOctTree / BuildOctTreeChildren, GigaVoxelsOctTree.cpp:1196-1306),
// each block occupies a 2x2x2 cell of the node-pool grid
// (OctTreeNodePool::create3DTexture, GigaVoxelsOctTreeNodePool.cpp:90-223) and
// each node is the two-word record of Node::GpuDataStruct.
#pragma once

#include <cstdint>
#include <memory>
#include <mutex>
#include <vector>

#include "gradients.h"
#include "terrain.h"

namespace vv {

constexpr uint32_t kBrickResidentBit = 0x80000000u;  // Node::setBrickIsOnGpuFlag
constexpr uint32_t kConstantBit = 0x40000000u;       // Node::setNodeTypeFlag(CONSTANT)
constexpr uint32_t kNoParent = 0xFFFFFFFFu;

inline uint32_t pack10(uint32_t x, uint32_t y, uint32_t z) { return (x << 20) | (y << 10) | z; }

class GigaVoxelsOctTree {
public:
    // GigaVoxelsOctTree::build for a terrain volume.  collapse = true makes
    // constant nodes leaves (the trees the reference reads from .gvx files);
    // false subdivides every node down to the leaf level as the raw-volume
    // build does.
    static std::unique_ptr<GigaVoxelsOctTree> build(std::shared_ptr<const TerrainVolume> vol,
                                                    bool collapse);

    int depth() const { return depth_; }                // L
    size_t node_count() const { return level_.size(); } // 8 per block
    const int* pool_dim() const { return pool_dim_; }
    const TerrainVolume& volume() const { return *vol_; }

    // Node index <-> node-pool grid position.
    void grid_of(uint32_t n, uint32_t& x, uint32_t& y, uint32_t& z) const;
    // Returns kNoParent if (x,y,z) is outside the pool.
    uint32_t index_of(uint32_t x, uint32_t y, uint32_t z) const;

    int level(uint32_t n) const { return level_[n]; }   // -1 = unused slot
    bool is_constant(uint32_t n) const { return (word0_[n] & kConstantBit) != 0; }
    bool has_children(uint32_t n) const { return (word0_[n] & 0x3FFFFFFFu & ~kConstantBit) != 0; }
    uint32_t parent(uint32_t n) const { return parent_[n]; }
    void origin(uint32_t n, int& i, int& j, int& k) const {
        i = ci_[n];
        j = cj_[n];
        k = ck_[n];
    }
    uint32_t word0(uint32_t n) const { return word0_[n]; }
    uint32_t word1(uint32_t n) const { return word1_[n]; }
    size_t nonconst_count() const { return nonconst_; }

    // Words in reference texture order (2 per grid cell), no brick resident.
    void words_grid(uint32_t* out) const;

    // Node::copyMipMapToBrick (GigaVoxelsOctTree.cpp:1428-1488): the 10^3
    // stored brick of node n, texels outside the volume are transparent black.
    void produce_brick_rgba8(uint32_t n, uint32_t* out) const;
    // Same, converted to fmt (vv_fmt) texels.
    void produce_brick(uint32_t n, int fmt, void* out) const;
    // The gradient brick of node n (gradients.h), fmt VV_FMT_FP32 (x, y, z,
    // 0) or VV_FMT_RGBA8 (unsigned mapping).  Builds the dense gradient
    // pyramid on first use; false when the tree is too deep for it.
    bool produce_gradient_brick(uint32_t n, int fmt, void* out) const;

private:
    mutable std::unique_ptr<GradientPyramid> grads_;
    mutable std::mutex grads_mu_;
    std::shared_ptr<const TerrainVolume> vol_;
    int depth_ = 0;
    int pool_dim_[3] = {0, 0, 0};
    std::vector<int8_t> level_;
    std::vector<uint16_t> ci_, cj_, ck_;
    std::vector<uint32_t> parent_;
    std::vector<uint32_t> word0_, word1_;
    size_t nonconst_ = 0;
};

// Node::computeNodeType (GigaVoxelsOctTree.cpp:1490-1609) for the node at
// level d with index (i,j,k): returns true if constant and its RGBA8 value.
bool classify_node(const TerrainVolume& vol, int d, int i, int j, int k, uint32_t& const_value);

// Store one normalized value v/255 (v in [0,255]) as the given format.
void convert_texel(uint32_t rgba8, int fmt, void* dst);
size_t texel_bytes(int fmt);
uint16_t float_to_half_rn(float f);
uint16_t float_to_bf16_rn(float f);

}  // namespace vv
