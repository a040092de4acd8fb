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
#include <string>
#include <vector>

#include "gradients.h"
#include "gvfile.h"
#include "terrain.h"

namespace vv {

constexpr uint32_t kBrickResidentBit = 0x80000000u;  // Node::setBrickIsOnGpuFlag
constexpr uint32_t kConstantBit = 0x40000000u;       // Node::setNodeTypeFlag(CONSTANT)
constexpr uint32_t kNoParent = 0xFFFFFFFFu;

inline uint32_t pack10(uint32_t x, uint32_t y, uint32_t z) { return (x << 20) | (y << 10) | z; }

// The nodes of one tree level in build order: cell (i,j,k), parent (index
// in the previous level), and the classification (constant flag and value).
struct TreeLevel {
    std::vector<uint16_t> i, j, k;
    std::vector<uint32_t> parent;  // kNoParent at the root level
    std::vector<uint8_t> isc;
    std::vector<uint32_t> cval;
    size_t size() const { return i.size(); }
};

class GigaVoxelsOctTree {
public:
    // GigaVoxelsOctTree::build for a terrain volume.  collapse = true makes
    // constant nodes leaves (the trees the reference reads from .gvx files);
    // false subdivides every node down to the leaf level as the raw-volume
    // build does.
    static std::unique_ptr<GigaVoxelsOctTree> build(std::shared_ptr<const TerrainVolume> vol,
                                                    bool collapse);
    // The same from classified levels computed elsewhere (the GPU builder):
    // level d+1 holds the 8 children of every node of level d that has
    // children (every node, or the non-constant ones with collapse), in the
    // order of their parents.
    static std::unique_ptr<GigaVoxelsOctTree> from_levels(std::shared_ptr<const TerrainVolume> vol,
                                                          std::vector<TreeLevel>&& levels, bool collapse);
    // GigaVoxelsReader::LoadOctTreeFile (GigaVoxelsReader.cpp:541-563) from
    // the records read_gvx produced.  Node::setConstantValue
    // (GigaVoxelsOctTree.cpp:1611-1621) computes a constant node's colour
    // but never stores it, so the reference renders constant nodes of a
    // .gvx as transparent black: constant_colors = false keeps that,
    // true stores the colour in word1 as the in-memory build does.
    static std::unique_ptr<GigaVoxelsOctTree> from_gvx(GvxFile&& f, bool constant_colors);
    // The tree as .gvx/.gvb files in dir (the offline voxelizer's layout).
    // A terrain tree writes 10^3 bricks with a 1-voxel border and, when
    // gradients is set and the tree is at most 6 levels deep, its
    // gradients; a file tree writes back what it read.
    bool save_gvx(const std::string& dir, bool gradients, std::string& err) const;

    int depth() const { return depth_; }                // L
    // Voxels per axis the ray step is derived from: 8 << L for the terrain,
    // the largest VolumeSize of a file tree (GigaVoxelsReader.cpp:430-440).
    int leaf_dim() const { return leaf_dim_; }
    bool has_volume() const { return vol_ != nullptr; }
    bool file_backed() const { return file_ != nullptr; }
    const GvxHeader* file_header() const { return file_ ? &file_->h : nullptr; }
    // Brick store of a file tree: brick b's stored texels at the origin of a
    // 10^3 RGBA8 block (1000 words from 1000 b), zero elsewhere.
    size_t file_brick_count() const { return file_ ? file_->border.size() / 3 : 0; }
    const uint32_t* file_texels() const { return file_ ? file_->texels.data() : nullptr; }
    bool file_has_normals() const { return file_ && !file_->normals.empty(); }
    int32_t file_brick(uint32_t n) const { return file_ ? file_->brick_of[n] : -1; }
    // The node's 8^3 voxels start `border` texels into its slot: the brick
    // pointer is slot origin + border (BrickPool::uploadBrick,
    // GigaVoxelsBrickPool.cpp:800-808); (1,1,1) for every terrain brick.
    void brick_border(uint32_t n, uint32_t b[3]) const {
        const int32_t k = file_ ? file_->brick_of[n] : -1;
        for (int a = 0; a < 3; ++a) b[a] = k < 0 ? 1u : file_->border[3 * (size_t)k + a];
    }
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
    // Start loading node n's records into the cache (the page-request
    // service walks nodes in request order, far apart in these arrays).
    void prefetch(uint32_t n) const {
        __builtin_prefetch(&parent_[n]);
        __builtin_prefetch(&word0_[n]);
        __builtin_prefetch(&level_[n]);
        __builtin_prefetch(&ci_[n]);
        __builtin_prefetch(&cj_[n]);
        __builtin_prefetch(&ck_[n]);
    }
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
    // Node-pool grid dimensions for num_nodes records
    // (OctTreeNodePool::create3DTexture, GigaVoxelsOctTreeNodePool.cpp:98-116).
    void set_pool_dim(size_t num_nodes);
    uint32_t child_pointer(size_t block) const;

    struct FileStore {
        GvxHeader h;
        std::vector<uint32_t> texels;       // 1000 RGBA8 per brick
        std::vector<uint32_t> normals;      // 1000 per brick: unsigned x, y, z bytes (or empty)
        std::vector<uint8_t> border, dims;  // 3 per brick
        std::vector<int32_t> brick_of;      // per node: brick, -1 none
        std::vector<int32_t> brick_index;   // per node: Brick attribute (index in its level)
        std::vector<uint32_t> color;        // per node: constant colour as read
        std::vector<uint8_t> type;          // per node: GvxNodeType
        std::vector<int32_t> mip;           // 3 per node: MipMapX..
    };
    std::unique_ptr<FileStore> file_;
    int leaf_dim_ = 8;
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

// The terrain volume and classified tree levels of GigaVoxelsOctTree::build
// computed on the current CUDA device (builder.cu); returns an error message,
// empty on success.
std::string gpu_build_terrain(const TerrainParams& p, bool collapse, std::shared_ptr<TerrainVolume>& vol_out,
                              std::vector<TreeLevel>& levels);

// Node::computeNodeType (GigaVoxelsOctTree.cpp:1490-1609) for the node at
// level d with index (i,j,k): returns true if constant and its RGBA8 value.
bool classify_node(const TerrainVolume& vol, int d, int i, int j, int k, uint32_t& const_value);

// Store one normalized value v/255 (v in [0,255]) as the given format.
void convert_texel(uint32_t rgba8, int fmt, void* dst);
size_t texel_bytes(int fmt);
// Bytes of one stored brick in fmt (1000 texels, or 90 blocks for DXT5 /
// DXT1); 0 for an unknown format.
size_t brick_bytes(int fmt);
uint16_t float_to_half_rn(float f);
uint16_t float_to_bf16_rn(float f);

}  // namespace vv
