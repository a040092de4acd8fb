// gvfile.h - the GigaVoxels dataset files: .gvx (XML octree), .gvb (binary
// bricks, one file per tree level) and .gvp (XML index of paged trees).
//
// Reader: GigaVoxelsReader (VoxViz/GigaVoxels/GigaVoxelsReader.cpp:35-101
// LoadGVP, :106-221 LoadBinaryBricks, :277-371 LoadOctTreeNode, :373-514
// LoadGVX).  Writer: the layout of the offline voxelizer
// (VoxViz/Voxelizer/Voxelizer/Voxelizer.cu:2840-3058 WriteOctTreeNode /
// writeOctTree, VoxelBrickWriter.cu:71-110 startBricksFile, :509-590
// WriteUByteBinaryBrick, :726-818 WriteBinaryBrick).
//
// Node order: the reader allocates node blocks of 8 in depth-first pre-order
// (a node's child block right before its children are read,
// OctTreeNodePool::allocateChildNodeBlock), the order the node pool keeps.
#pragma once

#include <cstdint>
#include <functional>
#include <string>
#include <vector>

namespace vv {

enum GvxNodeType : uint8_t { kGvxNonConst = 0, kGvxConst = 1, kGvxLeafConst = 2 };

struct GvxHeader {
    int max_depth = 0;            // MaxDepth: tree levels (depths 0 .. MaxDepth-1)
    float origin[3] = {0.f, 0.f, 0.f};   // X, Y, Z
    float delta[3] = {0.f, 0.f, 0.f};    // DeltaX.. : voxel size
    int volume_size[3] = {0, 0, 0};      // VolumeXSize..
    int brick_size[3] = {0, 0, 0};       // BrickXSize..
    bool binary = false;
    bool compressed = false;
};

struct GvxNode {
    int8_t level = -1;            // -1: an unused record of the root block
    uint8_t type = kGvxNonConst;
    int32_t mip[3] = {0, 0, 0};   // MipMapX.. : voxel origin in its mip level
    uint32_t parent = 0xFFFFFFFFu;
    int32_t child_block = -1;     // block index of the children, -1 none
    uint32_t color = 0;           // constant value as RGBA8 (setConstantValue's conversion)
    int32_t brick = -1;           // Brick attribute: index in its level's .gvb
};

// One brick of a .gvb file (uncompressed): dims include the border voxels,
// colours RGBA8 and gradients as unsigned bytes (x, y, z), x fastest.
struct GvxBrick {
    uint8_t dims[3] = {0, 0, 0};
    uint8_t border[3] = {0, 0, 0};
    std::vector<uint8_t> colors;   // 4 * dims product
    std::vector<uint8_t> normals;  // 3 * dims product, empty when not loaded
};

struct GvxFile {
    GvxHeader h;
    std::vector<GvxNode> nodes;                 // node-pool order, 8 per block
    std::vector<std::vector<GvxBrick>> bricks;  // per level, by brick index
};

// LoadGVX + LoadBinaryBricks.  load_normals = false skips the gradient
// payloads (GigaVoxelsReader::SetLoadNormals).  Returns false with a message
// on any error the reference rejects, and on the inputs this library cannot
// render (brick size other than 8, DXT-compressed bricks, trees deeper than
// 11 levels, brick indices with gaps or repeats).  Returns VV_OK, VV_ERR_IO
// (missing or malformed input, or one the reference rejects) or VV_ERR_ARG
// (content this library does not render), with the message in err.
int read_gvx(const std::string& path, bool load_normals, GvxFile& out, std::string& err);

// tree.gvx and voxels_<level>.gvb for every level that has bricks, in dir.
bool write_gvx(const std::string& dir, const GvxFile& f, std::string& err);
// The same with the bricks made one at a time by `source` (level, index):
// bricks_per_level[l] of them for level l; f.bricks is not used.  A brick
// without gradients is written with the zero vector (128, 128, 128).
using GvxBrickSource = std::function<void(size_t level, size_t index, GvxBrick& out)>;
bool write_gvx(const std::string& dir, const GvxFile& f, const std::vector<size_t>& bricks_per_level,
               const GvxBrickSource& source, std::string& err);

// The float a .gvx colour attribute needs so that the reader's conversion
// (unsigned char)(value * 255.0f) gives back v.
float gvx_color_value(uint32_t v);
// setConstantValue's conversion of one attribute value (truncation, clamped
// to [0, 255]).
uint32_t gvx_color_byte(float value);

struct GvpTile {
    float center[3] = {0.f, 0.f, 0.f};
    float radius = 0.f;
    float size_meters[3] = {0.f, 0.f, 0.f};
    std::string tree_file;  // path of the tile's .gvx (the .gvp's directory joined)
};

struct GvpFile {
    bool compressed = false;
    int brick_size[3] = {0, 0, 0};
    std::vector<GvpTile> tiles;
    float sphere_center[3] = {0.f, 0.f, 0.f};  // bounding sphere of all tiles
    double sphere_radius = -1.0;
};

// LoadGVP: the paged-tree index (the tiles are loaded on demand).
int read_gvp(const std::string& path, GvpFile& out, std::string& err);
bool write_gvp(const std::string& path, const GvpFile& f, std::string& err);

}  // namespace vv
