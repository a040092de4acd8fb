/*
 * voxviz_b200.hpp - the reference's host data-model API as C++ classes over
 * the C ABI of voxviz_b200.h (header-only; link libvoxviz_b200.so).
 *
 * The reference's renderer calls a C++ data model: GigaVoxelsOctTree
 * (VoxViz/GigaVoxels/GigaVoxelsOctTree.h:396-516), OctTreeNodePool
 * (GigaVoxelsOctTreeNodePool.h:28-44) and the BrickPool singleton
 * (GigaVoxelsBrickPool.h:136-191), and is itself a vox::Renderer plugin
 * (VoxViz/VoxVizCore/Renderer.h:64-79).  The classes below keep those names
 * and call semantics in namespace vv, with device pools owned by a vv_ctx
 * instead of GL textures:
 *
 *   GigaVoxelsOctTree  build / LoadOctTreeFile, getDepth, getBrickDimension,
 *                      getRayStepSize, getRootNode, node records
 *   OctTreeNodePool    allocateChildNodeBlock, getChild, create3DTexture,
 *                      get3DTextureDimensions, addToUpdateList, update
 *   BrickPool          instance, init, initSpecial, notifyUsed,
 *                      notifyDeleted, update, getUploadRequestList, plus
 *                      processNodeUsageList (NodeUsageListProcessor::run)
 *   GigaVoxelsRenderer the plugin frame protocol: init, draw, postDraw,
 *                      update, shutdown over vv_renderer_*
 *
 * Errors throw vv::Error (code + message); the C ABI itself never throws.
 */
#ifndef VOXVIZ_B200_HPP
#define VOXVIZ_B200_HPP

#include <cmath>
#include <cstdint>
#include <list>
#include <stdexcept>
#include <string>
#include <unordered_map>
#include <unordered_set>
#include <vector>

#include "voxviz_b200.h"

namespace vv {

class Error : public std::runtime_error {
public:
    Error(int code, const std::string& what) : std::runtime_error(what), code_(code) {}
    int code() const { return code_; }

private:
    int code_;
};

inline void check(int rc, const char* what, vv_ctx* ctx = nullptr) {
    if (rc == VV_OK) return;
    std::string msg = std::string(what) + ": " + vv_status_string(rc);
    const char* e = vv_last_error(ctx);
    if (e && *e) msg += std::string(" (") + e + ")";
    throw Error(rc, msg);
}

constexpr uint32_t kResidentBit = 0x80000000u;  // GpuDataStruct word0 bit 31
constexpr uint32_t kConstantBit = 0x40000000u;  // word0 bit 30

// ---------------------------------------------------------------------------
// GigaVoxelsOctTree: the octree of a dataset (terrain build or .gvx file).
class GigaVoxelsOctTree {
public:
    // GigaVoxelsOctTree::build (GigaVoxelsOctTree.cpp:1656-1701) over the
    // synthetic terrain.
    static GigaVoxelsOctTree build(const vv_terrain_desc& d) {
        vv_octree* t = nullptr;
        check(vv_octree_build_terrain(&d, &t), "GigaVoxelsOctTree::build");
        return GigaVoxelsOctTree(t);
    }
    // GigaVoxelsReader::LoadOctTreeFile (GigaVoxelsReader.cpp:373-514).
    static GigaVoxelsOctTree LoadOctTreeFile(const std::string& gvx, int32_t flags = 0) {
        vv_octree* t = nullptr;
        check(vv_octree_load_gvx(gvx.c_str(), flags, &t), "GigaVoxelsOctTree::LoadOctTreeFile");
        return GigaVoxelsOctTree(t);
    }
    GigaVoxelsOctTree(GigaVoxelsOctTree&& o) noexcept : t_(o.t_), info_(o.info_) { o.t_ = nullptr; }
    GigaVoxelsOctTree& operator=(GigaVoxelsOctTree&& o) noexcept {
        if (this != &o) {
            if (t_) vv_octree_destroy(t_);
            t_ = o.t_;
            info_ = o.info_;
            o.t_ = nullptr;
        }
        return *this;
    }
    GigaVoxelsOctTree(const GigaVoxelsOctTree&) = delete;
    GigaVoxelsOctTree& operator=(const GigaVoxelsOctTree&) = delete;
    ~GigaVoxelsOctTree() {
        if (t_) vv_octree_destroy(t_);
    }

    vv_octree* handle() const { return t_; }
    const vv_octree_info& info() const { return info_; }
    // getDepth: the number of levels (L + 1; GigaVoxelsOctTree.cpp:1668).
    int getDepth() const { return info_.depth + 1; }
    void getBrickDimension(size_t& x, size_t& y, size_t& z) const { x = y = z = VV_BRICK_DIM; }
    // getRayStepSize: one leaf voxel of the unit volume box.
    float getRayStepSize() const { return 1.0f / (float)info_.volume_dim; }
    // getRootNode: the root's grid position (node 0 of block 0).
    void getRootNode(uint32_t& x, uint32_t& y, uint32_t& z) const { x = y = z = 0u; }
    vv_node_info nodeInfo(uint32_t x, uint32_t y, uint32_t z) const {
        vv_node_info ni;
        check(vv_octree_node_info(t_, x, y, z, &ni), "GigaVoxelsOctTree::nodeInfo");
        return ni;
    }
    // The node pool as GigaVoxelsOctTree::build leaves it (texture order,
    // 2 words per node, nothing resident).
    std::vector<uint32_t> nodeWords() const {
        std::vector<uint32_t> w((size_t)info_.pool_dim[0] * info_.pool_dim[1] * info_.pool_dim[2] * 2);
        check(vv_octree_node_words(t_, w.data()), "GigaVoxelsOctTree::nodeWords");
        return w;
    }
    // Node::copyMipMapToBrick (GigaVoxelsOctTree.cpp:1428-1488) for nodes
    // given by grid position (3 words each), VV_BRICK_TEXELS texels each.
    void copyMipMapToBricks(const std::vector<uint32_t>& xyz, int32_t fmt, void* out) const {
        check(vv_octree_produce_bricks(t_, xyz.data(), (int32_t)(xyz.size() / 3), fmt, out),
              "GigaVoxelsOctTree::copyMipMapToBricks");
    }

private:
    explicit GigaVoxelsOctTree(vv_octree* t) : t_(t) { check(vv_octree_get_info(t_, &info_), "octree info"); }
    vv_octree* t_ = nullptr;
    vv_octree_info info_{};
};

// ---------------------------------------------------------------------------
// OctTreeNodePool: nodes in blocks of 8 (allocation order), laid out in a 3D
// grid by create3DTexture (GigaVoxelsOctTreeNodePool.cpp:49-223).
class OctTreeNodePool {
public:
    struct Node {                       // GigaVoxelsOctTree::Node's GPU data
        uint32_t word0 = 0, word1 = 0;  // GpuDataStruct (child pointer filled by create3DTexture)
        int64_t parent = -1;            // node index of the parent (-1: root)
        int64_t child_block = -1;       // block index of the children (-1: leaf)
        bool isConstant() const { return (word0 & kConstantBit) != 0; }
        bool isResident() const { return (word0 & kResidentBit) != 0; }
        // Node::setConstantValue with the colour stored (RGBA8)
        void setConstantValue(uint32_t rgba) {
            word0 |= kConstantBit;
            word1 = rgba;
        }
    };

    // allocateChildNodeBlock: append a block of 8 nodes, the children of
    // node `parent` (-1 for the root block); returns the block index.
    void allocateChildNodeBlock(int64_t parent, size_t& blockIndex) {
        blockIndex = nodes_.size() / 8;
        if (parent >= 0) nodes_.at((size_t)parent).child_block = (int64_t)blockIndex;
        for (int i = 0; i < 8; ++i) {
            Node n;
            n.parent = parent;
            nodes_.push_back(n);
        }
    }
    // getChild: node by allocation index (nullptr past the end).
    Node* getChild(size_t childIndex) { return childIndex < nodes_.size() ? &nodes_[childIndex] : nullptr; }
    const Node* getChild(size_t childIndex) const {
        return childIndex < nodes_.size() ? &nodes_[childIndex] : nullptr;
    }
    size_t getNodeCount() const { return nodes_.size(); }
    void get3DTextureDimensions(size_t& x, size_t& y, size_t& z) const {
        x = dim_[0];
        y = dim_[1];
        z = dim_[2];
    }

    // Grid position of node `i`: block b at (2(b mod bx), 2((b/bx) mod by),
    // 2(b/(bx by))), child k of the block at +(k&1, (k>>1)&1, k>>2).
    void gridPosition(size_t i, uint32_t& x, uint32_t& y, uint32_t& z) const {
        const size_t b = i / 8, k = i % 8, bx = dim_[0] / 2, by = dim_[1] / 2;
        x = (uint32_t)(2 * (b % bx) + (k & 1));
        y = (uint32_t)(2 * ((b / bx) % by) + ((k >> 1) & 1));
        z = (uint32_t)(2 * (b / (bx * by)) + (k >> 2));
    }
    size_t nodeIndexAt(uint32_t x, uint32_t y, uint32_t z) const {
        const size_t bx = dim_[0] / 2, by = dim_[1] / 2;
        const size_t b = (size_t)(z / 2) * bx * by + (size_t)(y / 2) * bx + (size_t)(x / 2);
        return b * 8 + (x & 1) + 2 * (y & 1) + 4 * (z & 1);
    }

    // create3DTexture: grid dimensions (even, the cube root rounded down to
    // even, then x grown by 2 until the nodes fit), child pointers as grid
    // positions, and the upload of every node word into tree `tree` of `ctx`
    // (ctx NULL: host layout only).  Returns the words in texture order.
    std::vector<uint32_t> create3DTexture(vv_ctx* ctx = nullptr, int32_t tree = 0) {
        const size_t n = nodes_.size();
        if (n == 0) throw Error(VV_ERR_STATE, "create3DTexture: no nodes");
        size_t cr = (size_t)std::pow((double)n, 1.0 / 3.0);
        if (cr % 2 != 0) {
            --cr;
            if (cr == 0) cr = 2;
        }
        dim_[0] = dim_[1] = dim_[2] = cr;
        while (dim_[0] * dim_[1] * dim_[2] < n) dim_[0] += 2;
        if (dim_[0] > 1024 || dim_[1] > 1024 || dim_[2] > 1024)
            throw Error(VV_ERR_ARG, "create3DTexture: the node grid exceeds the 10-bit pointers");
        for (Node& nd : nodes_) {
            nd.word0 &= kResidentBit | kConstantBit;
            if (nd.child_block >= 0) {
                uint32_t x, y, z;
                gridPosition((size_t)nd.child_block * 8, x, y, z);
                nd.word0 |= (x << 20) | (y << 10) | z;
            }
        }
        std::vector<uint32_t> w(dim_[0] * dim_[1] * dim_[2] * 2, 0u);
        for (size_t i = 0; i < n; ++i) {
            uint32_t x, y, z;
            gridPosition(i, x, y, z);
            const size_t t = ((size_t)z * dim_[1] + y) * dim_[0] + x;
            w[2 * t] = nodes_[i].word0;
            w[2 * t + 1] = nodes_[i].word1;
        }
        if (ctx) {
            check(vv_nodepool_upload(ctx, tree, w.data(), (int32_t)dim_[0], (int32_t)dim_[1], (int32_t)dim_[2]),
                  "OctTreeNodePool::create3DTexture", ctx);
            ctx_ = ctx;
            tree_ = tree;
        }
        return w;
    }
    // addToUpdateList / update: queue a node whose words changed, then patch
    // the queued nodes' words on the device (update3DTexture per node).
    void addToUpdateList(size_t i) {
        if (queued_.insert(i).second) update_list_.push_back(i);
    }
    void update() {
        if (update_list_.empty()) return;
        if (!ctx_) throw Error(VV_ERR_STATE, "OctTreeNodePool::update before create3DTexture on a context");
        std::vector<vv_node_patch> p(update_list_.size());
        for (size_t k = 0; k < update_list_.size(); ++k) {
            const Node& nd = nodes_[update_list_[k]];
            gridPosition(update_list_[k], p[k].x, p[k].y, p[k].z);
            p[k].word0 = nd.word0;
            p[k].word1 = nd.word1;
        }
        update_list_.clear();
        queued_.clear();
        check(vv_nodepool_patch(ctx_, tree_, p.data(), (int32_t)p.size()), "OctTreeNodePool::update", ctx_);
    }

    // The pool of a built octree: the nodes of `t` in the allocation order
    // GigaVoxelsOctTree::build uses (the root block, then each node's child
    // block depth first), read from its node words.
    static OctTreeNodePool fromOctree(const GigaVoxelsOctTree& t) {
        const std::vector<uint32_t> w = t.nodeWords();
        const vv_octree_info& in = t.info();
        const size_t dx = (size_t)in.pool_dim[0], dy = (size_t)in.pool_dim[1];
        OctTreeNodePool p;
        size_t b;
        p.allocateChildNodeBlock(-1, b);
        // DFS pre-order over (grid position of node, its pool index); the
        // root is record 0 of block 0 and records 1..7 stay unused, as in
        // the reference
        struct Item {
            uint32_t x, y, z;
            size_t idx;
        };
        std::vector<Item> stack{{0u, 0u, 0u, 0u}};
        while (!stack.empty()) {
            const Item it = stack.back();
            stack.pop_back();
            const size_t ti = ((size_t)it.z * dy + it.y) * dx + it.x;
            const uint32_t w0 = w[2 * ti], w1 = w[2 * ti + 1];
            Node& nd = p.nodes_[it.idx];
            nd.word0 = w0 & (kResidentBit | kConstantBit);
            nd.word1 = w1;
            const uint32_t cx = (w0 >> 20) & 0x3FFu, cy = (w0 >> 10) & 0x3FFu, cz = w0 & 0x3FFu;
            if (cx == 0u && cy == 0u && cz == 0u) continue;
            size_t blk;
            p.allocateChildNodeBlock((int64_t)it.idx, blk);
            for (int k = 7; k >= 0; --k)
                stack.push_back({cx + (uint32_t)(k & 1), cy + (uint32_t)((k >> 1) & 1), cz + (uint32_t)(k >> 2),
                                 blk * 8 + (size_t)k});
        }
        return p;
    }

private:
    std::vector<Node> nodes_;
    size_t dim_[3] = {0, 0, 0};
    std::vector<size_t> update_list_;
    std::unordered_set<size_t> queued_;
    vv_ctx* ctx_ = nullptr;
    int32_t tree_ = 0;
};

// ---------------------------------------------------------------------------
// BrickPool: the brick slots in HBM with the LRU of m_loadedBricks
// (GigaVoxelsBrickPool.cpp:330-424, 561-682).  A process-wide instance, as
// in the reference; nodes are OctTreeNodePool indices.
class BrickPool {
public:
    typedef std::vector<size_t> UploadRequestList;

    static BrickPool& instance() {
        static BrickPool p;
        return p;
    }
    static bool initialized() { return instance().ctx_ != nullptr; }

    // init: a pool of at least numGpuBricks slots of (brickDim + border)^3
    // RGBA8 texels; the slot grid is the cube root grown in x
    // (GigaVoxelsBrickPool.cpp:75-101).  Only 8^3 bricks with a border of 2
    // (one voxel per side) are supported.
    bool init(vv_ctx* ctx, size_t brickDimX, size_t brickDimY, size_t brickDimZ, size_t numGpuBricks,
              size_t /*numCpuBricks*/ = 0, size_t /*numPboBricks*/ = 0, size_t borderVoxels = 2u) {
        return initSpecial(ctx, VV_FMT_RGBA8, brickDimX, brickDimY, brickDimZ, numGpuBricks, borderVoxels);
    }
    // initSpecial: the same with another texel format (the reference picks
    // the GL internal format here).
    bool initSpecial(vv_ctx* ctx, int32_t fmt, size_t brickDimX, size_t brickDimY, size_t brickDimZ,
                     size_t numGpuBricks, size_t borderVoxels = 2u) {
        if (ctx_) return true;  // as the reference: the first init wins
        if (brickDimX != VV_BRICK_DIM || brickDimY != VV_BRICK_DIM || brickDimZ != VV_BRICK_DIM || borderVoxels != 2)
            throw Error(VV_ERR_ARG, "BrickPool::init: 8^3 bricks with a 1-voxel border only");
        size_t cr = (size_t)std::pow((double)numGpuBricks, 1.0 / 3.0);
        if (cr == 0) cr = 1;
        size_t s[3] = {cr, cr, cr};
        while (s[0] * s[1] * s[2] < numGpuBricks) ++s[0];
        check(vv_brickpool_create(ctx, (int32_t)s[0], (int32_t)s[1], (int32_t)s[2], fmt), "BrickPool::init", ctx);
        ctx_ = ctx;
        fmt_ = fmt;
        for (int a = 0; a < 3; ++a) slots_[a] = s[a];
        const size_t n = s[0] * s[1] * s[2];
        slot_node_.assign(n, -1);
        lru_.clear();
        where_.assign(n, lru_.end());
        for (size_t k = 0; k < n; ++k) where_[k] = lru_.insert(lru_.end(), k);  // empty slots first, in id order
        return true;
    }
    void reset() {
        ctx_ = nullptr;
        lru_.clear();
        where_.clear();
        slot_node_.clear();
        node_slot_.clear();
        requests_.clear();
        uploaded_ = 0;
    }

    size_t getDimX() const { return slots_[0] * (VV_BRICK_DIM + 2); }
    size_t getDimY() const { return slots_[1] * (VV_BRICK_DIM + 2); }
    size_t getDimZ() const { return slots_[2] * (VV_BRICK_DIM + 2); }
    size_t getBrickDimX() const { return VV_BRICK_DIM; }
    size_t getNumBricksUploaded() const { return uploaded_; }
    UploadRequestList& getUploadRequestList() { return requests_; }
    // slot of node i (-1: not resident)
    int64_t slotOf(size_t i) const {
        auto it = node_slot_.find(i);
        return it == node_slot_.end() ? -1 : (int64_t)it->second;
    }
    // the slots, least recently used first
    std::vector<uint32_t> lruOrder() const { return std::vector<uint32_t>(lru_.begin(), lru_.end()); }
    // (node, slot) of every resident brick, by slot
    std::vector<std::pair<size_t, size_t>> residency() const {
        std::vector<std::pair<size_t, size_t>> out;
        for (size_t s = 0; s < slot_node_.size(); ++s)
            if (slot_node_[s] >= 0) out.emplace_back((size_t)slot_node_[s], s);
        return out;
    }

    // notifyUsed: the node's brick was used this frame: its slot moves to
    // the back of the LRU order.
    void notifyUsed(size_t node) {
        const int64_t s = slotOf(node);
        if (s >= 0) lru_.splice(lru_.end(), lru_, where_[(size_t)s]);
    }
    // notifyDeleted: the node is gone: its slot is freed and goes to the
    // front (the next to be reused).
    void notifyDeleted(size_t node, OctTreeNodePool& pool) {
        const int64_t s = slotOf(node);
        if (s < 0) return;
        node_slot_.erase(node);
        slot_node_[(size_t)s] = -1;
        lru_.splice(lru_.begin(), lru_, where_[(size_t)s]);
        OctTreeNodePool::Node* nd = pool.getChild(node);
        if (nd) {
            nd->word0 &= ~kResidentBit;
            pool.addToUpdateList(node);
        }
    }

    // NodeUsageListProcessor::run (GigaVoxelsOctTree.cpp:430-657) on a
    // compacted request list (n x 4 words, node grid position + 1 packed
    // 10:10:10, 0 = empty): each node once in first-seen order, resident ones
    // touched, non-constant non-resident ones queued for upload; then the
    // root is touched (GigaVoxelsOctTree::update :1821-1850).
    void processNodeUsageList(const uint32_t* requests, size_t n, OctTreeNodePool& pool) {
        std::unordered_set<size_t> seen;
        size_t dx, dy, dz;
        pool.get3DTextureDimensions(dx, dy, dz);
        for (size_t k = 0; k < 4 * n; ++k) {
            const uint32_t v = requests[k];
            if (v == 0u) continue;
            const int64_t x = (int64_t)((v >> 20) & 1023u) - 1, y = (int64_t)((v >> 10) & 1023u) - 1,
                          z = (int64_t)(v & 1023u) - 1;
            if (x < 0 || y < 0 || z < 0 || x >= (int64_t)dx || y >= (int64_t)dy || z >= (int64_t)dz) continue;
            const size_t i = pool.nodeIndexAt((uint32_t)x, (uint32_t)y, (uint32_t)z);
            const OctTreeNodePool::Node* nd = pool.getChild(i);
            if (!nd || (i != 0 && nd->parent < 0)) continue;  // not a node of the tree
            if (!seen.insert(i).second) continue;
            if (slotOf(i) >= 0) notifyUsed(i);
            else if (!nd->isConstant()) requests_.push_back(i);
        }
        notifyUsed(0);
    }

    // update (GigaVoxelsBrickPool.cpp:561-682): every queued node that is
    // still not resident takes the least recently used slot (whose node
    // loses its brick), gets its brick from the octree and its pointer
    // (slot origin + border); a non-constant, non-resident parent follows.
    // Node words go to the node pool's update list; the list is emptied.
    void update(const GigaVoxelsOctTree& tree, OctTreeNodePool& pool) {
        std::vector<size_t> nodes;
        std::vector<uint32_t> slots;
        for (size_t i : requests_) {
            if (slotOf(i) >= 0) continue;
            upload(i, pool, nodes, slots);
            const OctTreeNodePool::Node* nd = pool.getChild(i);
            const int64_t p = nd ? nd->parent : -1;
            if (p >= 0) {
                const OctTreeNodePool::Node* pn = pool.getChild((size_t)p);
                if (pn && !pn->isConstant() && slotOf((size_t)p) < 0) upload((size_t)p, pool, nodes, slots);
            }
        }
        requests_.clear();
        if (nodes.empty()) return;
        // bricks of the uploaded nodes that are still resident, in upload order
        std::vector<uint32_t> xyz, keep_slots;
        for (size_t k = 0; k < nodes.size(); ++k) {
            if (slotOf(nodes[k]) != (int64_t)slots[k]) continue;  // evicted again within this update
            uint32_t x, y, z;
            pool.gridPosition(nodes[k], x, y, z);
            xyz.push_back(x);
            xyz.push_back(y);
            xyz.push_back(z);
            keep_slots.push_back(slots[k]);
        }
        const size_t bpt = fmt_ == VV_FMT_RGBA8 ? 4 : (fmt_ == VV_FMT_FP32 ? 16 : 8);
        std::vector<uint8_t> texels(keep_slots.size() * VV_BRICK_TEXELS * bpt);
        tree.copyMipMapToBricks(xyz, fmt_, texels.data());
        check(vv_upload_bricks(ctx_, keep_slots.data(), (int32_t)keep_slots.size(), texels.data()),
              "BrickPool::update", ctx_);
        uploaded_ += keep_slots.size();
    }

private:
    BrickPool() = default;
    void upload(size_t i, OctTreeNodePool& pool, std::vector<size_t>& nodes, std::vector<uint32_t>& slots) {
        const size_t s = lru_.front();
        lru_.splice(lru_.end(), lru_, where_[s]);
        const int64_t old = slot_node_[s];
        if (old >= 0) {
            node_slot_.erase((size_t)old);
            OctTreeNodePool::Node* on = pool.getChild((size_t)old);
            on->word0 &= ~kResidentBit;
            pool.addToUpdateList((size_t)old);
        }
        slot_node_[s] = (int64_t)i;
        node_slot_[i] = s;
        const uint32_t x = (uint32_t)(s % slots_[0]), y = (uint32_t)((s / slots_[0]) % slots_[1]),
                       z = (uint32_t)(s / (slots_[0] * slots_[1]));
        OctTreeNodePool::Node* nd = pool.getChild(i);
        nd->word0 |= kResidentBit;
        nd->word1 = ((x * 10u + 1u) << 20) | ((y * 10u + 1u) << 10) | (z * 10u + 1u);
        pool.addToUpdateList(i);
        nodes.push_back(i);
        slots.push_back((uint32_t)s);
    }

    vv_ctx* ctx_ = nullptr;
    int32_t fmt_ = VV_FMT_RGBA8;
    size_t slots_[3] = {0, 0, 0};
    std::list<size_t> lru_;
    std::vector<std::list<size_t>::iterator> where_;
    std::vector<int64_t> slot_node_;
    std::unordered_map<size_t, size_t> node_slot_;
    UploadRequestList requests_;
    size_t uploaded_ = 0;
};

// ---------------------------------------------------------------------------
// GigaVoxelsRenderer: the "gv" plugin's frame protocol (Renderer.h:64-79)
// over the library's renderer (octree, pools and paging on the device).
class GigaVoxelsRenderer {
public:
    // init: the context, the octree and the renderer (pools sized by the
    // descriptor; the root brick resident).
    void init(int32_t device, GigaVoxelsOctTree&& tree, const vv_renderer_desc& d) {
        vv_params p{};
        p.device = device;
        check(vv_ctx_create(&p, &ctx_), "GigaVoxelsRenderer::init");
        tree_ = new GigaVoxelsOctTree(std::move(tree));
        check(vv_renderer_create(ctx_, tree_->handle(), &d, &r_), "GigaVoxelsRenderer::init", ctx_);
    }
    // draw: ray cast and selection mask (and histopyramid) of the frame.
    void draw(const vv_camera& cam) {
        check(vv_renderer_draw_passes(r_, &cam, VV_PASS_RAYCAST), "GigaVoxelsRenderer::draw", ctx_);
    }
    // postDraw: compressNodeUsageList of the frame just drawn.
    void postDraw() { check(vv_renderer_post_draw(r_), "GigaVoxelsRenderer::postDraw", ctx_); }
    // update: the page-request service (UpdateBrickPool + UpdateOctTrees).
    void update() { check(vv_renderer_update(r_), "GigaVoxelsRenderer::update", ctx_); }
    void shutdown() {
        if (r_) vv_renderer_destroy(r_);
        r_ = nullptr;
        delete tree_;
        tree_ = nullptr;
        if (ctx_) vv_ctx_destroy(ctx_);
        ctx_ = nullptr;
    }
    ~GigaVoxelsRenderer() { shutdown(); }
    vv_renderer* handle() const { return r_; }
    vv_ctx* context() const { return ctx_; }

private:
    vv_ctx* ctx_ = nullptr;
    vv_renderer* r_ = nullptr;
    GigaVoxelsOctTree* tree_ = nullptr;
};

}  // namespace vv

#endif  // VOXVIZ_B200_HPP
