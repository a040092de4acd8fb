// octree.cpp - terrain octree builder, node-pool layout and brick production.
#include "octree.h"

#include "dxt.h"

#include <algorithm>
#include <climits>
#include <cmath>
#include <cstring>
#include <stdexcept>

#include "../../include/voxviz_b200.h"

namespace vv {

// Node::computeNodeType (GigaVoxelsOctTree.cpp:1490-1609).  The region is the
// node's 8^3 mip voxels plus a 1-voxel border on every side that is inside
// the level; a region that reaches the volume edge is compared against
// transparent black (:1556-1568).  Transparent voxels match any transparent
// value (:1577-1580).
bool classify_node(const TerrainVolume& vol, int d, int i, int j, int k, uint32_t& const_value) {
    const int L = vol.depth();
    const int m = L - d;
    const MipLevel& M = vol.mip(m);
    const int dim = M.dim;
    const int idx[3] = {i, j, k};
    int a0[3], a1[3];
    bool edge = false;
    for (int ax = 0; ax < 3; ++ax) {
        a0[ax] = 8 * idx[ax];
        a1[ax] = a0[ax] + 8;
        if (a0[ax] != 0) a0[ax] -= 1;
        if (a1[ax] <= dim - 1) a1[ax] += 1;
        if (a1[ax] > dim) a1[ax] = dim;
        if (a0[ax] == 0 || a1[ax] == dim) edge = true;
    }
    const uint32_t cv = edge ? 0u : vol.voxel(m, a0[0], a0[1], a0[2]);
    int minS = INT_MAX, maxE = 0;
    for (int y = a0[1]; y < a1[1]; ++y)
        for (int x = a0[0]; x < a1[0]; ++x) {
            size_t c = (size_t)y * dim + x;
            int s = M.s[c];
            minS = std::min(minS, s);
            maxE = std::max(maxE, s + (int)M.r[c]);
        }
    if (a0[2] >= maxE) {  // every voxel transparent black
        const_value = cv;
        return true;
    }
    if (a1[2] <= minS) {  // every voxel pure solid, colour by band
        if (edge) return false;
        if (vol.band(m, a0[2]) != vol.band(m, a1[2] - 1)) return false;
        const_value = cv;
        return true;
    }
    const bool cv_clear = (cv >> 24) == 0u;
    for (int z = a0[2]; z < a1[2]; ++z)
        for (int y = a0[1]; y < a1[1]; ++y)
            for (int x = a0[0]; x < a1[0]; ++x) {
                uint32_t v = vol.voxel(m, x, y, z);
                if ((v >> 24) == 0u && cv_clear) continue;
                if (v != cv) return false;
            }
    const_value = cv;
    return true;
}

std::unique_ptr<GigaVoxelsOctTree> GigaVoxelsOctTree::build(std::shared_ptr<const TerrainVolume> vol,
                                                            bool collapse) {
    const int L = vol->depth();
    std::vector<TreeLevel> lv((size_t)L + 1);
    lv[0].i.push_back(0);
    lv[0].j.push_back(0);
    lv[0].k.push_back(0);
    lv[0].parent.push_back(kNoParent);
    for (int d = 0; d <= L; ++d) {
        TreeLevel& cur = lv[(size_t)d];
        const size_t n = cur.size();
        cur.cval.assign(n, 0);
        cur.isc.assign(n, 0);
#pragma omp parallel for schedule(dynamic, 256)
        for (long q = 0; q < (long)n; ++q) {
            uint32_t cv = 0;
            bool c = classify_node(*vol, d, cur.i[(size_t)q], cur.j[(size_t)q], cur.k[(size_t)q], cv);
            cur.isc[(size_t)q] = c ? 1 : 0;
            cur.cval[(size_t)q] = cv;
        }
        if (d == L) break;
        TreeLevel& nxt = lv[(size_t)d + 1];
        for (size_t q = 0; q < n; ++q) {
            if (collapse && cur.isc[q]) continue;
            for (int c = 0; c < 8; ++c) {
                nxt.i.push_back((uint16_t)(2 * cur.i[q] + (c & 1)));
                nxt.j.push_back((uint16_t)(2 * cur.j[q] + ((c >> 1) & 1)));
                nxt.k.push_back((uint16_t)(2 * cur.k[q] + (c >> 2)));
                nxt.parent.push_back((uint32_t)q);
            }
        }
    }
    return from_levels(std::move(vol), std::move(lv), collapse);
}

std::unique_ptr<GigaVoxelsOctTree> GigaVoxelsOctTree::from_levels(std::shared_ptr<const TerrainVolume> vol,
                                                                  std::vector<TreeLevel>&& lv, bool collapse) {
    std::unique_ptr<GigaVoxelsOctTree> t(new GigaVoxelsOctTree());
    t->vol_ = vol;
    const int L = vol->depth();
    t->depth_ = L;
    if (lv.size() != (size_t)L + 1 || lv[0].size() != 1) throw std::invalid_argument("bad tree levels");
    // each node's first child in the next level (children come 8 per parent,
    // in parent order)
    std::vector<std::vector<uint32_t>> first_child(lv.size()), nidx(lv.size());
    for (int d = 0; d <= L; ++d) {
        const TreeLevel& cur = lv[(size_t)d];
        if (cur.isc.size() != cur.size() || cur.cval.size() != cur.size() || cur.parent.size() != cur.size())
            throw std::invalid_argument("bad tree level arrays");
        first_child[(size_t)d].assign(cur.size(), UINT32_MAX);
        nidx[(size_t)d].assign(cur.size(), 0);
        if (d == L) break;
        uint32_t next = 0;
        for (size_t q = 0; q < cur.size(); ++q) {
            if (collapse && cur.isc[q]) continue;
            first_child[(size_t)d][q] = next;
            next += 8;
        }
        if ((size_t)next != lv[(size_t)d + 1].size()) throw std::invalid_argument("tree level sizes disagree");
    }
    // Depth-first pre-order block numbering (BuildOctTreeChildren allocates a
    // child's block right before recursing into it).
    size_t blocks = 1;
    {
        std::vector<std::pair<int, uint32_t>> stack;
        nidx[0][0] = 0;
        stack.push_back({0, 0u});
        while (!stack.empty()) {
            auto [d, q] = stack.back();
            stack.pop_back();
            uint32_t fc = first_child[(size_t)d][q];
            if (fc == UINT32_MAX) continue;
            size_t B = blocks++;
            for (int c = 0; c < 8; ++c) nidx[(size_t)d + 1][fc + (uint32_t)c] = (uint32_t)(8 * B + (size_t)c);
            for (int c = 7; c >= 0; --c) stack.push_back({d + 1, fc + (uint32_t)c});
        }
    }
    const size_t num_nodes = 8 * blocks;
    t->set_pool_dim(num_nodes);
    t->leaf_dim_ = 8 << L;

    t->level_.assign(num_nodes, -1);
    t->ci_.assign(num_nodes, 0);
    t->cj_.assign(num_nodes, 0);
    t->ck_.assign(num_nodes, 0);
    t->parent_.assign(num_nodes, kNoParent);
    t->word0_.assign(num_nodes, 0);
    t->word1_.assign(num_nodes, 0);
    size_t nonconst = 0;
    for (int d = 0; d <= L; ++d) {
        const TreeLevel& cur = lv[(size_t)d];
        for (size_t q = 0; q < cur.size(); ++q) {
            uint32_t n = nidx[(size_t)d][q];
            t->level_[n] = (int8_t)d;
            t->ci_[n] = cur.i[q];
            t->cj_[n] = cur.j[q];
            t->ck_[n] = cur.k[q];
            t->parent_[n] = d == 0 ? kNoParent : nidx[(size_t)d - 1][cur.parent[q]];
            uint32_t w0 = 0, w1 = 0;
            if (cur.isc[q]) {
                w0 |= kConstantBit;
                w1 = cur.cval[q];
            } else {
                ++nonconst;
            }
            const uint32_t fc = first_child[(size_t)d][q];
            if (fc != UINT32_MAX) w0 |= t->child_pointer(nidx[(size_t)d + 1][fc] / 8);
            t->word0_[n] = w0;
            t->word1_[n] = w1;
        }
    }
    t->nonconst_ = nonconst;
    return t;
}

void GigaVoxelsOctTree::set_pool_dim(size_t num_nodes) {
    size_t cube_root = (size_t)std::pow((double)num_nodes, 1.0 / 3.0);
    if (cube_root % 2 != 0) {
        --cube_root;
        if (cube_root == 0) cube_root = 2;
    }
    size_t dx = cube_root, dy = cube_root, dz = cube_root;
    while (dx * dy * dz < num_nodes) dx += 2;
    if (dx > 1022 || dy > 1022 || dz > 1022)
        throw std::runtime_error("node pool exceeds the 10-bit grid of the node encoding");
    pool_dim_[0] = (int)dx;
    pool_dim_[1] = (int)dy;
    pool_dim_[2] = (int)dz;
}

// The child pointer of word0 for child block `block`: the block's first grid
// cell, blocks laid x-major over the grid's 2x2x2 cells.
uint32_t GigaVoxelsOctTree::child_pointer(size_t block) const {
    const size_t bx = (size_t)pool_dim_[0] / 2, by = (size_t)pool_dim_[1] / 2;
    return pack10((uint32_t)(2 * (block % bx)), (uint32_t)(2 * ((block / bx) % by)), (uint32_t)(2 * (block / (bx * by))));
}

std::unique_ptr<GigaVoxelsOctTree> GigaVoxelsOctTree::from_gvx(GvxFile&& f, bool constant_colors) {
    std::unique_ptr<GigaVoxelsOctTree> t(new GigaVoxelsOctTree());
    const size_t nn = f.nodes.size();
    if (nn == 0 || nn % 8 != 0 || f.nodes[0].level != 0) throw std::runtime_error("the file has no root node");
    t->depth_ = f.h.max_depth - 1;
    const int vmax = std::max(f.h.volume_size[0], std::max(f.h.volume_size[1], f.h.volume_size[2]));
    t->leaf_dim_ = vmax > 0 ? vmax : 8 << t->depth_;
    t->set_pool_dim(nn);
    auto st = std::make_unique<FileStore>();
    st->h = f.h;
    t->level_.assign(nn, -1);
    t->ci_.assign(nn, 0);
    t->cj_.assign(nn, 0);
    t->ck_.assign(nn, 0);
    t->parent_.assign(nn, kNoParent);
    t->word0_.assign(nn, 0);
    t->word1_.assign(nn, 0);
    st->brick_of.assign(nn, -1);
    st->brick_index.assign(nn, -1);
    st->color.assign(nn, 0);
    st->type.assign(nn, 0);
    st->mip.assign(3 * nn, 0);
    // global brick ids: the levels' bricks one after another
    std::vector<size_t> first(f.bricks.size() + 1, 0);
    for (size_t lv = 0; lv < f.bricks.size(); ++lv) first[lv + 1] = first[lv] + f.bricks[lv].size();
    const size_t nb = first.back();
    bool normals = nb > 0;
    for (const auto& lv : f.bricks)
        for (const GvxBrick& b : lv)
            if (b.normals.empty()) normals = false;
    st->texels.assign(nb * VV_BRICK_TEXELS, 0u);
    if (normals) st->normals.assign(nb * VV_BRICK_TEXELS, 0u);
    st->border.assign(3 * nb, 1);
    st->dims.assign(3 * nb, 10);
    size_t nonconst = 0;
    for (size_t n = 0; n < nn; ++n) {
        const GvxNode& r = f.nodes[n];
        if (r.level < 0) continue;
        t->level_[n] = r.level;
        for (int a = 0; a < 3; ++a) st->mip[3 * n + a] = r.mip[a];
        t->ci_[n] = (uint16_t)std::max(0, r.mip[0] / 8);
        t->cj_[n] = (uint16_t)std::max(0, r.mip[1] / 8);
        t->ck_[n] = (uint16_t)std::max(0, r.mip[2] / 8);
        t->parent_[n] = r.parent;
        st->type[n] = r.type;
        st->color[n] = r.color;
        uint32_t w0 = 0, w1 = 0;
        if (r.type != kGvxNonConst) {
            w0 |= kConstantBit;
            if (constant_colors) w1 = r.color;
        } else {
            ++nonconst;
            if (r.brick < 0 || (size_t)r.level >= f.bricks.size() || (size_t)r.brick >= f.bricks[(size_t)r.level].size())
                throw std::runtime_error("a non-constant node has no brick");
            st->brick_of[n] = (int32_t)(first[(size_t)r.level] + (size_t)r.brick);
            st->brick_index[n] = r.brick;
        }
        if (r.child_block >= 0) w0 |= t->child_pointer((size_t)r.child_block);
        t->word0_[n] = w0;
        t->word1_[n] = w1;
    }
    for (size_t lv = 0; lv < f.bricks.size(); ++lv)
        for (size_t i = 0; i < f.bricks[lv].size(); ++i) {
            GvxBrick& b = f.bricks[lv][i];
            const size_t id = first[lv] + i;
            uint32_t* out = st->texels.data() + id * VV_BRICK_TEXELS;
            uint32_t* nout = normals ? st->normals.data() + id * VV_BRICK_TEXELS : nullptr;
            size_t q = 0;
            for (int z = 0; z < b.dims[2]; ++z)
                for (int y = 0; y < b.dims[1]; ++y)
                    for (int x = 0; x < b.dims[0]; ++x, ++q) {
                        const size_t o = (size_t)(z * 100 + y * 10 + x);
                        std::memcpy(out + o, b.colors.data() + 4 * q, 4);
                        if (nout)
                            nout[o] = (uint32_t)b.normals[3 * q] | ((uint32_t)b.normals[3 * q + 1] << 8) |
                                      ((uint32_t)b.normals[3 * q + 2] << 16);
                    }
            for (int a = 0; a < 3; ++a) {
                st->border[3 * id + a] = b.border[a];
                st->dims[3 * id + a] = b.dims[a];
            }
            std::vector<uint8_t>().swap(b.colors);
            std::vector<uint8_t>().swap(b.normals);
        }
    t->nonconst_ = nonconst;
    t->file_ = std::move(st);
    return t;
}

bool GigaVoxelsOctTree::save_gvx(const std::string& dir, bool gradients, std::string& err) const {
    GvxFile f;
    const size_t nn = level_.size();
    if (file_) {
        f.h = file_->h;
    } else {
        f.h.max_depth = depth_ + 1;
        for (int a = 0; a < 3; ++a) {
            f.h.delta[a] = 1.0f / (float)(8 << depth_);
            f.h.volume_size[a] = 8 << depth_;
            f.h.brick_size[a] = 8;
        }
        f.h.binary = true;
    }
    f.h.compressed = false;
    f.nodes.assign(nn, GvxNode());
    std::vector<size_t> per_level((size_t)f.h.max_depth, 0);
    std::vector<std::pair<int, int32_t>> brick_slot(nn, {-1, -1});  // (level, index) of node n's brick
    for (size_t n = 0; n < nn; ++n) {
        if (level_[n] < 0) continue;
        GvxNode& r = f.nodes[n];
        r.level = level_[n];
        r.parent = parent_[n];
        if (file_) {
            for (int a = 0; a < 3; ++a) r.mip[a] = file_->mip[3 * n + a];
        } else {
            r.mip[0] = 8 * ci_[n];
            r.mip[1] = 8 * cj_[n];
            r.mip[2] = 8 * ck_[n];
        }
        if (has_children((uint32_t)n)) {
            const uint32_t c = word0_[n] & 0x3FFFFFFFu & ~kConstantBit;
            r.child_block = (int32_t)(index_of((c >> 20) & 0x3FFu, (c >> 10) & 0x3FFu, c & 0x3FFu) / 8);
        }
        if (is_constant((uint32_t)n)) {
            r.type = file_ ? file_->type[n] : (uint8_t)(r.child_block >= 0 ? kGvxConst : kGvxLeafConst);
            r.color = file_ ? file_->color[n] : word1_[n];
        } else {
            r.type = kGvxNonConst;
            r.brick = file_ ? file_->brick_index[n] : (int32_t)per_level[(size_t)r.level];
            per_level[(size_t)r.level] = std::max(per_level[(size_t)r.level], (size_t)r.brick + 1);
            brick_slot[n] = {r.level, r.brick};
        }
    }
    // node of each (level, brick index)
    std::vector<std::vector<uint32_t>> node_of(per_level.size());
    for (size_t lv = 0; lv < per_level.size(); ++lv) node_of[lv].assign(per_level[lv], kNoParent);
    for (size_t n = 0; n < nn; ++n)
        if (brick_slot[n].first >= 0) node_of[(size_t)brick_slot[n].first][(size_t)brick_slot[n].second] = (uint32_t)n;
    const bool grads = gradients && (file_ ? file_has_normals() : depth_ <= 6);
    auto source = [&](size_t lv, size_t i, GvxBrick& b) {
        const uint32_t n = node_of[lv][i];
        uint32_t tex[VV_BRICK_TEXELS], nrm[VV_BRICK_TEXELS];
        if (file_) {
            const size_t id = (size_t)file_->brick_of[n];
            for (int a = 0; a < 3; ++a) {
                b.dims[a] = file_->dims[3 * id + a];
                b.border[a] = file_->border[3 * id + a];
            }
            std::memcpy(tex, file_->texels.data() + id * VV_BRICK_TEXELS, sizeof(tex));
            if (grads) std::memcpy(nrm, file_->normals.data() + id * VV_BRICK_TEXELS, sizeof(nrm));
        } else {
            for (int a = 0; a < 3; ++a) {
                b.dims[a] = 10;
                b.border[a] = 1;
            }
            produce_brick_rgba8(n, tex);
            if (grads) produce_gradient_brick(n, VV_FMT_RGBA8, nrm);
        }
        const size_t count = (size_t)b.dims[0] * b.dims[1] * b.dims[2];
        b.colors.resize(4 * count);
        b.normals.clear();
        if (grads) b.normals.resize(3 * count);
        size_t q = 0;
        for (int z = 0; z < b.dims[2]; ++z)
            for (int y = 0; y < b.dims[1]; ++y)
                for (int x = 0; x < b.dims[0]; ++x, ++q) {
                    const size_t o = (size_t)(z * 100 + y * 10 + x);
                    std::memcpy(b.colors.data() + 4 * q, tex + o, 4);
                    if (grads)
                        for (int c = 0; c < 3; ++c) b.normals[3 * q + c] = (uint8_t)(nrm[o] >> (8 * c));
                }
    };
    return write_gvx(dir, f, per_level, source, err);
}

void GigaVoxelsOctTree::grid_of(uint32_t n, uint32_t& x, uint32_t& y, uint32_t& z) const {
    const uint32_t bx = (uint32_t)pool_dim_[0] / 2, by = (uint32_t)pool_dim_[1] / 2;
    uint32_t k = n >> 3, c = n & 7u;
    x = 2 * (k % bx) + (c & 1u);
    y = 2 * ((k / bx) % by) + ((c >> 1) & 1u);
    z = 2 * (k / (bx * by)) + (c >> 2);
}

uint32_t GigaVoxelsOctTree::index_of(uint32_t x, uint32_t y, uint32_t z) const {
    if (x >= (uint32_t)pool_dim_[0] || y >= (uint32_t)pool_dim_[1] || z >= (uint32_t)pool_dim_[2])
        return kNoParent;
    const uint32_t bx = (uint32_t)pool_dim_[0] / 2, by = (uint32_t)pool_dim_[1] / 2;
    uint64_t k = ((uint64_t)(z / 2) * by + (y / 2)) * bx + (x / 2);
    uint64_t n = 8 * k + ((x & 1u) | ((y & 1u) << 1) | ((z & 1u) << 2));
    if (n >= level_.size()) return kNoParent;
    return (uint32_t)n;
}

void GigaVoxelsOctTree::words_grid(uint32_t* out) const {
    const size_t cells = (size_t)pool_dim_[0] * pool_dim_[1] * pool_dim_[2];
    std::memset(out, 0, cells * 2 * sizeof(uint32_t));
    for (size_t n = 0; n < level_.size(); ++n) {
        uint32_t x, y, z;
        grid_of((uint32_t)n, x, y, z);
        size_t g = ((size_t)z * pool_dim_[1] + y) * pool_dim_[0] + x;
        out[2 * g] = word0_[n];
        out[2 * g + 1] = word1_[n];
    }
}

void GigaVoxelsOctTree::produce_brick_rgba8(uint32_t n, uint32_t* out) const {
    if (file_) {
        const int32_t k = file_->brick_of[n];
        if (k < 0) std::memset(out, 0, VV_BRICK_TEXELS * sizeof(uint32_t));
        else std::memcpy(out, file_->texels.data() + (size_t)k * VV_BRICK_TEXELS, VV_BRICK_TEXELS * sizeof(uint32_t));
        return;
    }
    const int d = level_[n];
    const int m = depth_ - d;
    const MipLevel& M = vol_->mip(m);
    const int dim = M.dim;
    const int x0 = 8 * ci_[n] - 1, y0 = 8 * cj_[n] - 1, z0 = 8 * ck_[n] - 1;
    for (int by = 0; by < 10; ++by) {
        const int y = y0 + by;
        for (int bx = 0; bx < 10; ++bx) {
            const int x = x0 + bx;
            if (x < 0 || y < 0 || x >= dim || y >= dim) {
                for (int bz = 0; bz < 10; ++bz) out[(bz * 10 + by) * 10 + bx] = 0u;
                continue;
            }
            const size_t c = (size_t)y * dim + x;
            const int s = M.s[c], e = s + M.r[c];
            const uint32_t* run = M.data.empty() ? nullptr : M.data.data() + M.off[c];
            for (int bz = 0; bz < 10; ++bz) {
                const int z = z0 + bz;
                uint32_t v;
                if (z < 0 || z >= dim) v = 0u;
                else if (z < s) v = band_colour(vol_->band(m, z));
                else if (z < e) v = run[z - s];
                else v = 0u;
                out[(bz * 10 + by) * 10 + bx] = v;
            }
        }
    }
}

size_t texel_bytes(int fmt) {
    switch (fmt) {
        case VV_FMT_RGBA8: return 4;
        case VV_FMT_FP16: return 8;
        case VV_FMT_BF16: return 8;
        case VV_FMT_FP32: return 16;
        default: return 0;
    }
}

size_t brick_bytes(int fmt) {
    if (fmt == VV_FMT_DXT5) return (size_t)dxt::kDxt5SlotBytes;
    if (fmt == VV_FMT_DXT1) return (size_t)dxt::kDxt1SlotBytes;
    return VV_BRICK_TEXELS * texel_bytes(fmt);
}

// The 90 blocks of a brick (10^3 RGBA8 texels) in DXT5 or DXT1.
static void encode_brick_dxt(const uint32_t* rgba, int fmt, void* out) {
    for (int b = 0; b < dxt::kBlocksPerSlot; ++b) {
        uint32_t px[16], valid;
        dxt::gather_block(rgba, b, px, valid);
        if (fmt == VV_FMT_DXT5) dxt::encode_dxt5(px, valid, (uint32_t*)out + 4 * b);
        else dxt::encode_dxt1(px, valid, (uint32_t*)out + 2 * b);
    }
}

uint16_t float_to_half_rn(float f) {
    uint32_t x;
    std::memcpy(&x, &f, 4);
    const uint32_t sign = (x >> 16) & 0x8000u;
    const uint32_t ax = x & 0x7FFFFFFFu;
    if (ax >= 0x7F800000u) return (uint16_t)(sign | (ax > 0x7F800000u ? 0x7E00u : 0x7C00u));
    if (ax >= 0x477FF000u) return (uint16_t)(sign | 0x7C00u);
    if (ax < 0x38800000u) {
        const int e = (int)(ax >> 23);
        if (e < 102) return (uint16_t)sign;
        const uint32_t mant = (ax & 0x7FFFFFu) | 0x800000u;
        const int shift = 126 - e;
        uint32_t q = mant >> shift;
        const uint32_t rem = mant & ((1u << shift) - 1u), half = 1u << (shift - 1);
        if (rem > half || (rem == half && (q & 1u))) ++q;
        return (uint16_t)(sign | q);
    }
    const uint32_t e = (ax >> 23) - 127u + 15u;
    uint32_t q = (e << 10) | ((ax & 0x7FFFFFu) >> 13);
    const uint32_t rem = ax & 0x1FFFu;
    if (rem > 0x1000u || (rem == 0x1000u && (q & 1u))) ++q;
    return (uint16_t)(sign | q);
}

uint16_t float_to_bf16_rn(float f) {
    uint32_t x;
    std::memcpy(&x, &f, 4);
    if ((x & 0x7FFFFFFFu) > 0x7F800000u) return (uint16_t)((x >> 16) | 0x40u);
    x += 0x7FFFu + ((x >> 16) & 1u);
    return (uint16_t)(x >> 16);
}

void convert_texel(uint32_t v, int fmt, void* dst) {
    float c[4];
    for (int ch = 0; ch < 4; ++ch) c[ch] = (float)((v >> (8 * ch)) & 255u) / 255.0f;
    switch (fmt) {
        case VV_FMT_RGBA8: std::memcpy(dst, &v, 4); break;
        case VV_FMT_FP16: {
            uint16_t h[4];
            for (int ch = 0; ch < 4; ++ch) h[ch] = float_to_half_rn(c[ch]);
            std::memcpy(dst, h, 8);
            break;
        }
        case VV_FMT_BF16: {
            uint16_t h[4];
            for (int ch = 0; ch < 4; ++ch) h[ch] = float_to_bf16_rn(c[ch]);
            std::memcpy(dst, h, 8);
            break;
        }
        case VV_FMT_FP32: std::memcpy(dst, c, 16); break;
        default: break;
    }
}

void GigaVoxelsOctTree::produce_brick(uint32_t n, int fmt, void* out) const {
    uint32_t tmp[VV_BRICK_TEXELS];
    produce_brick_rgba8(n, tmp);
    if (fmt == VV_FMT_DXT5) {
        encode_brick_dxt(tmp, fmt, out);
        return;
    }
    const size_t tb = texel_bytes(fmt);
    unsigned char* o = (unsigned char*)out;
    for (int t = 0; t < VV_BRICK_TEXELS; ++t) convert_texel(tmp[t], fmt, o + (size_t)t * tb);
}

bool GigaVoxelsOctTree::produce_gradient_brick(uint32_t n, int fmt, void* out) const {
    if (fmt == VV_FMT_DXT1) {  // the unsigned RGBA8 gradients, block-compressed
        uint32_t tmp[VV_BRICK_TEXELS];
        if (!produce_gradient_brick(n, VV_FMT_RGBA8, tmp)) return false;
        encode_brick_dxt(tmp, fmt, out);
        return true;
    }
    if (fmt != VV_FMT_FP32 && fmt != VV_FMT_RGBA8) return false;
    if (file_) {
        // the file's unsigned bytes (GradientsAreUnsigned is set for every
        // file tree, GigaVoxelsReader.cpp:419-420); FP32 holds them as b/255
        const int32_t k = file_->brick_of[n];
        if (file_->normals.empty() || k < 0) return false;
        const uint32_t* src = file_->normals.data() + (size_t)k * VV_BRICK_TEXELS;
        if (fmt == VV_FMT_RGBA8) {
            std::memcpy(out, src, VV_BRICK_TEXELS * sizeof(uint32_t));
        } else {
            float* o = (float*)out;
            for (int t = 0; t < VV_BRICK_TEXELS; ++t) {
                for (int c = 0; c < 3; ++c) o[4 * t + c] = (float)((src[t] >> (8 * c)) & 255u) / 255.0f;
                o[4 * t + 3] = 0.0f;
            }
        }
        return true;
    }
    {
        std::lock_guard<std::mutex> lock(grads_mu_);
        if (!grads_) {
            if (depth_ > 6) return false;
            grads_ = std::make_unique<GradientPyramid>(*vol_);
        }
    }
    const int d = level_[n], m = depth_ - d;
    const int i = ci_[n], j = cj_[n], k = ck_[n];
    // copyMipMapToBrick: texel (bx,by,bz) is mip voxel (8i-1+bx, 8j-1+by,
    // 8k-1+bz), zero outside the level (the brick is cleared first)
    for (int bz = 0; bz < 10; ++bz)
        for (int by = 0; by < 10; ++by)
            for (int bx = 0; bx < 10; ++bx) {
                float g[3];
                grads_->at(m, 8 * i - 1 + bx, 8 * j - 1 + by, 8 * k - 1 + bz, g);
                const size_t t = (size_t)(bz * 100 + by * 10 + bx);
                if (fmt == VV_FMT_FP32) {
                    float* o = (float*)out + 4 * t;
                    o[0] = g[0];
                    o[1] = g[1];
                    o[2] = g[2];
                    o[3] = 0.0f;
                } else {
                    uint32_t w = 0;
                    for (int c = 0; c < 3; ++c) {
                        const float u = std::floor(((g[c] + 1.0f) * 0.5f) * 255.0f + 0.5f);
                        const uint32_t b = u < 0.0f ? 0u : (u > 255.0f ? 255u : (uint32_t)u);
                        w |= b << (8 * c);
                    }
                    ((uint32_t*)out)[t] = w;
                }
            }
    return true;
}

}  // namespace vv
