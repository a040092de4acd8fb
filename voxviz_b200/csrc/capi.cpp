// capi.cpp - C ABI of the host data model (octree, camera, renderer).
#include <cuda_runtime.h>

#include <cstring>
#include <exception>
#include <memory>
#include <new>
#include <string>

#include "ctx.h"
#include "gvfile.h"
#include "handles.h"
#include "octree.h"
#include "renderer.h"
#include "scene.h"


struct vv_scene {
    std::unique_ptr<vv::PagedScene> impl;
};

extern "C" {

int vv_octree_build_terrain(const vv_terrain_desc* d, vv_octree** out) {
    if (!d || !out) return VV_ERR_ARG;
    *out = nullptr;
    if (d->depth < 0 || d->depth > 10 || d->octaves < 1 || d->base_cells < 1) return VV_ERR_ARG;
    try {
        vv::TerrainParams p;
        p.seed = d->seed;
        p.depth = d->depth;
        p.octaves = d->octaves;
        p.lacunarity = d->lacunarity;
        p.gain = d->gain;
        p.base_cells = d->base_cells;
        p.threads = d->threads;
        auto o = std::make_unique<vv_octree>();
        o->volume = std::make_shared<vv::TerrainVolume>(p);
        o->tree = vv::GigaVoxelsOctTree::build(o->volume, d->collapse_constant != 0);
        *out = o.release();
        return VV_OK;
    } catch (const std::bad_alloc&) {
        return VV_ERR_OOM;
    } catch (const std::exception&) {
        return VV_ERR_ARG;
    }
}

int vv_octree_build_terrain_gpu(const vv_terrain_desc* d, int32_t device, vv_octree** out) {
    if (!d || !out) return VV_ERR_ARG;
    *out = nullptr;
    if (d->depth < 0 || d->depth > 10 || d->octaves < 1 || d->base_cells < 1) return VV_ERR_ARG;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || device < 0 || device >= ndev) {
        vv::set_thread_error("vv_octree_build_terrain_gpu: no such CUDA device");
        return VV_ERR_NODEV;
    }
    if (cudaSetDevice(device) != cudaSuccess) return VV_ERR_CUDA;
    try {
        vv::TerrainParams p;
        p.seed = d->seed;
        p.depth = d->depth;
        p.octaves = d->octaves;
        p.lacunarity = d->lacunarity;
        p.gain = d->gain;
        p.base_cells = d->base_cells;
        p.threads = d->threads;
        std::shared_ptr<vv::TerrainVolume> vol;
        std::vector<vv::TreeLevel> levels;
        const std::string err = vv::gpu_build_terrain(p, d->collapse_constant != 0, vol, levels);
        if (!err.empty()) {
            vv::set_thread_error("vv_octree_build_terrain_gpu: " + err);
            return VV_ERR_CUDA;
        }
        auto o = std::make_unique<vv_octree>();
        o->volume = vol;
        o->tree = vv::GigaVoxelsOctTree::from_levels(o->volume, std::move(levels), d->collapse_constant != 0);
        *out = o.release();
        return VV_OK;
    } catch (const std::bad_alloc&) {
        return VV_ERR_OOM;
    } catch (const std::exception& e) {
        vv::set_thread_error(std::string("vv_octree_build_terrain_gpu: ") + e.what());
        return VV_ERR_ARG;
    }
}

void vv_octree_destroy(vv_octree* t) { delete t; }

int vv_octree_get_info(const vv_octree* t, vv_octree_info* info) {
    if (!t || !info) return VV_ERR_ARG;
    std::memset(info, 0, sizeof(*info));
    info->depth = t->tree->depth();
    info->volume_dim = t->tree->leaf_dim();
    info->node_count = (int64_t)t->tree->node_count();
    for (int a = 0; a < 3; ++a) info->pool_dim[a] = t->tree->pool_dim()[a];
    info->nonconst_count = (int64_t)t->tree->nonconst_count();
    info->root_is_constant = t->tree->is_constant(0) ? 1 : 0;
    info->root_word0 = t->tree->word0(0);
    info->root_word1 = t->tree->word1(0);
    return VV_OK;
}

int vv_octree_node_words(const vv_octree* t, uint32_t* words) {
    if (!t || !words) return VV_ERR_ARG;
    t->tree->words_grid(words);
    return VV_OK;
}

int vv_octree_node_info(const vv_octree* t, uint32_t x, uint32_t y, uint32_t z, vv_node_info* info) {
    if (!t || !info) return VV_ERR_ARG;
    std::memset(info, 0, sizeof(*info));
    const uint32_t n = t->tree->index_of(x, y, z);
    if (n == vv::kNoParent || t->tree->level(n) < 0) return VV_OK;
    info->valid = 1;
    info->level = t->tree->level(n);
    int i, j, k;
    t->tree->origin(n, i, j, k);
    info->origin[0] = 8 * i;
    info->origin[1] = 8 * j;
    info->origin[2] = 8 * k;
    info->is_constant = t->tree->is_constant(n) ? 1 : 0;
    info->has_children = t->tree->has_children(n) ? 1 : 0;
    const uint32_t p = t->tree->parent(n);
    if (p == vv::kNoParent) {
        info->parent[0] = info->parent[1] = info->parent[2] = -1;
    } else {
        uint32_t px, py, pz;
        t->tree->grid_of(p, px, py, pz);
        info->parent[0] = (int32_t)px;
        info->parent[1] = (int32_t)py;
        info->parent[2] = (int32_t)pz;
    }
    return VV_OK;
}

int vv_octree_produce_bricks(const vv_octree* t, const uint32_t* xyz, int32_t n, int32_t fmt, void* out) {
    if (!t || n < 0 || (n > 0 && (!xyz || !out))) return VV_ERR_ARG;
    const size_t bb = vv::brick_bytes(fmt);
    if (!bb || fmt == VV_FMT_DXT1) return VV_ERR_ARG;
    for (int32_t i = 0; i < n; ++i) {
        const uint32_t idx = t->tree->index_of(xyz[3 * i], xyz[3 * i + 1], xyz[3 * i + 2]);
        if (idx == vv::kNoParent || t->tree->level(idx) < 0) return VV_ERR_ARG;
    }
    unsigned char* o = (unsigned char*)out;
#pragma omp parallel for schedule(dynamic, 16)
    for (int32_t i = 0; i < n; ++i) {
        const uint32_t idx = t->tree->index_of(xyz[3 * i], xyz[3 * i + 1], xyz[3 * i + 2]);
        t->tree->produce_brick(idx, fmt, o + (size_t)i * bb);
    }
    return VV_OK;
}

int vv_octree_produce_gradients(const vv_octree* t, const uint32_t* xyz, int32_t n, int32_t fmt, void* out) {
    if (!t || n < 0 || (n > 0 && (!xyz || !out))) return VV_ERR_ARG;
    if (fmt != VV_FMT_FP32 && fmt != VV_FMT_RGBA8 && fmt != VV_FMT_DXT1) return VV_ERR_ARG;
    if (t->tree->file_backed() ? !t->tree->file_has_normals() : t->tree->depth() > 6) return VV_ERR_ARG;
    const size_t tb = vv::brick_bytes(fmt);
    for (int32_t i = 0; i < n; ++i) {
        const uint32_t idx = t->tree->index_of(xyz[3 * i], xyz[3 * i + 1], xyz[3 * i + 2]);
        if (idx == vv::kNoParent || t->tree->level(idx) < 0) return VV_ERR_ARG;
    }
    if (n > 0) {  // build the pyramid once, outside the parallel loop
        const uint32_t idx = t->tree->index_of(xyz[0], xyz[1], xyz[2]);
        if (!t->tree->produce_gradient_brick(idx, fmt, out)) return VV_ERR_ARG;
    }
    unsigned char* o = (unsigned char*)out;
#pragma omp parallel for schedule(dynamic, 16)
    for (int32_t i = 1; i < n; ++i) {
        const uint32_t idx = t->tree->index_of(xyz[3 * i], xyz[3 * i + 1], xyz[3 * i + 2]);
        t->tree->produce_gradient_brick(idx, fmt, o + (size_t)i * tb);
    }
    return VV_OK;
}

int vv_octree_mip_level(const vv_octree* t, int32_t level, uint32_t* out, size_t out_words) {
    if (!t || !out || level < 0 || level > t->tree->depth() || !t->tree->has_volume()) return VV_ERR_ARG;
    const vv::TerrainVolume& v = t->tree->volume();
    const int d = v.mip(level).dim;
    if (out_words < (size_t)d * d * d) return VV_ERR_ARG;
#pragma omp parallel for schedule(static)
    for (int z = 0; z < d; ++z)
        for (int y = 0; y < d; ++y)
            for (int x = 0; x < d; ++x) out[((size_t)z * d + y) * d + x] = v.voxel(level, x, y, z);
    return VV_OK;
}

int vv_octree_heights(const vv_octree* t, int32_t* out) {
    if (!t || !out || !t->tree->has_volume()) return VV_ERR_ARG;
    const auto& h = t->tree->volume().heights();
    std::memcpy(out, h.data(), h.size() * sizeof(int32_t));
    return VV_OK;
}

int vv_octree_load_gvx(const char* path, int32_t flags, vv_octree** out) {
    if (!path || !out) {
        vv::set_thread_error("vv_octree_load_gvx: path and out are required");
        return VV_ERR_ARG;
    }
    *out = nullptr;
    try {
        vv::GvxFile f;
        std::string err;
        const int rc = vv::read_gvx(path, (flags & VV_GVX_SKIP_GRADIENTS) == 0, f, err);
        if (rc) {
            vv::set_thread_error(err);
            return rc;
        }
        auto o = std::make_unique<vv_octree>();
        o->tree = vv::GigaVoxelsOctTree::from_gvx(std::move(f), (flags & VV_GVX_CONSTANT_COLORS) != 0);
        *out = o.release();
        return VV_OK;
    } catch (const std::bad_alloc&) {
        vv::set_thread_error("vv_octree_load_gvx: out of host memory");
        return VV_ERR_OOM;
    } catch (const std::exception& e) {
        vv::set_thread_error(std::string("vv_octree_load_gvx: ") + e.what());
        return VV_ERR_ARG;
    }
}

int vv_octree_save_gvx(const vv_octree* t, const char* dir, int32_t flags) {
    if (!t || !dir) return VV_ERR_ARG;
    try {
        std::string err;
        if (!t->tree->save_gvx(dir, (flags & VV_GVX_SKIP_GRADIENTS) == 0, err)) {
            vv::set_thread_error(err);
            return VV_ERR_IO;
        }
        return VV_OK;
    } catch (const std::bad_alloc&) {
        return VV_ERR_OOM;
    }
}

int vv_octree_gvx_info(const vv_octree* t, vv_gvx_info* info) {
    if (!t || !info) return VV_ERR_ARG;
    std::memset(info, 0, sizeof(*info));
    const vv::GvxHeader* h = t->tree->file_header();
    info->file_backed = h ? 1 : 0;
    info->max_depth = t->tree->depth() + 1;
    for (int a = 0; a < 3; ++a) {
        info->origin[a] = h ? h->origin[a] : 0.0f;
        info->delta[a] = h ? h->delta[a] : 1.0f / (float)(8 << t->tree->depth());
        info->volume_size[a] = h ? h->volume_size[a] : 8 << t->tree->depth();
        info->brick_size[a] = h ? h->brick_size[a] : 8;
    }
    info->bricks = h ? (int64_t)t->tree->file_brick_count() : (int64_t)t->tree->nonconst_count();
    info->has_gradients = h ? (t->tree->file_has_normals() ? 1 : 0) : (t->tree->depth() <= 6 ? 1 : 0);
    info->ray_step_size = 1.0f / (float)t->tree->leaf_dim();
    return VV_OK;
}

int vv_gvp_read(const char* path, vv_gvp_info* info, vv_gvp_tile* tiles, int32_t cap) {
    if (!path || !info || cap < 0 || (cap > 0 && !tiles)) return VV_ERR_ARG;
    try {
        vv::GvpFile f;
        std::string err;
        const int rc = vv::read_gvp(path, f, err);
        if (rc) {
            vv::set_thread_error(err);
            return rc;
        }
        std::memset(info, 0, sizeof(*info));
        info->compressed = f.compressed ? 1 : 0;
        for (int a = 0; a < 3; ++a) {
            info->brick_size[a] = f.brick_size[a];
            info->sphere_center[a] = f.sphere_center[a];
        }
        info->tiles = (int32_t)f.tiles.size();
        info->sphere_radius = f.sphere_radius;
        for (int32_t i = 0; i < cap && (size_t)i < f.tiles.size(); ++i) {
            const vv::GvpTile& s = f.tiles[(size_t)i];
            vv_gvp_tile& d = tiles[i];
            std::memset(&d, 0, sizeof(d));
            for (int a = 0; a < 3; ++a) {
                d.center[a] = s.center[a];
                d.size_meters[a] = s.size_meters[a];
            }
            d.radius = s.radius;
            if (s.tree_file.size() >= sizeof(d.tree_file)) {
                vv::set_thread_error("vv_gvp_read: a TreeFile path is longer than 1023 bytes");
                return VV_ERR_ARG;
            }
            std::memcpy(d.tree_file, s.tree_file.c_str(), s.tree_file.size() + 1);
        }
        return VV_OK;
    } catch (const std::bad_alloc&) {
        return VV_ERR_OOM;
    }
}

int vv_gvp_write(const char* path, const vv_gvp_info* info, const vv_gvp_tile* tiles, int32_t n) {
    if (!path || !info || n < 0 || (n > 0 && !tiles)) return VV_ERR_ARG;
    vv::GvpFile f;
    f.compressed = info->compressed != 0;
    for (int a = 0; a < 3; ++a) f.brick_size[a] = info->brick_size[a];
    for (int32_t i = 0; i < n; ++i) {
        vv::GvpTile t;
        for (int a = 0; a < 3; ++a) {
            t.center[a] = tiles[i].center[a];
            t.size_meters[a] = tiles[i].size_meters[a];
        }
        t.radius = tiles[i].radius;
        t.tree_file.assign(tiles[i].tree_file, strnlen(tiles[i].tree_file, sizeof(tiles[i].tree_file)));
        f.tiles.push_back(std::move(t));
    }
    std::string err;
    if (!vv::write_gvp(path, f, err)) {
        vv::set_thread_error(err);
        return VV_ERR_IO;
    }
    return VV_OK;
}

int vv_scene_create(vv_ctx* ctx, const char* gvp_path, const vv_scene_desc* d, vv_scene** out) {
    if (!gvp_path || !d || !out) return VV_ERR_ARG;
    *out = nullptr;
    if (!ctx && !(d->flags & VV_SCENE_HOST_ONLY)) {
        vv::set_thread_error("vv_scene_create: a context is required unless VV_SCENE_HOST_ONLY");
        return VV_ERR_ARG;
    }
    if (!(d->flags & VV_SCENE_HOST_ONLY) && (!vv::brick_bytes(d->fmt) || d->fmt == VV_FMT_DXT1)) return VV_ERR_ARG;
    try {
        vv::GvpFile f;
        std::string err;
        const int rc = vv::read_gvp(gvp_path, f, err);
        if (rc) {
            vv::set_thread_error(err);
            return rc;
        }
        auto sc = std::make_unique<vv_scene>();
        sc->impl = std::make_unique<vv::PagedScene>(ctx, std::move(f), *d);
        const int r = sc->impl->init();
        if (r) return r;
        *out = sc.release();
        return VV_OK;
    } catch (const std::bad_alloc&) {
        return VV_ERR_OOM;
    } catch (const std::exception& e) {
        vv::set_thread_error(std::string("vv_scene_create: ") + e.what());
        return VV_ERR_ARG;
    }
}

void vv_scene_destroy(vv_scene* s) { delete s; }

int vv_scene_draw(vv_scene* s, const vv_camera* cam) {
    if (!s || !cam) return VV_ERR_ARG;
    return s->impl->draw(*cam);
}

int vv_scene_update(vv_scene* s) {
    if (!s) return VV_ERR_ARG;
    return s->impl->update();
}

int vv_scene_wait_loads(vv_scene* s) {
    if (!s) return VV_ERR_ARG;
    return s->impl->wait_loads();
}

int vv_scene_read_color(vv_scene* s, float* host_rgba) {
    if (!s || !host_rgba) return VV_ERR_ARG;
    return s->impl->read_color(host_rgba);
}

int vv_scene_tile_states(const vv_scene* s, vv_scene_tile_state* out, int32_t cap) {
    if (!s || cap < 0 || (cap > 0 && !out)) return VV_ERR_ARG;
    s->impl->tile_states(out, cap);
    return VV_OK;
}

int vv_scene_get_stats(const vv_scene* s, vv_scene_stats* out) {
    if (!s || !out) return VV_ERR_ARG;
    s->impl->stats(*out);
    return VV_OK;
}

vv_renderer* vv_scene_tile_renderer(vv_scene* s, int32_t tile) { return s ? s->impl->tile_renderer(tile) : nullptr; }

int vv_compute_uniforms(const vv_octree_info* tree, const vv_camera* cam, int32_t sx, int32_t sy, int32_t sz,
                        float lod_scalar, float alpha_stop, vv_uniforms* out) {
    if (!tree || !cam || !out || cam->width <= 0 || cam->height <= 0) return VV_ERR_ARG;
    const int slots[3] = {sx, sy, sz};
    vv::compute_uniforms(tree->depth, tree->volume_dim, tree->root_is_constant != 0, *cam, slots, lod_scalar,
                         alpha_stop, *out);
    return VV_OK;
}

float vv_camera_pixel_size(const vv_camera* cam) { return cam ? vv::camera_pixel_size(*cam) : 0.0f; }

int vv_make_jitter(uint32_t seed, int32_t size, uint8_t* out) {
    if (!out || size <= 0 || size > 256) return VV_ERR_ARG;
    vv::make_jitter(seed, size, out);
    return VV_OK;
}

int vv_renderer_create(vv_ctx* ctx, vv_octree* tree, const vv_renderer_desc* d, vv_renderer** out) {
    if (!ctx || !tree || !d || !out) return VV_ERR_ARG;
    *out = nullptr;
    try {
        auto r = std::make_unique<vv_renderer>();
        r->ctx = ctx;
        r->impl = std::make_unique<vv::GigaVoxelsRenderer>(ctx, tree, tree->tree.get(), *d);
        int rc = r->impl->init();
        if (rc) return rc;
        *out = r.release();
        return VV_OK;
    } catch (const std::bad_alloc&) {
        return VV_ERR_OOM;
    }
}

void vv_renderer_destroy(vv_renderer* r) { delete r; }

int vv_renderer_draw(vv_renderer* r, const vv_camera* cam) {
    if (!r || !cam) return VV_ERR_ARG;
    return r->impl->draw(*cam);
}

int vv_renderer_update(vv_renderer* r) {
    if (!r) return VV_ERR_ARG;
    return r->impl->update();
}

int vv_renderer_draw_passes(vv_renderer* r, const vv_camera* cam, int32_t passes) {
    if (!r || !cam) return VV_ERR_ARG;
    return r->impl->draw_passes(*cam, passes);
}

int vv_renderer_post_draw(vv_renderer* r) {
    if (!r) return VV_ERR_ARG;
    return r->impl->post_draw();
}

int vv_renderer_service(vv_renderer* r, const uint32_t* requests, const uint32_t* count, int32_t cap) {
    if (!r) return VV_ERR_ARG;
    return r->impl->service(requests, count, cap);
}

int vv_renderer_set_deferred(vv_renderer* r, int32_t on) {
    if (!r) return VV_ERR_ARG;
    return r->impl->set_deferred(on != 0);
}

int vv_renderer_stage_uploads(vv_renderer* r) {
    if (!r) return VV_ERR_ARG;
    return r->impl->stage_uploads();
}

int vv_renderer_enqueue_uploads(vv_renderer* r) {
    if (!r) return VV_ERR_ARG;
    return r->impl->enqueue_uploads();
}

int vv_renderer_get_stats(const vv_renderer* r, vv_renderer_stats* out) {
    if (!r || !out) return VV_ERR_ARG;
    r->impl->stats(*out);
    return VV_OK;
}

int vv_renderer_frame_buffers(vv_renderer* r, float** color, uint32_t** usage, uint32_t** mask, uint32_t** requests,
                              uint32_t** request_count) {
    if (!r) return VV_ERR_ARG;
    if (color) *color = r->impl->d_color;
    if (usage) *usage = r->impl->d_usage;
    if (mask) *mask = r->impl->d_mask;
    if (requests) *requests = r->impl->d_requests;
    if (request_count) *request_count = r->impl->d_count;
    return VV_OK;
}

int vv_renderer_read_color(vv_renderer* r, float* host_rgba) {
    if (!r || !host_rgba || !r->impl->d_color) return VV_ERR_ARG;
    const size_t bytes = (size_t)r->impl->width * r->impl->height * r->impl->color_bytes();
    if (cudaMemcpyAsync(host_rgba, r->impl->d_color, bytes, cudaMemcpyDeviceToHost, r->ctx->stream) != cudaSuccess)
        return VV_ERR_CUDA;
    if (cudaStreamSynchronize(r->ctx->stream) != cudaSuccess) return VV_ERR_CUDA;
    return VV_OK;
}

int vv_renderer_read_color_async(vv_renderer* r, float* host_rgba) {
    if (!r || !host_rgba) return VV_ERR_ARG;
    return r->impl->read_color_async(host_rgba);
}

int vv_renderer_wait_readback(vv_renderer* r) {
    if (!r) return VV_ERR_ARG;
    return r->impl->wait_readback();
}

int vv_renderer_read_lists(vv_renderer* r, uint32_t* host_usage, uint32_t* host_mask) {
    if (!r || !r->impl->d_usage) return VV_ERR_ARG;
    const size_t np = (size_t)r->impl->width * r->impl->height;
    cudaStream_t s = r->ctx->stream;
    if (host_usage && cudaMemcpyAsync(host_usage, r->impl->d_usage, np * 48, cudaMemcpyDeviceToHost, s) != cudaSuccess)
        return VV_ERR_CUDA;
    if (host_mask && cudaMemcpyAsync(host_mask, r->impl->d_mask, np * 4, cudaMemcpyDeviceToHost, s) != cudaSuccess)
        return VV_ERR_CUDA;
    if (cudaStreamSynchronize(s) != cudaSuccess) return VV_ERR_CUDA;
    return VV_OK;
}

int vv_renderer_last_requests(const vv_renderer* r, uint32_t* out, int32_t cap, int32_t* n) {
    if (!r || !n) return VV_ERR_ARG;
    std::vector<uint32_t> q;
    const int rc = const_cast<vv_renderer*>(r)->impl->last_requests(q);
    if (rc) return rc;
    const int32_t cnt = (int32_t)(q.size() / 4);
    *n = cnt;
    if (out) std::memcpy(out, q.data(), (size_t)std::min(cnt, cap) * 16);
    return VV_OK;
}

int vv_renderer_residency(const vv_renderer* r, uint32_t* out_xyz, uint32_t* out_slot, int64_t cap, int64_t* n) {
    if (!r || !n) return VV_ERR_ARG;
    std::vector<uint32_t> xyz, slot;
    r->impl->residency(xyz, slot);
    *n = (int64_t)slot.size();
    const size_t m = (size_t)std::min<int64_t>(cap, (int64_t)slot.size());
    if (out_xyz) std::memcpy(out_xyz, xyz.data(), m * 3 * 4);
    if (out_slot) std::memcpy(out_slot, slot.data(), m * 4);
    return VV_OK;
}

int vv_renderer_lru_order(vv_renderer* r, uint32_t* out, int64_t cap, int64_t* n) {
    if (!r || !n || cap < 0) return VV_ERR_ARG;
    std::vector<uint32_t> order;
    const int rc = r->impl->lru_order(order);
    if (rc) return rc;
    *n = (int64_t)order.size();
    if (out) std::memcpy(out, order.data(), (size_t)std::min<int64_t>(cap, (int64_t)order.size()) * 4);
    return VV_OK;
}

int vv_renderer_last_uniforms(const vv_renderer* r, vv_uniforms* out) {
    if (!r || !out) return VV_ERR_ARG;
    *out = r->impl->last_uniforms();
    return VV_OK;
}

vv_ctx* vv_renderer_ctx(vv_renderer* r) { return r ? r->ctx : nullptr; }

}  // extern "C"
