// renderer.cpp - GigaVoxels renderer frame protocol and page-request service.
#include "renderer.h"

#include "ctx.h"
#include "kernels.cuh"

#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <stdexcept>

#ifdef _OPENMP
#include <omp.h>
#endif

namespace vv {

namespace {

struct D3 {
    double x, y, z;
};
D3 d3(const float* a) { return D3{a[0], a[1], a[2]}; }
D3 operator+(D3 a, D3 b) { return D3{a.x + b.x, a.y + b.y, a.z + b.z}; }
D3 operator-(D3 a, D3 b) { return D3{a.x - b.x, a.y - b.y, a.z - b.z}; }
D3 operator*(D3 a, double s) { return D3{a.x * s, a.y * s, a.z * s}; }
double dot(D3 a, D3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
D3 cross(D3 a, D3 b) { return D3{a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }
D3 unit(D3 a) { return a * (1.0 / std::sqrt(dot(a, a))); }

// ComputePerspective (Camera.cpp:74-89): ymax = near * tanf(fovy * pi / 360).
void frustum_extent(const vv_camera& cam, double& xmax, double& ymax) {
    const double PI = 3.14159265358979323846;
    ymax = (double)cam.near_dist * (double)std::tan((float)((double)cam.fov_y_deg * PI / 360.0));
    const float aspect = (float)cam.width / (float)cam.height;
    xmax = ymax * (double)aspect;
}

}  // namespace

float camera_pixel_size(const vv_camera& cam) {
    // Unproject window points (W/2,H/2) and (W/2+1,H/2+1) on the near plane and
    // take 1 - cos of the angle between the two eye rays.  In eye space the
    // points are (x_ndc*xmax, y_ndc*ymax, -near).
    double xmax, ymax;
    frustum_extent(cam, xmax, ymax);
    const double n = cam.near_dist;
    D3 a{0.0, 0.0, -n};
    D3 b{(2.0 / cam.width) * xmax, (2.0 / cam.height) * ymax, -n};
    return (float)(1.0 - dot(unit(a), unit(b)));
}

void make_jitter(uint32_t seed, int size, uint8_t* out) {
    for (int i = 0; i < size * size; ++i) {
        uint32_t h = lattice_hash((uint32_t)i, 0x51ED27u, seed ^ 0xA5A5A5A5u);
        // rand()/RAND_MAX scaled to 255, zero bumped to one (GLUtils.cpp:478-485)
        float f = (float)(h >> 8) * (1.0f / 16777215.0f);
        unsigned char v = (unsigned char)(255.0f * f);
        if (v == 0) v = 1;
        out[i] = v;
    }
}

void compute_uniforms(int depth, int leaf_dim, bool root_is_constant, const vv_camera& cam, const int slots[3],
                      float lod_scalar, float alpha_stop, vv_uniforms& u) {
    std::memset(&u, 0, sizeof(u));
    // The volume box is [0,1]^3: translation 0.5, scale 1 (:1655-1672).
    const float trans = 0.5f, scale = 1.0f;
    for (int a = 0; a < 3; ++a) {
        u.vol_extent_min[a] = ((0.0f - trans) / scale) + 0.5f;
        u.vol_extent_max[a] = ((1.0f - trans) / scale) + 0.5f;
        u.camera_position[a] = ((cam.position[a] - trans) / scale) + 0.5f;
    }
    D3 look = unit(d3(cam.look)), up = unit(d3(cam.up));
    D3 left = unit(cross(up, look));  // vox::Camera keeps left = up x look
    const float upf[3] = {(float)up.x, (float)up.y, (float)up.z};
    const float leftf[3] = {(float)left.x, (float)left.y, (float)left.z};
    std::memcpy(u.camera_up, upf, sizeof(upf));
    std::memcpy(u.camera_left, leftf, sizeof(leftf));
    // RayStepSize = getRayStepSize() * 0.5 with getRayStepSize = one leaf
    // voxel (GigaVoxelsReader.cpp:430-440; GigaVoxelsRenderer.cpp:1705).
    const int N = leaf_dim > 0 ? leaf_dim : 8 << depth;
    const float leaf = (1.0f / (float)N) / (1.0f - 0.0f);
    const float rs = leaf * 0.5f;
    u.ray_step_size = rs;
    // BrickStepVector (:1728-1751)
    const float pow2 = std::pow(2.0f, (float)depth);
    const float bd[3] = {8.0f, 8.0f, 8.0f};
    for (int a = 0; a < 3; ++a) {
        float root_step = (scale * rs) * pow2;
        float root_voxel = scale / bd[a];
        float ratio = root_step / root_voxel;
        float pool_dim = (float)(slots[a] * 10);
        float pool_voxel = 1.0f / pool_dim;
        u.brick_step_vector[a] = pool_voxel * ratio;
        u.brick_dimension[a] = bd[a];
        u.brick_pool_dimension[a] = pool_dim;
    }
    u.root_voxel_half_size = (1.0f / 8.0f) * 0.5f;  // (:1780-1787)
    // LightPosition: world (0, 100, 0) / volScale + 0.5 (:1695-1699); lighting off
    const float light[3] = {0.0f, 100.0f, 0.0f};
    for (int a = 0; a < 3; ++a) u.light_position[a] = (light[a] / scale) + 0.5f;
    u.compute_lighting = 0;
    u.gradients_unsigned = 0;
    u.pixel_size = camera_pixel_size(cam);
    u.lod_scalar = lod_scalar;
    u.alpha_stop = alpha_stop;
    u.oct_tree_depth_minus_one = depth;
    u.max_nodes_to_push = 12 * ((cam.frame % 2) + 1);  // (:1813-1816)
    u.root_node_is_constant = root_is_constant ? 1 : 0;
    u.jitter_tex_size = 32;
    u.width = cam.width;
    u.height = cam.height;
    const D3 C = d3(cam.position);
    u.camera_inside = (C.x > 0.0 && C.x < 1.0 && C.y > 0.0 && C.y < 1.0 && C.z > 0.0 && C.z < 1.0) ? 1 : 0;
    double xmax, ymax;
    frustum_extent(cam, xmax, ymax);
    D3 right = left * -1.0;
    // camera-relative near-plane corner of window coordinate (0,0)
    D3 O = look * (double)cam.near_dist - right * xmax - up * ymax;
    D3 dx = right * (2.0 * xmax / cam.width), dy = up * (2.0 * ymax / cam.height);
    const double o[3] = {O.x, O.y, O.z}, ddx[3] = {dx.x, dx.y, dx.z}, ddy[3] = {dy.x, dy.y, dy.z};
    for (int a = 0; a < 3; ++a) {
        u.near_origin[a] = (float)o[a];
        u.near_dx[a] = (float)ddx[a];
        u.near_dy[a] = (float)ddy[a];
    }
}

GigaVoxelsRenderer::GigaVoxelsRenderer(vv_ctx* ctx, vv_octree*, const GigaVoxelsOctTree* tree,
                                       const vv_renderer_desc& d)
    : ctx_(ctx), tree_(tree), d_(d) {}

GigaVoxelsRenderer::~GigaVoxelsRenderer() {
    if (ctx_) vv_ctx_synchronize(ctx_);
    if (copy_stream_) {
        cudaStreamSynchronize(copy_stream_);
        cudaStreamDestroy(copy_stream_);
        for (cudaEvent_t e : {ev_copied_[0], ev_copied_[1], ev_drawn_})
            if (e) cudaEventDestroy(e);
    }
    void* bufs[] = {color_buf_[0], color_buf_[1], d_usage, d_mask, d_requests, d_count};
    for (void* b : bufs)
        if (b) cudaFree(b);
    if (h_stage_) cudaFreeHost(h_stage_);
    if (h_small_) cudaFreeHost(h_small_);
    if (h_cand_) cudaFreeHost(h_cand_);
    if (h_unique_) cudaFreeHost(h_unique_);
    if (h_win_) cudaFreeHost(h_win_);
    if (h_seq_) cudaFreeHost(h_seq_);
    if (ev_seq_) cudaEventDestroy(ev_seq_);
    void* dbufs[] = {dd_.first, dd_.block_sums, dd_.unique, d_fjobs_, d_fpatch_,  // dd_.count: order_.counters
                     d_def_jobs_, d_def_patches_, d_def_counts_};
    for (void* b : dbufs)
        if (b) cudaFree(b);
    slot_order_free(order_);
    if (ev_flush_) cudaEventDestroy(ev_flush_);
    void* hbufs[] = {h_def_jobs_, h_def_patches_, (void*)h_def_counts_, h_fjobs_, h_fpatch_};
    for (void* b : hbufs)
        if (b) cudaFreeHost(b);
}

int GigaVoxelsRenderer::init() {
    const size_t bb = brick_bytes(d_.fmt);
    if (!bb || d_.fmt == VV_FMT_DXT1) return VV_ERR_ARG;
    brick_bytes_ = bb;
    size_t want;
    if (d_.pool_bytes > 0) want = (size_t)d_.pool_bytes / bb;
    else want = tree_->nonconst_count() + 1;
    if (want < 1) want = 1;
    // BrickPool::init slot grid (GigaVoxelsBrickPool.cpp:75-87)
    size_t cr = (size_t)std::pow((double)want, 1.0 / 3.0);
    if (cr < 1) cr = 1;
    size_t sx = cr, sy = cr, sz = cr;
    while (sx * sy * sz < want) ++sx;
    if (sx > 102 || sy > 102 || sz > 102) return VV_ERR_ARG;
    slots_[0] = (int)sx;
    slots_[1] = (int)sy;
    slots_[2] = (int)sz;
    total_slots_ = (uint32_t)(sx * sy * sz);
    int rc = vv_brickpool_create(ctx_, slots_[0], slots_[1], slots_[2], d_.fmt);
    if (rc) return rc;
    // LRU order: slot-id order on the device, and the same in the host window
    if (slot_order_init(order_, total_slots_, ctx_->stream) != cudaSuccess) return VV_ERR_OOM;
    if (cudaHostAlloc((void**)&h_win_, (size_t)total_slots_ * 4, cudaHostAllocMapped) != cudaSuccess ||
        cudaMallocHost((void**)&h_seq_, (size_t)total_slots_ * 4) != cudaSuccess)
        return VV_ERR_OOM;
    if (cudaHostGetDevicePointer((void**)&dh_win_, h_win_, 0) != cudaSuccess) return VV_ERR_CUDA;
    rc = ensure_small();
    if (rc) return rc;
    if (cudaEventCreateWithFlags(&ev_seq_, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&ev_flush_, cudaEventDisableTiming) != cudaSuccess)
        return VV_ERR_CUDA;
    for (uint32_t i = 0; i < total_slots_; ++i) h_win_[i] = i;
    head_ = 0;
    epoch_ = 1;
    win_start_ = 0;
    win_len_ = total_slots_;
    touch_seen_.assign(total_slots_, 0u);
    if (d_.device_paging) {
        device_paging_ = true;
        if (tree_->file_backed()) {
            dstore_ = std::make_unique<DeviceBrickStore>();
            if (dstore_->upload(tree_->file_texels(), tree_->file_brick_count()) != cudaSuccess) return VV_ERR_OOM;
        } else {
            dterrain_ = std::make_unique<DeviceTerrain>();
            if (dterrain_->upload(tree_->volume()) != cudaSuccess) return VV_ERR_OOM;
        }
        const int* g = tree_->pool_dim();
        dd_.first_cells = (size_t)g[0] * g[1] * g[2];
        if (cudaMalloc((void**)&dd_.first, dd_.first_cells * 4) != cudaSuccess) return VV_ERR_OOM;
        if (cudaMemset(dd_.first, 0xFF, dd_.first_cells * 4) != cudaSuccess) return VV_ERR_CUDA;
        dd_.count = order_.counters;  // counters[0]: the distinct count
    }
    const size_t nn = tree_->node_count();
    w0_.resize(nn);
    w1_.resize(nn);
    for (size_t i = 0; i < nn; ++i) {
        w0_[i] = tree_->word0((uint32_t)i);
        w1_[i] = tree_->word1((uint32_t)i);
    }
    const int* pd = tree_->pool_dim();
    std::vector<uint32_t> words((size_t)pd[0] * pd[1] * pd[2] * 2);
    tree_->words_grid(words.data());
    rc = vv_nodepool_upload(ctx_, 0, words.data(), pd[0], pd[1], pd[2]);
    if (rc) return rc;
    std::vector<uint8_t> jit(32 * 32);
    make_jitter(d_.jitter_seed, 32, jit.data());
    rc = vv_set_jitter(ctx_, jit.data(), 32);
    if (rc) return rc;
    slot_node_.assign(total_slots_, -1);
    node_slot_.assign(nn, -1);
    touched_mark_.assign(nn, 0);
    seen_mark_.assign(nn, 0);
    // BrickPool::initBricks (GigaVoxelsBrickPool.cpp:270-354): the root
    // brick, or every brick when the pool holds them all.
    if (d_.preload_all) {
        for (size_t n = 0; n < nn; ++n)
            if (tree_->level((uint32_t)n) >= 0 && !tree_->is_constant((uint32_t)n)) {
                if (pending_nodes_.size() >= total_slots_) break;
                rc = upload_nodes((uint32_t)n);
                if (rc) return rc;
            }
    } else if (!tree_->is_constant(0)) {
        rc = upload_nodes(0);
        if (rc) return rc;
    }
    rc = flush_uploads();
    uploaded_ = 0;
    return rc;
}

int GigaVoxelsRenderer::alloc_frame(int w, int h) {
    if (w == width && h == height && d_color) return VV_OK;
    void** bufs[] = {(void**)&color_buf_[0], (void**)&color_buf_[1], (void**)&d_usage, (void**)&d_mask,
                     (void**)&d_requests, (void**)&d_count};
    vv_ctx_synchronize(ctx_);
    if (copy_stream_) cudaStreamSynchronize(copy_stream_);
    copy_pending_[0] = copy_pending_[1] = false;
    for (void** b : bufs)
        if (*b) {
            cudaFree(*b);
            *b = nullptr;
        }
    d_color = nullptr;
    const size_t np = (size_t)w * h;
    cap_ = d_.request_cap > 0 ? d_.request_cap : (int)np;
    // two colour buffers: a frame's read-back may run while the next is drawn
    if (cudaMalloc((void**)&color_buf_[0], np * color_bytes()) != cudaSuccess) return VV_ERR_OOM;
    if (cudaMalloc((void**)&color_buf_[1], np * color_bytes()) != cudaSuccess) return VV_ERR_OOM;
    d_color = color_buf_[cur_color_];
    if (cudaMalloc((void**)&d_usage, np * 48) != cudaSuccess) return VV_ERR_OOM;
    if (cudaMalloc((void**)&d_mask, np * 4) != cudaSuccess) return VV_ERR_OOM;
    if (cudaMalloc((void**)&d_requests, (size_t)cap_ * 16) != cudaSuccess) return VV_ERR_OOM;
    if (cudaMalloc((void**)&d_count, 4) != cudaSuccess) return VV_ERR_OOM;
    width = w;
    height = h;
    return VV_OK;
}

int GigaVoxelsRenderer::draw(const vv_camera& cam) { return draw_passes(cam, VV_PASS_ALL); }

int GigaVoxelsRenderer::draw_passes(const vv_camera& cam, int passes) {
    if ((passes & VV_PASS_RAYCAST) == 0 || (passes & ~VV_PASS_ALL) != 0) return VV_ERR_ARG;
    const int rc = prepare_draw(cam);
    if (rc) return rc;
    // the selection mask and histopyramid belong to the draw (drawVolume,
    // GigaVoxelsRenderer.cpp:1070-1088); the compaction to postDraw (:1150-1186)
    compact_pending_ = false;
    const int rc2 = finish_draw(passes | VV_PASS_SELECT);
    if (rc2) return rc2;
    compact_pending_ = (passes & VV_PASS_COMPACT) == 0;
    return VV_OK;
}

int GigaVoxelsRenderer::post_draw() {
    if (!compact_pending_) return VV_OK;
    compact_pending_ = false;
    return finish_draw(VV_PASS_COMPACT);
}

int GigaVoxelsRenderer::prepare_draw(const vv_camera& cam) {
    int rc = start_readback();  // a read-back requested without a service since
    if (rc) return rc;
    rc = alloc_frame(cam.width, cam.height);
    if (rc) return rc;
    // alternate colour buffers; wait for a pending read-back of the one reused
    cur_color_ ^= 1;
    if (copy_pending_[cur_color_]) {
        if (cudaStreamWaitEvent(ctx_->stream, ev_copied_[cur_color_], 0) != cudaSuccess) return VV_ERR_CUDA;
        copy_pending_[cur_color_] = false;
    }
    d_color = color_buf_[cur_color_];
    compute_uniforms(tree_->depth(), tree_->leaf_dim(), tree_->is_constant(0), cam, slots_, d_.lod_scalar,
                     d_.alpha_stop, last_u_);
    frame_ = cam.frame;
    return VV_OK;
}

int GigaVoxelsRenderer::finish_draw(int passes) {
    if (!d_color) return VV_ERR_STATE;
    vv_frame_out o;
    std::memset(&o, 0, sizeof(o));
    o.color = d_color;
    o.usage = d_usage;
    o.mask = d_mask;
    o.requests = d_requests;
    o.request_count = d_count;
    o.request_cap = cap_;
    o.compress_max_push = 4 * ((int)(frame_ % 3) + 1);  // (GigaVoxelsRenderer.cpp:2093-2098)
    o.passes = passes | (d_.color_rgba8 ? VV_PASS_COLOR_RGBA8 : 0);
    return vv_render(ctx_, 0, &last_u_, &o);
}

int GigaVoxelsRenderer::read_color_async(void* host) {
    if (!d_color || !host) return VV_ERR_ARG;
    if (!copy_stream_) {
        if (cudaStreamCreateWithFlags(&copy_stream_, cudaStreamNonBlocking) != cudaSuccess) return VV_ERR_CUDA;
        for (int i = 0; i < 2; ++i)
            if (cudaEventCreateWithFlags(&ev_copied_[i], cudaEventDisableTiming) != cudaSuccess) return VV_ERR_CUDA;
        if (cudaEventCreateWithFlags(&ev_drawn_, cudaEventDisableTiming) != cudaSuccess) return VV_ERR_CUDA;
    }
    int rc = start_readback();  // an earlier request goes out first
    if (rc) return rc;
    if (cudaEventRecord(ev_drawn_, ctx_->stream) != cudaSuccess) return VV_ERR_CUDA;
    // The copy starts at the end of the page-request service (update or
    // service), or at the next draw or wait: the bulk transfer would
    // otherwise hold the device-to-host direction of the bus while the
    // service waits for its small read-outs.  It then overlaps the next ray
    // cast instead.
    readback_host_ = host;
    readback_buf_ = cur_color_;
    copy_pending_[cur_color_] = true;
    return VV_OK;
}

int GigaVoxelsRenderer::start_readback() {
    if (!readback_host_) return VV_OK;
    void* host = readback_host_;
    readback_host_ = nullptr;
    if (cudaStreamWaitEvent(copy_stream_, ev_drawn_, 0) != cudaSuccess) return VV_ERR_CUDA;
    if (cudaMemcpyAsync(host, color_buf_[readback_buf_], (size_t)width * height * color_bytes(), cudaMemcpyDeviceToHost,
                        copy_stream_) != cudaSuccess)
        return VV_ERR_CUDA;
    if (cudaEventRecord(ev_copied_[readback_buf_], copy_stream_) != cudaSuccess) return VV_ERR_CUDA;
    return VV_OK;
}

int GigaVoxelsRenderer::wait_readback() {
    int rc = start_readback();
    if (rc) return rc;
    if (copy_stream_ && cudaStreamSynchronize(copy_stream_) != cudaSuccess) return VV_ERR_CUDA;
    return VV_OK;
}

int GigaVoxelsRenderer::ensure_small() {
    if (h_small_) return VV_OK;
    if (cudaHostAlloc((void**)&h_small_, 32, cudaHostAllocMapped) != cudaSuccess) return VV_ERR_OOM;
    std::memset(h_small_, 0, 32);
    if (cudaHostGetDevicePointer((void**)&dh_small_, h_small_, 0) != cudaSuccess) return VV_ERR_CUDA;
    return VV_OK;
}

int GigaVoxelsRenderer::read_count(const uint32_t* count, uint32_t& out) {
    int rc = ensure_small();
    if (rc) return rc;
    if (launch_read_word(count, dh_small_, ctx_->stream) != cudaSuccess) return VV_ERR_CUDA;
    if (cudaStreamSynchronize(ctx_->stream) != cudaSuccess) return VV_ERR_CUDA;
    out = h_small_[0];
    return VV_OK;
}

int GigaVoxelsRenderer::next_epoch() {
    if (++epoch_ == 0) {  // marks of every earlier epoch would collide: clear them
        if (cudaMemsetAsync(order_.mark, 0, (size_t)total_slots_ * 4, ctx_->stream) != cudaSuccess)
            return VV_ERR_CUDA;
        epoch_ = 1;
    }
    return VV_OK;
}

int GigaVoxelsRenderer::flush_touches() {
    if (pending_touch_.empty()) return VV_OK;
    const uint32_t n = total_slots_;
    if (++touch_stamp_ == 0) {
        std::fill(touch_seen_.begin(), touch_seen_.end(), 0u);
        touch_stamp_ = 1;
    }
    // the previous partition's copy out of h_seq_ must have been read
    if (cudaEventSynchronize(ev_seq_) != cudaSuccess) return VV_ERR_CUDA;
    // a slot touched more than once keeps its last touch
    uint32_t m = 0;
    for (size_t i = pending_touch_.size(); i-- > 0;) {
        const uint32_t s = pending_touch_[i];
        if (s >= n) return ctx_fail(ctx_, VV_ERR_BOUNDS, "touch of a slot outside the brick pool");
        if (touch_seen_[s] == touch_stamp_) continue;
        touch_seen_[s] = touch_stamp_;
        h_seq_[m++] = s;
    }
    std::reverse(h_seq_, h_seq_ + m);
    pending_touch_.clear();
    if (cudaMemcpyAsync(order_.seq, h_seq_, (size_t)m * 4, cudaMemcpyHostToDevice, ctx_->stream) != cudaSuccess ||
        cudaEventRecord(ev_seq_, ctx_->stream) != cudaSuccess)
        return VV_ERR_CUDA;
    if (launch_mark_touched(order_, m, epoch_, ctx_->d_status, ctx_->stream) != cudaSuccess ||
        launch_order_partition(order_, head_, epoch_, false, m, m, 0xFFFFFFFFu, ctx_->d_status, ctx_->stream) !=
            cudaSuccess)
        return VV_ERR_CUDA;
    head_ = 0;
    win_len_ = 0;
    return next_epoch();
}

int GigaVoxelsRenderer::fetch_order(uint32_t want) {
    const uint32_t n = total_slots_;
    const uint32_t len = std::min<uint32_t>(n, std::max<uint32_t>(want, 65536u));
    const uint32_t first = std::min<uint32_t>(len, n - head_);
    const uint32_t* d = order_.order[order_.cur];
    if (cudaMemcpyAsync(h_win_, d + head_, (size_t)first * 4, cudaMemcpyDeviceToHost, ctx_->stream) != cudaSuccess)
        return VV_ERR_CUDA;
    if (len > first &&
        cudaMemcpyAsync(h_win_ + first, d, (size_t)(len - first) * 4, cudaMemcpyDeviceToHost, ctx_->stream) !=
            cudaSuccess)
        return VV_ERR_CUDA;
    if (cudaStreamSynchronize(ctx_->stream) != cudaSuccess) return VV_ERR_CUDA;
    win_start_ = head_;
    win_len_ = len;
    return VV_OK;
}

int GigaVoxelsRenderer::evict_front(uint32_t& s) {
    int rc = flush_touches();  // touches made so far come before this eviction
    if (rc) return rc;
    const uint32_t n = total_slots_;
    uint32_t off = head_ >= win_start_ ? head_ - win_start_ : head_ + n - win_start_;
    if (off >= win_len_) {
        rc = fetch_order(evict_hint_);
        if (rc) return rc;
        off = 0;
    }
    s = h_win_[off];
    if (s >= n) return ctx_fail(ctx_, VV_ERR_BOUNDS, "the LRU order holds a slot outside the brick pool");
    // the front slot goes to the back: in the full circular order, the head advances
    head_ = head_ + 1 == n ? 0 : head_ + 1;
    if (evict_hint_) --evict_hint_;
    return VV_OK;
}

// The device production job of node `node` into slot `slot`: the terrain
// node's level and brick index, or the file tree's store brick.
uint4 GigaVoxelsRenderer::production_job(uint32_t slot, uint32_t node) const {
    if (tree_->file_backed()) return make_uint4(slot, (uint32_t)tree_->file_brick(node), 0u, 0u);
    int ci, cj, ck;
    tree_->origin(node, ci, cj, ck);
    return make_uint4(slot, (uint32_t)tree_->level(node), ((uint32_t)ci << 20) | ((uint32_t)cj << 10) | (uint32_t)ck,
                      0u);
}

int GigaVoxelsRenderer::upload_nodes(uint32_t n) {
    // BrickPool::update body (GigaVoxelsBrickPool.cpp:583-629): evict the
    // LRU front, upload into its slot, move it to the back.
    uint32_t s;
    const int rc = evict_front(s);
    if (rc) return rc;
    const int32_t old = slot_node_[s];
    if (old >= 0) {
        node_slot_[(size_t)old] = -1;
        w0_[(size_t)old] &= ~kBrickResidentBit;
        if (!touched_mark_[(size_t)old]) {
            touched_mark_[(size_t)old] = 1;
            touched_.push_back((uint32_t)old);
        }
        ++evictions_;
        --resident_;
    }
    slot_node_[s] = (int32_t)n;
    node_slot_[n] = (int32_t)s;
    const uint32_t sx = s % (uint32_t)slots_[0], sy = (s / (uint32_t)slots_[0]) % (uint32_t)slots_[1],
                   sz = s / ((uint32_t)slots_[0] * (uint32_t)slots_[1]);
    // uploadBrick (:800-810): pointer = slot origin + border
    uint32_t b[3];
    tree_->brick_border(n, b);
    w1_[n] = pack10(sx * 10 + b[0], sy * 10 + b[1], sz * 10 + b[2]);
    w0_[n] |= kBrickResidentBit;
    if (!touched_mark_[n]) {
        touched_mark_[n] = 1;
        touched_.push_back(n);
    }
    pending_nodes_.push_back(n);
    pending_slots_.push_back(s);
    ++uploaded_;
    ++uploaded_total_;
    ++resident_;
    return VV_OK;
}

int GigaVoxelsRenderer::flush_uploads() {
    int rc = VV_OK;
    ms_produce_ = 0.0f;
    const auto t0 = std::chrono::steady_clock::now();
    // One upload per slot, the latest: a slot re-used within a service holds
    // its last node, and the bricks of one launch are written in no fixed
    // order.  keep_ lists those pending uploads, latest first.
    if (slot_job_.size() != total_slots_) slot_job_.assign(total_slots_, -1);
    keep_.clear();
    for (size_t i = pending_nodes_.size(); i-- > 0;) {
        const uint32_t s = pending_slots_[i];
        if (slot_job_[s] >= 0) continue;
        slot_job_[s] = (int32_t)i;
        keep_.push_back((uint32_t)i);
    }
    for (uint32_t i : keep_) slot_job_[pending_slots_[i]] = -1;
    const size_t n = keep_.size();
    if (device_paging_) {
        rc = flush_device();
        ms_upload_ = std::chrono::duration<float, std::milli>(std::chrono::steady_clock::now() - t0).count();
        return rc;
    }
    if (n) {
        const size_t bb = brick_bytes_;
        const size_t bytes = n * bb;
        if (h_stage_cap_ < bytes) {
            // pinned memory is slow to allocate: grow geometrically, at least 4096 bricks
            const size_t want = std::max(std::max(bytes, 2 * h_stage_cap_), 4096 * bb);
            if (h_stage_) cudaFreeHost(h_stage_);
            h_stage_ = nullptr;
            h_stage_cap_ = 0;
            if (cudaMallocHost(&h_stage_, want) != cudaSuccess) return VV_ERR_OOM;
            h_stage_cap_ = want;
        }
        unsigned char* st = (unsigned char*)h_stage_;
        const int fmt = d_.fmt;
        up_slots_.resize(n);
        for (size_t k = 0; k < n; ++k) up_slots_[k] = pending_slots_[keep_[k]];
#pragma omp parallel for schedule(dynamic, 16) num_threads(d_.producer_threads > 0 ? d_.producer_threads : omp_get_max_threads())
        for (long k = 0; k < (long)n; ++k)
            tree_->produce_brick(pending_nodes_[keep_[(size_t)k]], fmt, st + (size_t)k * bb);
        ms_produce_ = std::chrono::duration<float, std::milli>(std::chrono::steady_clock::now() - t0).count();
    }
    const auto t2 = std::chrono::steady_clock::now();
    if (n) {
        rc = vv_upload_bricks(ctx_, up_slots_.data(), (int32_t)n, h_stage_);
        if (rc) return rc;
    }
    if (!touched_.empty()) {
        std::vector<vv_node_patch> patches;
        patches.reserve(touched_.size());
        for (uint32_t t : touched_) {
            vv_node_patch q;
            tree_->grid_of(t, q.x, q.y, q.z);
            q.word0 = w0_[t];
            q.word1 = w1_[t];
            patches.push_back(q);
            touched_mark_[t] = 0;
        }
        touched_.clear();
        rc = vv_nodepool_patch(ctx_, 0, patches.data(), (int32_t)patches.size());
        if (rc) return rc;
    }
    pending_nodes_.clear();
    pending_slots_.clear();
    ms_upload_ = std::chrono::duration<float, std::milli>(std::chrono::steady_clock::now() - t2).count();
    return rc;
}

// Device paging: brick production on the GPU, straight into the slots, and
// the node patches.  Jobs and patches are written to mapped pinned memory;
// one coalesced kernel pulls them into device memory, so the service queues
// no transfer on the copy engines (which a frame's colour read-back may
// hold), and the production and patch kernels read device memory.
int GigaVoxelsRenderer::flush_device() {
    const size_t n = keep_.size(), np = touched_.size();
    if (n == 0 && np == 0) {
        pending_nodes_.clear();
        pending_slots_.clear();
        return VV_OK;
    }
    // the previous flush's pull has finished reading the mapped buffers
    if (cudaEventSynchronize(ev_flush_) != cudaSuccess) return VV_ERR_CUDA;
    if (fjobs_cap_ < n) {  // pinned allocations are slow: grow geometrically
        if (h_fjobs_) cudaFreeHost(h_fjobs_);
        if (d_fjobs_) cudaFree(d_fjobs_);
        h_fjobs_ = d_fjobs_ = nullptr;
        fjobs_cap_ = std::max<size_t>(std::max(n, 2 * fjobs_cap_), 16384);
        if (cudaHostAlloc((void**)&h_fjobs_, fjobs_cap_ * sizeof(uint4), cudaHostAllocMapped) != cudaSuccess ||
            cudaMalloc((void**)&d_fjobs_, fjobs_cap_ * sizeof(uint4)) != cudaSuccess) {
            fjobs_cap_ = 0;
            return VV_ERR_OOM;
        }
        if (cudaHostGetDevicePointer((void**)&dh_fjobs_, h_fjobs_, 0) != cudaSuccess) return VV_ERR_CUDA;
    }
    if (fpatch_cap_ < np) {
        if (h_fpatch_) cudaFreeHost(h_fpatch_);
        if (d_fpatch_) cudaFree(d_fpatch_);
        h_fpatch_ = d_fpatch_ = nullptr;
        fpatch_cap_ = std::max<size_t>(std::max(np, 2 * fpatch_cap_), 32768);
        // whole 16-byte words: the pull reads the last partial one
        const size_t bytes = (fpatch_cap_ * sizeof(vv_node_patch) + 15) / 16 * 16;
        if (cudaHostAlloc((void**)&h_fpatch_, bytes, cudaHostAllocMapped) != cudaSuccess ||
            cudaMalloc((void**)&d_fpatch_, bytes) != cudaSuccess) {
            fpatch_cap_ = 0;
            return VV_ERR_OOM;
        }
        if (cudaHostGetDevicePointer((void**)&dh_fpatch_, h_fpatch_, 0) != cudaSuccess) return VV_ERR_CUDA;
    }
    constexpr size_t kAhead = 16;  // records prefetched ahead (far apart in the arrays)
    for (size_t k = 0; k < n; ++k) {
        if (k + kAhead < n) tree_->prefetch(pending_nodes_[keep_[k + kAhead]]);
        const uint32_t i = keep_[k];
        h_fjobs_[k] = production_job(pending_slots_[i], pending_nodes_[i]);
    }
    for (size_t k = 0; k < np; ++k) {
        if (k + kAhead < np) {
            const uint32_t f = touched_[k + kAhead];
            __builtin_prefetch(&w0_[f]);
            __builtin_prefetch(&w1_[f]);
            __builtin_prefetch(&touched_mark_[f]);
        }
        const uint32_t t = touched_[k];
        vv_node_patch& q = h_fpatch_[k];
        tree_->grid_of(t, q.x, q.y, q.z);
        q.word0 = w0_[t];
        q.word1 = w1_[t];
        touched_mark_[t] = 0;
    }
    void* pool = nullptr;
    size_t pool_bytes = 0;
    vv_brickpool_device_ptr(ctx_, &pool, &pool_bytes);
    const DeviceTree& t = ctx_->trees[0];
    const size_t patch_words = (np * sizeof(vv_node_patch) + 15) / 16;
    if (launch_pull(dh_fjobs_, d_fjobs_, n, (const uint4*)dh_fpatch_, (uint4*)d_fpatch_, patch_words,
                    ctx_->stream) != cudaSuccess ||
        cudaEventRecord(ev_flush_, ctx_->stream) != cudaSuccess ||
        (dstore_ ? launch_copy_bricks(dstore_->view(), d_fjobs_, (int)n, pool, d_.fmt, ctx_cell_mask_rw(ctx_),
                                      (long long)total_slots_, ctx_->d_status, ctx_->stream)
                 : launch_produce_bricks(dterrain_->view(), d_fjobs_, (int)n, pool, d_.fmt, ctx_cell_mask_rw(ctx_),
                                         (long long)total_slots_, ctx_->d_status, ctx_->stream)) != cudaSuccess ||
        launch_node_patch(d_fpatch_, (int)np, t.nodes, t.dim, ctx_->d_status, ctx_->stream) != cudaSuccess)
        return VV_ERR_CUDA;
    touched_.clear();
    pending_nodes_.clear();
    pending_slots_.clear();
    return VV_OK;
}

// One distinct requested node, in first-seen order (NodeUsageListProcessor::run,
// GigaVoxelsOctTree.cpp:509-523): touch its brick if resident, else queue a
// non-constant node for upload.
void GigaVoxelsRenderer::visit(uint32_t nidx, std::vector<uint32_t>& upload) {
    if (node_slot_[nidx] >= 0) touch((uint32_t)node_slot_[nidx]);
    else if (!tree_->is_constant(nidx)) upload.push_back(nidx);
}

int GigaVoxelsRenderer::update_host(uint32_t n, std::vector<uint32_t>& upload) {
    host_requests_.resize((size_t)n * 4);
    if (n) {
        if (cudaMemcpyAsync(host_requests_.data(), d_requests, (size_t)n * 16, cudaMemcpyDeviceToHost,
                            ctx_->stream) != cudaSuccess)
            return VV_ERR_CUDA;
        if (cudaStreamSynchronize(ctx_->stream) != cudaSuccess) return VV_ERR_CUDA;
    }
    requests_on_host_ = true;
    if (++seen_epoch_ == 0) {
        std::fill(seen_mark_.begin(), seen_mark_.end(), 0u);
        seen_epoch_ = 1;
    }
    for (size_t i = 0; i < host_requests_.size(); ++i) {
        const uint32_t id = host_requests_[i];
        if (id == 0u) continue;
        const uint32_t x = ((id >> 20) & 0x3FFu) - 1u, y = ((id >> 10) & 0x3FFu) - 1u, z = (id & 0x3FFu) - 1u;
        const uint32_t nidx = tree_->index_of(x, y, z);
        if (nidx == kNoParent || tree_->level(nidx) < 0) continue;
        if (seen_mark_[nidx] == seen_epoch_) continue;
        seen_mark_[nidx] = seen_epoch_;
        visit(nidx, upload);
    }
    return VV_OK;
}

int GigaVoxelsRenderer::update_device(uint32_t n, std::vector<uint32_t>& upload, const uint32_t* requests) {
    requests_on_host_ = false;
    root_on_device_ = false;
    if (!n) return VV_OK;
    const size_t ids = (size_t)n * 4, blocks = (ids + 1023) / 1024;
    if (dd_.block_cap < blocks) {
        if (dd_.block_sums) cudaFree(dd_.block_sums);
        dd_.block_sums = nullptr;
        dd_.block_cap = std::max(blocks, 2 * dd_.block_cap);
        if (cudaMalloc((void**)&dd_.block_sums, dd_.block_cap * 4) != cudaSuccess) return VV_ERR_OOM;
    }
    if (dd_.unique_cap < ids) {
        if (dd_.unique) cudaFree(dd_.unique);
        dd_.unique = nullptr;
        dd_.unique_cap = std::max(ids + ids / 4, 2 * dd_.unique_cap);  // headroom: counts vary a little
        if (cudaMalloc((void**)&dd_.unique, dd_.unique_cap * 4) != cudaSuccess) return VV_ERR_OOM;
    }
    const int* pd = tree_->pool_dim();
    if (launch_dedupe(requests, (int)n, pd, dd_, ctx_->stream) != cudaSuccess) return VV_ERR_CUDA;
    // When the device node words hold this renderer's state (no node-word
    // change is pending on the host), the distinct nodes are classified on
    // the device, whose LRU order takes their touches and the root's; the
    // host reads back only the upload candidates and the order's front.
    // (deferred uploads: once the device has applied the last staging)
    const bool classified = touched_.empty() && (!deferred_ || h_def_counts_[3] == h_def_counts_[2]);
    uint32_t root_slot = 0xFFFFFFFFu;
    if (classified) {
        int rc = flush_touches();  // earlier host touches come first
        if (rc) return rc;
        if (order_.cand_cap < ids) {
            if (order_.cand) cudaFree(order_.cand);
            order_.cand = nullptr;
            order_.cand_cap = std::max(ids + ids / 4, 2 * order_.cand_cap);
            if (cudaMalloc((void**)&order_.cand, order_.cand_cap * 4) != cudaSuccess) {
                order_.cand_cap = 0;
                return VV_ERR_OOM;
            }
        }
        if (order_.cand_sums_cap < blocks) {
            if (order_.cand_sums) cudaFree(order_.cand_sums);
            order_.cand_sums = nullptr;
            order_.cand_sums_cap = dd_.block_cap;
            if (cudaMalloc((void**)&order_.cand_sums, order_.cand_sums_cap * 4) != cudaSuccess) {
                order_.cand_sums_cap = 0;
                return VV_ERR_OOM;
            }
        }
        if (node_slot_[0] >= 0) root_slot = (uint32_t)node_slot_[0];
        const DeviceTree& t = ctx_->trees[0];
        if (launch_classify_split(dd_, (uint32_t)ids, t.nodes, t.dim, slots_, root_slot, epoch_, order_,
                                  ctx_->d_status, ctx_->stream) != cudaSuccess ||
            launch_order_partition(order_, head_, epoch_, true, 0, (uint32_t)std::min<size_t>(ids, total_slots_),
                                   root_slot, ctx_->d_status, ctx_->stream) != cudaSuccess)
            return VV_ERR_CUDA;
        head_ = 0;
        win_len_ = 0;
        rc = next_epoch();
        if (rc) return rc;
    }
    uint32_t u = 0, back = 0;
    const uint32_t* list = nullptr;
    if (classified) {
        // one read-out: counters, candidates and the order's front, enough
        // for every upload a candidate can cause (itself and its parent)
        if (h_cand_cap_ < ids) {
            if (h_cand_) cudaFreeHost(h_cand_);
            h_cand_ = nullptr;
            h_cand_cap_ = std::max(ids + ids / 4, 2 * h_cand_cap_);
            if (cudaHostAlloc((void**)&h_cand_, h_cand_cap_ * 4, cudaHostAllocMapped) != cudaSuccess) {
                h_cand_cap_ = 0;
                return VV_ERR_OOM;
            }
            if (cudaHostGetDevicePointer((void**)&dh_cand_, h_cand_, 0) != cudaSuccess) return VV_ERR_CUDA;
        }
        if (launch_service_readout(order_, dh_small_ + 4, dh_cand_, (uint32_t)h_cand_cap_, dh_win_, ctx_->stream) !=
            cudaSuccess)
            return VV_ERR_CUDA;
        if (cudaStreamSynchronize(ctx_->stream) != cudaSuccess) return VV_ERR_CUDA;
        u = h_small_[4];
        back = h_small_[6];
        const uint32_t m = h_small_[5], untouched = h_small_[7];
        if (m > u || back > u || back > h_cand_cap_ || untouched > total_slots_ ||
            m + (root_slot < total_slots_ ? 1u : 0u) != total_slots_ - untouched)
            return ctx_fail(ctx_, VV_ERR_BOUNDS, "LRU order partition: touched and untouched counts disagree");
        win_start_ = 0;
        win_len_ = (uint32_t)std::min<size_t>(total_slots_, 2 * (size_t)back + 2);
        list = h_cand_;
    } else {
        // every distinct node comes back for the host's visit
        int rc = read_count(order_.counters, u);
        if (rc) return rc;
        back = u;
        if (h_unique_cap_ < back) {
            if (h_unique_) cudaFreeHost(h_unique_);
            h_unique_ = nullptr;
            h_unique_cap_ = std::max((size_t)back, 2 * h_unique_cap_);
            if (cudaMallocHost((void**)&h_unique_, h_unique_cap_ * 4) != cudaSuccess) {
                h_unique_cap_ = 0;
                return VV_ERR_OOM;
            }
        }
        if (back) {
            if (cudaMemcpyAsync(h_unique_, dd_.unique, (size_t)back * 4, cudaMemcpyDeviceToHost, ctx_->stream) !=
                    cudaSuccess ||
                cudaStreamSynchronize(ctx_->stream) != cudaSuccess)
                return VV_ERR_CUDA;
        }
        list = h_unique_;
    }
    const auto tv = std::chrono::steady_clock::now();
    const uint32_t dx = (uint32_t)pd[0], dy = (uint32_t)pd[1];
    for (uint32_t k = 0; k < back; ++k) {
        const uint32_t g = list[k];
        const uint32_t nidx = tree_->index_of(g % dx, (g / dx) % dy, g / (dx * dy));
        if (nidx == kNoParent || tree_->level(nidx) < 0) continue;
        visit(nidx, upload);
    }
    ms_visit_ = std::chrono::duration<float, std::milli>(std::chrono::steady_clock::now() - tv).count();
    unique_ = (int32_t)u;
    root_on_device_ = classified;
    return VV_OK;
}

int GigaVoxelsRenderer::update() {
    if (!d_count) return VV_ERR_STATE;
    int prc = post_draw();  // a frame drawn without compaction is compacted first
    if (prc) return prc;
    uploaded_ = 0;
    uint32_t count = 0;
    int rc = read_count(d_count, count);
    if (rc) return rc;
    const auto t0 = std::chrono::steady_clock::now();  // the draw has finished here
    active_ = count;
    const uint32_t n = std::min<uint32_t>(count, (uint32_t)cap_);
    req_count_ = n;
    std::vector<uint32_t> upload;
    rc = device_paging_ ? update_device(n, upload, d_requests) : update_host(n, upload);
    if (rc) return rc;
    const auto t1 = std::chrono::steady_clock::now();
    ms_readback_ = std::chrono::duration<float, std::milli>(t1 - t0).count();
    rc = apply_policy(upload);
    if (rc) return rc;
    ms_policy_ = std::chrono::duration<float, std::milli>(std::chrono::steady_clock::now() - t1).count();
    rc = deferred_ ? VV_OK : flush_uploads();
    if (rc) return rc;
    return start_readback();  // the service's last read-out is done
}

int GigaVoxelsRenderer::apply_policy(std::vector<uint32_t>& upload) {
    // GigaVoxelsOctTree::update touches the root every frame (:1821-1850);
    // after a device classification that touch is already in the order.
    if (!root_on_device_ && node_slot_[0] >= 0) touch((uint32_t)node_slot_[0]);
    root_on_device_ = false;
    evict_hint_ = 2 * (uint32_t)upload.size() + 1;
    // BrickPool::update (GigaVoxelsBrickPool.cpp:561-682), including the
    // upload of a non-resident non-constant parent (:629-673).  The records
    // of the node kAhead uploads on, and of the parent of the one half as
    // far, are prefetched: the nodes are far apart in the host arrays.
    constexpr size_t kAhead = 16;
    for (size_t i = 0; i < upload.size(); ++i) {
        if (i + kAhead < upload.size()) {
            const uint32_t f = upload[i + kAhead];
            __builtin_prefetch(&node_slot_[f]);
            __builtin_prefetch(&w0_[f]);
            __builtin_prefetch(&w1_[f]);
            __builtin_prefetch(&touched_mark_[f]);
            tree_->prefetch(f);
        }
        if (i + kAhead / 2 < upload.size()) {
            const uint32_t par = tree_->parent(upload[i + kAhead / 2]);
            if (par != kNoParent) {
                __builtin_prefetch(&node_slot_[par]);
                tree_->prefetch(par);
            }
        }
        const uint32_t nidx = upload[i];
        if (node_slot_[nidx] >= 0) continue;
        int rc = upload_nodes(nidx);
        if (rc) return rc;
        const uint32_t par = tree_->parent(nidx);
        if (par != kNoParent && !tree_->is_constant(par) && node_slot_[par] < 0) {
            rc = upload_nodes(par);
            if (rc) return rc;
        }
    }
    evict_hint_ = 0;
    return flush_touches();  // touches that no eviction followed
}

int GigaVoxelsRenderer::service(const uint32_t* requests, const uint32_t* count, int cap) {
    if (!device_paging_) return VV_ERR_STATE;
    if (!requests || !count || cap < 0) return VV_ERR_ARG;
    uploaded_ = 0;
    uint32_t c = 0;
    int rc = read_count(count, c);
    if (rc) return rc;
    const auto t0 = std::chrono::steady_clock::now();
    active_ = c;
    const uint32_t n = std::min<uint32_t>(c, (uint32_t)cap);
    req_count_ = n;
    std::vector<uint32_t> upload;
    rc = update_device(n, upload, requests);
    if (rc) return rc;
    const auto t1 = std::chrono::steady_clock::now();
    ms_readback_ = std::chrono::duration<float, std::milli>(t1 - t0).count();
    rc = apply_policy(upload);
    if (rc) return rc;
    ms_policy_ = std::chrono::duration<float, std::milli>(std::chrono::steady_clock::now() - t1).count();
    rc = deferred_ ? VV_OK : flush_uploads();
    if (rc) return rc;
    return start_readback();  // the service's last read-out is done
}

int GigaVoxelsRenderer::set_deferred(bool on) {
    if (on == deferred_) return VV_OK;
    if (!on) {
        deferred_ = false;
        return flush_uploads();  // whatever was pending goes out now
    }
    if (!device_paging_) return VV_ERR_STATE;
    if (!h_def_jobs_) {
        // a slot holds at most one job per staging (later jobs replace
        // earlier ones); a node is patched at most once
        def_job_cap_ = total_slots_;
        def_patch_cap_ = (uint32_t)std::min<size_t>(w0_.size(), 2 * (size_t)total_slots_ + 4096);
        // patches in whole 16-byte words: the pull reads the last partial one
        const size_t patch_bytes = ((size_t)def_patch_cap_ * sizeof(vv_node_patch) + 15) / 16 * 16;
        if (cudaHostAlloc((void**)&h_def_jobs_, (size_t)def_job_cap_ * sizeof(uint4), cudaHostAllocMapped) !=
                cudaSuccess ||
            cudaHostAlloc((void**)&h_def_patches_, patch_bytes, cudaHostAllocMapped) != cudaSuccess ||
            cudaHostAlloc((void**)const_cast<uint32_t**>(&h_def_counts_), 4 * sizeof(uint32_t), cudaHostAllocMapped) != cudaSuccess ||
            cudaMalloc((void**)&d_def_jobs_, (size_t)def_job_cap_ * sizeof(uint4)) != cudaSuccess ||
            cudaMalloc((void**)&d_def_patches_, patch_bytes) != cudaSuccess ||
            cudaMalloc((void**)&d_def_counts_, 2 * sizeof(uint32_t)) != cudaSuccess)
            return VV_ERR_OOM;
        h_def_counts_[0] = h_def_counts_[1] = h_def_counts_[2] = h_def_counts_[3] = 0;
        slot_job_.assign(total_slots_, -1);
    }
    deferred_ = true;
    return VV_OK;
}

int GigaVoxelsRenderer::stage_uploads() {
    if (!deferred_) return VV_ERR_STATE;
    // the latest job per slot: an earlier job for the same slot belongs to a
    // node that was evicted again before this staging
    std::vector<uint32_t> keep;
    keep.reserve(pending_nodes_.size());
    for (size_t i = pending_nodes_.size(); i-- > 0;) {
        const uint32_t s = pending_slots_[i];
        if (slot_job_[s] >= 0) continue;
        slot_job_[s] = (int32_t)i;
        keep.push_back((uint32_t)i);
    }
    for (uint32_t i : keep) slot_job_[pending_slots_[i]] = -1;
    if (keep.size() > def_job_cap_ || touched_.size() > def_patch_cap_) {
        // does not fit the staging: apply at once on the stream instead
        h_def_counts_[0] = h_def_counts_[1] = 0;
        return flush_uploads();
    }
    uint32_t nj = 0;
    for (size_t k = keep.size(); k-- > 0;) {  // back to first-seen order
        const uint32_t i = keep[k];
        h_def_jobs_[nj++] = production_job(pending_slots_[i], pending_nodes_[i]);
    }
    uint32_t np = 0;
    for (uint32_t t : touched_) {
        vv_node_patch& q = h_def_patches_[np++];
        tree_->grid_of(t, q.x, q.y, q.z);
        q.word0 = w0_[t];
        q.word1 = w1_[t];
        touched_mark_[t] = 0;
    }
    touched_.clear();
    pending_nodes_.clear();
    pending_slots_.clear();
    h_def_counts_[0] = nj;
    h_def_counts_[1] = np;
    if (nj || np) h_def_counts_[2] = ++stage_gen_;  // applied once the enqueued work has run
    return VV_OK;
}

int GigaVoxelsRenderer::enqueue_uploads() {
    if (!deferred_) return VV_ERR_STATE;
    uint4* jobs = nullptr;
    vv_node_patch* patches = nullptr;
    uint32_t* counts = nullptr;
    if (cudaHostGetDevicePointer((void**)&jobs, h_def_jobs_, 0) != cudaSuccess ||
        cudaHostGetDevicePointer((void**)&patches, h_def_patches_, 0) != cudaSuccess ||
        cudaHostGetDevicePointer((void**)&counts, (void*)h_def_counts_, 0) != cudaSuccess)
        return VV_ERR_CUDA;
    void* pool = nullptr;
    size_t pool_bytes = 0;
    vv_brickpool_device_ptr(ctx_, &pool, &pool_bytes);
    // counts, jobs and patches into device memory, then production and
    // patches from there
    if (launch_pull_staged(counts, jobs, def_job_cap_, patches, def_patch_cap_, d_def_counts_, d_def_jobs_,
                           d_def_patches_, ctx_->stream) != cudaSuccess)
        return VV_ERR_CUDA;
    const cudaError_t pe =
        dstore_ ? launch_copy_staged(dstore_->view(), d_def_jobs_, d_def_counts_, def_job_cap_, pool, d_.fmt,
                                     ctx_cell_mask_rw(ctx_), (long long)total_slots_, ctx_->d_status, ctx_->stream)
                : launch_produce_staged(dterrain_->view(), d_def_jobs_, d_def_counts_, def_job_cap_, pool, d_.fmt,
                                        ctx_cell_mask_rw(ctx_), (long long)total_slots_, ctx_->d_status, ctx_->stream);
    if (pe != cudaSuccess) return VV_ERR_CUDA;
    const DeviceTree& t = ctx_->trees[0];
    if (launch_node_patch_staged(d_def_patches_, d_def_counts_ + 1, def_patch_cap_, t.nodes, t.dim, ctx_->d_status,
                                 ctx_->stream) != cudaSuccess)
        return VV_ERR_CUDA;
    // the staging's generation, recorded as applied after its patches
    if (launch_read_word(counts + 2, counts + 3, ctx_->stream) != cudaSuccess) return VV_ERR_CUDA;
    return VV_OK;
}

int GigaVoxelsRenderer::last_requests(std::vector<uint32_t>& out) {
    if (requests_on_host_) {
        out = host_requests_;
        return VV_OK;
    }
    out.resize((size_t)req_count_ * 4);
    if (req_count_) {
        if (cudaMemcpyAsync(out.data(), d_requests, (size_t)req_count_ * 16, cudaMemcpyDeviceToHost, ctx_->stream) !=
            cudaSuccess)
            return VV_ERR_CUDA;
        if (cudaStreamSynchronize(ctx_->stream) != cudaSuccess) return VV_ERR_CUDA;
    }
    return VV_OK;
}

void GigaVoxelsRenderer::stats(vv_renderer_stats& s) const {
    s.frame = frame_;
    s.requests = req_count_;
    s.active_pixels = active_;
    s.bricks_uploaded = uploaded_;
    s.bricks_uploaded_total = uploaded_total_;
    s.resident_bricks = resident_;
    s.evictions_total = evictions_;
    s.pool_slots = (int32_t)total_slots_;
    s.ms_readback = ms_readback_;
    s.ms_policy = ms_policy_;
    s.ms_produce = ms_produce_;
    s.ms_upload = ms_upload_;
    s.ms_visit = ms_visit_;
    s.unique_nodes = unique_;
}

int GigaVoxelsRenderer::lru_order(std::vector<uint32_t>& out) {
    int rc = flush_touches();
    if (rc) return rc;
    const uint32_t n = total_slots_;
    out.resize(n);
    const uint32_t* d = order_.order[order_.cur];
    if (cudaMemcpyAsync(out.data(), d + head_, (size_t)(n - head_) * 4, cudaMemcpyDeviceToHost, ctx_->stream) !=
            cudaSuccess ||
        (head_ && cudaMemcpyAsync(out.data() + (n - head_), d, (size_t)head_ * 4, cudaMemcpyDeviceToHost,
                                  ctx_->stream) != cudaSuccess) ||
        cudaStreamSynchronize(ctx_->stream) != cudaSuccess)
        return VV_ERR_CUDA;
    return VV_OK;
}

void GigaVoxelsRenderer::residency(std::vector<uint32_t>& xyz, std::vector<uint32_t>& slot) const {
    xyz.clear();
    slot.clear();
    for (uint32_t s = 0; s < total_slots_; ++s) {
        if (slot_node_[s] < 0) continue;
        uint32_t x, y, z;
        tree_->grid_of((uint32_t)slot_node_[s], x, y, z);
        xyz.push_back(x);
        xyz.push_back(y);
        xyz.push_back(z);
        slot.push_back(s);
    }
}

}  // namespace vv
