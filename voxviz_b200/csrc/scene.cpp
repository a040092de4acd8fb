// scene.cpp - paged scenes of .gvx tiles (see scene.h).
#include "scene.h"

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <exception>
#include <new>

#include "kernels.cuh"

namespace vv {

namespace {

void normalize(double v[3]) {
    const double l = std::sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
    if (l > 0.0)
        for (int a = 0; a < 3; ++a) v[a] /= l;
}

void cross(const double a[3], const double b[3], double out[3]) {
    out[0] = a[1] * b[2] - a[2] * b[1];
    out[1] = a[2] * b[0] - a[0] * b[2];
    out[2] = a[0] * b[1] - a[1] * b[0];
}

}  // namespace

void Frustum::set(const vv_camera& cam, double far_dist) {
    double look[3] = {cam.look[0], cam.look[1], cam.look[2]};
    double up[3] = {cam.up[0], cam.up[1], cam.up[2]};
    normalize(look);
    normalize(up);
    double left[3];
    cross(up, look, left);
    normalize(left);
    const double e[3] = {cam.position[0], cam.position[1], cam.position[2]};
    const double u[3] = {-left[0], -left[1], -left[2]}, *v = up, n[3] = {-look[0], -look[1], -look[2]};
    auto dot = [](const double* a, const double* b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; };
    // FlyCamera::computeViewMatrix, column-major
    const double modl[16] = {u[0], v[0], n[0], 0.0, u[1], v[1], n[1], 0.0,
                             u[2], v[2], n[2], 0.0, -dot(e, u), -dot(e, v), -dot(e, n), 1.0};
    // ComputePerspective / ComputeFrustum (symmetric frustum)
    const double znear = cam.near_dist, zfar = far_dist;
    const float aspect = (float)cam.width / (float)cam.height;
    const double ymax = znear * (double)tanf((float)(cam.fov_y_deg * 3.14159265358979323846 / 360.0));
    const double xmax = ymax * aspect;
    double proj[16] = {0.0};
    proj[0] = 2.0 * znear / (2.0 * xmax);
    proj[5] = 2.0 * znear / (2.0 * ymax);
    proj[10] = (-zfar - znear) / (zfar - znear);
    proj[11] = -1.0;
    proj[14] = (-2.0 * znear * zfar) / (zfar - znear);
    double clip[16];
    for (int i = 0; i < 4; ++i)
        for (int j = 0; j < 4; ++j)
            clip[4 * i + j] = modl[4 * i] * proj[j] + modl[4 * i + 1] * proj[4 + j] + modl[4 * i + 2] * proj[8 + j] +
                              modl[4 * i + 3] * proj[12 + j];
    // right, left, bottom, top, far, near (Frustum.cpp:47-118)
    const int col[6] = {0, 0, 1, 1, 2, 2};
    const double sgn[6] = {-1.0, 1.0, 1.0, -1.0, -1.0, 1.0};
    for (int p = 0; p < 6; ++p) {
        for (int k = 0; k < 4; ++k) plane[p][k] = clip[4 * k + 3] + sgn[p] * clip[4 * k + col[p]];
        const double t = std::sqrt(plane[p][0] * plane[p][0] + plane[p][1] * plane[p][1] + plane[p][2] * plane[p][2]);
        for (int k = 0; k < 4; ++k) plane[p][k] /= t;
    }
}

bool Frustum::sphere(const float c[3], float radius, float& distance) const {
    double d = 0.0;
    for (int p = 0; p < 6; ++p) {
        d = plane[p][0] * c[0] + plane[p][1] * c[1] + plane[p][2] * c[2] + plane[p][3];
        if (d <= -(double)radius) return false;
    }
    distance = (float)d;  // the near plane's
    return true;
}

PagedScene::PagedScene(vv_ctx* ctx, GvpFile&& gvp, const vv_scene_desc& d) : ctx_(ctx), d_(d), gvp_(std::move(gvp)) {
    if (d_.stale_frames <= 0) d_.stale_frames = 100;
    if (!(d_.far_dist > 0.0f)) d_.far_dist = 10000.0f;
    host_only_ = (d_.flags & VV_SCENE_HOST_ONLY) != 0;
    tiles_.reserve(gvp_.tiles.size());
    for (const GvpTile& g : gvp_.tiles) {
        tiles_.push_back(std::make_unique<SceneTile>());
        tiles_.back()->info = g;
    }
}

PagedScene::~PagedScene() {
    {
        std::lock_guard<std::mutex> lock(mu_);
        done_ = true;
    }
    cv_.notify_all();
    if (thread_.joinable()) thread_.join();
    for (auto& t : tiles_) release_tile(*t);
    if (d_color_) cudaFree(d_color_);
    if (ev_blended_) cudaEventDestroy(ev_blended_);
    if (ev_cast_) cudaEventDestroy(ev_cast_);
}

int PagedScene::init() {
    if (!host_only_) {
        if (!ctx_) return VV_ERR_ARG;
        if (cudaEventCreateWithFlags(&ev_blended_, cudaEventDisableTiming) != cudaSuccess ||
            cudaEventCreateWithFlags(&ev_cast_, cudaEventDisableTiming) != cudaSuccess)
            return VV_ERR_CUDA;
    }
    if (!(d_.flags & VV_SCENE_SYNCHRONOUS)) thread_ = std::thread([this] { loader_main(); });
    return VV_OK;
}

// requestLoadOctTree (GigaVoxelsDatabasePager.cpp:340-372): once per tile
// until it is merged.
void PagedScene::request_load(size_t t, float dist) {
    std::lock_guard<std::mutex> lock(mu_);
    SceneTile& s = *tiles_[t];
    if (s.on_request_list) return;
    s.on_request_list = true;
    requests_.push_back(Request{t, dist});
    cv_.notify_all();
}

// DatabasePagerThread::run's body (:238-331): the requests sorted by last
// access (latest first) then distance to the near plane (nearest first),
// each tree read and handed over for merging.
void PagedScene::load_requests(std::vector<Request>& reqs) {
    std::stable_sort(reqs.begin(), reqs.end(), [this](const Request& a, const Request& b) {
        const uint64_t la = tiles_[a.tile]->last_access.load(), lb = tiles_[b.tile]->last_access.load();
        if (la != lb) return la > lb;
        return a.dist < b.dist;
    });
    for (const Request& r : reqs) {
        SceneTile& s = *tiles_[r.tile];
        {
            std::lock_guard<std::mutex> lock(mu_);
            if (done_) break;          // the scene is being destroyed
            if (s.tree || s.loaded) {  // loaded already
                s.on_request_list = false;
                continue;
            }
        }
        const auto t0 = std::chrono::steady_clock::now();
        std::unique_ptr<vv_octree> o;
        std::string err;
        try {
            GvxFile f;
            if (read_gvx(s.info.tree_file, (d_.load_flags & VV_GVX_SKIP_GRADIENTS) == 0, f, err) == VV_OK) {
                o = std::make_unique<vv_octree>();
                o->tree = GigaVoxelsOctTree::from_gvx(std::move(f), (d_.load_flags & VV_GVX_CONSTANT_COLORS) != 0);
            }
        } catch (const std::exception& e) {
            err = e.what();
            o.reset();
        }
        const double ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
        std::lock_guard<std::mutex> lock(mu_);
        load_ms_total_ += ms;
        load_ms_max_ = std::max(load_ms_max_, ms);
        if (!o) {
            // the reference prints the failure and leaves the tile on its
            // request list: it is not tried again
            s.load_failed = true;
            s.error = err;
            ++load_failures_;
            continue;
        }
        s.loaded = std::move(o);
        handled_.push_back(r.tile);
    }
    reqs.clear();
}

void PagedScene::loader_main() {
    std::vector<Request> reqs;
    for (;;) {
        {
            std::unique_lock<std::mutex> lock(mu_);
            busy_ = false;
            idle_cv_.notify_all();
            cv_.wait(lock, [this] { return done_ || !requests_.empty(); });
            if (done_) return;
            reqs.swap(requests_);
            busy_ = true;
        }
        load_requests(reqs);
    }
}

int PagedScene::wait_loads() {
    if (d_.flags & VV_SCENE_SYNCHRONOUS) {
        std::vector<Request> reqs;
        {
            std::lock_guard<std::mutex> lock(mu_);
            reqs.swap(requests_);
        }
        load_requests(reqs);
        return VV_OK;
    }
    std::unique_lock<std::mutex> lock(mu_);
    idle_cv_.wait(lock, [this] { return requests_.empty() && !busy_; });
    return VV_OK;
}

// mergeHandledRequests (:378-415): a loaded tree becomes the tile's
// drawable tree with its device resources.
int PagedScene::merge_handled() {
    std::vector<size_t> h;
    {
        std::lock_guard<std::mutex> lock(mu_);
        h.swap(handled_);
    }
    int rc = VV_OK;
    for (size_t t : h) {
        SceneTile& s = *tiles_[t];
        {
            std::lock_guard<std::mutex> lock(mu_);
            s.tree = std::move(s.loaded);
            s.on_request_list = false;
        }
        const int r = attach_tile(s);
        if (r) {
            s.load_failed = true;
            {
                std::lock_guard<std::mutex> lock(mu_);
                if (s.error.empty()) s.error = "could not create the tile's renderer";
            }
            release_tile(s);
            if (!rc) rc = r;
            continue;
        }
        ++loads_;
    }
    return rc;
}

// unloadStalePagedOctTreeNodes (:425-453): a tile unseen for more than
// stale_frames frames is released (unsigned frame difference, as there).
int PagedScene::unload_stale(uint64_t frame) {
    for (auto& tp : tiles_) {
        SceneTile& s = *tp;
        if (!s.tree) continue;
        const uint64_t stale = frame - s.last_access.load();
        if (stale > (uint64_t)d_.stale_frames) {
            release_tile(s);
            ++unloads_;
        }
    }
    return VV_OK;
}

int PagedScene::attach_tile(SceneTile& s) {
    const GvxHeader* h = s.tree->tree->file_header();
    for (int a = 0; a < 3; ++a) {
        s.box_min[a] = h ? h->origin[a] : 0.0f;
        s.box_max[a] = h ? h->origin[a] + h->delta[a] * (float)h->volume_size[a] : 1.0f;
    }
    if (host_only_) return VV_OK;
    const float sx = s.box_max[0] - s.box_min[0], sy = s.box_max[1] - s.box_min[1], sz = s.box_max[2] - s.box_min[2];
    if (!(sx > 0.0f) || std::fabs(sy - sx) > 1e-5f * sx || std::fabs(sz - sx) > 1e-5f * sx) {
        std::lock_guard<std::mutex> lock(mu_);
        s.error = "the tile's box is not a cube";
        return VV_ERR_ARG;
    }
    vv_params p{};
    p.device = ctx_->device;
    int rc = vv_ctx_create(&p, &s.ctx);
    if (rc) return rc;
    vv_renderer_desc rd{};
    rd.fmt = d_.fmt;
    rd.pool_bytes = d_.pool_bytes_per_tile;
    rd.request_cap = d_.request_cap;
    rd.lod_scalar = d_.lod_scalar > 0.0f ? d_.lod_scalar : 1.0f;
    rd.alpha_stop = d_.alpha_stop > 0.0f ? d_.alpha_stop : 0.99f;
    rd.jitter_seed = d_.jitter_seed;
    rd.device_paging = d_.device_paging;
    try {
        auto r = std::make_unique<vv_renderer>();
        r->ctx = s.ctx;
        r->impl = std::make_unique<GigaVoxelsRenderer>(s.ctx, s.tree.get(), s.tree->tree.get(), rd);
        rc = r->impl->init();
        if (rc) return rc;
        s.renderer = std::move(r);
    } catch (const std::bad_alloc&) {
        return VV_ERR_OOM;
    }
    if (cudaEventCreateWithFlags(&s.drawn, cudaEventDisableTiming) != cudaSuccess) return VV_ERR_CUDA;
    return VV_OK;
}

void PagedScene::release_tile(SceneTile& s) {
    if (s.ctx) vv_ctx_synchronize(s.ctx);
    s.renderer.reset();
    if (s.drawn) cudaEventDestroy(s.drawn);
    s.drawn = nullptr;
    if (s.ctx) vv_ctx_destroy(s.ctx);
    s.ctx = nullptr;
    std::unique_ptr<vv_octree> gone;
    {
        std::lock_guard<std::mutex> lock(mu_);
        gone = std::move(s.tree);
    }
}

// drawVolume's volume transform (GigaVoxelsRenderer.cpp:1655-1690): the
// camera in the tile's unit box, (p - centre) / scale + 0.5; directions keep
// their values and distances scale with the (cubic) box.
int PagedScene::tile_camera(const SceneTile& s, const vv_camera& w, vv_camera& out) const {
    out = w;
    for (int a = 0; a < 3; ++a) {
        const float centre = (s.box_min[a] + s.box_max[a]) * 0.5f;
        const float scale = s.box_max[a] - s.box_min[a];
        out.position[a] = ((w.position[a] - centre) / scale) + 0.5f;
    }
    out.near_dist = w.near_dist / (s.box_max[0] - s.box_min[0]);
    return VV_OK;
}

int PagedScene::draw(const vv_camera& cam) {
    if (cam.width <= 0 || cam.height <= 0) return VV_ERR_ARG;
    frame_ = (uint64_t)(int64_t)cam.frame;
    Frustum fr;
    fr.set(cam, d_.far_dist);
    render_list_.clear();
    // the cull visitor (GigaVoxelsRenderer.cpp:785-798): visible tiles are
    // stamped; loaded ones go into the render list, farthest first (equal
    // distances keep the tile order), the others are requested
    for (size_t t = 0; t < tiles_.size(); ++t) {
        SceneTile& s = *tiles_[t];
        s.visible = false;
        s.drawn_order = -1;
        float dist;
        if (!fr.sphere(s.info.center, s.info.radius, dist)) continue;
        s.visible = true;
        s.last_access.store(frame_);
        if (!s.tree) {
            s.dist = dist;
            if (!s.load_failed) request_load(t, dist);
            continue;
        }
        s.dist = dist - s.info.radius;
        size_t k = 0;
        while (k < render_list_.size() && !(tiles_[render_list_[k]]->dist < s.dist)) ++k;
        render_list_.insert(render_list_.begin() + (long)k, t);
    }
    for (size_t k = 0; k < render_list_.size(); ++k) tiles_[render_list_[k]]->drawn_order = (int)k;
    update_list_ = render_list_;
    if (host_only_) return VV_OK;
    // the scene colour: cleared, then each tile blended over it
    if (cam.width != width_ || cam.height != height_ || !d_color_) {
        vv_ctx_synchronize(ctx_);
        if (d_color_) cudaFree(d_color_);
        d_color_ = nullptr;
        if (cudaMalloc((void**)&d_color_, (size_t)cam.width * cam.height * 16) != cudaSuccess) return VV_ERR_OOM;
        width_ = cam.width;
        height_ = cam.height;
    }
    const size_t np = (size_t)width_ * height_;
    if (cudaMemsetAsync(d_color_, 0, np * 16, ctx_->stream) != cudaSuccess) return VV_ERR_CUDA;
    if ((d_.flags & VV_SCENE_BATCHED) && !render_list_.empty()) return draw_batched(cam);
    for (size_t t : render_list_) {
        SceneTile& s = *tiles_[t];
        vv_camera tc;
        tile_camera(s, cam, tc);
        // the tile's colour buffers are reused every other frame: the last
        // blend that read them must be done
        if (blended_once_ && cudaStreamWaitEvent(s.ctx->stream, ev_blended_, 0) != cudaSuccess) return VV_ERR_CUDA;
        int rc = s.renderer->impl->draw(tc);
        if (rc) return rc;
        if (cudaEventRecord(s.drawn, s.ctx->stream) != cudaSuccess ||
            cudaStreamWaitEvent(ctx_->stream, s.drawn, 0) != cudaSuccess)
            return VV_ERR_CUDA;
        if (launch_blend_over((float4*)d_color_, (const float4*)s.renderer->impl->d_color, np, ctx_->stream) !=
            cudaSuccess)
            return VV_ERR_CUDA;
    }
    if (cudaEventRecord(ev_blended_, ctx_->stream) != cudaSuccess) return VV_ERR_CUDA;
    blended_once_ = true;
    return VV_OK;
}

// The drawn tiles' ray casts as one persistent launch on the scene's stream
// (the batched kernel: one queue of pixel tiles over all views), then each
// tile's selection and compaction on its own stream, and the blends.
int PagedScene::draw_batched(const vv_camera& cam) {
    const size_t np = (size_t)width_ * height_;
    views_.resize(render_list_.size());
    for (size_t k = 0; k < render_list_.size(); ++k) {
        SceneTile& s = *tiles_[render_list_[k]];
        vv_camera tc;
        tile_camera(s, cam, tc);
        if (blended_once_ && cudaStreamWaitEvent(s.ctx->stream, ev_blended_, 0) != cudaSuccess) return VV_ERR_CUDA;
        GigaVoxelsRenderer& r = *s.renderer->impl;
        int rc = r.prepare_draw(tc);
        if (rc) return rc;
        // the tile's pools and node words as its stream left them
        if (cudaEventRecord(s.drawn, s.ctx->stream) != cudaSuccess ||
            cudaStreamWaitEvent(ctx_->stream, s.drawn, 0) != cudaSuccess)
            return VV_ERR_CUDA;
        vv_batch_view& v = views_[k];
        std::memset(&v, 0, sizeof(v));
        v.ctx = s.ctx;
        v.tree = 0;
        v.u = r.last_uniforms();
        v.color = r.d_color;
        v.usage = r.d_usage;
    }
    const vv_batch_config cfg{8, 8, 1, 0};
    int rc = vv_render_batch(ctx_, views_.data(), (int32_t)views_.size(), &cfg);
    if (rc) return rc;
    if (cudaEventRecord(ev_cast_, ctx_->stream) != cudaSuccess) return VV_ERR_CUDA;
    for (size_t t : render_list_) {
        SceneTile& s = *tiles_[t];
        if (cudaStreamWaitEvent(s.ctx->stream, ev_cast_, 0) != cudaSuccess) return VV_ERR_CUDA;
        rc = s.renderer->impl->finish_draw(VV_PASS_SELECT | VV_PASS_COMPACT);
        if (rc) return rc;
        if (launch_blend_over((float4*)d_color_, (const float4*)s.renderer->impl->d_color, np, ctx_->stream) !=
            cudaSuccess)
            return VV_ERR_CUDA;
    }
    if (cudaEventRecord(ev_blended_, ctx_->stream) != cudaSuccess) return VV_ERR_CUDA;
    blended_once_ = true;
    return VV_OK;
}

int PagedScene::update() {
    int rc = VV_OK;
    if (d_.flags & VV_SCENE_SYNCHRONOUS) {
        std::vector<Request> reqs;
        {
            std::lock_guard<std::mutex> lock(mu_);
            reqs.swap(requests_);
        }
        load_requests(reqs);
    }
    // GigaVoxelsRenderer::update (:1520-1570): merge, unload, then the
    // drawn trees' page-request services
    rc = merge_handled();
    unload_stale(frame_);
    if (!host_only_)
        for (size_t t : update_list_) {
            SceneTile& s = *tiles_[t];
            if (!s.renderer) continue;
            const int r = s.renderer->impl->update();
            if (r && !rc) rc = r;
        }
    return rc;
}

int PagedScene::read_color(float* host) {
    if (host_only_ || !d_color_) return VV_ERR_STATE;
    if (cudaMemcpyAsync(host, d_color_, (size_t)width_ * height_ * 16, cudaMemcpyDeviceToHost, ctx_->stream) !=
            cudaSuccess ||
        cudaStreamSynchronize(ctx_->stream) != cudaSuccess)
        return VV_ERR_CUDA;
    return VV_OK;
}

vv_renderer* PagedScene::tile_renderer(int t) {
    if (t < 0 || (size_t)t >= tiles_.size()) return nullptr;
    return tiles_[(size_t)t]->renderer.get();
}

void PagedScene::tile_states(vv_scene_tile_state* out, int cap) const {
    std::lock_guard<std::mutex> lock(mu_);
    for (int i = 0; i < cap && (size_t)i < tiles_.size(); ++i) {
        const SceneTile& s = *tiles_[(size_t)i];
        vv_scene_tile_state& o = out[i];
        std::memset(&o, 0, sizeof(o));
        o.loaded = s.tree ? 1 : 0;
        o.pending = (s.on_request_list || s.loaded) ? 1 : 0;
        o.visible = s.visible ? 1 : 0;
        o.drawn_order = s.drawn_order;
        o.failed = s.load_failed ? 1 : 0;
        o.dist_to_near_plane = s.dist;
        o.last_access = (int64_t)s.last_access.load();
    }
}

void PagedScene::stats(vv_scene_stats& st) const {
    std::lock_guard<std::mutex> lock(mu_);
    std::memset(&st, 0, sizeof(st));
    st.tiles = (int32_t)tiles_.size();
    for (const auto& t : tiles_) {
        if (t->tree) ++st.loaded;
        if (t->on_request_list || t->loaded) ++st.pending;
    }
    st.drawn = (int32_t)render_list_.size();
    st.loads = loads_;
    st.unloads = unloads_;
    st.load_failures = load_failures_;
    const int64_t attempts = loads_ + load_failures_ + (int64_t)handled_.size();
    st.load_ms_avg = attempts > 0 ? (float)(load_ms_total_ / (double)attempts) : 0.0f;
    st.load_ms_max = (float)load_ms_max_;
}

std::string PagedScene::tile_error(int t) const {
    if (t < 0 || (size_t)t >= tiles_.size()) return std::string();
    std::lock_guard<std::mutex> lock(mu_);
    return tiles_[(size_t)t]->error;
}

}  // namespace vv
