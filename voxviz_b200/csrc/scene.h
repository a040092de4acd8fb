// scene.h - paged scenes: tiles of .gvx trees listed by a .gvp, culled
// against the camera frustum, loaded and unloaded by a pager, drawn back to
// front and blended.
//
// Mirrors the reference's paged-scene path: the cull visitor of
// GigaVoxelsRenderer (GigaVoxels/GigaVoxelsRenderer.cpp:667-798) with
// vox::Frustum (VoxVizCore/Frustum.cpp), the render-list draw with
// GL_SRC_ALPHA / GL_ONE_MINUS_SRC_ALPHA blending (:997-1090), and
// gv::DatabasePager (GigaVoxels/GigaVoxelsDatabasePager.cpp: request list
// sorted by last access then distance :226-236, load thread :238-331,
// mergeHandledRequests :378-415, unloadStalePagedOctTreeNodes :425-453).
#pragma once

#include <cuda_runtime.h>

#include <atomic>
#include <condition_variable>
#include <cstdint>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "../../include/voxviz_b200.h"
#include "gvfile.h"
#include "handles.h"

namespace vv {


// vox::Frustum::setFromCamera (Frustum.cpp:13-120) for a vox::Camera whose
// projection is ComputePerspective (Camera.cpp:44-89: fov_y, aspect
// width/height, near, far) and whose view matrix is FlyCamera's
// (Camera.cpp:365-395: u = -left, v = up, n = -look, eye = position), in
// double arithmetic.  The camera's left is up x look.
struct Frustum {
    double plane[6][4];  // right, left, bottom, top, far, near; unit normals
    void set(const vv_camera& cam, double far_dist);
    // sphereInFrustum (Frustum.cpp:122-135): false when the sphere is
    // outside a plane; distance = the centre's signed distance to the near
    // plane.
    bool sphere(const float c[3], float radius, float& distance) const;
};

struct SceneTile {
    GvpTile info;
    std::atomic<uint64_t> last_access{0};   // PagedOctTreeNode::m_lastAccessFrameIndex
    // guarded by the scene's mutex (the pager thread reads or writes them)
    bool on_request_list = false;
    std::atomic<bool> load_failed{false};
    std::string error;
    std::unique_ptr<vv_octree> tree;        // merged (drawable) tree; set and reset under the mutex
    std::unique_ptr<vv_octree> loaded;      // loaded by the pager, not merged yet
    vv_ctx* ctx = nullptr;                  // the tile's device context and renderer
    std::unique_ptr<vv_renderer> renderer;
    cudaEvent_t drawn = nullptr;            // the tile's colour of this frame is complete
    float box_min[3] = {0, 0, 0}, box_max[3] = {0, 0, 0};
    // this frame
    bool visible = false;
    int drawn_order = -1;
    float dist = 0.0f;
};

class PagedScene {
public:
    PagedScene(vv_ctx* ctx, GvpFile&& gvp, const vv_scene_desc& d);
    ~PagedScene();
    int init();
    int draw(const vv_camera& world_cam);  // cull, request loads, draw and blend
    int update();                          // merge loads, unload stale, tile services
    int wait_loads();                      // until the pager has no request left
    int read_color(float* host);
    void tile_states(vv_scene_tile_state* out, int cap) const;
    void stats(vv_scene_stats& s) const;
    size_t tile_count() const { return tiles_.size(); }
    vv_renderer* tile_renderer(int tile);
    std::string tile_error(int tile) const;

private:
    struct Request {
        size_t tile;
        float dist;
    };
    void request_load(size_t t, float dist);
    void load_requests(std::vector<Request>& reqs);  // sort and load (the pager thread's body)
    void loader_main();
    int merge_handled();
    int unload_stale(uint64_t frame);
    int attach_tile(SceneTile& t);
    void release_tile(SceneTile& t);
    int tile_camera(const SceneTile& t, const vv_camera& world, vv_camera& out) const;

    vv_ctx* ctx_;
    vv_scene_desc d_;
    GvpFile gvp_;
    std::vector<std::unique_ptr<SceneTile>> tiles_;
    std::vector<size_t> render_list_;   // this frame, first drawn first (farthest)
    std::vector<size_t> update_list_;   // the render list of the last draw
    uint64_t frame_ = 0;
    int width_ = 0, height_ = 0;
    float* d_color_ = nullptr;
    cudaEvent_t ev_blended_ = nullptr;  // the last frame's blends are done
    cudaEvent_t ev_cast_ = nullptr;     // the batched ray cast is done
    std::vector<vv_batch_view> views_;
    int draw_batched(const vv_camera& cam);
    bool blended_once_ = false;
    bool host_only_ = false;
    // pager
    mutable std::mutex mu_;
    std::condition_variable cv_, idle_cv_;
    std::vector<Request> requests_;
    std::vector<size_t> handled_;
    bool done_ = false, busy_ = false;
    std::thread thread_;
    int64_t loads_ = 0, unloads_ = 0, load_failures_ = 0;
    double load_ms_total_ = 0.0, load_ms_max_ = 0.0;
};

}  // namespace vv
