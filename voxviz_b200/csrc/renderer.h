// renderer.h - host side of the "gv" renderer plugin: uniform derivation,
// frame protocol and the page-request service with a deterministic LRU.
#pragma once

#include <cstdint>
#include <memory>
#include <vector>

#include "../../include/voxviz_b200.h"
#include "octree.h"
#include "production.h"

namespace vv {

// GigaVoxelsRenderer::drawVolume uniform derivation
// (GigaVoxelsRenderer.cpp:1630-1816) for a volume box [0,1]^3.
void compute_uniforms(int depth, bool root_is_constant, const vv_camera& cam, const int slots[3],
                      float lod_scalar, float alpha_stop, vv_uniforms& u);
// Camera::getPixelSize (Camera.cpp:128-196) restated without GLU.
float camera_pixel_size(const vv_camera& cam);
// GLUtils::Create2DJitterTexture (GLUtils.cpp:455-497) with a seeded hash
// instead of srand(time): values in [1,255].
void make_jitter(uint32_t seed, int size, uint8_t* out);

// The brick pool's slot bookkeeping: an LRU list over slot ids
// (BrickPool::m_loadedBricks, GigaVoxelsBrickPool.cpp:330-424) made
// deterministic: touching a slot moves it to the back, eviction takes the
// front, and initially the empty slots lead in slot-id order.
class SlotLRU {
public:
    void init(uint32_t slots);
    uint32_t front() const { return head_; }
    void touch(uint32_t s);  // move to back
    uint32_t size() const { return n_; }

private:
    std::vector<uint32_t> prev_, next_;
    uint32_t head_ = 0, tail_ = 0, n_ = 0;
};

class GigaVoxelsRenderer {
public:
    GigaVoxelsRenderer(vv_ctx* ctx, vv_octree* tree_handle, const GigaVoxelsOctTree* tree,
                       const vv_renderer_desc& d);
    ~GigaVoxelsRenderer();
    int init();                          // Renderer::init
    int draw(const vv_camera& cam);      // Renderer::draw
    int update();                        // Renderer::postDraw + Renderer::update
    // The page-request service for a compacted list drawn elsewhere (device
    // pointers); uploads are applied at once, or staged when deferred.
    int service(const uint32_t* requests, const uint32_t* count, int cap);
    // Deferred uploads: service() only stages; stage_uploads() writes this
    // frame's jobs and node patches to pinned mapped memory and
    // enqueue_uploads() launches the count-independent device side.
    int set_deferred(bool on);
    int stage_uploads();
    int enqueue_uploads();
    void stats(vv_renderer_stats& s) const;

    vv_ctx* ctx() { return ctx_; }
    const vv_uniforms& last_uniforms() const { return last_u_; }
    int slots(int a) const { return slots_[a]; }
    // The last compacted request list (host copy; read back from the device
    // when the device-side service did not need it on the host).
    int last_requests(std::vector<uint32_t>& out);
    void residency(std::vector<uint32_t>& xyz, std::vector<uint32_t>& slot) const;

    float* d_color = nullptr;
    uint32_t* d_usage = nullptr;
    uint32_t* d_mask = nullptr;
    uint32_t* d_requests = nullptr;
    uint32_t* d_count = nullptr;
    int width = 0, height = 0;

private:
    int alloc_frame(int w, int h);
    int upload_nodes(uint32_t node);     // upload the brick of node, evicting the LRU slot
    int flush_uploads();
    int update_host(uint32_t n, std::vector<uint32_t>& upload);
    int update_device(uint32_t n, std::vector<uint32_t>& upload, const uint32_t* requests);
    int apply_policy(std::vector<uint32_t>& upload);
    void visit(uint32_t nidx, std::vector<uint32_t>& upload);

    vv_ctx* ctx_;
    const GigaVoxelsOctTree* tree_;
    vv_renderer_desc d_;
    int slots_[3] = {0, 0, 0};
    uint32_t total_slots_ = 0;
    size_t texel_bytes_ = 4;
    SlotLRU lru_;
    std::vector<int32_t> slot_node_;     // node index held by slot, -1 empty
    std::vector<int32_t> node_slot_;     // slot of node index, -1 not resident
    std::vector<uint32_t> w0_, w1_;      // current node words
    std::vector<uint32_t> pending_nodes_, pending_slots_;
    std::vector<uint32_t> touched_;      // node indices whose words changed
    std::vector<uint8_t> touched_mark_;
    std::vector<uint32_t> host_requests_;
    std::vector<uint32_t> seen_mark_;
    uint32_t seen_epoch_ = 0;
    vv_uniforms last_u_{};
    int cap_ = 0;
    int64_t frame_ = -1;
    int32_t frame_for_compress_ = 0;
    int64_t req_count_ = 0, active_ = 0, uploaded_ = 0, uploaded_total_ = 0, evictions_ = 0, resident_ = 0;
    float ms_readback_ = 0.f, ms_policy_ = 0.f, ms_produce_ = 0.f, ms_upload_ = 0.f, ms_visit_ = 0.f;
    int32_t unique_ = 0;
    // device-side service
    bool device_paging_ = false;
    std::unique_ptr<DeviceTerrain> dterrain_;
    DedupeBuffers dd_;
    uint32_t* h_small_ = nullptr;   // pinned: request count, distinct count
    uint32_t* h_unique_ = nullptr;  // pinned: distinct node cells of the last frame
    size_t h_unique_cap_ = 0;
    std::vector<uint4> jobs_;
    uint4* d_jobs_ = nullptr;
    size_t jobs_cap_ = 0;
    bool requests_on_host_ = false;
    void* h_stage_ = nullptr;            // pinned brick staging
    size_t h_stage_cap_ = 0;
    // deferred uploads (pinned, mapped): jobs, node patches, their counts
    bool deferred_ = false;
    uint4* h_def_jobs_ = nullptr;
    vv_node_patch* h_def_patches_ = nullptr;
    uint32_t* h_def_counts_ = nullptr;   // [0] jobs, [1] patches
    uint32_t def_job_cap_ = 0, def_patch_cap_ = 0;
    std::vector<int32_t> slot_job_;      // staging: latest job index per slot
};

}  // namespace vv
