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
// (GigaVoxelsRenderer.cpp:1630-1816) for a volume box [0,1]^3; leaf_dim is
// the voxel count per axis the ray step is one voxel of (8 << depth when 0).
void compute_uniforms(int depth, int leaf_dim, bool root_is_constant, const vv_camera& cam, const int slots[3],
                      float lod_scalar, float alpha_stop, vv_uniforms& u);
// Camera::getPixelSize (Camera.cpp:128-196) restated without GLU.
float camera_pixel_size(const vv_camera& cam);
// GLUtils::Create2DJitterTexture (GLUtils.cpp:455-497) with a seeded hash
// instead of srand(time): values in [1,255].
void make_jitter(uint32_t seed, int size, uint8_t* out);

class GigaVoxelsRenderer {
public:
    GigaVoxelsRenderer(vv_ctx* ctx, vv_octree* tree_handle, const GigaVoxelsOctTree* tree,
                       const vv_renderer_desc& d);
    ~GigaVoxelsRenderer();
    int init();                          // Renderer::init
    int draw(const vv_camera& cam);      // Renderer::draw
    // Renderer::draw with the chosen passes of vv_render; a frame drawn
    // without VV_PASS_COMPACT is compacted by post_draw (Renderer::postDraw:
    // compressNodeUsageList) or, at the latest, by update.
    int draw_passes(const vv_camera& cam, int passes);
    int post_draw();
    // draw() in two halves, for a ray cast made elsewhere (a batched launch
    // over several renderers): prepare_draw sets up the frame buffers and
    // uniforms, finish_draw runs the given passes of vv_render on them.
    int prepare_draw(const vv_camera& cam);
    int finish_draw(int passes);
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
    // Read-back of the last frame's colour on a copy stream, started once
    // the page-request service is done (overlapping the next draw);
    // wait_readback completes it.
    int read_color_async(void* host);
    int wait_readback();
    void stats(vv_renderer_stats& s) const;
    size_t color_bytes() const { return d_.color_rgba8 ? 4 : 16; }  // per pixel

    vv_ctx* ctx() { return ctx_; }
    const vv_uniforms& last_uniforms() const { return last_u_; }
    int slots(int a) const { return slots_[a]; }
    // The last compacted request list (host copy; read back from the device
    // when the device-side service did not need it on the host).
    int last_requests(std::vector<uint32_t>& out);
    void residency(std::vector<uint32_t>& xyz, std::vector<uint32_t>& slot) const;
    // The brick pool's slots, least recently used first (pending host
    // touches applied first).
    int lru_order(std::vector<uint32_t>& out);

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
    // The brick pool's LRU order (BrickPool::m_loadedBricks,
    // GigaVoxelsBrickPool.cpp:330-424, made deterministic: touching a slot
    // moves it to the back, eviction takes the front, initially the empty
    // slots lead in slot-id order) lives on the device; touches made on the
    // host wait in pending_touch_ until the next partition.
    void touch(uint32_t s) { pending_touch_.push_back(s); }
    int flush_touches();
    int evict_front(uint32_t& s);      // the LRU slot, moved to the back
    int fetch_order(uint32_t want);    // order entries from head_ into h_win_
    int next_epoch();

    vv_ctx* ctx_;
    const GigaVoxelsOctTree* tree_;
    vv_renderer_desc d_;
    int slots_[3] = {0, 0, 0};
    uint32_t total_slots_ = 0;
    size_t brick_bytes_ = 4000;          // one stored brick in the pool's format
    SlotOrderBuffers order_;
    uint32_t head_ = 0;                  // position of the LRU front in order_.order[order_.cur]
    uint32_t epoch_ = 1;                 // mark of the next partition's touches
    uint32_t* h_win_ = nullptr;          // pinned: order entries from win_start_ on (circular)
    uint32_t win_start_ = 0, win_len_ = 0;
    uint32_t evict_hint_ = 0;            // evictions still expected in this service
    bool root_on_device_ = false;        // this service's root touch is in the device partition
    std::vector<uint32_t> pending_touch_;
    std::vector<uint32_t> touch_seen_;   // per slot: stamp of its last de-duplication
    uint32_t touch_stamp_ = 0;
    uint32_t* h_seq_ = nullptr;          // pinned: de-duplicated pending touches
    cudaEvent_t ev_seq_ = nullptr;       // the last copy out of h_seq_ has been read
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
    bool compact_pending_ = false;       // drawn without the compaction pass
    int64_t frame_ = -1;
    int32_t frame_for_compress_ = 0;
    int64_t req_count_ = 0, active_ = 0, uploaded_ = 0, uploaded_total_ = 0, evictions_ = 0, resident_ = 0;
    float ms_readback_ = 0.f, ms_policy_ = 0.f, ms_produce_ = 0.f, ms_upload_ = 0.f, ms_visit_ = 0.f;
    int32_t unique_ = 0;
    // device-side service
    bool device_paging_ = false;
    std::unique_ptr<DeviceTerrain> dterrain_;
    std::unique_ptr<DeviceBrickStore> dstore_;  // file trees: every brick in device memory
    uint4 production_job(uint32_t slot, uint32_t node) const;
    DedupeBuffers dd_;
    // Read-backs of the service go to mapped pinned memory, written by
    // kernels (dh_* are the device views), so that they do not wait behind
    // a colour read-back on the copy engines.
    // [0] request count, [1] distinct count, [4..7] order_.counters
    uint32_t* h_small_ = nullptr;
    uint32_t* dh_small_ = nullptr;
    uint32_t* h_cand_ = nullptr;    // upload candidates of a classified service
    uint32_t* dh_cand_ = nullptr;
    size_t h_cand_cap_ = 0;
    uint32_t* dh_win_ = nullptr;
    int ensure_small();
    int read_count(const uint32_t* count, uint32_t& out);
    // pinned: distinct node cells of the last frame (unclassified service)
    uint32_t* h_unique_ = nullptr;
    size_t h_unique_cap_ = 0;
    // eager device uploads: production jobs and node patches in mapped
    // pinned memory (h_*, device views dh_*) pulled into device copies
    // (d_*); ev_flush_ marks the end of the pull
    int flush_device();
    uint4* h_fjobs_ = nullptr;
    uint4* dh_fjobs_ = nullptr;
    uint4* d_fjobs_ = nullptr;
    size_t fjobs_cap_ = 0;
    vv_node_patch* h_fpatch_ = nullptr;
    vv_node_patch* dh_fpatch_ = nullptr;
    vv_node_patch* d_fpatch_ = nullptr;
    size_t fpatch_cap_ = 0;
    cudaEvent_t ev_flush_ = nullptr;
    bool requests_on_host_ = false;
    void* h_stage_ = nullptr;            // pinned brick staging
    size_t h_stage_cap_ = 0;
    // deferred uploads (pinned, mapped): jobs, node patches, their counts
    bool deferred_ = false;
    uint4* h_def_jobs_ = nullptr;
    vv_node_patch* h_def_patches_ = nullptr;
    // [0] jobs, [1] patches, [2] the staging's generation (host), [3] the
    // generation the device last applied (written by the enqueued work)
    volatile uint32_t* h_def_counts_ = nullptr;
    uint32_t stage_gen_ = 0;
    // their device copies, pulled at the start of each enqueue
    uint4* d_def_jobs_ = nullptr;
    vv_node_patch* d_def_patches_ = nullptr;
    uint32_t* d_def_counts_ = nullptr;
    uint32_t def_job_cap_ = 0, def_patch_cap_ = 0;
    std::vector<int32_t> slot_job_;      // latest pending upload per slot (-1 between uses)
    std::vector<uint32_t> keep_;         // pending uploads kept by a flush
    std::vector<uint32_t> up_slots_;     // their slots (host production)
    // colour buffers (alternating per draw) and their read-back
    float* color_buf_[2] = {nullptr, nullptr};
    int cur_color_ = 0;
    cudaStream_t copy_stream_ = nullptr;
    cudaEvent_t ev_copied_[2] = {nullptr, nullptr};
    cudaEvent_t ev_drawn_ = nullptr;
    bool copy_pending_[2] = {false, false};
    void* readback_host_ = nullptr;      // a requested read-back not started yet
    int readback_buf_ = 0;
    int start_readback();
};

}  // namespace vv
