// ctx.h - the device context behind the vv_ctx handle.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <string>

#include "../../include/voxviz_b200.h"

namespace vv {

struct DeviceTree {
    uint2* nodes = nullptr;  // block-linear node pool
    int dim[3] = {0, 0, 0};
    size_t cells = 0;
};

int vv_max_iterations(const vv_uniforms* u);

// Error and scratch helpers of ctx.cu for the other translation units.
int ctx_fail(vv_ctx* c, int code, const std::string& msg);
int ctx_ensure(vv_ctx* c, void** ptr, size_t* cap, size_t bytes, const char* what);
int ctx_ensure_host(vv_ctx* c, void** ptr, size_t* cap, size_t bytes);
// The pool's empty-cell masks when valid, else nullptr (no skipping).
const uint32_t* ctx_cell_mask(const vv_ctx* c);
uint32_t* ctx_cell_mask_rw(vv_ctx* c);
// The message vv_last_error(NULL) returns on this thread.
void set_thread_error(const std::string& msg);

}  // namespace vv

struct vv_ctx {
    int device = 0;
    cudaStream_t stream = nullptr;
    std::string err;
    int* d_status = nullptr;
    vv::DeviceTree trees[VV_MAX_TREES];
    // brick pool
    void* bricks = nullptr;
    bool bricks_external = false;  // attached caller memory: never freed here
    int slots[3] = {0, 0, 0};
    long long total_slots = 0;
    int fmt = VV_FMT_RGBA8;
    size_t brick_bytes = 0;
    size_t pool_bytes = 0;
    // empty-cell masks of the brick pool (cellmask.cuh), 32 words per slot;
    // valid while every write to the pool went through this library
    uint32_t* cell_mask = nullptr;
    long long cell_mask_slots = 0;
    bool cell_mask_valid = false;
    // gradient pool (lighting): same slots as the brick pool
    void* grads = nullptr;
    int grad_fmt = VV_FMT_FP32;
    size_t grad_brick_bytes = 0;
    size_t grad_pool_bytes = 0;
    // jitter
    uint8_t* d_jitter = nullptr;
    int jitter_size = 0;
    // scratch
    uint32_t* d_usage = nullptr;
    size_t usage_cap = 0;
    uint32_t* d_mask = nullptr;
    size_t mask_cap = 0;
    uint32_t* d_counts = nullptr;
    size_t counts_cap = 0;
    uint32_t* d_offsets = nullptr;
    size_t offsets_cap = 0;
    uint32_t* d_up_slots = nullptr;
    size_t up_slots_cap = 0;
    void* d_up_bricks = nullptr;
    size_t up_bricks_cap = 0;
    vv_node_patch* d_patches = nullptr;
    size_t patches_cap = 0;
    uint32_t* d_grid_words = nullptr;
    size_t grid_words_cap = 0;
    void* h_stage = nullptr;
    size_t h_stage_cap = 0;
    // batched launch: the launch-parameter block of the views (host) and one
    // tile-queue counter per launch (device)
    void* h_batch = nullptr;
    size_t h_batch_cap = 0;
    void* d_batch = nullptr;
    size_t d_batch_cap = 0;
    // extra copies of a sparse gradient's rows (VV_GRAD_SPREAD), all zero
    // between calls
    float4* d_spread = nullptr;
    size_t spread_elems = 0;
    long long spread_rows_kept = 0;  // rows per copy of sums kept by VV_GRAD_SPREAD_KEEP, else 0
    // compaction in one launch per pyramid level instead of compact.cu's three
    bool per_level_compaction = false;
    // ray-cast form (VV_RAYCAST_TILES / VV_RAYCAST_REFILL) and the refill
    // form's tile counter
    int raycast_mode = 0;
    unsigned int* d_refill_counter = nullptr;
    // profiling
    bool profiling = false;
    bool timed = false;
    cudaEvent_t ev[3] = {nullptr, nullptr, nullptr};
};
