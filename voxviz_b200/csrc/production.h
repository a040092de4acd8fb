// production.h - device side of the page-request service.
//
// * Brick production on the GPU: a device copy of the terrain's column-run
//   mip pyramid and a kernel that writes Node::copyMipMapToBrick's 10^3
//   stored brick (GigaVoxelsOctTree.cpp:1428-1488) straight into its pool
//   slot, in the pool's format.
// * Request de-duplication on the GPU: the node ids of the compacted list in
//   first-seen order, each once (the std::map of NodeUsageListProcessor::run,
//   GigaVoxelsOctTree.cpp:515, made deterministic).
#pragma once

#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>
#include <vector>

namespace vv {

class TerrainVolume;

struct DeviceMipLevel {
    int dim;
    const uint16_t* s;     // pure-solid count per column
    const uint16_t* r;     // explicit run length per column (nullptr at level 0)
    const uint32_t* off;   // run offset per column
    const uint32_t* data;  // explicit RGBA8 voxels
};

struct DeviceTerrainView {
    int depth;
    uint32_t band[8];
    DeviceMipLevel lv[11];
};

class DeviceTerrain {
public:
    ~DeviceTerrain();
    cudaError_t upload(const TerrainVolume& v);
    const DeviceTerrainView& view() const { return v_; }
    size_t bytes() const { return bytes_; }

private:
    void* alloc_copy(const void* src, size_t bytes, cudaError_t& e);
    DeviceTerrainView v_{};
    std::vector<void*> allocs_;
    size_t bytes_ = 0;
};

// jobs[i] = {slot, node level, i<<20 | j<<10 | k, 0}: produce the stored
// brick of node (level, i, j, k) into brick-pool slot `slot`.
cudaError_t launch_produce_bricks(const DeviceTerrainView& t, const uint4* jobs, int n, void* pool, int fmt,
                                  long long total_slots, int* status, cudaStream_t s);

// The same with jobs and their count read on the device from pinned, mapped
// host memory (at most max_jobs): a count-independent launch for CUDA graphs.
cudaError_t launch_produce_staged(const DeviceTerrainView& t, const uint4* jobs, const uint32_t* count,
                                  uint32_t max_jobs, void* pool, int fmt, long long total_slots, int* status,
                                  cudaStream_t s);

struct DedupeBuffers {
    uint32_t* first = nullptr;       // per node-pool grid cell, all 0xFFFFFFFF between calls
    size_t first_cells = 0;
    uint32_t* block_sums = nullptr;  // one per 1024 ids
    size_t block_cap = 0;
    uint32_t* unique = nullptr;      // grid cell index of each distinct node, first-seen order
    size_t unique_cap = 0;
    uint32_t* count = nullptr;       // number of distinct nodes
};

// State of each distinct node in the device node pool (block-linear, grid
// dims `dim`): its brick slot when resident, 0x80000000 | cell when neither
// resident nor constant, 0xFFFFFFFF when constant.  `count` is read on the
// device; at most max_n entries.
cudaError_t launch_classify(const uint32_t* unique, const uint32_t* count, uint32_t max_n, const uint2* nodes,
                            const int dim[3], const int slots[3], uint32_t* codes, cudaStream_t s);

// De-duplicate the node ids of `n_entries` compacted entries (4 ids each).
cudaError_t launch_dedupe(const uint32_t* requests, int n_entries, const int grid_dim[3], const DedupeBuffers& b,
                          cudaStream_t s);

}  // namespace vv
