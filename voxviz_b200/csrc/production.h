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
// masks: the pool's empty-cell masks (32 words per slot), written for each
// produced slot, or nullptr.
cudaError_t launch_produce_bricks(const DeviceTerrainView& t, const uint4* jobs, int n, void* pool, int fmt,
                                  uint32_t* masks, long long total_slots, int* status, cudaStream_t s);

// The same with the job count read on the device (at most max_jobs): a
// count-independent launch for CUDA graphs.  Jobs and count should be in
// device memory (launch_pull_staged puts them there).
cudaError_t launch_produce_staged(const DeviceTerrainView& t, const uint4* jobs, const uint32_t* count,
                                  uint32_t max_jobs, void* pool, int fmt, uint32_t* masks, long long total_slots,
                                  int* status, cudaStream_t s);

// The bricks of a tree read from files, resident in device memory: brick b
// is the 10^3 RGBA8 block at texels + 1000 b.  Paging such a tree copies a
// brick from here into its pool slot (a device-to-device gather) instead of
// the host-to-PBO upload of BrickPool::uploadBrick
// (GigaVoxelsBrickPool.cpp:729-813).
struct DeviceBrickStoreView {
    const uint32_t* texels;
    uint32_t bricks;
};

class DeviceBrickStore {
public:
    ~DeviceBrickStore();
    cudaError_t upload(const uint32_t* texels, size_t bricks);
    DeviceBrickStoreView view() const { return DeviceBrickStoreView{d_, (uint32_t)bricks_}; }
    size_t bytes() const { return bricks_ * 4000u; }

private:
    uint32_t* d_ = nullptr;
    size_t bricks_ = 0;
};

// jobs[i] = {slot, brick, 0, 0}: copy store brick `brick` into pool slot
// `slot`, in the pool's format, and write the slot's empty-cell mask (masks
// may be nullptr).  The staged form reads the job count on the device.
cudaError_t launch_copy_bricks(const DeviceBrickStoreView& st, const uint4* jobs, int n, void* pool, int fmt,
                               uint32_t* masks, long long total_slots, int* status, cudaStream_t s);
cudaError_t launch_copy_staged(const DeviceBrickStoreView& st, const uint4* jobs, const uint32_t* count,
                               uint32_t max_jobs, void* pool, int fmt, uint32_t* masks, long long total_slots,
                               int* status, cudaStream_t s);

struct DedupeBuffers {
    uint32_t* first = nullptr;       // per node-pool grid cell, all 0xFFFFFFFF between calls
    size_t first_cells = 0;
    uint32_t* block_sums = nullptr;  // one per 1024 ids
    size_t block_cap = 0;
    uint32_t* unique = nullptr;      // grid cell index of each distinct node, first-seen order
    size_t unique_cap = 0;
    uint32_t* count = nullptr;       // number of distinct nodes
};

// The brick pool's LRU order on the device (BrickPool::m_loadedBricks,
// GigaVoxelsBrickPool.cpp:330-424, made deterministic): order[cur] lists
// every slot once, least recently used first, read circularly from a head
// position the host keeps.  Evicting the front and re-using its slot moves it
// to the back, which in a full circular list is advancing the head, so only
// touches of other slots move data: a partition keeps the untouched slots in
// their order and appends the touched ones in touch order.
struct SlotOrderBuffers {
    uint32_t* order[2] = {nullptr, nullptr};
    int cur = 0;
    uint32_t n = 0;                  // slots
    uint32_t* mark = nullptr;        // per slot: epoch of the partition that last touched it
    uint32_t* block_sums = nullptr;  // partition scan, one per 1024 slots
    uint32_t* seq = nullptr;         // touched slots in touch order (n entries)
    uint32_t* cand = nullptr;        // upload candidates: grid cells, first-seen order
    size_t cand_cap = 0;
    uint32_t* cand_sums = nullptr;   // candidate scan, one per 1024 distinct nodes
    size_t cand_sums_cap = 0;
    // device counters: [0] distinct nodes, [1] touched, [2] candidates, [3] untouched
    uint32_t* counters = nullptr;
};

// Identity order (slot-id order: the empty slots lead), marks cleared.
cudaError_t slot_order_init(SlotOrderBuffers& b, uint32_t n, cudaStream_t s);
void slot_order_free(SlotOrderBuffers& b);

// For the distinct requested nodes (dd.unique, dd.count: grid cells in
// first-seen order) against the device node pool: the resident nodes' slots
// go to seq in first-seen order, except root_slot (0xFFFFFFFF when the root
// is not resident), and are marked with `epoch`, together with root_slot;
// the cells of the non-resident, non-constant nodes go to cand.  Counts land
// in counters[1] and [2].  At most max_n distinct nodes; dd.unique is
// overwritten with each node's state (slot, 0x80000000 | cell, 0xFFFFFFFF).
cudaError_t launch_classify_split(const DedupeBuffers& dd, uint32_t max_n, const uint2* nodes, const int dim[3],
                                  const int slots[3], uint32_t root_slot, uint32_t epoch, SlotOrderBuffers& b,
                                  int* status, cudaStream_t s);

// Mark the m touched slots already in b.seq (host-known m) with `epoch`.
cudaError_t launch_mark_touched(SlotOrderBuffers& b, uint32_t m, uint32_t epoch, int* status, cudaStream_t s);

// Partition the order read from `head`: the slots not marked with `epoch`
// keep their order, then the touched ones follow: seq's first m entries (m
// from counters[1] when seq_on_device, else m_host) and root_slot last when
// it is a slot.  Writes order[cur ^ 1] from position 0 and flips cur;
// counters[3] receives the untouched count.  A touched count that does not
// complete the list (a repeated or invalid slot) sets VV_ERR_BOUNDS.
cudaError_t launch_order_partition(SlotOrderBuffers& b, uint32_t head, uint32_t epoch, bool seq_on_device,
                                   uint32_t m_host, uint32_t max_m, uint32_t root_slot, int* status,
                                   cudaStream_t s);

// Read-out of a classified service into mapped host memory, written by the
// SMs so that it does not queue behind copies on the copy engines (such as a
// frame's colour read-back): counters[0..3] to h_counters, the candidates to
// h_cand (at most cand_cap) and the order's first min(n, 2 * candidates + 2)
// entries from position 0 to h_win.  All three are device views of mapped
// host allocations.
cudaError_t launch_service_readout(const SlotOrderBuffers& b, uint32_t* h_counters, uint32_t* h_cand,
                                   uint32_t cand_cap, uint32_t* h_win, cudaStream_t s);

// Copy two ranges of 16-byte words from mapped host memory into device
// memory, coalesced (a service's production jobs and node patches): the SMs
// read over the bus, so nothing queues on the copy engines.
cudaError_t launch_pull(const uint4* src_a, uint4* dst_a, size_t n_a, const uint4* src_b, uint4* dst_b, size_t n_b,
                        cudaStream_t s);

// The same for staged uploads, whose counts are read on the device (a
// count-independent launch for CUDA graphs): h_counts[0] jobs (at most
// max_jobs) and h_counts[1] node patches (at most max_patches, 20 bytes
// each, the mapped allocation rounded up to whole 16-byte words) are pulled
// into d_jobs / d_patches, the clamped counts into d_counts[0..1].  A few
// CTAs, each reading the counts once.
cudaError_t launch_pull_staged(const uint32_t* h_counts, const uint4* h_jobs, uint32_t max_jobs,
                               const void* h_patches, uint32_t max_patches, uint32_t* d_counts, uint4* d_jobs,
                               void* d_patches, cudaStream_t s);

// One word from device memory to mapped host memory.
cudaError_t launch_read_word(const uint32_t* src, uint32_t* h_dst, cudaStream_t s);

// De-duplicate the node ids of `n_entries` compacted entries (4 ids each);
// the distinct count goes to b.count.
cudaError_t launch_dedupe(const uint32_t* requests, int n_entries, const int grid_dim[3], const DedupeBuffers& b,
                          cudaStream_t s);

}  // namespace vv
