// production.cu - GPU brick production and request de-duplication.
#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include <algorithm>
#include <cstring>

#include "../../include/voxviz_b200.h"
#include "cellmask.cuh"
#include "dxt.h"
#include "production.h"
#include "terrain.h"

namespace vv {

DeviceTerrain::~DeviceTerrain() {
    for (void* p : allocs_) cudaFree(p);
}

void* DeviceTerrain::alloc_copy(const void* src, size_t bytes, cudaError_t& e) {
    if (e != cudaSuccess) return nullptr;
    void* p = nullptr;
    e = cudaMalloc(&p, bytes ? bytes : 4);
    if (e != cudaSuccess) return nullptr;
    allocs_.push_back(p);
    bytes_ += bytes;
    if (bytes) e = cudaMemcpy(p, src, bytes, cudaMemcpyHostToDevice);
    return p;
}

cudaError_t DeviceTerrain::upload(const TerrainVolume& vol) {
    cudaError_t e = cudaSuccess;
    v_.depth = vol.depth();
    for (int b = 0; b < 8; ++b) v_.band[b] = band_colour(b);
    for (int m = 0; m <= vol.depth(); ++m) {
        const MipLevel& L = vol.mip(m);
        DeviceMipLevel& d = v_.lv[m];
        d.dim = L.dim;
        d.s = (const uint16_t*)alloc_copy(L.s.data(), L.s.size() * sizeof(uint16_t), e);
        if (m == 0) {  // the leaf level has no explicit voxels
            d.r = nullptr;
            d.off = nullptr;
            d.data = nullptr;
            continue;
        }
        d.r = (const uint16_t*)alloc_copy(L.r.data(), L.r.size() * sizeof(uint16_t), e);
        std::vector<uint32_t> off32(L.off.size());
        for (size_t i = 0; i < off32.size(); ++i) off32[i] = (uint32_t)L.off[i];
        d.off = (const uint32_t*)alloc_copy(off32.data(), off32.size() * sizeof(uint32_t), e);
        d.data = (const uint32_t*)alloc_copy(L.data.data(), L.data.size() * sizeof(uint32_t), e);
    }
    return e;
}

namespace {

template <int FMT>
__device__ __forceinline__ void store_texel(void* pool, size_t i, uint32_t v) {
    if (FMT == VV_FMT_RGBA8) {
        ((uint32_t*)pool)[i] = v;
        return;
    }
    // the same v/255 values as the host producer, rounded to nearest even
    const float c0 = (float)(v & 255u) / 255.0f, c1 = (float)((v >> 8) & 255u) / 255.0f;
    const float c2 = (float)((v >> 16) & 255u) / 255.0f, c3 = (float)(v >> 24) / 255.0f;
    if (FMT == VV_FMT_FP32) {
        ((float4*)pool)[i] = make_float4(c0, c1, c2, c3);
    } else if (FMT == VV_FMT_FP16) {
        const uint32_t a = (uint32_t)__half_as_ushort(__float2half_rn(c0)) |
                           ((uint32_t)__half_as_ushort(__float2half_rn(c1)) << 16);
        const uint32_t b = (uint32_t)__half_as_ushort(__float2half_rn(c2)) |
                           ((uint32_t)__half_as_ushort(__float2half_rn(c3)) << 16);
        ((uint2*)pool)[i] = make_uint2(a, b);
    } else {
        const uint32_t a = (uint32_t)__bfloat16_as_ushort(__float2bfloat16_rn(c0)) |
                           ((uint32_t)__bfloat16_as_ushort(__float2bfloat16_rn(c1)) << 16);
        const uint32_t b = (uint32_t)__bfloat16_as_ushort(__float2bfloat16_rn(c2)) |
                           ((uint32_t)__bfloat16_as_ushort(__float2bfloat16_rn(c3)) << 16);
        ((uint2*)pool)[i] = make_uint2(a, b);
    }
}

// A DXT5 pool slot from the brick's RGBA8 texels in shared memory (all
// threads of the CTA, after a barrier): one 16-byte block per thread.
__device__ __forceinline__ void encode_dxt5_slot(const uint32_t* rgba, void* pool, size_t slot) {
    for (int b = threadIdx.x; b < dxt::kBlocksPerSlot; b += blockDim.x) {
        uint32_t px[16], valid, w[4];
        dxt::gather_block(rgba, b, px, valid);
        dxt::encode_dxt5(px, valid, w);
        ((uint4*)pool)[slot * dxt::kBlocksPerSlot + (size_t)b] = make_uint4(w[0], w[1], w[2], w[3]);
    }
}

// One CTA per brick.  Texel (bx,by,bz) of node (d; i,j,k) is the mip-level
// (L-d) voxel (8i-1+bx, 8j-1+by, 8k-1+bz), transparent black outside the level.
template <int FMT>
__device__ __forceinline__ void produce_one(const DeviceTerrainView& t, const uint4 job, void* __restrict__ pool,
                                            uint32_t* __restrict__ masks, long long total_slots, int* status) {
    __shared__ uint8_t zero[VV_BRICK_TEXELS];  // texel all-zero flags for the slot's cell mask
    __shared__ uint32_t rgba[FMT == VV_FMT_DXT5 ? VV_BRICK_TEXELS : 1];  // the brick before compression
    if ((long long)job.x >= total_slots || (int)job.y > t.depth) {
        if (threadIdx.x == 0 && status) atomicCAS(status, 0, VV_ERR_BOUNDS);
        return;
    }
    const int m = t.depth - (int)job.y;
    const DeviceMipLevel L = t.lv[m];
    const int i = (int)((job.z >> 20) & 1023u), j = (int)((job.z >> 10) & 1023u), k = (int)(job.z & 1023u);
    const size_t base = (size_t)job.x * 1000u;
    for (int q = threadIdx.x; q < 1000; q += blockDim.x) {
        const int bz = q / 100, by = (q / 10) % 10, bx = q % 10;
        const int x = 8 * i - 1 + bx, y = 8 * j - 1 + by, z = 8 * k - 1 + bz;
        uint32_t v = 0u;
        if (x >= 0 && y >= 0 && z >= 0 && x < L.dim && y < L.dim && z < L.dim) {
            const size_t c = (size_t)y * L.dim + x;
            const int s = L.s[c];
            if (z < s) {
                v = t.band[((z << m) >> t.depth) & 7];
            } else if (L.r) {
                const int r = L.r[c];
                if (z < s + r) v = L.data[L.off[c] + (uint32_t)(z - s)];
            }
        }
        if constexpr (FMT == VV_FMT_DXT5) rgba[q] = v;
        else store_texel<FMT>(pool, base + (size_t)q, v);
        zero[q] = v == 0u ? 1 : 0;  // RGBA8 zero stores (and DXT-decodes) as zero in every format
    }
    if constexpr (FMT == VV_FMT_DXT5) {
        __syncthreads();
        encode_dxt5_slot(rgba, pool, (size_t)job.x);
    }
    if (masks) {  // the same for the whole CTA
        __syncthreads();
        write_cell_mask(zero, masks + (size_t)job.x * kCellMaskWords);
    }
    __syncthreads();  // zero[] and rgba[] serve the CTA's next job
}

template <int FMT>
__global__ void produce_kernel(const __grid_constant__ DeviceTerrainView t, const uint4* __restrict__ jobs,
                               void* __restrict__ pool, uint32_t* __restrict__ masks, long long total_slots,
                               int* status) {
    produce_one<FMT>(t, jobs[blockIdx.x], pool, masks, total_slots, status);
}

// Staged form: the job count is read on the device, so the launch itself
// does not depend on it (it can sit in a CUDA graph replayed every frame).
// Jobs and count are device copies (see launch_pull_staged): a read of
// mapped host memory from every CTA costs a bus round trip each.
template <int FMT>
__global__ void produce_staged_kernel(const __grid_constant__ DeviceTerrainView t, const uint4* jobs,
                                      const volatile uint32_t* count, uint32_t max_jobs, void* __restrict__ pool,
                                      uint32_t* __restrict__ masks, long long total_slots, int* status) {
    __shared__ uint32_t s_n;  // one read of the count per CTA
    if (threadIdx.x == 0) s_n = min(*count, max_jobs);
    __syncthreads();
    const uint32_t n = s_n;
    __shared__ uint4 s_job;  // and one per job
    for (uint32_t j = blockIdx.x; j < n; j += gridDim.x) {
        if (threadIdx.x == 0) s_job = jobs[j];
        __syncthreads();
        produce_one<FMT>(t, s_job, pool, masks, total_slots, status);
        __syncthreads();
    }
}

// One CTA per job: store brick job.y into slot job.x.  The store holds
// RGBA8, so an RGBA8 pool takes 16-byte words as they are (a slot and a
// store brick are 4000 bytes, 16-byte aligned).
template <int FMT>
__device__ __forceinline__ void copy_one(const DeviceBrickStoreView& st, const uint4 job, void* __restrict__ pool,
                                         uint32_t* __restrict__ masks, long long total_slots, int* status) {
    __shared__ uint8_t zero[VV_BRICK_TEXELS];
    __shared__ uint32_t rgba[FMT == VV_FMT_DXT5 ? VV_BRICK_TEXELS : 1];
    if ((long long)job.x >= total_slots || job.y >= st.bricks) {
        if (threadIdx.x == 0 && status) atomicCAS(status, 0, VV_ERR_BOUNDS);
        return;
    }
    const uint32_t* src = st.texels + (size_t)job.y * VV_BRICK_TEXELS;
    const size_t base = (size_t)job.x * VV_BRICK_TEXELS;
    if (FMT == VV_FMT_RGBA8) {
        const uint4* s4 = (const uint4*)src;
        uint4* d4 = (uint4*)((uint32_t*)pool + base);
        for (int q = threadIdx.x; q < VV_BRICK_TEXELS / 4; q += blockDim.x) {
            const uint4 v = __ldg(s4 + q);
            d4[q] = v;
            zero[4 * q] = v.x == 0u;
            zero[4 * q + 1] = v.y == 0u;
            zero[4 * q + 2] = v.z == 0u;
            zero[4 * q + 3] = v.w == 0u;
        }
    } else {
        for (int q = threadIdx.x; q < VV_BRICK_TEXELS; q += blockDim.x) {
            const uint32_t v = __ldg(src + q);
            if constexpr (FMT == VV_FMT_DXT5) rgba[q] = v;
            else store_texel<FMT>(pool, base + (size_t)q, v);
            zero[q] = v == 0u;
        }
        if constexpr (FMT == VV_FMT_DXT5) {
            __syncthreads();
            encode_dxt5_slot(rgba, pool, (size_t)job.x);
        }
    }
    if (masks) {
        __syncthreads();
        write_cell_mask(zero, masks + (size_t)job.x * kCellMaskWords);
        __syncthreads();
    }
}

template <int FMT>
__global__ void copy_kernel(const DeviceBrickStoreView st, const uint4* __restrict__ jobs, void* __restrict__ pool,
                            uint32_t* __restrict__ masks, long long total_slots, int* status) {
    copy_one<FMT>(st, jobs[blockIdx.x], pool, masks, total_slots, status);
}

template <int FMT>
__global__ void copy_staged_kernel(const DeviceBrickStoreView st, const uint4* jobs, const volatile uint32_t* count,
                                   uint32_t max_jobs, void* __restrict__ pool, uint32_t* __restrict__ masks,
                                   long long total_slots, int* status) {
    __shared__ uint32_t s_n;
    if (threadIdx.x == 0) s_n = min(*count, max_jobs);
    __syncthreads();
    const uint32_t n = s_n;
    __shared__ uint4 s_job;
    for (uint32_t j = blockIdx.x; j < n; j += gridDim.x) {
        if (threadIdx.x == 0) s_job = jobs[j];
        __syncthreads();
        copy_one<FMT>(st, s_job, pool, masks, total_slots, status);
        __syncthreads();
    }
}

__device__ __forceinline__ bool decode_cell(uint32_t id, int dx, int dy, int dz, uint32_t& g) {
    if (id == 0u) return false;
    const uint32_t x = ((id >> 20) & 0x3FFu) - 1u, y = ((id >> 10) & 0x3FFu) - 1u, z = (id & 0x3FFu) - 1u;
    if (x >= (uint32_t)dx || y >= (uint32_t)dy || z >= (uint32_t)dz) return false;
    g = (z * (uint32_t)dy + y) * (uint32_t)dx + x;
    return true;
}

__global__ void dedupe_first_kernel(const uint32_t* __restrict__ ids, int n, int dx, int dy, int dz,
                                    uint32_t* __restrict__ first) {
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= n) return;
    uint32_t g;
    if (decode_cell(ids[q], dx, dy, dz, g)) atomicMin(first + g, (uint32_t)q);
}

__global__ void __launch_bounds__(1024) dedupe_count_kernel(const uint32_t* __restrict__ ids, int n, int dx, int dy,
                                                            int dz, const uint32_t* __restrict__ first,
                                                            uint32_t* __restrict__ block_sums) {
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    uint32_t g = 0;
    const bool f = q < n && decode_cell(ids[q], dx, dy, dz, g) && first[g] == (uint32_t)q;
    const int c = __syncthreads_count(f);
    if (threadIdx.x == 0) block_sums[blockIdx.x] = (uint32_t)c;
}

// Exclusive scan of the block sums in place, total to *count (one CTA of
// 1024 threads).
__device__ void scan_sums(uint32_t* __restrict__ sums, int nb, uint32_t* __restrict__ count) {
    __shared__ uint32_t warp_tot[32];
    __shared__ uint32_t carry;
    if (threadIdx.x == 0) carry = 0u;
    __syncthreads();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int base = 0; base < nb; base += 1024) {
        const int i = base + (int)threadIdx.x;
        const uint32_t v = i < nb ? sums[i] : 0u;
        uint32_t x = v;
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, x, o);
            if (lane >= o) x += y;
        }
        if (lane == 31) warp_tot[warp] = x;
        __syncthreads();
        if (warp == 0) {
            uint32_t w = warp_tot[lane];
            for (int o = 1; o < 32; o <<= 1) {
                const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, w, o);
                if (lane >= o) w += y;
            }
            warp_tot[lane] = w;  // inclusive
        }
        __syncthreads();
        const uint32_t before = carry + (warp > 0 ? warp_tot[warp - 1] : 0u) + (x - v);
        if (i < nb) sums[i] = before;
        __syncthreads();
        if (threadIdx.x == 0) carry += warp_tot[31];
        __syncthreads();
    }
    if (threadIdx.x == 0) *count = carry;
}

__global__ void __launch_bounds__(1024) scan_sums_kernel(uint32_t* __restrict__ sums, int nb,
                                                         uint32_t* __restrict__ count) {
    scan_sums(sums, nb, count);
}

// Two independent scans, one per CTA.
__global__ void __launch_bounds__(1024) scan_sums2_kernel(uint32_t* __restrict__ sums_a, uint32_t* __restrict__ sums_b,
                                                          int nb, uint32_t* __restrict__ count_a,
                                                          uint32_t* __restrict__ count_b) {
    if (blockIdx.x == 0) scan_sums(sums_a, nb, count_a);
    else scan_sums(sums_b, nb, count_b);
}

__global__ void __launch_bounds__(1024) dedupe_scatter_kernel(const uint32_t* __restrict__ ids, int n, int dx,
                                                              int dy, int dz, uint32_t* __restrict__ first,
                                                              const uint32_t* __restrict__ block_off,
                                                              uint32_t* __restrict__ out) {
    __shared__ uint32_t warp_cnt[32];
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint32_t g = 0;
    const bool f = q < n && decode_cell(ids[q], dx, dy, dz, g) && first[g] == (uint32_t)q;
    const unsigned b = __ballot_sync(0xFFFFFFFFu, f);
    if (lane == 0) warp_cnt[warp] = (uint32_t)__popc(b);
    __syncthreads();
    if (f) {
        uint32_t off = block_off[blockIdx.x];
        for (int w = 0; w < warp; ++w) off += warp_cnt[w];
        off += (uint32_t)__popc(b & ((1u << lane) - 1u));
        out[off] = g;
        first[g] = 0xFFFFFFFFu;  // ready for the next frame
    }
}

// State of a distinct requested node (grid cell g) in the device node pool
// (block-linear, 2x2x2 node blocks): the brick-pool slot if resident,
// 0x80000000 | g if neither resident nor constant (an upload candidate),
// 0xFFFFFFFF otherwise.
__device__ __forceinline__ uint32_t node_state(uint32_t g, const uint2* __restrict__ nodes, int dx, int dy, int sx,
                                               int sy) {
    const uint32_t x = g % (uint32_t)dx, y = (g / (uint32_t)dx) % (uint32_t)dy, z = g / ((uint32_t)dx * dy);
    const uint32_t blk = ((z >> 1) * ((uint32_t)dy >> 1) + (y >> 1)) * ((uint32_t)dx >> 1) + (x >> 1);
    const uint2 w = nodes[(size_t)blk * 8u + ((x & 1u) | ((y & 1u) << 1) | ((z & 1u) << 2))];
    if (w.x & 0x80000000u) {
        // brick pointer = slot origin + border (0..2 per axis), 10 texels per slot
        const uint32_t px = (w.y >> 20) & 0x3FFu, py = (w.y >> 10) & 0x3FFu, pz = w.y & 0x3FFu;
        return ((pz / 10u) * (uint32_t)sy + py / 10u) * (uint32_t)sx + px / 10u;
    }
    return (w.x & 0x40000000u) ? 0xFFFFFFFFu : (0x80000000u | g);
}

__device__ __forceinline__ bool is_touch(uint32_t st, uint32_t root_slot) {
    return st < 0x80000000u && st != root_slot;
}
__device__ __forceinline__ bool is_candidate(uint32_t st) { return (st & 0x80000000u) && st != 0xFFFFFFFFu; }

// Per 1024 distinct nodes: their states (in place) and the block counts of
// resident nodes other than the root's slot and of upload candidates.
__global__ void __launch_bounds__(1024) classify_count_kernel(uint32_t* __restrict__ unique,
                                                              const uint32_t* __restrict__ count, uint32_t max_n,
                                                              const uint2* __restrict__ nodes, int dx, int dy, int sx,
                                                              int sy, uint32_t root_slot,
                                                              uint32_t* __restrict__ sums_touch,
                                                              uint32_t* __restrict__ sums_cand) {
    const uint32_t n = min(*count, max_n);
    const uint32_t k = blockIdx.x * 1024u + threadIdx.x;
    bool t = false, c = false;
    if (k < n) {
        const uint32_t st = node_state(unique[k], nodes, dx, dy, sx, sy);
        unique[k] = st;
        t = is_touch(st, root_slot);
        c = is_candidate(st);
    }
    const int nt = __syncthreads_count(t);
    const int nc = __syncthreads_count(c);
    if (threadIdx.x == 0) {
        sums_touch[blockIdx.x] = (uint32_t)nt;
        sums_cand[blockIdx.x] = (uint32_t)nc;
    }
}

// Offset of this lane's flagged element inside its CTA, from per-warp counts.
__device__ __forceinline__ uint32_t warp_offset(const uint32_t* warp_cnt, int warp, int lane, unsigned ballot) {
    uint32_t off = 0;
    for (int w = 0; w < warp; ++w) off += warp_cnt[w];
    return off + (uint32_t)__popc(ballot & ((1u << lane) - 1u));
}

// Scatter of the touched slots (first-seen order, marked with `epoch`) and of
// the upload candidates' cells, from the scanned block counts.
__global__ void __launch_bounds__(1024) split_scatter_kernel(const uint32_t* __restrict__ states,
                                                             const uint32_t* __restrict__ count, uint32_t max_n,
                                                             uint32_t root_slot, const uint32_t* __restrict__ off_touch,
                                                             const uint32_t* __restrict__ off_cand, uint32_t n_slots,
                                                             uint32_t epoch, uint32_t* __restrict__ seq,
                                                             uint32_t* __restrict__ mark, uint32_t* __restrict__ cand,
                                                             int* status) {
    __shared__ uint32_t wt[32], wc[32];
    if (blockIdx.x == 0 && threadIdx.x == 0 && root_slot < n_slots) mark[root_slot] = epoch;
    const uint32_t n = min(*count, max_n);
    if (blockIdx.x * 1024u >= n) return;  // whole CTA
    const uint32_t k = blockIdx.x * 1024u + threadIdx.x;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const uint32_t st = k < n ? states[k] : 0xFFFFFFFFu;
    const bool t = is_touch(st, root_slot), c = is_candidate(st);
    const unsigned bt = __ballot_sync(0xFFFFFFFFu, t), bc = __ballot_sync(0xFFFFFFFFu, c);
    if (lane == 0) {
        wt[warp] = (uint32_t)__popc(bt);
        wc[warp] = (uint32_t)__popc(bc);
    }
    __syncthreads();
    if (t) {
        const uint32_t off = off_touch[blockIdx.x] + warp_offset(wt, warp, lane, bt);
        if (st < n_slots && off < n_slots) {
            seq[off] = st;
            mark[st] = epoch;
        } else {
            atomicCAS(status, 0, VV_ERR_BOUNDS);
        }
    }
    if (c) cand[off_cand[blockIdx.x] + warp_offset(wc, warp, lane, bc)] = st & 0x7FFFFFFFu;
}

__global__ void mark_touched_kernel(const uint32_t* __restrict__ seq, uint32_t m, uint32_t n_slots, uint32_t epoch,
                                    uint32_t* __restrict__ mark, int* status) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < m; i += gridDim.x * blockDim.x) {
        const uint32_t s = seq[i];
        if (s < n_slots) mark[s] = epoch;
        else atomicCAS(status, 0, VV_ERR_BOUNDS);
    }
}

__device__ __forceinline__ uint32_t ring(uint32_t head, uint32_t j, uint32_t n) {
    const uint32_t p = head + j;
    return p >= n ? p - n : p;
}

__global__ void __launch_bounds__(1024) order_count_kernel(const uint32_t* __restrict__ order, uint32_t n,
                                                           uint32_t head, const uint32_t* __restrict__ mark,
                                                           uint32_t epoch, uint32_t* __restrict__ sums) {
    const uint32_t j = blockIdx.x * 1024u + threadIdx.x;
    const uint32_t slot = j < n ? order[ring(head, j, n)] : n;
    const bool f = slot < n && mark[slot] != epoch;  // a slot out of range drops out: the counts then disagree
    const int c = __syncthreads_count(f);
    if (threadIdx.x == 0) sums[blockIdx.x] = (uint32_t)c;
}

// CTAs [0, nb_order): the untouched slots in their order; the CTAs after
// them: the touched slots (seq's m entries, then root_slot when it is a
// slot) after the untouched ones.
__global__ void __launch_bounds__(1024) order_scatter_kernel(const uint32_t* __restrict__ order, uint32_t n,
                                                             uint32_t head, const uint32_t* __restrict__ mark,
                                                             uint32_t epoch, const uint32_t* __restrict__ off,
                                                             uint32_t nb_order, const uint32_t* __restrict__ counters,
                                                             bool seq_on_device, uint32_t m_host, uint32_t root_slot,
                                                             const uint32_t* __restrict__ seq,
                                                             uint32_t* __restrict__ out, int* status) {
    __shared__ uint32_t wcnt[32];
    if (blockIdx.x < nb_order) {
        const uint32_t j = blockIdx.x * 1024u + threadIdx.x;
        const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
        uint32_t slot = 0;
        bool f = false;
        if (j < n) {
            slot = order[ring(head, j, n)];
            f = slot < n && mark[slot] != epoch;
        }
        const unsigned b = __ballot_sync(0xFFFFFFFFu, f);
        if (lane == 0) wcnt[warp] = (uint32_t)__popc(b);
        __syncthreads();
        if (f) out[off[blockIdx.x] + warp_offset(wcnt, warp, lane, b)] = slot;
        return;
    }
    const uint32_t m = seq_on_device ? counters[1] : m_host;
    const uint32_t u = counters[3];
    const uint32_t total = m + (root_slot < n ? 1u : 0u);
    if (u > n || total != n - u) {
        if (blockIdx.x == nb_order && threadIdx.x == 0) atomicCAS(status, 0, VV_ERR_BOUNDS);
        return;
    }
    const uint32_t stride = (gridDim.x - nb_order) * 1024u;
    for (uint32_t i = (blockIdx.x - nb_order) * 1024u + threadIdx.x; i < total; i += stride)
        out[u + i] = i < m ? seq[i] : root_slot;
}

__global__ void service_readout_kernel(const uint32_t* __restrict__ counters, const uint32_t* __restrict__ cand,
                                       const uint32_t* __restrict__ order, uint32_t n_slots,
                                       uint32_t* __restrict__ h_counters, uint32_t* __restrict__ h_cand,
                                       uint32_t cand_cap, uint32_t* __restrict__ h_win) {
    const uint32_t c = min(counters[2], cand_cap);
    const uint32_t len = (uint32_t)min((unsigned long long)n_slots, 2ull * c + 2ull);
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x, stride = gridDim.x * blockDim.x;
    if (t < 4) h_counters[t] = counters[t];
    for (uint32_t i = t; i < c; i += stride) h_cand[i] = cand[i];
    for (uint32_t i = t; i < len; i += stride) h_win[i] = order[i];
}

__global__ void read_word_kernel(const uint32_t* __restrict__ src, uint32_t* __restrict__ dst) { *dst = *src; }

__global__ void pull_staged_kernel(const volatile uint32_t* h_counts, const uint4* __restrict__ h_jobs,
                                   uint32_t max_jobs, const uint4* __restrict__ h_patch_words, uint32_t max_patches,
                                   uint32_t* __restrict__ d_counts, uint4* __restrict__ d_jobs,
                                   uint4* __restrict__ d_patch_words) {
    __shared__ uint32_t s_n[2];
    if (threadIdx.x < 2) s_n[threadIdx.x] = min(h_counts[threadIdx.x], threadIdx.x ? max_patches : max_jobs);
    __syncthreads();
    const uint32_t nj = s_n[0], np = s_n[1];
    if (blockIdx.x == 0 && threadIdx.x < 2) d_counts[threadIdx.x] = s_n[threadIdx.x];
    const size_t nw = ((size_t)np * 20u + 15u) / 16u;
    const size_t stride = (size_t)gridDim.x * blockDim.x;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < nj + nw; i += stride) {
        if (i < nj) d_jobs[i] = h_jobs[i];
        else d_patch_words[i - nj] = h_patch_words[i - nj];
    }
}

__global__ void pull_kernel(const uint4* __restrict__ src_a, uint4* __restrict__ dst_a, size_t n_a,
                            const uint4* __restrict__ src_b, uint4* __restrict__ dst_b, size_t n_b) {
    const size_t stride = (size_t)gridDim.x * blockDim.x;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n_a + n_b; i += stride) {
        if (i < n_a) dst_a[i] = src_a[i];
        else dst_b[i - n_a] = src_b[i - n_a];
    }
}

__global__ void iota_kernel(uint32_t* __restrict__ o, uint32_t n) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) o[i] = i;
}

}  // namespace

cudaError_t slot_order_init(SlotOrderBuffers& b, uint32_t n, cudaStream_t s) {
    slot_order_free(b);
    if (n == 0) return cudaErrorInvalidValue;
    const size_t nb = (n + 1023u) / 1024u;
    cudaError_t e;
    if ((e = cudaMalloc((void**)&b.order[0], (size_t)n * 4)) != cudaSuccess ||
        (e = cudaMalloc((void**)&b.order[1], (size_t)n * 4)) != cudaSuccess ||
        (e = cudaMalloc((void**)&b.mark, (size_t)n * 4)) != cudaSuccess ||
        (e = cudaMalloc((void**)&b.seq, (size_t)n * 4)) != cudaSuccess ||
        (e = cudaMalloc((void**)&b.block_sums, nb * 4)) != cudaSuccess ||
        (e = cudaMalloc((void**)&b.counters, 4 * 4)) != cudaSuccess)
        return e;
    b.n = n;
    b.cur = 0;
    if ((e = cudaMemsetAsync(b.mark, 0, (size_t)n * 4, s)) != cudaSuccess) return e;
    if ((e = cudaMemsetAsync(b.counters, 0, 16, s)) != cudaSuccess) return e;
    // both buffers start as valid slot lists, so no stale entry is ever out of range
    const unsigned grid = (unsigned)std::min<size_t>((n + 255u) / 256u, 4096u);
    iota_kernel<<<grid, 256, 0, s>>>(b.order[0], n);
    iota_kernel<<<grid, 256, 0, s>>>(b.order[1], n);
    return cudaGetLastError();
}

void slot_order_free(SlotOrderBuffers& b) {
    void* bufs[] = {b.order[0], b.order[1], b.mark, b.seq, b.block_sums, b.counters, b.cand, b.cand_sums};
    for (void* p : bufs)
        if (p) cudaFree(p);
    b = SlotOrderBuffers{};
}

cudaError_t launch_classify_split(const DedupeBuffers& dd, uint32_t max_n, const uint2* nodes, const int dim[3],
                                  const int slots[3], uint32_t root_slot, uint32_t epoch, SlotOrderBuffers& b,
                                  int* status, cudaStream_t s) {
    if (max_n == 0) return cudaMemsetAsync(b.counters + 1, 0, 8, s);
    const size_t nb = (max_n + 1023u) / 1024u;
    if (nb > dd.block_cap || nb > b.cand_sums_cap || max_n > dd.unique_cap || max_n > b.cand_cap)
        return cudaErrorInvalidValue;
    classify_count_kernel<<<(unsigned)nb, 1024, 0, s>>>(dd.unique, dd.count, max_n, nodes, dim[0], dim[1], slots[0],
                                                         slots[1], root_slot, dd.block_sums, b.cand_sums);
    scan_sums2_kernel<<<2, 1024, 0, s>>>(dd.block_sums, b.cand_sums, (int)nb, b.counters + 1, b.counters + 2);
    split_scatter_kernel<<<(unsigned)nb, 1024, 0, s>>>(dd.unique, dd.count, max_n, root_slot, dd.block_sums,
                                                        b.cand_sums, b.n, epoch, b.seq, b.mark, b.cand, status);
    return cudaGetLastError();
}

cudaError_t launch_service_readout(const SlotOrderBuffers& b, uint32_t* h_counters, uint32_t* h_cand,
                                   uint32_t cand_cap, uint32_t* h_win, cudaStream_t s) {
    service_readout_kernel<<<64, 256, 0, s>>>(b.counters, b.cand, b.order[b.cur], b.n, h_counters, h_cand, cand_cap,
                                              h_win);
    return cudaGetLastError();
}

cudaError_t launch_pull(const uint4* src_a, uint4* dst_a, size_t n_a, const uint4* src_b, uint4* dst_b, size_t n_b,
                        cudaStream_t s) {
    const size_t n = n_a + n_b;
    if (n == 0) return cudaSuccess;
    // every read in flight at once: one 16-byte word per thread up to 148 x 8 CTAs
    const unsigned grid = (unsigned)std::min<size_t>((n + 255) / 256, 1184);
    pull_kernel<<<grid, 256, 0, s>>>(src_a, dst_a, n_a, src_b, dst_b, n_b);
    return cudaGetLastError();
}

cudaError_t launch_pull_staged(const uint32_t* h_counts, const uint4* h_jobs, uint32_t max_jobs,
                               const void* h_patches, uint32_t max_patches, uint32_t* d_counts, uint4* d_jobs,
                               void* d_patches, cudaStream_t s) {
    pull_staged_kernel<<<64, 256, 0, s>>>(h_counts, h_jobs, max_jobs, (const uint4*)h_patches, max_patches, d_counts,
                                          d_jobs, (uint4*)d_patches);
    return cudaGetLastError();
}

cudaError_t launch_read_word(const uint32_t* src, uint32_t* h_dst, cudaStream_t s) {
    read_word_kernel<<<1, 1, 0, s>>>(src, h_dst);
    return cudaGetLastError();
}

cudaError_t launch_mark_touched(SlotOrderBuffers& b, uint32_t m, uint32_t epoch, int* status, cudaStream_t s) {
    if (m == 0) return cudaSuccess;
    if (m > b.n) return cudaErrorInvalidValue;
    mark_touched_kernel<<<(unsigned)std::min<uint32_t>((m + 255u) / 256u, 2048u), 256, 0, s>>>(b.seq, m, b.n, epoch,
                                                                                             b.mark, status);
    return cudaGetLastError();
}

cudaError_t launch_order_partition(SlotOrderBuffers& b, uint32_t head, uint32_t epoch, bool seq_on_device,
                                   uint32_t m_host, uint32_t max_m, uint32_t root_slot, int* status,
                                   cudaStream_t s) {
    if (b.n == 0 || head >= b.n) return cudaErrorInvalidValue;
    const uint32_t nb = (b.n + 1023u) / 1024u;
    const uint32_t bound = std::min<uint32_t>((seq_on_device ? max_m : m_host) + 1u, b.n);
    const uint32_t append_blocks = std::max<uint32_t>(1u, std::min<uint32_t>((bound + 1023u) / 1024u, 148u));
    order_count_kernel<<<nb, 1024, 0, s>>>(b.order[b.cur], b.n, head, b.mark, epoch, b.block_sums);
    scan_sums_kernel<<<1, 1024, 0, s>>>(b.block_sums, (int)nb, b.counters + 3);
    order_scatter_kernel<<<nb + append_blocks, 1024, 0, s>>>(b.order[b.cur], b.n, head, b.mark, epoch, b.block_sums,
                                                             nb, b.counters, seq_on_device, m_host, root_slot, b.seq,
                                                             b.order[b.cur ^ 1], status);
    const cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) b.cur ^= 1;
    return e;
}

cudaError_t launch_produce_bricks(const DeviceTerrainView& t, const uint4* jobs, int n, void* pool, int fmt,
                                  uint32_t* masks, long long total_slots, int* status, cudaStream_t s) {
    if (n <= 0) return cudaSuccess;
    switch (fmt) {
        case VV_FMT_RGBA8: produce_kernel<VV_FMT_RGBA8><<<n, 256, 0, s>>>(t, jobs, pool, masks, total_slots, status); break;
        case VV_FMT_FP16: produce_kernel<VV_FMT_FP16><<<n, 256, 0, s>>>(t, jobs, pool, masks, total_slots, status); break;
        case VV_FMT_BF16: produce_kernel<VV_FMT_BF16><<<n, 256, 0, s>>>(t, jobs, pool, masks, total_slots, status); break;
        case VV_FMT_FP32: produce_kernel<VV_FMT_FP32><<<n, 256, 0, s>>>(t, jobs, pool, masks, total_slots, status); break;
        case VV_FMT_DXT5: produce_kernel<VV_FMT_DXT5><<<n, 256, 0, s>>>(t, jobs, pool, masks, total_slots, status); break;
        default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

cudaError_t launch_produce_staged(const DeviceTerrainView& t, const uint4* jobs, const uint32_t* count,
                                  uint32_t max_jobs, void* pool, int fmt, uint32_t* masks, long long total_slots,
                                  int* status, cudaStream_t s) {
    if (max_jobs == 0) return cudaSuccess;
    int dev = 0, sms = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const unsigned grid = (unsigned)std::min<long long>((long long)max_jobs, (long long)std::max(sms, 1) * 8);
    switch (fmt) {
        case VV_FMT_RGBA8:
            produce_staged_kernel<VV_FMT_RGBA8><<<grid, 256, 0, s>>>(t, jobs, count, max_jobs, pool, masks, total_slots, status);
            break;
        case VV_FMT_FP16:
            produce_staged_kernel<VV_FMT_FP16><<<grid, 256, 0, s>>>(t, jobs, count, max_jobs, pool, masks, total_slots, status);
            break;
        case VV_FMT_BF16:
            produce_staged_kernel<VV_FMT_BF16><<<grid, 256, 0, s>>>(t, jobs, count, max_jobs, pool, masks, total_slots, status);
            break;
        case VV_FMT_FP32:
            produce_staged_kernel<VV_FMT_FP32><<<grid, 256, 0, s>>>(t, jobs, count, max_jobs, pool, masks, total_slots, status);
            break;
        case VV_FMT_DXT5:
            produce_staged_kernel<VV_FMT_DXT5><<<grid, 256, 0, s>>>(t, jobs, count, max_jobs, pool, masks, total_slots, status);
            break;
        default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

DeviceBrickStore::~DeviceBrickStore() {
    if (d_) cudaFree(d_);
}

cudaError_t DeviceBrickStore::upload(const uint32_t* texels, size_t bricks) {
    if (d_) cudaFree(d_);
    d_ = nullptr;
    bricks_ = 0;
    if (bricks > 0xFFFFFFFFull) return cudaErrorInvalidValue;
    const size_t bytes = std::max<size_t>(bricks, 1) * VV_BRICK_TEXELS * sizeof(uint32_t);
    cudaError_t e = cudaMalloc((void**)&d_, bytes);
    if (e != cudaSuccess) {
        d_ = nullptr;
        return e;
    }
    bricks_ = bricks;
    if (bricks) e = cudaMemcpy(d_, texels, bricks * VV_BRICK_TEXELS * sizeof(uint32_t), cudaMemcpyHostToDevice);
    return e;
}

cudaError_t launch_copy_bricks(const DeviceBrickStoreView& st, const uint4* jobs, int n, void* pool, int fmt,
                               uint32_t* masks, long long total_slots, int* status, cudaStream_t s) {
    if (n <= 0) return cudaSuccess;
    switch (fmt) {
        case VV_FMT_RGBA8: copy_kernel<VV_FMT_RGBA8><<<n, 256, 0, s>>>(st, jobs, pool, masks, total_slots, status); break;
        case VV_FMT_FP16: copy_kernel<VV_FMT_FP16><<<n, 256, 0, s>>>(st, jobs, pool, masks, total_slots, status); break;
        case VV_FMT_BF16: copy_kernel<VV_FMT_BF16><<<n, 256, 0, s>>>(st, jobs, pool, masks, total_slots, status); break;
        case VV_FMT_FP32: copy_kernel<VV_FMT_FP32><<<n, 256, 0, s>>>(st, jobs, pool, masks, total_slots, status); break;
        case VV_FMT_DXT5: copy_kernel<VV_FMT_DXT5><<<n, 256, 0, s>>>(st, jobs, pool, masks, total_slots, status); break;
        default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

cudaError_t launch_copy_staged(const DeviceBrickStoreView& st, const uint4* jobs, const uint32_t* count,
                               uint32_t max_jobs, void* pool, int fmt, uint32_t* masks, long long total_slots,
                               int* status, cudaStream_t s) {
    if (max_jobs == 0) return cudaSuccess;
    int dev = 0, sms = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const unsigned grid = (unsigned)std::min<long long>((long long)max_jobs, (long long)std::max(sms, 1) * 8);
    switch (fmt) {
        case VV_FMT_RGBA8:
            copy_staged_kernel<VV_FMT_RGBA8><<<grid, 256, 0, s>>>(st, jobs, count, max_jobs, pool, masks, total_slots, status);
            break;
        case VV_FMT_FP16:
            copy_staged_kernel<VV_FMT_FP16><<<grid, 256, 0, s>>>(st, jobs, count, max_jobs, pool, masks, total_slots, status);
            break;
        case VV_FMT_BF16:
            copy_staged_kernel<VV_FMT_BF16><<<grid, 256, 0, s>>>(st, jobs, count, max_jobs, pool, masks, total_slots, status);
            break;
        case VV_FMT_FP32:
            copy_staged_kernel<VV_FMT_FP32><<<grid, 256, 0, s>>>(st, jobs, count, max_jobs, pool, masks, total_slots, status);
            break;
        case VV_FMT_DXT5:
            copy_staged_kernel<VV_FMT_DXT5><<<grid, 256, 0, s>>>(st, jobs, count, max_jobs, pool, masks, total_slots, status);
            break;
        default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

cudaError_t launch_dedupe(const uint32_t* requests, int n_entries, const int grid_dim[3], const DedupeBuffers& b,
                          cudaStream_t s) {
    const int n = 4 * n_entries;
    if (n <= 0) return cudaMemsetAsync(b.count, 0, sizeof(uint32_t), s);
    const int nb = (n + 1023) / 1024;
    if ((size_t)nb > b.block_cap || (size_t)n > b.unique_cap) return cudaErrorInvalidValue;
    dedupe_first_kernel<<<(n + 255) / 256, 256, 0, s>>>(requests, n, grid_dim[0], grid_dim[1], grid_dim[2], b.first);
    dedupe_count_kernel<<<nb, 1024, 0, s>>>(requests, n, grid_dim[0], grid_dim[1], grid_dim[2], b.first,
                                            b.block_sums);
    scan_sums_kernel<<<1, 1024, 0, s>>>(b.block_sums, nb, b.count);
    dedupe_scatter_kernel<<<nb, 1024, 0, s>>>(requests, n, grid_dim[0], grid_dim[1], grid_dim[2], b.first,
                                              b.block_sums, b.unique);
    return cudaGetLastError();
}

}  // namespace vv
