// kernels.cu - sm_100a kernels of the GigaVoxels hot path.
//
// raycast_kernel      GigaVoxelsNoLighting.frag main (:490-751) per pixel
// select_kernel       GenerateSelectionMask.frag + ComputeActiveTexels.frag
// pyramid_up_kernel   GenerateHistoPyramid.frag (one launch per level)
// pyramid_down_kernel the key walk of CompressNodeUsageList.frag (:55-105),
//                     run top-down as exclusive offsets instead of per key
// compact_kernel      CompressNodeUsageList.frag (:107-149), scattered by rank
//
// Floating point: this file is compiled with -fmad=false -prec-div=true
// -prec-sqrt=true and without fast-math, so every +,-,*,/ and sqrt below is
// one IEEE binary32 operation in the written order.  The only fused
// operation is the explicit fmaf() of lerp().  The host oracle performs the
// same sequence, which makes descent decisions, step counts, LOD choices and
// node-usage lists bit-identical.
#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include <algorithm>

#include "raycast_common.cuh"
#include "select.cuh"

namespace vv {

using namespace rc;

// LIT: GigaVoxels.frag with ComputeLighting (gradient pool in p.grads).
// 7 resident CTAs (28 warps) per SM: at most 72 registers per thread.  The
// walk is bound by dependency latency, and more warps hide more of it:
// 1080p paged frames measured 3.74 ms uncapped (82 registers, 5 CTAs),
// 3.56 ms at 6 CTAs, 3.43 ms at 7 (a few bytes spilled), 3.48 ms at 8.
template <int FMT, bool COUNT, bool LIT>
__global__ void __launch_bounds__(128, 7) raycast_kernel(const __grid_constant__ RaycastParams p) {
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int px = blockIdx.x * 16 + (warp & 1) * 8 + (lane & 7);
    const int py = blockIdx.y * 8 + (warp >> 1) * 4 + (lane >> 3);
    if (px >= p.u.width || py >= p.u.height) return;
    __shared__ uint2 path_w[kPathLevels][128];
    __shared__ uint32_t path_p[kPathLevels][128];
    render_pixel<FMT, COUNT, 1, !COUNT, LIT>(p, px, py,
                                             PathSlots{&path_w[0][threadIdx.x], &path_p[0][threadIdx.x], 128, nullptr});
}

// The brick-staging form (RGBA8 pools): the pixels and walk of raycast_kernel,
// each warp with one slot copy in shared memory (StageBuf).  33 KB of shared
// memory per CTA allow 6 resident CTAs, hence the register cap of 6.
__global__ void __launch_bounds__(128, 6) raycast_staged_kernel(const __grid_constant__ RaycastParams p) {
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    __shared__ StageBuf stage[4];
    if (lane == 0) stage_init(&stage[warp]);
    __syncwarp();
    const int px = blockIdx.x * 16 + (warp & 1) * 8 + (lane & 7);
    const int py = blockIdx.y * 8 + (warp >> 1) * 4 + (lane >> 3);
    if (px >= p.u.width || py >= p.u.height) return;
    __shared__ uint2 path_w[kPathLevels][128];
    __shared__ uint32_t path_p[kPathLevels][128];
    render_pixel<VV_FMT_RGBA8, false, 1, true, false, true>(
        p, px, py, PathSlots{&path_w[0][threadIdx.x], &path_p[0][threadIdx.x], 128, &stage[warp]});
}

cudaError_t launch_raycast_staged(int fmt, const RaycastParams& p, cudaStream_t s) {
    if (fmt != VV_FMT_RGBA8) return cudaErrorInvalidValue;
    dim3 block(128);
    dim3 grid((unsigned)((p.u.width + 15) / 16), (unsigned)((p.u.height + 7) / 8));
    raycast_staged_kernel<<<grid, block, 0, s>>>(p);
    return cudaGetLastError();
}

// The lane-refill form (render_refill): a persistent grid of as many CTAs
// as are resident at once, pixels handed out in 8x4 tiles from `counter`
// (zeroed before the launch).
template <int FMT>
__global__ void __launch_bounds__(128, 7) raycast_refill_kernel(const __grid_constant__ RaycastParams p,
                                                                unsigned int* counter) {
    __shared__ uint2 path_w[kPathLevels][128];
    __shared__ uint32_t path_p[kPathLevels][128];
    render_refill<FMT>(p, counter, PathSlots{&path_w[0][threadIdx.x], &path_p[0][threadIdx.x], 128, nullptr});
}

cudaError_t launch_raycast_refill(int fmt, const RaycastParams& p, unsigned int* counter, cudaStream_t s) {
    static int ctas[5] = {0, 0, 0, 0, 0};  // resident CTAs on the device (per format)
    if (fmt < 0 || fmt > VV_FMT_DXT5) return cudaErrorInvalidValue;
    cudaError_t e = cudaSuccess;
    if (!ctas[fmt]) {
        int dev = 0, sms = 0, per_sm = 0;
        e = cudaGetDevice(&dev);
        if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        if (e == cudaSuccess) {
            switch (fmt) {
                case VV_FMT_RGBA8:
                    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, raycast_refill_kernel<VV_FMT_RGBA8>, 128, 0);
                    break;
                case VV_FMT_FP16:
                    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, raycast_refill_kernel<VV_FMT_FP16>, 128, 0);
                    break;
                case VV_FMT_BF16:
                    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, raycast_refill_kernel<VV_FMT_BF16>, 128, 0);
                    break;
                case VV_FMT_DXT5:
                    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, raycast_refill_kernel<VV_FMT_DXT5>, 128, 0);
                    break;
                default:
                    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, raycast_refill_kernel<VV_FMT_FP32>, 128, 0);
                    break;
            }
        }
        if (e != cudaSuccess) return e;
        ctas[fmt] = std::max(1, sms * per_sm);
    }
    e = cudaMemsetAsync(counter, 0, sizeof(unsigned int), s);
    if (e != cudaSuccess) return e;
    dim3 block(128), grid((unsigned)ctas[fmt]);
    switch (fmt) {
        case VV_FMT_RGBA8: raycast_refill_kernel<VV_FMT_RGBA8><<<grid, block, 0, s>>>(p, counter); break;
        case VV_FMT_FP16: raycast_refill_kernel<VV_FMT_FP16><<<grid, block, 0, s>>>(p, counter); break;
        case VV_FMT_BF16: raycast_refill_kernel<VV_FMT_BF16><<<grid, block, 0, s>>>(p, counter); break;
        case VV_FMT_DXT5: raycast_refill_kernel<VV_FMT_DXT5><<<grid, block, 0, s>>>(p, counter); break;
        default: raycast_refill_kernel<VV_FMT_FP32><<<grid, block, 0, s>>>(p, counter); break;
    }
    return cudaGetLastError();
}

cudaError_t launch_raycast(int fmt, const RaycastParams& p, cudaStream_t s) {
    dim3 block(128);
    dim3 grid((unsigned)((p.u.width + 15) / 16), (unsigned)((p.u.height + 7) / 8));
    const bool count = p.node_touch && p.brick_touch;
    const bool lit = p.u.compute_lighting && p.grads && !count;
#define VV_LAUNCH(F)                                                           \
    if (count) raycast_kernel<F, true, false><<<grid, block, 0, s>>>(p);       \
    else if (lit) raycast_kernel<F, false, true><<<grid, block, 0, s>>>(p);    \
    else raycast_kernel<F, false, false><<<grid, block, 0, s>>>(p);
    switch (fmt) {
        case VV_FMT_RGBA8: VV_LAUNCH(VV_FMT_RGBA8) break;
        case VV_FMT_FP16: VV_LAUNCH(VV_FMT_FP16) break;
        case VV_FMT_BF16: VV_LAUNCH(VV_FMT_BF16) break;
        case VV_FMT_FP32: VV_LAUNCH(VV_FMT_FP32) break;
        case VV_FMT_DXT5: VV_LAUNCH(VV_FMT_DXT5) break;
        default: return cudaErrorInvalidValue;
    }
#undef VV_LAUNCH
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// GenerateSelectionMask.frag (:15-187) + ComputeActiveTexels.frag (:9-25)

__global__ void select_kernel(const uint4* __restrict__ usage, uint32_t* __restrict__ mask,
                              uint32_t* __restrict__ level0, int w, int h) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= w || y >= h) return;
    const size_t pix = (size_t)y * w + x;
    const uint32_t bits = select_bits(usage, x, y, w, h);
    if (mask) mask[pix] = bits;
    level0[pix] = bits != 0u ? 1u : 0u;
}

cudaError_t launch_select(const uint4* usage, uint32_t* mask, uint32_t* level0, int w, int h,
                          cudaStream_t s) {
    dim3 block(32, 4);
    dim3 grid((unsigned)((w + 31) / 32), (unsigned)((h + 3) / 4));
    select_kernel<<<grid, block, 0, s>>>(usage, mask, level0, w, h);
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Histopyramid.  Children of parent (X,Y) at the finer level (w,h), in the
// order CompressNodeUsageList walks them: the 2x2 block, then for an odd last
// row (x,y+2),(x+1,y+2) and for an odd last column the (x+2,*) cells.

__device__ __forceinline__ int child_list(int X, int Y, int w, int h, int* cx, int* cy) {
    const int x = 2 * X, y = 2 * Y;
    int n = 0;
    cx[n] = x; cy[n++] = y;
    cx[n] = x + 1; cy[n++] = y;
    cx[n] = x; cy[n++] = y + 1;
    cx[n] = x + 1; cy[n++] = y + 1;
    if (y + 2 == h - 1) {
        cx[n] = x; cy[n++] = y + 2;
        cx[n] = x + 1; cy[n++] = y + 2;
        if (x + 2 == w - 1) {
            cx[n] = x + 2; cy[n++] = y + 2;
            cx[n] = x + 2; cy[n++] = y + 1;
            cx[n] = x + 2; cy[n++] = y;
        }
    } else if (x + 2 == w - 1) {
        cx[n] = x + 2; cy[n++] = y + 1;
        cx[n] = x + 2; cy[n++] = y;
    }
    return n;
}

__device__ __forceinline__ uint32_t cell(const uint32_t* lvl, int x, int y, int w, int h) {
    return (x < w && y < h) ? lvl[(size_t)y * w + x] : 0u;
}

__global__ void pyramid_up_kernel(const uint32_t* __restrict__ fine, uint32_t* __restrict__ coarse, int w,
                                  int h, int cw, int ch) {
    const int X = blockIdx.x * blockDim.x + threadIdx.x;
    const int Y = blockIdx.y * blockDim.y + threadIdx.y;
    if (X >= cw || Y >= ch) return;
    int cx[9], cy[9];
    const int n = child_list(X, Y, w, h, cx, cy);
    uint32_t sum = 0u;
    for (int i = 0; i < n; ++i) sum += cell(fine, cx[i], cy[i], w, h);
    coarse[(size_t)Y * cw + X] = sum;
}

// Offsets at the finer level from the coarser level's offsets: each child
// finds its parent and adds the counts of the siblings walked before it.
__global__ void pyramid_down_kernel(const uint32_t* __restrict__ fine_cnt, uint32_t* __restrict__ fine_off,
                                    const uint32_t* __restrict__ coarse_off, int w, int h, int cw, int ch) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= w || y >= h) return;
    const int X = min(x >> 1, cw - 1), Y = min(y >> 1, ch - 1);
    int cx[9], cy[9];
    const int n = child_list(X, Y, w, h, cx, cy);
    uint32_t off = coarse_off[(size_t)Y * cw + X];
    for (int i = 0; i < n; ++i) {
        if (cx[i] == x && cy[i] == y) break;
        off += cell(fine_cnt, cx[i], cy[i], w, h);
    }
    fine_off[(size_t)y * w + x] = off;
}

__global__ void compact_kernel(const __grid_constant__ CompactParams p) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= p.width || y >= p.height) return;
    const size_t pix = (size_t)y * p.width + x;
    uint32_t bits = p.mask[pix];
    if (bits == 0u) return;
    const uint32_t rank = p.offsets[pix];
    if (rank >= (uint32_t)p.cap) return;
    const uint4* o = p.usage + pix * 3;
    uint4 a = o[0], b = o[1], c = o[2];
    const uint32_t list[12] = {a.x, a.y, a.z, a.w, b.x, b.y, b.z, b.w, c.x, c.y, c.z, c.w};
    uint32_t out[4] = {0u, 0u, 0u, 0u};
    int pushed = 0;
    for (int item = 0; item < 12 && bits != 0u && pushed < p.max_push; ++item, bits >>= 1) {
        if (bits & 1u) {
            out[pushed & 3] = list[item];
            ++pushed;
        }
    }
    reinterpret_cast<uint4*>(p.requests)[rank] = make_uint4(out[0], out[1], out[2], out[3]);
}

__global__ void copy_total_kernel(const uint32_t* top, uint32_t* dst) {
    if (threadIdx.x == 0 && blockIdx.x == 0) *dst = *top;
}

cudaError_t launch_pyramid_levels(uint32_t* counts, uint32_t* offsets, const int* lw, const int* lh,
                                  const long long* loff, int first, int levels, cudaStream_t s) {
    dim3 block(32, 4);
    for (int l = first; l + 1 < levels; ++l) {
        const int cw = lw[l + 1], ch = lh[l + 1];
        dim3 grid((unsigned)((cw + 31) / 32), (unsigned)((ch + 3) / 4));
        pyramid_up_kernel<<<grid, block, 0, s>>>(counts + loff[l], counts + loff[l + 1], lw[l], lh[l], cw, ch);
    }
    cudaError_t e = cudaMemsetAsync(offsets + loff[levels - 1], 0, sizeof(uint32_t), s);
    if (e != cudaSuccess) return e;
    for (int l = levels - 2; l >= first; --l) {
        dim3 grid((unsigned)((lw[l] + 31) / 32), (unsigned)((lh[l] + 3) / 4));
        pyramid_down_kernel<<<grid, block, 0, s>>>(counts + loff[l], offsets + loff[l], offsets + loff[l + 1], lw[l],
                                                   lh[l], lw[l + 1], lh[l + 1]);
    }
    return cudaGetLastError();
}

cudaError_t launch_compact(const CompactParams& p, cudaStream_t s) {
    dim3 block(32, 4);
    for (int l = 0; l + 1 < p.levels; ++l) {
        const int cw = p.level_w[l + 1], ch = p.level_h[l + 1];
        dim3 grid((unsigned)((cw + 31) / 32), (unsigned)((ch + 3) / 4));
        pyramid_up_kernel<<<grid, block, 0, s>>>(p.counts + p.level_off[l], p.counts + p.level_off[l + 1],
                                                 p.level_w[l], p.level_h[l], cw, ch);
    }
    const int top = p.levels - 1;
    cudaMemsetAsync(p.offsets + p.level_off[top], 0, sizeof(uint32_t), s);
    for (int l = top - 1; l >= 0; --l) {
        const int w = p.level_w[l], h = p.level_h[l];
        dim3 grid((unsigned)((w + 31) / 32), (unsigned)((h + 3) / 4));
        pyramid_down_kernel<<<grid, block, 0, s>>>(p.counts + p.level_off[l], p.offsets + p.level_off[l],
                                                   p.offsets + p.level_off[l + 1], w, h, p.level_w[l + 1],
                                                   p.level_h[l + 1]);
    }
    if (p.request_count) copy_total_kernel<<<1, 32, 0, s>>>(p.counts + p.level_off[top], p.request_count);
    if (p.requests && p.cap > 0) {
        dim3 grid((unsigned)((p.width + 31) / 32), (unsigned)((p.height + 3) / 4));
        compact_kernel<<<grid, block, 0, s>>>(p);
    }
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Node pool: reference texture order <-> block-linear device layout.

__device__ __forceinline__ size_t block_linear(uint32_t x, uint32_t y, uint32_t z, int dx, int dy) {
    const uint32_t bx = (uint32_t)dx >> 1, by = (uint32_t)dy >> 1;
    size_t blk = ((size_t)(z >> 1) * by + (y >> 1)) * bx + (x >> 1);
    return blk * 8u + ((x & 1u) | ((y & 1u) << 1) | ((z & 1u) << 2));
}

__global__ void node_upload_kernel(const uint2* __restrict__ grid, uint2* __restrict__ nodes, int dx, int dy,
                                   int dz) {
    const size_t total = (size_t)dx * dy * dz;
    for (size_t g = blockIdx.x * (size_t)blockDim.x + threadIdx.x; g < total; g += (size_t)gridDim.x * blockDim.x) {
        uint32_t x = (uint32_t)(g % dx), y = (uint32_t)((g / dx) % dy), z = (uint32_t)(g / ((size_t)dx * dy));
        nodes[block_linear(x, y, z, dx, dy)] = grid[g];
    }
}

__global__ void node_download_kernel(const uint2* __restrict__ nodes, uint2* __restrict__ grid, int dx, int dy,
                                     int dz) {
    const size_t total = (size_t)dx * dy * dz;
    for (size_t g = blockIdx.x * (size_t)blockDim.x + threadIdx.x; g < total; g += (size_t)gridDim.x * blockDim.x) {
        uint32_t x = (uint32_t)(g % dx), y = (uint32_t)((g / dx) % dy), z = (uint32_t)(g / ((size_t)dx * dy));
        grid[g] = nodes[block_linear(x, y, z, dx, dy)];
    }
}

__global__ void node_patch_kernel(const vv_node_patch* __restrict__ patches, int n, uint2* __restrict__ nodes,
                                  int dx, int dy, int dz, int* status) {
    // The host hands over at most one patch per node (the last one it made),
    // so the parallel writes are order-independent.
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const vv_node_patch q = patches[i];
    if (q.x >= (uint32_t)dx || q.y >= (uint32_t)dy || q.z >= (uint32_t)dz) {
        set_status(status, VV_ERR_BOUNDS);
        return;
    }
    nodes[block_linear(q.x, q.y, q.z, dx, dy)] = make_uint2(q.word0, q.word1);
}

__global__ void node_patch_staged_kernel(const vv_node_patch* patches, const volatile uint32_t* count,
                                         uint32_t max_patches, uint2* __restrict__ nodes, int dx, int dy, int dz,
                                         int* status) {
    __shared__ uint32_t s_n;  // one read of the count per CTA
    if (threadIdx.x == 0) s_n = min(*count, max_patches);
    __syncthreads();
    const uint32_t n = s_n;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const vv_node_patch q = patches[i];
        if (q.x >= (uint32_t)dx || q.y >= (uint32_t)dy || q.z >= (uint32_t)dz) {
            set_status(status, VV_ERR_BOUNDS);
            continue;
        }
        nodes[block_linear(q.x, q.y, q.z, dx, dy)] = make_uint2(q.word0, q.word1);
    }
}

cudaError_t launch_node_patch_staged(const vv_node_patch* patches, const uint32_t* count, uint32_t max_patches,
                                     uint2* nodes, const int dim[3], int* status, cudaStream_t s) {
    if (max_patches == 0) return cudaSuccess;
    const unsigned grid = (unsigned)std::min<uint32_t>((max_patches + 255) / 256, 1184u);
    node_patch_staged_kernel<<<grid, 256, 0, s>>>(patches, count, max_patches, nodes, dim[0], dim[1], dim[2],
                                                  status);
    return cudaGetLastError();
}

cudaError_t launch_node_upload(const uint32_t* grid_words, uint2* nodes, const int dim[3], cudaStream_t s) {
    node_upload_kernel<<<592, 256, 0, s>>>((const uint2*)grid_words, nodes, dim[0], dim[1], dim[2]);
    return cudaGetLastError();
}

cudaError_t launch_node_download(const uint2* nodes, uint32_t* grid_words, const int dim[3], cudaStream_t s) {
    node_download_kernel<<<592, 256, 0, s>>>(nodes, (uint2*)grid_words, dim[0], dim[1], dim[2]);
    return cudaGetLastError();
}

cudaError_t launch_node_patch(const vv_node_patch* patches, int n, uint2* nodes, const int dim[3], int* status,
                              cudaStream_t s) {
    if (n <= 0) return cudaSuccess;
    node_patch_kernel<<<(n + 255) / 256, 256, 0, s>>>(patches, n, nodes, dim[0], dim[1], dim[2], status);
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Brick upload: scatter n staged bricks into their pool slots, 16-byte
// vectors, one CTA per brick.

__global__ void brick_scatter_kernel(const uint32_t* __restrict__ slots, const uint4* __restrict__ src,
                                     uint4* __restrict__ pool, int vec_per_brick, long long total_slots,
                                     int* status) {
    const int b = blockIdx.x;
    const uint32_t slot = slots[b];
    if ((long long)slot >= total_slots) {
        if (threadIdx.x == 0) set_status(status, VV_ERR_BOUNDS);
        return;
    }
    const uint4* s = src + (size_t)b * vec_per_brick;
    uint4* d = pool + (size_t)slot * vec_per_brick;
    for (int i = threadIdx.x; i < vec_per_brick; i += blockDim.x) d[i] = __ldg(s + i);
}

template <int FMT>
__global__ void cell_mask_kernel(const uint32_t* __restrict__ slots, const void* __restrict__ pool,
                                 long long total_slots, uint32_t* __restrict__ masks) {
    __shared__ uint8_t zero[VV_BRICK_TEXELS];
    const long long slot = slots ? (long long)slots[blockIdx.x] : (long long)blockIdx.x;
    if (slot >= total_slots) return;  // whole CTA (a bad slot was reported by the upload)
    for (int q = threadIdx.x; q < VV_BRICK_TEXELS; q += blockDim.x)
        zero[q] = texel_is_zero<FMT>(pool, (size_t)slot * VV_BRICK_TEXELS + q) ? 1 : 0;
    __syncthreads();
    write_cell_mask(zero, masks + (size_t)slot * kCellMaskWords);
}

cudaError_t launch_cell_masks(const uint32_t* slots, long long n, const void* pool, int fmt, long long total_slots,
                              uint32_t* masks, cudaStream_t s) {
    if (n <= 0) return cudaSuccess;
    if (n > 0x7FFFFFFFLL) return cudaErrorInvalidValue;
    const unsigned grid = (unsigned)n;
    switch (fmt) {
        case VV_FMT_RGBA8: cell_mask_kernel<VV_FMT_RGBA8><<<grid, 256, 0, s>>>(slots, pool, total_slots, masks); break;
        case VV_FMT_FP16: cell_mask_kernel<VV_FMT_FP16><<<grid, 256, 0, s>>>(slots, pool, total_slots, masks); break;
        case VV_FMT_BF16: cell_mask_kernel<VV_FMT_BF16><<<grid, 256, 0, s>>>(slots, pool, total_slots, masks); break;
        case VV_FMT_FP32: cell_mask_kernel<VV_FMT_FP32><<<grid, 256, 0, s>>>(slots, pool, total_slots, masks); break;
        case VV_FMT_DXT5: cell_mask_kernel<VV_FMT_DXT5><<<grid, 256, 0, s>>>(slots, pool, total_slots, masks); break;
        default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

// One pixel per thread; 48 bytes moved per pixel (HBM-bound).  Separate
// rounded products and sum (no contraction), the order the formula reads.
__global__ void blend_over_kernel(float4* __restrict__ dst, const float4* __restrict__ src, size_t n) {
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float4 s = src[i];
    float4 d = dst[i];
    const float a = s.w, ia = __fsub_rn(1.0f, s.w);
    d.x = __fadd_rn(__fmul_rn(s.x, a), __fmul_rn(d.x, ia));
    d.y = __fadd_rn(__fmul_rn(s.y, a), __fmul_rn(d.y, ia));
    d.z = __fadd_rn(__fmul_rn(s.z, a), __fmul_rn(d.z, ia));
    d.w = __fadd_rn(__fmul_rn(s.w, a), __fmul_rn(d.w, ia));
    dst[i] = d;
}

cudaError_t launch_blend_over(float4* dst, const float4* src, size_t n, cudaStream_t s) {
    if (n == 0) return cudaSuccess;
    const size_t blocks = (n + 255) / 256;
    if (blocks > 0x7FFFFFFFull) return cudaErrorInvalidValue;
    blend_over_kernel<<<(unsigned)blocks, 256, 0, s>>>(dst, src, n);
    return cudaGetLastError();
}

cudaError_t launch_brick_scatter(const uint32_t* slots, int n, const void* src, void* pool, size_t brick_bytes,
                                 long long total_slots, int* status, cudaStream_t s) {
    if (n <= 0) return cudaSuccess;
    brick_scatter_kernel<<<n, 256, 0, s>>>(slots, (const uint4*)src, (uint4*)pool, (int)(brick_bytes / 16),
                                           total_slots, status);
    return cudaGetLastError();
}

}  // namespace vv
