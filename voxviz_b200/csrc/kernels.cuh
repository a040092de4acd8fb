// kernels.cuh - device-side launch interfaces of the GigaVoxels hot path.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include <cmath>

#include "../../include/voxviz_b200.h"

namespace vv {

// Everything one ray-cast launch reads (kernel parameter, __grid_constant__).
struct RaycastParams {
    vv_uniforms u;
    const uint2* nodes;      // node pool, block-linear: 8 nodes of a 2x2x2 cell contiguous
    int node_dim[3];         // node-pool grid dims (even)
    const void* bricks;      // brick pool, slot-major brick-linear texels
    int slots[3];            // slots per axis
    const uint8_t* jitter;   // jitter_tex_size^2 bytes
    float4* color;           // [H*W] or nullptr
    uint4* usage;            // [H*W*3] (12 uint32 per pixel)
    int* status;             // sticky device status word
    const void* grads;       // gradient pool (lighting), same slots as bricks, or nullptr
    int grad_fmt;            // VV_FMT_FP32 or VV_FMT_RGBA8
    int max_iter;            // bound on outer-loop iterations per ray
    uint32_t* node_touch;    // footprint mode: bit per node (block-linear index)
    uint32_t* brick_touch;   // footprint mode: bit per brick-pool slot
    const uint32_t* cell_mask;  // empty-cell masks of the pool (cellmask.cuh), or nullptr
    // set_divisors: RN(1 / brick_pool_dimension) per axis (fixed_div.h), and
    // 1 / ray_step_size when that is a power of two (else 0: divide)
    float rpdim[3];
    float rstep;
    int color8;              // colour as RGBA8 unorm: color is read as uint32_t[H*W]
};

// The reciprocals of RaycastParams from its uniforms (host).
inline void set_divisors(RaycastParams& p) {
    for (int a = 0; a < 3; ++a) p.rpdim[a] = 1.0f / p.u.brick_pool_dimension[a];
    int e = 0;
    const float m = std::frexp(p.u.ray_step_size, &e);
    p.rstep = (m == 0.5f) ? 1.0f / p.u.ray_step_size : 0.0f;
}

// Pyramid/compaction launch state.
struct CompactParams {
    int width, height;
    int levels;                       // pyramid levels (level 0 = full res)
    int level_w[24], level_h[24];
    long long level_off[24];          // element offset of each level in counts/offsets
    uint32_t* counts;                 // pyramid counts (all levels)
    uint32_t* offsets;                // exclusive offsets (all levels)
    const uint4* usage;
    const uint32_t* mask;
    uint32_t* requests;               // [cap][4]
    uint32_t* request_count;
    int cap;
    int max_push;
};

cudaError_t launch_raycast(int fmt, const RaycastParams& p, cudaStream_t s);
// The persistent lane-refill ray cast (same results; plain unlit draws only).
cudaError_t launch_raycast_refill(int fmt, const RaycastParams& p, unsigned int* counter, cudaStream_t s);
cudaError_t launch_raycast_staged(int fmt, const RaycastParams& p, cudaStream_t s);
// Differentiable forward (colour + per-ray checkpoints) and its adjoint.
size_t ckpt_bytes(int w, int h, int per_ray);
cudaError_t launch_forward_ckpt(int fmt, const RaycastParams& p, void* ckpt, int per_ray, cudaStream_t s);
// Where the adjoint adds dL/d(texel): `grad` holds 4 floats (or, with f64,
// 4 doubles) per texel, 1000 texels per row; row = brick-pool slot (dense,
// slot_map NULL) or the row the slot map assigns (claimed on first touch
// from rows_used, at most rows_cap rows).  With copies > 1 (binary32 rows)
// warp w of CTA b adds to copy (w + 4 (b.x mod 2)) mod copies: copy 0 is
// `grad`, copy k > 0 starts at spread + (k - 1) * spread_rows * 1000
// (spread_rows = rows_cap, or the pool's slots for dense rows; all zero
// before the first launch; launch_spread_reduce adds the rows in use into
// `grad` and zeroes them).
struct GradTarget {
    void* grad;
    int f64;
    int warp_sum;  // sum the lanes that add to the same texel before the atomic
    int* slot_map;
    int* rows_used;
    int rows_cap;
    int copies;       // 1, 2, 4 or 8
    float4* spread;   // copies 1..copies-1
    int spread_rows;  // rows per copy
};
cudaError_t launch_backward(int fmt, const RaycastParams& p, const void* ckpt, int per_ray, const float4* dl_dcolor,
                            const GradTarget& grad, cudaStream_t s);
cudaError_t launch_spread_reduce(const GradTarget& grad, cudaStream_t s);
cudaError_t launch_select(const uint4* usage, uint32_t* mask, uint32_t* level0, int w, int h,
                          cudaStream_t s);
cudaError_t launch_compact(const CompactParams& p, cudaStream_t s);
// Histopyramid up-sweep from level `first` to the top and down-sweep of the
// exclusive offsets back to level `first` (level arrays at counts/offsets +
// loff[l], dims lw[l] x lh[l]).
cudaError_t launch_pyramid_levels(uint32_t* counts, uint32_t* offsets, const int* lw, const int* lh,
                                  const long long* loff, int first, int levels, cudaStream_t s);
cudaError_t launch_node_upload(const uint32_t* grid_words, uint2* nodes, const int dim[3],
                               cudaStream_t s);
cudaError_t launch_node_download(const uint2* nodes, uint32_t* grid_words, const int dim[3],
                                 cudaStream_t s);
// Patches and their count read on the device (at most max_patches): a
// count-independent launch for CUDA graphs.  Device copies of both make it
// fast (mapped host memory costs a bus round trip per CTA).
cudaError_t launch_node_patch_staged(const vv_node_patch* patches, const uint32_t* count, uint32_t max_patches,
                                     uint2* nodes, const int dim[3], int* status, cudaStream_t s);
cudaError_t launch_node_patch(const vv_node_patch* patches, int n, uint2* nodes, const int dim[3],
                              int* status, cudaStream_t s);
cudaError_t launch_brick_scatter(const uint32_t* slots, int n, const void* src, void* pool,
                                 size_t brick_bytes, long long total_slots, int* status,
                                 cudaStream_t s);
// glBlendFunc(GL_SRC_ALPHA, GL_ONE_MINUS_SRC_ALPHA) of one tile's colour
// over the scene's, per channel in FP32: dst = src * src.a + dst * (1 - src.a).
cudaError_t launch_blend_over(float4* dst, const float4* src, size_t n, cudaStream_t s);
// Empty-cell masks (cellmask.cuh) of n slots (slots[i], or slot i when slots
// is null) from the pool's current contents: 32 words per slot.
cudaError_t launch_cell_masks(const uint32_t* slots, long long n, const void* pool, int fmt, long long total_slots,
                              uint32_t* masks, cudaStream_t s);

}  // namespace vv
