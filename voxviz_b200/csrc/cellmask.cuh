// cellmask.cuh - per brick-pool slot, one bit per 2x2x2 texel cell that is
// entirely zero.
//
// A trilinear sample whose eight taps lie in the slot is addressed by its
// first tap (x, y, z) in [0,8]^3; cell (x, y, z) is bit (z*9 + y)*9 + x of
// the slot's 32-word mask and is set when all eight texels have every
// channel's bit pattern zero.  Such a sample is exactly (0,0,0,0) whatever
// its weights, and compositing it leaves the destination unchanged, so the
// walk may take the zero without loading the texels.  729 cells in words
// 0..22; words 23..31 are zero (128 bytes per slot, one L1 line).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/voxviz_b200.h"
#include "dxt.h"

namespace vv {

constexpr int kCellMaskWords = 32;
constexpr int kCellsPerAxis = 9;

// Whether texel i of the pool (format FMT, 1000 texels per slot) is zero in
// every bit.
template <int FMT>
__device__ __forceinline__ bool texel_is_zero(const void* pool, size_t i) {
    if (FMT == VV_FMT_RGBA8) return ((const uint32_t*)pool)[i] == 0u;
    if (FMT == VV_FMT_DXT5) {  // the decoded texel
        const size_t slot = i / 1000u;
        const int r = (int)(i - slot * 1000u), z = r / 100, y = (r / 10) % 10, x = r % 10;
        const uint4 v = ((const uint4*)pool)[slot * dxt::kBlocksPerSlot + (size_t)dxt::block_of(x, y, z)];
        const uint32_t w[4] = {v.x, v.y, v.z, v.w};
        return dxt::decode_dxt5(w, dxt::texel_of(x, y)) == 0u;
    }
    if (FMT == VV_FMT_FP32) {
        const uint4 v = ((const uint4*)pool)[i];
        return (v.x | v.y | v.z | v.w) == 0u;
    }
    const uint2 v = ((const uint2*)pool)[i];  // FP16, BF16
    return (v.x | v.y) == 0u;
}

// All threads of a CTA (blockDim.x a multiple of 32): zero[q] (shared, 1000
// flags) holds texel q of the slot and the CTA has synchronised; writes the
// slot's 32 mask words.
__device__ __forceinline__ void write_cell_mask(const uint8_t* zero, uint32_t* __restrict__ out) {
    for (int base = 0; base < 32 * kCellMaskWords; base += blockDim.x) {
        const int c = base + (int)threadIdx.x;
        bool z = false;
        if (c < kCellsPerAxis * kCellsPerAxis * kCellsPerAxis) {
            const int x = c % 9, y = (c / 9) % 9, zz = c / 81;
            const int t = (zz * 10 + y) * 10 + x;
            z = (zero[t] & zero[t + 1] & zero[t + 10] & zero[t + 11] & zero[t + 100] & zero[t + 101] &
                 zero[t + 110] & zero[t + 111]) != 0;
        }
        const unsigned b = __ballot_sync(0xFFFFFFFFu, z);
        // each warp covers the 32 cells of one mask word
        if ((threadIdx.x & 31u) == 0u && c < 32 * kCellMaskWords) out[c >> 5] = b;
    }
}

}  // namespace vv
