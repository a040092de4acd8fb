// select.cuh - the per-pixel selection of GenerateSelectionMask.frag
// (:15-187): which of a pixel's node-usage entries are kept, shared by the
// selection kernel and the fused compaction.
#pragma once

#include <cstdint>

namespace vv {

// Bit i set: entry i of pixel (x, y) is non-zero, no earlier entry was zero,
// and the same node id is not at entry i-1, i or i+1 (cyclically) of the
// pixels two to the top, two to the top-right or two to the right (those
// pixels request it; frame edges have no such neighbour).
__device__ __forceinline__ uint32_t select_bits(const uint4* __restrict__ usage, int x, int y, int w, int h) {
    const size_t pix = (size_t)y * w + x;
    uint32_t own[12];
    {
        const uint4* o = usage + pix * 3;
        const uint4 a = o[0], b = o[1], c = o[2];
        own[0] = a.x; own[1] = a.y; own[2] = a.z; own[3] = a.w;
        own[4] = b.x; own[5] = b.y; own[6] = b.z; own[7] = b.w;
        own[8] = c.x; own[9] = c.y; own[10] = c.z; own[11] = c.w;
    }
    uint32_t bits = 0u;
    if (own[0] == 0u) return bits;
    uint32_t top[12], tr[12], rt[12];
    const bool has_top = y < h - 2, has_right = x < w - 2;
    auto load = [&](uint32_t* dstl, bool cond, int nx, int ny) {
        if (cond) {
            const uint4* o = usage + ((size_t)ny * w + nx) * 3;
            const uint4 a = o[0], b = o[1], c = o[2];
            dstl[0] = a.x; dstl[1] = a.y; dstl[2] = a.z; dstl[3] = a.w;
            dstl[4] = b.x; dstl[5] = b.y; dstl[6] = b.z; dstl[7] = b.w;
            dstl[8] = c.x; dstl[9] = c.y; dstl[10] = c.z; dstl[11] = c.w;
        } else {
#pragma unroll
            for (int i = 0; i < 12; ++i) dstl[i] = 0u;
        }
    };
    load(top, has_top, x, y + 2);
    load(tr, has_top && has_right, x + 2, y + 2);
    load(rt, has_right, x + 2, y);
#pragma unroll
    for (int i = 0; i < 12; ++i) {
        const uint32_t v = own[i];
        if (v == 0u) break;
        const int pi = (i + 11) % 12, ni = (i + 1) % 12;
        if (v == top[i] || v == top[pi] || v == top[ni]) continue;
        if (v == tr[i] || v == tr[pi] || v == tr[ni]) continue;
        if (v == rt[i] || v == rt[pi] || v == rt[ni]) continue;
        bits |= 1u << i;
    }
    return bits;
}

}  // namespace vv
