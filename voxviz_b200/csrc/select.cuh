// select.cuh - the per-pixel selection of GenerateSelectionMask.frag
// (:15-187): which of a pixel's node-usage entries are kept, shared by the
// selection kernel and the fused compaction.
#pragma once

#include <cstdint>

namespace vv {

// Bit i set: entry i of pixel (x, y) is non-zero, no earlier entry was zero,
// and the same node id is not at entry i-1, i or i+1 (cyclically) of the
// pixels two to the top, two to the top-right or two to the right (those
// pixels request it; frame edges have no such neighbour).  Entries past the
// first zero may match a neighbour's zero: they are masked by `valid`.
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
    if (own[0] == 0u) return 0u;
    // the entries before the first zero
    uint32_t valid = 0u;
    bool open = true;
#pragma unroll
    for (int i = 0; i < 12; ++i) {
        open = open && own[i] != 0u;
        valid |= open ? 1u << i : 0u;
    }
    // an entry is dropped when a neighbour holds its node at the same
    // position or one to either side (cyclically); one neighbour record at
    // a time keeps 24 words live instead of 48
    uint32_t drop = 0u;
    auto test = [&](int nx, int ny) {
        const uint4* o = usage + ((size_t)ny * w + nx) * 3;
        const uint4 a = o[0], b = o[1], c = o[2];
        const uint32_t nb[12] = {a.x, a.y, a.z, a.w, b.x, b.y, b.z, b.w, c.x, c.y, c.z, c.w};
#pragma unroll
        for (int i = 0; i < 12; ++i) {
            const int pi = (i + 11) % 12, ni = (i + 1) % 12;
            const uint32_t v = own[i];
            drop |= (v == nb[i] || v == nb[pi] || v == nb[ni]) ? 1u << i : 0u;
        }
    };
    const bool has_top = y < h - 2, has_right = x < w - 2;
    if (has_top) test(x, y + 2);
    if (has_top && has_right) test(x + 2, y + 2);
    if (has_right) test(x + 2, y);
    return valid & ~drop;
}

}  // namespace vv
