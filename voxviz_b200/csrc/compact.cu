// compact.cu - the page-request compaction in three launches.
//
// GenerateSelectionMask.frag, GenerateHistoPyramid.frag and
// CompressNodeUsageList.frag (GigaVoxelsRenderer.cpp:1937-2135) as the
// per-level kernels of kernels.cu run them: a histopyramid whose levels halve
// the frame (a level of odd size folds its last row / column into the last
// parent), counts summed upwards, exclusive offsets handed downwards in each
// parent's child order, and every selected pixel's entries written at its
// offset.  Here the pyramid is cut at level 5:
//   tile_up_kernel   one CTA per level-5 node: the selection of the pixels
//                    under it (written to the mask) and the counts of its
//                    subtree up to the node, in shared memory;
//   top_kernel       one CTA: the pyramid above level 5, counts up and
//                    offsets down, and the request count;
//   tile_down_kernel one CTA per level-5 node: its subtree's counts again
//                    (from the mask), the offsets down from the node's, and
//                    the compaction of its pixels.
// The pixels under a level-k node form a rectangle: a node range [a, b) at
// level k+1 covers [2a, 2b) at level k, extended to the level's width when
// b is the level-(k+1) width (the fold).  Same parents, same child order,
// same sums: the offsets, and so the request order, equal the per-level
// kernels' (integer arithmetic).
#include <algorithm>

#include "compact.h"
#include "select.cuh"

namespace vv {
namespace {

constexpr int kCut = 5;              // the level whose nodes the tile kernels own
constexpr int kFoot = 2 << kCut;     // at most 2^(kCut+1) - 1 cells per axis under one node, at level 0
constexpr int kTileThreads = 256;
constexpr int kTile = 1 << kCut;     // pixels per axis under a level-kCut node without folds
constexpr int kTopThreads = 1024;
constexpr int kTopMaxCells = 16384;  // level-5 nodes one top CTA takes (with the levels above)

struct Levels {
    int n;                 // levels in the pyramid
    int w[24], h[24];
};

// Children of parent (X, Y) at the finer level (w, h), in the order the
// compaction walks them: the 2x2 block, then for an odd last row (x, y+2),
// (x+1, y+2) and for an odd last column the (x+2, *) cells.  Child j is
// computed from j (no arrays: registers only).
struct Kids {
    int x, y, n;
    bool row, col;  // the parent takes the odd last row / column
    __device__ __forceinline__ Kids(int X, int Y, int w, int h) {
        x = 2 * X;
        y = 2 * Y;
        row = y + 2 == h - 1;
        col = x + 2 == w - 1;
        n = 4 + (row ? 2 : 0) + (col ? (row ? 3 : 2) : 0);
    }
    __device__ __forceinline__ void at(int j, int& cx, int& cy) const {
        if (j < 4) {
            cx = x + (j & 1);
            cy = y + (j >> 1);
        } else if (row && j < 6) {
            cx = x + (j - 4);
            cy = y + 2;
        } else {
            // the column cells, bottom up: (x+2, y+2) after a folded row, then (x+2, y+1), (x+2, y)
            const int r = j - (row ? 6 : 4);
            cx = x + 2;
            cy = y + (row ? 2 : 1) - r;
        }
    }
};

// The subtree of level-kCut node (X, Y): its node rectangle at every level
// k <= kCut, [x0[k], x1[k]) x [y0[k], y1[k]), and where level k's cells sit
// in the shared arrays (base[k], row pitch x1[k] - x0[k]).
struct Subtree {
    int x0[kCut + 1], x1[kCut + 1], y0[kCut + 1], y1[kCut + 1];
    int base[kCut + 2];
};

__device__ __forceinline__ void subtree(const Levels& L, int X, int Y, Subtree& t) {
    t.x0[kCut] = X;
    t.x1[kCut] = X + 1;
    t.y0[kCut] = Y;
    t.y1[kCut] = Y + 1;
    for (int k = kCut - 1; k >= 0; --k) {
        t.x0[k] = 2 * t.x0[k + 1];
        t.x1[k] = t.x1[k + 1] == L.w[k + 1] ? L.w[k] : 2 * t.x1[k + 1];
        t.y0[k] = 2 * t.y0[k + 1];
        t.y1[k] = t.y1[k + 1] == L.h[k + 1] ? L.h[k] : 2 * t.y1[k + 1];
    }
    t.base[0] = 0;
    for (int k = 0; k <= kCut; ++k) t.base[k + 1] = t.base[k] + (t.x1[k] - t.x0[k]) * (t.y1[k] - t.y0[k]);
}

// cells of a subtree at levels 0..kCut: at most the sum of kFoot^2 / 4^k
constexpr int kSubtreeCells = kFoot * kFoot + (kFoot / 2) * (kFoot / 2) + (kFoot / 4) * (kFoot / 4) +
                              (kFoot / 8) * (kFoot / 8) + (kFoot / 16) * (kFoot / 16) + 4 + 1;

__device__ __forceinline__ uint32_t sub_cell(const uint16_t* a, const Subtree& t, int k, int x, int y) {
    if (x < t.x0[k] || x >= t.x1[k] || y < t.y0[k] || y >= t.y1[k]) return 0u;  // outside the level
    return a[t.base[k] + (y - t.y0[k]) * (t.x1[k] - t.x0[k]) + (x - t.x0[k])];
}

__device__ __forceinline__ int level_cells(const Subtree& t, int k) {
    return (t.x1[k] - t.x0[k]) * (t.y1[k] - t.y0[k]);
}

// The upper levels of a subtree hold few cells: from the first level (going
// up) with at most kWarpCells cells one warp does the rest, with warp
// barriers only.
constexpr int kWarpCells = 64;

// Level k+1 of the subtree's counts from level k's (cells i = first, first
// + step, ...).
__device__ __forceinline__ void up_level(const Levels& L, const Subtree& t, uint16_t* cnt, int k, int first,
                                         int step) {
    const int w = t.x1[k + 1] - t.x0[k + 1], n = level_cells(t, k + 1);
    for (int i = first; i < n; i += step) {
        const Kids kids(t.x0[k + 1] + i % w, t.y0[k + 1] + i / w, L.w[k], L.h[k]);
        uint32_t sum = 0u;
        for (int j = 0; j < kids.n; ++j) {
            int cx, cy;
            kids.at(j, cx, cy);
            sum += sub_cell(cnt, t, k, cx, cy);
        }
        cnt[t.base[k + 1] + i] = (uint16_t)sum;
    }
}

// counts of levels 1..kCut of the subtree from level 0's (in cnt); on
// return warp 0 has every level, the other warps the block-swept ones
__device__ __forceinline__ void sweep_up(const Levels& L, const Subtree& t, uint16_t* cnt) {
    int k = 0;
    for (; k < kCut && level_cells(t, k + 1) > kWarpCells; ++k) {
        up_level(L, t, cnt, k, threadIdx.x, blockDim.x);
        __syncthreads();
    }
    if (threadIdx.x < 32) {
        for (; k < kCut; ++k) {
            up_level(L, t, cnt, k, threadIdx.x, 32);
            __syncwarp();
        }
    }
}

__global__ void __launch_bounds__(kTileThreads) tile_up_kernel(const __grid_constant__ Levels L,
                                                                const uint4* __restrict__ usage,
                                                                uint32_t* __restrict__ mask,
                                                                uint32_t* __restrict__ cut_counts) {
    __shared__ uint16_t cnt[kSubtreeCells];  // counts of at most 63 x 63 pixels fit in 16 bits
    __shared__ Subtree t;
    __shared__ uint32_t wsum[kTileThreads / 32];
    const int X = blockIdx.x, Y = blockIdx.y;
    if (threadIdx.x == 0) subtree(L, X, Y, t);
    __syncthreads();
    const int W = L.w[0], H = L.h[0];
    const int w0 = t.x1[0] - t.x0[0], n0 = w0 * (t.y1[0] - t.y0[0]);
    if (w0 == kTile && n0 == kTile * kTile) {
        // no fold under this node: its count is a plain sum
        uint32_t c = 0u;
        for (int i = threadIdx.x; i < n0; i += blockDim.x) {
            const int x = t.x0[0] + (i & (kTile - 1)), y = t.y0[0] + i / kTile;
            const uint32_t bits = select_bits(usage, x, y, W, H);
            mask[(size_t)y * W + x] = bits;
            c += bits != 0u ? 1u : 0u;
        }
        c = __reduce_add_sync(0xFFFFFFFFu, c);
        if ((threadIdx.x & 31u) == 0u) wsum[threadIdx.x >> 5] = c;
        __syncthreads();
        if (threadIdx.x == 0) {
            uint32_t s = 0u;
            for (int w = 0; w < kTileThreads / 32; ++w) s += wsum[w];
            cut_counts[(size_t)Y * L.w[kCut] + X] = s;
        }
        return;
    }
    for (int i = threadIdx.x; i < n0; i += blockDim.x) {
        const int x = t.x0[0] + i % w0, y = t.y0[0] + i / w0;
        const uint32_t bits = select_bits(usage, x, y, W, H);
        mask[(size_t)y * W + x] = bits;
        cnt[i] = bits != 0u ? 1 : 0;
    }
    __syncthreads();
    sweep_up(L, t, cnt);
    if (threadIdx.x == 0) cut_counts[(size_t)Y * L.w[kCut] + X] = cnt[t.base[kCut]];
}

// The pyramid from level kCut up: counts, then offsets down to level kCut.
// Shared arrays: counts and offsets of levels kCut..n-1, one after another.
__global__ void __launch_bounds__(kTopThreads) top_kernel(const __grid_constant__ Levels L,
                                                           const uint32_t* __restrict__ cut_counts,
                                                           uint32_t* __restrict__ cut_offsets,
                                                           uint32_t* __restrict__ request_count) {
    extern __shared__ uint32_t sm[];
    int base[25];
    base[kCut] = 0;
    for (int k = kCut; k < L.n; ++k) base[k + 1] = base[k] + L.w[k] * L.h[k];
    uint32_t* cnt = sm;
    uint32_t* off = sm + base[L.n];
    const int n_cut = L.w[kCut] * L.h[kCut];
    for (int i = threadIdx.x; i < n_cut; i += blockDim.x) cnt[i] = cut_counts[i];
    __syncthreads();
    for (int k = kCut; k + 1 < L.n; ++k) {
        const int cw = L.w[k + 1], n = cw * L.h[k + 1];
        for (int i = threadIdx.x; i < n; i += blockDim.x) {
            const Kids kids(i % cw, i / cw, L.w[k], L.h[k]);
            uint32_t sum = 0u;
            for (int j = 0; j < kids.n; ++j) {
                int cx, cy;
                kids.at(j, cx, cy);
                if (cx < L.w[k] && cy < L.h[k]) sum += cnt[base[k] + cy * L.w[k] + cx];
            }
            cnt[base[k + 1] + i] = sum;
        }
        __syncthreads();
    }
    const int top = L.n - 1;
    if (threadIdx.x == 0) {
        off[base[top]] = 0u;
        if (request_count) *request_count = cnt[base[top]];
    }
    __syncthreads();
    // offsets down, per parent: each child gets the parent's offset plus the
    // counts of the children before it
    for (int k = top - 1; k >= kCut; --k) {
        const int w = L.w[k], cw = L.w[k + 1], n = cw * L.h[k + 1];
        for (int i = threadIdx.x; i < n; i += blockDim.x) {
            const Kids kids(i % cw, i / cw, w, L.h[k]);
            uint32_t o = off[base[k + 1] + i];
            for (int j = 0; j < kids.n; ++j) {
                int cx, cy;
                kids.at(j, cx, cy);
                if (cx >= w || cy >= L.h[k]) continue;
                const int c = base[k] + cy * w + cx;
                off[c] = o;
                o += cnt[c];
            }
        }
        __syncthreads();
    }
    for (int i = threadIdx.x; i < n_cut; i += blockDim.x) cut_offsets[i] = off[i];
}

// Level k of the subtree's offsets from level k+1's: each parent (i = first,
// first + step, ...) hands its offset plus the counts of the children before
// each child down.
__device__ __forceinline__ void down_level(const Levels& L, const Subtree& t, const uint16_t* cnt, uint32_t* off,
                                           int k, int first, int step) {
    const int pw = t.x1[k + 1] - t.x0[k + 1], n = level_cells(t, k + 1);
    const int w = t.x1[k] - t.x0[k];
    for (int i = first; i < n; i += step) {
        const Kids kids(t.x0[k + 1] + i % pw, t.y0[k + 1] + i / pw, L.w[k], L.h[k]);
        uint32_t o = off[t.base[k + 1] + i];
        for (int j = 0; j < kids.n; ++j) {
            int cx, cy;
            kids.at(j, cx, cy);
            if (cx >= L.w[k] || cy >= L.h[k]) continue;
            const int c = t.base[k] + (cy - t.y0[k]) * w + (cx - t.x0[k]);
            off[c] = o;
            o += cnt[c];
        }
    }
}

// The position of x in a Morton index (the even bits).
__device__ __forceinline__ int even_bits(uint32_t m) {
    m &= 0x55555555u;
    m = (m | (m >> 1)) & 0x33333333u;
    m = (m | (m >> 2)) & 0x0F0F0F0Fu;
    m = (m | (m >> 4)) & 0x00FF00FFu;
    m = (m | (m >> 8)) & 0x0000FFFFu;
    return (int)m;
}

struct TileDown {
    Levels L;
    const uint4* usage;
    const uint32_t* mask;
    const uint32_t* cut_offsets;
    uint32_t* requests;
    int cap;
    int max_push;
};

// CompressNodeUsageList.frag (:107-149): the kept entries of a selected
// pixel in order, at most max_push, each into entry (pushed mod 4) - the
// last four pushed stay (registers throughout) - at the pixel's offset.
__device__ __forceinline__ void write_request(const TileDown& p, size_t pix, uint32_t bits, uint32_t rank) {
    if (rank >= (uint32_t)p.cap) return;
    const uint4* o = p.usage + pix * 3;
    const uint4 a = o[0], b = o[1], c = o[2];
    const uint32_t list[12] = {a.x, a.y, a.z, a.w, b.x, b.y, b.z, b.w, c.x, c.y, c.z, c.w};
    uint32_t o0 = 0u, o1 = 0u, o2 = 0u, o3 = 0u;
    int pushed = 0;
#pragma unroll
    for (int item = 0; item < 12; ++item) {
        if (((bits >> item) & 1u) && pushed < p.max_push) {
            const uint32_t v = list[item];
            const int s = pushed & 3;
            o0 = s == 0 ? v : o0;
            o1 = s == 1 ? v : o1;
            o2 = s == 2 ? v : o2;
            o3 = s == 3 ? v : o3;
            ++pushed;
        }
    }
    reinterpret_cast<uint4*>(p.requests)[rank] = make_uint4(o0, o1, o2, o3);
}

__global__ void __launch_bounds__(kTileThreads) tile_down_kernel(const __grid_constant__ TileDown p) {
    __shared__ uint16_t cnt[kSubtreeCells];  // counts of at most 63 x 63 pixels fit in 16 bits
    __shared__ uint32_t off[kSubtreeCells];
    __shared__ Subtree t;
    __shared__ uint32_t wtot[kTileThreads / 32];
    const Levels& L = p.L;
    const int X = blockIdx.x, Y = blockIdx.y;
    if (threadIdx.x == 0) subtree(L, X, Y, t);
    __syncthreads();
    const int W = L.w[0];
    const int w0 = t.x1[0] - t.x0[0], n0 = w0 * (t.y1[0] - t.y0[0]);
    if (w0 == kTile && n0 == kTile * kTile) {
        // no fold under this node: the order under it is the Morton order
        // of its 32x32 pixels (children (x,y), (x+1,y), (x,y+1), (x+1,y+1)
        // at every level), so a pixel's offset is the node's plus the
        // selected pixels before it in that order - one block-wide scan.
        // Thread i takes Morton indices 4i..4i+3.
        constexpr int kPer = kTile * kTile / kTileThreads;
        uint32_t bits[kPer];
        size_t pix[kPer];
        uint32_t c = 0u;
#pragma unroll
        for (int j = 0; j < kPer; ++j) {
            const uint32_t m = (uint32_t)(threadIdx.x * kPer + j);
            pix[j] = (size_t)(t.y0[0] + even_bits(m >> 1)) * W + (size_t)(t.x0[0] + even_bits(m));
            bits[j] = p.mask[pix[j]];
            c += bits[j] != 0u ? 1u : 0u;
        }
        const unsigned lane = threadIdx.x & 31u;
        uint32_t incl = c;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            const uint32_t v = __shfl_up_sync(0xFFFFFFFFu, incl, d);
            if (lane >= (unsigned)d) incl += v;
        }
        if (lane == 31u) wtot[threadIdx.x >> 5] = incl;
        __syncthreads();
        uint32_t r = p.cut_offsets[(size_t)Y * L.w[kCut] + X] + incl - c;
        for (int w = 0; w < (int)(threadIdx.x >> 5); ++w) r += wtot[w];
        if (!p.requests || p.cap <= 0) return;
#pragma unroll
        for (int j = 0; j < kPer; ++j) {
            if (bits[j] != 0u) {
                write_request(p, pix[j], bits[j], r);
                ++r;
            }
        }
        return;
    }
    for (int i = threadIdx.x; i < n0; i += blockDim.x) {
        const int x = t.x0[0] + i % w0, y = t.y0[0] + i / w0;
        cnt[i] = p.mask[(size_t)y * W + x] != 0u ? 1 : 0;
    }
    __syncthreads();
    sweep_up(L, t, cnt);
    if (threadIdx.x == 0) off[t.base[kCut]] = p.cut_offsets[(size_t)Y * L.w[kCut] + X];
    __syncthreads();
    // offsets down, per parent (the children of a node of the subtree are
    // in the subtree, or outside the level): the small upper levels by warp
    // 0, which holds their counts, then the rest by the block
    int k = kCut - 1;
    if (threadIdx.x < 32) {
        for (; k >= 0 && level_cells(t, k + 1) <= kWarpCells; --k) {
            down_level(L, t, cnt, off, k, threadIdx.x, 32);
            __syncwarp();
        }
    }
    __syncthreads();
    k = kCut - 1;
    while (k >= 0 && level_cells(t, k + 1) <= kWarpCells) --k;
    for (; k >= 0; --k) {
        down_level(L, t, cnt, off, k, threadIdx.x, blockDim.x);
        __syncthreads();
    }
    if (!p.requests || p.cap <= 0) return;
    for (int i = threadIdx.x; i < n0; i += blockDim.x) {
        const int x = t.x0[0] + i % w0, y = t.y0[0] + i / w0;
        const size_t pix = (size_t)y * W + x;
        const uint32_t bits = p.mask[pix];
        if (bits != 0u) write_request(p, pix, bits, off[i]);
    }
}

}  // namespace

cudaError_t launch_compact_fused(const CompactParams& p, uint32_t* mask, cudaStream_t s) {
    if (p.levels <= kCut + 1 || p.levels > 24 || !mask) return cudaErrorNotSupported;
    Levels L;
    L.n = p.levels;
    for (int k = 0; k < p.levels; ++k) {
        L.w[k] = p.level_w[k];
        L.h[k] = p.level_h[k];
    }
    const int n_cut = L.w[kCut] * L.h[kCut];
    if (n_cut > kTopMaxCells) return cudaErrorNotSupported;
    long long top_cells = 0;
    for (int k = kCut; k < L.n; ++k) top_cells += (long long)L.w[k] * L.h[k];
    const size_t top_bytes = (size_t)top_cells * 2 * sizeof(uint32_t);
    if (top_bytes > 200 * 1024) return cudaErrorNotSupported;
    if (top_bytes > 48 * 1024) {  // (on the current device; only frames above ~2.5 K x 2 K need it)
        const cudaError_t e = cudaFuncSetAttribute(top_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                   (int)top_bytes);
        if (e != cudaSuccess) return e;
    }
    // the per-level scratch of CompactParams: level-5 counts and offsets
    uint32_t* cut_counts = p.counts;
    uint32_t* cut_offsets = p.offsets;
    const dim3 grid((unsigned)L.w[kCut], (unsigned)L.h[kCut]);
    tile_up_kernel<<<grid, kTileThreads, 0, s>>>(L, p.usage, mask, cut_counts);
    top_kernel<<<1, kTopThreads, top_bytes, s>>>(L, cut_counts, cut_offsets, p.request_count);
    TileDown d;
    d.L = L;
    d.usage = p.usage;
    d.mask = mask;
    d.cut_offsets = cut_offsets;
    d.requests = p.requests;
    d.cap = p.cap;
    d.max_push = p.max_push;
    tile_down_kernel<<<grid, kTileThreads, 0, s>>>(d);
    return cudaGetLastError();
}

}  // namespace vv
