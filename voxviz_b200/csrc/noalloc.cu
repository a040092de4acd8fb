// noalloc.cu - page-request compaction that allocates nothing.
//
// vv_compact_requests_noalloc runs the selection mask, the histopyramid and
// the compaction of a frame's node-usage lists like vv_render's
// VV_PASS_SELECT | VV_PASS_COMPACT, but keeps its pyramid in a file-scope
// device array instead of memory the context allocates.  It is meant for
// callers that must not call cudaMalloc: code running inside an allocator or
// a memory-pool callback, real-time render threads that may not block on the
// driver's allocator, and processes whose device memory is handed out by a
// framework that forbids side allocations.  Level 0 of the pyramid is read
// straight from the selection mask the caller passes, so only levels >= 1
// (at most width*height cells each for counts and offsets) live in the array.
#include <cuda_runtime.h>

#include <mutex>
#include <string>

#include "kernels.cuh"

namespace vv {
void set_thread_error(const std::string& msg);
}

namespace {

// Pyramid counts [0, MAX) and exclusive offsets [MAX, 2*MAX) of levels >= 1.
// Every GPU that loads the library holds these 16 MiB until the process exits.
__device__ __align__(256) uint32_t g_compact_scratch[2u * VV_NOALLOC_MAX_PIXELS];

std::mutex g_scratch_mu;
uint32_t* g_scratch_ptr[1024] = {};

// Device address of the scratch array on the current device.  The array's
// name is only a host-side stand-in; the address comes from
// cudaGetSymbolAddress, once per device, with that device current.  The
// first lookup can load the module on that device (lazy loading), which may
// allocate; the kept address does not survive a reset of the device's
// primary context (cudaDeviceReset).
int scratch_address(uint32_t** out) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess || dev < 0 || dev >= 1024) {
        vv::set_thread_error(std::string("cudaGetDevice: ") + cudaGetErrorString(e));
        return VV_ERR_CUDA;
    }
    std::lock_guard<std::mutex> lk(g_scratch_mu);
    if (!g_scratch_ptr[dev]) {
        void* p = nullptr;
        e = cudaGetSymbolAddress(&p, g_compact_scratch);
        if (e != cudaSuccess || !p) {
            vv::set_thread_error(std::string("cudaGetSymbolAddress(compaction scratch): ") + cudaGetErrorString(e));
            return VV_ERR_CUDA;
        }
        g_scratch_ptr[dev] = (uint32_t*)p;
    }
    *out = g_scratch_ptr[dev];
    return VV_OK;
}

__device__ __forceinline__ void load12(const uint4* __restrict__ usage, size_t pix, uint32_t* v) {
    const uint4* o = usage + pix * 3;
    const uint4 a = o[0], b = o[1], c = o[2];
    v[0] = a.x; v[1] = a.y; v[2] = a.z; v[3] = a.w;
    v[4] = b.x; v[5] = b.y; v[6] = b.z; v[7] = b.w;
    v[8] = c.x; v[9] = c.y; v[10] = c.z; v[11] = c.w;
}

// GenerateSelectionMask.frag (:15-187): keep item i unless the list two
// pixels up, up-right or right holds it at i-1, i or i+1.
__global__ void na_select_kernel(const uint4* __restrict__ usage, uint32_t* __restrict__ mask, int w, int h) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= w || y >= h) return;
    uint32_t own[12], nb[3][12];
    load12(usage, (size_t)y * w + x, own);
    uint32_t bits = 0u;
    if (own[0] != 0u) {
        const bool up = y < h - 2, right = x < w - 2;
        const bool has[3] = {up, up && right, right};
        const int nx[3] = {x, x + 2, x + 2}, ny[3] = {y + 2, y + 2, y};
        for (int k = 0; k < 3; ++k) {
            if (has[k]) load12(usage, (size_t)ny[k] * w + nx[k], nb[k]);
            else
                for (int i = 0; i < 12; ++i) nb[k][i] = 0u;
        }
        for (int i = 0; i < 12; ++i) {
            const uint32_t v = own[i];
            if (v == 0u) break;
            const int p = (i + 11) % 12, n = (i + 1) % 12;
            bool dup = false;
            for (int k = 0; k < 3; ++k) dup |= v == nb[k][i] || v == nb[k][p] || v == nb[k][n];
            if (!dup) bits |= 1u << i;
        }
    }
    mask[(size_t)y * w + x] = bits;
}

// Children of level-1 cell (X,Y) in the walk order of CompressNodeUsageList.frag.
__device__ __forceinline__ int na_children(int X, int Y, int w, int h, int* cx, int* cy) {
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

__device__ __forceinline__ uint32_t active(const uint32_t* mask, int x, int y, int w, int h) {
    return (x < w && y < h && mask[(size_t)y * w + x] != 0u) ? 1u : 0u;
}

// Level 1 of ComputeActiveTexels + GenerateHistoPyramid, from the mask.
__global__ void na_level1_kernel(const uint32_t* __restrict__ mask, uint32_t* __restrict__ l1, int w, int h, int w1,
                                 int h1) {
    const int X = blockIdx.x * blockDim.x + threadIdx.x, Y = blockIdx.y * blockDim.y + threadIdx.y;
    if (X >= w1 || Y >= h1) return;
    int cx[9], cy[9];
    const int n = na_children(X, Y, w, h, cx, cy);
    uint32_t s = 0u;
    for (int i = 0; i < n; ++i) s += active(mask, cx[i], cy[i], w, h);
    l1[(size_t)Y * w1 + X] = s;
}

// CompressNodeUsageList.frag (:107-149) for each active pixel at its rank:
// the level-1 parent's offset plus the active siblings walked before it.
__global__ void na_compact_kernel(const uint4* __restrict__ usage, const uint32_t* __restrict__ mask,
                                  const uint32_t* __restrict__ off1, int w, int h, int w1, int h1,
                                  uint4* __restrict__ requests, int cap, int max_push) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= w || y >= h) return;
    const size_t pix = (size_t)y * w + x;
    uint32_t bits = mask[pix];
    if (bits == 0u) return;
    uint32_t rank = 0u;
    if (off1) {
        const int X = min(x >> 1, w1 - 1), Y = min(y >> 1, h1 - 1);
        int cx[9], cy[9];
        const int n = na_children(X, Y, w, h, cx, cy);
        rank = off1[(size_t)Y * w1 + X];
        for (int i = 0; i < n; ++i) {
            if (cx[i] == x && cy[i] == y) break;
            rank += active(mask, cx[i], cy[i], w, h);
        }
    }
    if (rank >= (uint32_t)cap) return;
    uint32_t list[12];
    load12(usage, pix, list);
    uint32_t out[4] = {0u, 0u, 0u, 0u};
    int pushed = 0;
    for (int item = 0; item < 12 && bits != 0u && pushed < max_push; ++item, bits >>= 1) {
        if (bits & 1u) {
            out[pushed & 3] = list[item];
            ++pushed;
        }
    }
    requests[rank] = make_uint4(out[0], out[1], out[2], out[3]);
}

__global__ void na_total_kernel(const uint32_t* top, const uint32_t* mask, uint32_t* count) {
    if (threadIdx.x == 0 && blockIdx.x == 0) *count = top ? *top : (mask[0] != 0u ? 1u : 0u);
}

}  // namespace

extern "C" int vv_compact_requests_noalloc(const uint32_t* usage, uint32_t* mask, int32_t width, int32_t height,
                                           uint32_t* requests, uint32_t* request_count, int32_t request_cap,
                                           int32_t compress_max_push, void* cuda_stream) {
    if (!usage || !mask || width <= 0 || height <= 0 || request_cap < 0 || (request_cap > 0 && !requests)) {
        vv::set_thread_error("vv_compact_requests_noalloc: usage and mask are required, sizes must be positive");
        return VV_ERR_ARG;
    }
    if ((long long)width * height > (long long)VV_NOALLOC_MAX_PIXELS) {
        vv::set_thread_error("vv_compact_requests_noalloc: width*height exceeds VV_NOALLOC_MAX_PIXELS (2^21); "
                             "use vv_render for larger frames");
        return VV_ERR_ARG;
    }
    uint32_t* scratch = nullptr;
    int rc = scratch_address(&scratch);
    if (rc) return rc;
    cudaStream_t s = (cudaStream_t)cuda_stream;
    // Level dims as GigaVoxelsRenderer::generateSelectionMaskHistoPyramid shrinks the viewport.
    int lw[32], lh[32];
    long long loff[32];
    int levels = 0;
    {
        int w = width, h = height;
        long long off = 0;
        while (true) {
            lw[levels] = w;
            lh[levels] = h;
            loff[levels] = levels == 0 ? 0 : off;
            if (levels > 0) off += (long long)w * h;
            ++levels;
            if (w == 1 && h == 1) break;
            if (w != 1) w >>= 1;
            if (h != 1) h >>= 1;
        }
    }
    uint32_t* counts = scratch;
    uint32_t* offsets = scratch + VV_NOALLOC_MAX_PIXELS;
    const int max_push = compress_max_push > 0 ? compress_max_push : 4;
    dim3 block(32, 4);
    dim3 grid0((unsigned)((width + 31) / 32), (unsigned)((height + 3) / 4));
    na_select_kernel<<<grid0, block, 0, s>>>((const uint4*)usage, mask, width, height);
    if (levels > 1) {
        dim3 grid1((unsigned)((lw[1] + 31) / 32), (unsigned)((lh[1] + 3) / 4));
        na_level1_kernel<<<grid1, block, 0, s>>>(mask, counts + loff[1], width, height, lw[1], lh[1]);
        cudaError_t e = vv::launch_pyramid_levels(counts, offsets, lw, lh, loff, 1, levels, s);
        if (e != cudaSuccess) {
            vv::set_thread_error(std::string("vv_compact_requests_noalloc: ") + cudaGetErrorString(e));
            return VV_ERR_CUDA;
        }
    }
    if (request_count)
        na_total_kernel<<<1, 32, 0, s>>>(levels > 1 ? counts + loff[levels - 1] : nullptr, mask, request_count);
    if (request_cap > 0)
        na_compact_kernel<<<grid0, block, 0, s>>>((const uint4*)usage, mask, levels > 1 ? offsets + loff[1] : nullptr,
                                                  width, height, levels > 1 ? lw[1] : 1, levels > 1 ? lh[1] : 1,
                                                  (uint4*)requests, request_cap, max_push);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        vv::set_thread_error(std::string("vv_compact_requests_noalloc: ") + cudaGetErrorString(e));
        return VV_ERR_CUDA;
    }
    return VV_OK;
}
