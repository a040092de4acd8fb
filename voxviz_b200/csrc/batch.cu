// batch.cu - many views of many octrees in one persistent launch.
//
// A persistent grid (resident CTAs per SM x SM count) pulls pixel tiles of
// all views from a device work queue (one atomic counter; tiles numbered view
// by view, row-major inside a view).  The views' RaycastParams (uniforms +
// the pools of each view's octree) travel by value in the kernel's parameter
// space, up to kMaxLaunchViews views per launch (88 with the 360-byte view
// record; larger batches launch in chunks), so a
// CTA reads its view's parameters from the constant bank as the single-view
// ray cast does, and runs render_pixel, the vv_render ray cast, on every
// pixel of the tile.  Tile shape and the march-loop
// unroll (samples per loop trip) are template parameters; the compiled
// variants are listed in kVariants and picked per batch by the autotuner.
//
// Floating point: compiled with the same flags as kernels.cu, so a pixel's
// colour and usage list are those of vv_render, bit for bit.
#include <algorithm>
#include <cstring>
#include <string>

#include "ctx.h"
#include "raycast_common.cuh"

namespace vv {

using namespace rc;

// One view of a batch, as the kernel reads it (device memory).
struct BatchView {
    RaycastParams p;
    int tiles_x;     // tiles per row of this view
    int tile_begin;  // index of its first tile in the queue
};

// The views of one launch.  Kernel parameters may take 32,764 bytes.
constexpr int kMaxLaunchViews = 88;  // 360 bytes each
struct BatchParams {
    int n;            // views
    int total_tiles;  // tiles of all n views
    BatchView v[kMaxLaunchViews];
};
static_assert(sizeof(BatchParams) <= 32000, "batch views must fit the kernel parameter space");

namespace {

template <int FMT, int TW, int TH, int STEPS>
// about 28 warps per SM (896 / tile threads CTAs): at most ~72 registers per
// thread.  Copying a view's parameters to shared memory instead left ~120
// registers per thread and spilled heavily above 16 warps per SM.
__global__ void __launch_bounds__(TW * TH, 896 / (TW * TH))
    batch_raycast_kernel(const __grid_constant__ BatchParams bp, unsigned* __restrict__ counter) {
    static_assert(TW % 8 == 0 && TH % 4 == 0, "a tile is made of 8x4 warp tiles");
    const BatchView* views = bp.v;
    const int nviews = bp.n, total_tiles = bp.total_tiles;
    __shared__ int s_tile, s_view, s_tx, s_ty;
    __shared__ uint2 path_w[kPathLevels][TW * TH];
    __shared__ uint32_t path_p[kPathLevels][TW * TH];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    // each warp covers an 8x4 block of the tile (coherent descents)
    const int wx = (warp % (TW / 8)) * 8 + (lane & 7);
    const int wy = (warp / (TW / 8)) * 4 + (lane >> 3);
    for (;;) {
        if (threadIdx.x == 0) {
            const int t = (int)atomicAdd(counter, 1u);
            s_tile = t;
            if (t < total_tiles) {
                int lo = 0, hi = nviews - 1;
                while (lo < hi) {
                    const int mid = (lo + hi + 1) >> 1;
                    if (views[mid].tile_begin <= t) lo = mid;
                    else hi = mid - 1;
                }
                const int local = t - views[lo].tile_begin;
                s_view = lo;
                s_tx = local % views[lo].tiles_x;
                s_ty = local / views[lo].tiles_x;
            }
        }
        __syncthreads();
        if (s_tile >= total_tiles) return;
        const RaycastParams& sp = views[s_view].p;
        const int px = s_tx * TW + wx, py = s_ty * TH + wy;
        if (px < sp.u.width && py < sp.u.height)
            render_pixel<FMT, false, STEPS, true>(sp, px, py,
                                                  PathSlots{&path_w[0][threadIdx.x], &path_p[0][threadIdx.x], TW * TH, nullptr});
        // every thread is done with s_* before thread 0 takes the next tile
        __syncthreads();
    }
}

struct Variant {
    int tw, th, steps;
};
constexpr Variant kVariants[] = {{8, 8, 1},   {8, 8, 2},   {8, 8, 4},   {16, 8, 1}, {16, 8, 2}, {16, 8, 4},
                                 {16, 16, 1}, {16, 16, 2}, {16, 16, 4}, {32, 8, 1}, {32, 8, 2}, {32, 8, 4}};
constexpr int kNumVariants = (int)(sizeof(kVariants) / sizeof(kVariants[0]));

using BatchKernel = void (*)(BatchParams, unsigned*);

template <int FMT>
BatchKernel kernel_for(int tw, int th, int steps) {
#define VV_V(W, H, S) \
    if (tw == W && th == H && steps == S) return batch_raycast_kernel<FMT, W, H, S>;
    VV_V(8, 8, 1) VV_V(8, 8, 2) VV_V(8, 8, 4)
    VV_V(16, 8, 1) VV_V(16, 8, 2) VV_V(16, 8, 4)
    VV_V(16, 16, 1) VV_V(16, 16, 2) VV_V(16, 16, 4)
    VV_V(32, 8, 1) VV_V(32, 8, 2) VV_V(32, 8, 4)
#undef VV_V
    return nullptr;
}

BatchKernel find_kernel(int fmt, int tw, int th, int steps) {
    switch (fmt) {
        case VV_FMT_RGBA8: return kernel_for<VV_FMT_RGBA8>(tw, th, steps);
        case VV_FMT_FP16: return kernel_for<VV_FMT_FP16>(tw, th, steps);
        case VV_FMT_BF16: return kernel_for<VV_FMT_BF16>(tw, th, steps);
        case VV_FMT_FP32: return kernel_for<VV_FMT_FP32>(tw, th, steps);
        default: return nullptr;
    }
}

int batch_fail(vv_ctx* c, int code, const std::string& msg) { return ctx_fail(c, code, msg); }

#define VV_CUDA(c, expr)                                                                          \
    do {                                                                                          \
        cudaError_t e_ = (expr);                                                                  \
        if (e_ != cudaSuccess) return batch_fail(c, VV_ERR_CUDA, std::string(#expr) + ": " + cudaGetErrorString(e_)); \
    } while (0)

bool stream_capturing(cudaStream_t s) {
    cudaStreamCaptureStatus st = cudaStreamCaptureStatusNone;
    return cudaStreamIsCapturing(s, &st) == cudaSuccess && st != cudaStreamCaptureStatusNone;
}

}  // namespace

// Shared by vv_render_batch and the autotuner: validate the views, fill the
// launch parameters and launch one persistent grid per chunk of at most
// kMaxLaunchViews views.
static int batch_launch(vv_ctx* c, const vv_batch_view* views, int32_t n, const vv_batch_config* cfg) {
    if (!c || !views || n <= 0 || !cfg) return batch_fail(c, VV_ERR_ARG, "bad batch arguments");
    const int tw = cfg->tile_w, th = cfg->tile_h, steps = cfg->steps;
    int fmt = -1;
    for (int i = 0; i < n; ++i) {
        const vv_batch_view& bv = views[i];
        if (!bv.ctx) return batch_fail(c, VV_ERR_ARG, "batch view without a context");
        if (bv.ctx->device != c->device) return batch_fail(c, VV_ERR_ARG, "batch views span devices");
        if (!bv.ctx->bricks) return batch_fail(c, VV_ERR_STATE, "brick pool not created");
        if (fmt < 0) fmt = bv.ctx->fmt;
        else if (fmt != bv.ctx->fmt) return batch_fail(c, VV_ERR_ARG, "batch views mix brick formats");
    }
    BatchKernel kern = find_kernel(fmt, tw, th, steps);
    if (!kern) return batch_fail(c, VV_ERR_ARG, "no compiled batch variant for this tile shape / steps");
    cudaSetDevice(c->device);
    // launch parameters are copied when the launch is made: one host block serves every chunk
    int rc = ctx_ensure_host(c, &c->h_batch, &c->h_batch_cap, sizeof(BatchParams));
    if (rc) return rc;
    const int chunks = (n + kMaxLaunchViews - 1) / kMaxLaunchViews;
    rc = ctx_ensure(c, &c->d_batch, &c->d_batch_cap, (size_t)chunks * 16, "batch queue counters");
    if (rc) return rc;
    int per_sm = cfg->ctas_per_sm;
    if (per_sm <= 0) {
        VV_CUDA(c, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, tw * th, 0));
        per_sm = std::max(per_sm, 1);
    }
    int sms = 0;
    VV_CUDA(c, cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, c->device));
    BatchParams& bp = *(BatchParams*)c->h_batch;
    for (int k = 0; k < chunks; ++k) {
        const int first = k * kMaxLaunchViews, cnt = std::min(kMaxLaunchViews, n - first);
        long long tiles = 0;
        for (int i = 0; i < cnt; ++i) {
            const vv_batch_view& bv = views[first + i];
            const vv_uniforms* u = &bv.u;
            if (bv.tree < 0 || bv.tree >= VV_MAX_TREES) return batch_fail(c, VV_ERR_ARG, "bad tree index");
            const DeviceTree& t = bv.ctx->trees[bv.tree];
            if (!t.nodes) return batch_fail(c, VV_ERR_STATE, "node pool not uploaded");
            const int W = u->width, H = u->height;
            if (W <= 0 || H <= 0 || W > 16384 || H > 16384) return batch_fail(c, VV_ERR_ARG, "bad viewport");
            if (u->jitter_tex_size != bv.ctx->jitter_size)
                return batch_fail(c, VV_ERR_ARG, "jitter_tex_size does not match the table");
            if (!(u->ray_step_size > 0.0f)) return batch_fail(c, VV_ERR_ARG, "ray_step_size must be > 0");
            if (u->compute_lighting) return batch_fail(c, VV_ERR_ARG, "the batched launch covers the unlit ray cast");
            for (int a = 0; a < 3; ++a)
                if (u->brick_pool_dimension[a] != (float)(bv.ctx->slots[a] * 10))
                    return batch_fail(c, VV_ERR_ARG, "brick_pool_dimension does not match the brick pool");
            BatchView& v = bp.v[i];
            std::memset(&v, 0, sizeof(v));
            v.p.u = *u;
            set_divisors(v.p);
            v.p.nodes = t.nodes;
            for (int a = 0; a < 3; ++a) {
                v.p.node_dim[a] = t.dim[a];
                v.p.slots[a] = bv.ctx->slots[a];
            }
            v.p.bricks = bv.ctx->bricks;
            v.p.cell_mask = ctx_cell_mask(bv.ctx);
            v.p.jitter = bv.ctx->d_jitter;
            v.p.color = (float4*)bv.color;
            v.p.usage = (uint4*)bv.usage;
            v.p.status = bv.ctx->d_status;
            v.p.max_iter = vv_max_iterations(u);
            v.tiles_x = (W + tw - 1) / tw;
            v.tile_begin = (int)tiles;
            tiles += (long long)v.tiles_x * ((H + th - 1) / th);
            if (tiles > 0x7FFFFFFFLL) return batch_fail(c, VV_ERR_ARG, "batch has too many tiles");
        }
        bp.n = cnt;
        bp.total_tiles = (int)tiles;
        unsigned* counter = (unsigned*)((char*)c->d_batch + (size_t)k * 16);
        VV_CUDA(c, cudaMemsetAsync(counter, 0, sizeof(unsigned), c->stream));
        const long long want = (long long)sms * per_sm;
        const int grid = (int)std::max(1LL, std::min(want, tiles));
        kern<<<grid, tw * th, 0, c->stream>>>(bp, counter);
        VV_CUDA(c, cudaGetLastError());
    }
    return VV_OK;
}

}  // namespace vv

using namespace vv;

extern "C" {

int32_t vv_batch_variants(vv_batch_config* out, int32_t cap) {
    for (int i = 0; i < kNumVariants && out && i < cap; ++i) {
        out[i].tile_w = kVariants[i].tw;
        out[i].tile_h = kVariants[i].th;
        out[i].steps = kVariants[i].steps;
        out[i].ctas_per_sm = 0;
    }
    return kNumVariants;
}

int vv_render_batch(vv_ctx* c, const vv_batch_view* views, int32_t n, const vv_batch_config* cfg) {
    return batch_launch(c, views, n, cfg);
}

int vv_batch_autotune(vv_ctx* c, const vv_batch_view* views, int32_t n, int32_t reps, vv_batch_config* best,
                      float* ms) {
    if (!c || !views || n <= 0 || !best || reps <= 0) return batch_fail(c, VV_ERR_ARG, "bad autotune arguments");
    cudaSetDevice(c->device);
    if (stream_capturing(c->stream)) return batch_fail(c, VV_ERR_STATE, "cannot autotune inside a stream capture");
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    VV_CUDA(c, cudaEventCreate(&e0));
    VV_CUDA(c, cudaEventCreate(&e1));
    float best_ms = 0.0f;
    int best_i = -1, rc = VV_OK;
    for (int i = 0; i < kNumVariants; ++i) {
        vv_batch_config cfg{kVariants[i].tw, kVariants[i].th, kVariants[i].steps, 0};
        rc = batch_launch(c, views, n, &cfg);
        if (rc) break;
        cudaEventRecord(e0, c->stream);
        for (int r = 0; r < reps && !rc; ++r) rc = batch_launch(c, views, n, &cfg);
        if (rc) break;
        cudaEventRecord(e1, c->stream);
        if (cudaEventSynchronize(e1) != cudaSuccess) {
            rc = batch_fail(c, VV_ERR_CUDA, "autotune synchronize failed");
            break;
        }
        float t = 0.0f;
        cudaEventElapsedTime(&t, e0, e1);
        t /= (float)reps;
        if (ms) ms[i] = t;
        if (best_i < 0 || t < best_ms) {
            best_ms = t;
            best_i = i;
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (rc) return rc;
    best->tile_w = kVariants[best_i].tw;
    best->tile_h = kVariants[best_i].th;
    best->steps = kVariants[best_i].steps;
    best->ctas_per_sm = 0;
    return VV_OK;
}

}  // extern "C"
