// ctx.cu - device context, pools and the render entry point of the C ABI.
#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "compact.h"
#include "ctx.h"
#include "dxt.h"
#include "cellmask.cuh"
#include "kernels.cuh"

using namespace vv;

namespace {

thread_local std::string g_global_error;

int fail(vv_ctx* c, int code, const std::string& msg) {
    if (c) c->err = msg;
    else g_global_error = msg;
    return code;
}

int cuda_fail(vv_ctx* c, cudaError_t e, const char* where) {
    return fail(c, VV_ERR_CUDA, std::string(where) + ": " + cudaGetErrorString(e));
}

#define VV_CUDA(c, expr)                                  \
    do {                                                  \
        cudaError_t e_ = (expr);                          \
        if (e_ != cudaSuccess) return cuda_fail(c, e_, #expr); \
    } while (0)

// Bytes of one stored brick (slot) of a pool in `fmt`; 0 for a format the
// brick pool (grad false) or the gradient pool (grad true) cannot hold.
size_t fmt_brick_bytes(int fmt, bool grad) {
    switch (fmt) {
        case VV_FMT_RGBA8: return 4u * VV_BRICK_TEXELS;
        case VV_FMT_FP16: return grad ? 0u : 8u * VV_BRICK_TEXELS;
        case VV_FMT_BF16: return grad ? 0u : 8u * VV_BRICK_TEXELS;
        case VV_FMT_FP32: return 16u * VV_BRICK_TEXELS;
        case VV_FMT_DXT5: return grad ? 0u : (size_t)dxt::kDxt5SlotBytes;
        case VV_FMT_DXT1: return grad ? (size_t)dxt::kDxt1SlotBytes : 0u;
        default: return 0;
    }
}

// Grow a device buffer to at least `bytes`.
cudaError_t launch_raycast_any(vv_ctx* c, const RaycastParams& p) { return launch_raycast(c->fmt, p, c->stream); }

// Grow a device buffer to at least `bytes` (geometrically, so that a run of
// slowly growing requests does not re-allocate every call).
int ensure(vv_ctx* c, void** ptr, size_t* cap, size_t bytes, const char* what) {
    if (*cap >= bytes && *ptr) return VV_OK;
    const size_t grown = *cap * 2;
    if (*ptr) cudaFree(*ptr);
    *ptr = nullptr;
    *cap = 0;
    size_t want = std::max(std::max(bytes, grown), (size_t)256);
    cudaError_t e = cudaMalloc(ptr, want);
    if (e != cudaSuccess) {
        *ptr = nullptr;
        return fail(c, VV_ERR_OOM, std::string("cudaMalloc ") + what + ": " + cudaGetErrorString(e));
    }
    *cap = want;
    return VV_OK;
}

int ensure_host(vv_ctx* c, void** ptr, size_t* cap, size_t bytes) {
    if (*cap >= bytes && *ptr) return VV_OK;
    const size_t grown = *cap * 2;
    if (*ptr) cudaFreeHost(*ptr);
    *ptr = nullptr;
    *cap = 0;
    size_t want = std::max(std::max(bytes, grown), (size_t)4096);
    cudaError_t e = cudaMallocHost(ptr, want);
    if (e != cudaSuccess) {
        *ptr = nullptr;
        return fail(c, VV_ERR_OOM, std::string("cudaMallocHost: ") + cudaGetErrorString(e));
    }
    *cap = want;
    return VV_OK;
}

}  // namespace

namespace vv {
int ctx_fail(vv_ctx* c, int code, const std::string& msg) { return fail(c, code, msg); }
int ctx_ensure(vv_ctx* c, void** ptr, size_t* cap, size_t bytes, const char* what) {
    return ensure(c, ptr, cap, bytes, what);
}
int ctx_ensure_host(vv_ctx* c, void** ptr, size_t* cap, size_t bytes) { return ensure_host(c, ptr, cap, bytes); }
const uint32_t* ctx_cell_mask(const vv_ctx* c) { return c->cell_mask_valid ? c->cell_mask : nullptr; }
uint32_t* ctx_cell_mask_rw(vv_ctx* c) { return c->cell_mask_valid ? c->cell_mask : nullptr; }
}  // namespace vv

namespace {

// Cell masks sized for the pool's current slots (contents not yet valid).
int alloc_cell_masks(vv_ctx* c) {
    c->cell_mask_valid = false;
    if (c->cell_mask && c->cell_mask_slots == c->total_slots) return VV_OK;
    if (c->cell_mask) {
        VV_CUDA(c, cudaStreamSynchronize(c->stream));
        cudaFree(c->cell_mask);
        c->cell_mask = nullptr;
        c->cell_mask_slots = 0;
    }
    const size_t bytes = (size_t)c->total_slots * vv::kCellMaskWords * sizeof(uint32_t);
    if (cudaMalloc((void**)&c->cell_mask, bytes) != cudaSuccess) {
        c->cell_mask = nullptr;
        return fail(c, VV_ERR_OOM, "cudaMalloc cell masks");
    }
    c->cell_mask_slots = c->total_slots;
    return VV_OK;
}

// Every slot's mask from the pool's current contents.
int rebuild_cell_masks(vv_ctx* c) {
    int rc = alloc_cell_masks(c);
    if (rc) return rc;
    VV_CUDA(c, vv::launch_cell_masks(nullptr, c->total_slots, c->bricks, c->fmt, c->total_slots, c->cell_mask,
                                     c->stream));
    c->cell_mask_valid = true;
    return VV_OK;
}

}  // namespace

extern "C" {

int vv_abi_version(void) { return VV_ABI_VERSION; }

const char* vv_status_string(int s) {
    switch (s) {
        case VV_OK: return "ok";
        case VV_ERR_ARG: return "invalid argument";
        case VV_ERR_OOM: return "out of memory";
        case VV_ERR_CUDA: return "CUDA error";
        case VV_ERR_TIMEOUT: return "device loop bound reached";
        case VV_ERR_BOUNDS: return "device index out of bounds";
        case VV_ERR_STATE: return "call out of order";
        case VV_ERR_NODEV: return "no CUDA device";
        case VV_ERR_IO: return "file missing, unreadable or malformed";
        default: return "unknown status";
    }
}

int vv_ctx_create(const vv_params* params, vv_ctx** out) {
    if (!out) return fail(nullptr, VV_ERR_ARG, "out is NULL");
    *out = nullptr;
    int n = 0;
    cudaError_t e = cudaGetDeviceCount(&n);
    if (e != cudaSuccess || n == 0) return fail(nullptr, VV_ERR_NODEV, "no CUDA device available");
    int dev = params ? params->device : 0;
    if (dev < 0 || dev >= n) return fail(nullptr, VV_ERR_ARG, "device ordinal out of range");
    e = cudaSetDevice(dev);
    if (e != cudaSuccess) return fail(nullptr, VV_ERR_CUDA, cudaGetErrorString(e));
    vv_ctx* c = new vv_ctx();
    c->device = dev;
    e = cudaMalloc(&c->d_status, sizeof(int));
    if (e != cudaSuccess) {
        delete c;
        return fail(nullptr, VV_ERR_OOM, "cudaMalloc status word");
    }
    cudaMemset(c->d_status, 0, sizeof(int));
    // default jitter: constant 128 (1/2 step) until the caller sets a table
    std::vector<uint8_t> jit(32 * 32, 128);
    if (cudaMalloc(&c->d_jitter, jit.size()) != cudaSuccess) {
        cudaFree(c->d_status);
        delete c;
        return fail(nullptr, VV_ERR_OOM, "cudaMalloc jitter");
    }
    cudaMemcpy(c->d_jitter, jit.data(), jit.size(), cudaMemcpyHostToDevice);
    c->jitter_size = 32;
    *out = c;
    return VV_OK;
}

int vv_ctx_destroy(vv_ctx* c) {
    if (!c) return VV_OK;
    cudaSetDevice(c->device);
    cudaStreamSynchronize(c->stream);
    for (auto& t : c->trees)
        if (t.nodes) cudaFree(t.nodes);
    if (c->bricks && !c->bricks_external) cudaFree(c->bricks);
    void* bufs[] = {c->d_status, c->d_jitter, c->d_usage, c->d_mask, c->d_counts, c->d_offsets,
                    c->d_up_slots, c->d_up_bricks, c->d_patches, c->d_grid_words, c->d_batch, c->grads,
                    c->cell_mask, c->d_refill_counter, c->d_spread};
    for (void* b : bufs)
        if (b) cudaFree(b);
    if (c->h_stage) cudaFreeHost(c->h_stage);
    if (c->h_batch) cudaFreeHost(c->h_batch);
    for (auto& e : c->ev)
        if (e) cudaEventDestroy(e);
    delete c;
    return VV_OK;
}

const char* vv_last_error(const vv_ctx* c) { return c ? c->err.c_str() : g_global_error.c_str(); }

int vv_ctx_set_stream(vv_ctx* c, void* s) {
    if (!c) return VV_ERR_ARG;
    c->stream = (cudaStream_t)s;
    return VV_OK;
}

int vv_ctx_synchronize(vv_ctx* c) {
    if (!c) return VV_ERR_ARG;
    cudaSetDevice(c->device);
    VV_CUDA(c, cudaStreamSynchronize(c->stream));
    return VV_OK;
}

int vv_ctx_device_status(vv_ctx* c, int32_t* status, int32_t clear) {
    if (!c || !status) return VV_ERR_ARG;
    cudaSetDevice(c->device);
    int v = 0;
    VV_CUDA(c, cudaMemcpyAsync(&v, c->d_status, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
    VV_CUDA(c, cudaStreamSynchronize(c->stream));
    *status = v;
    if (clear) VV_CUDA(c, cudaMemsetAsync(c->d_status, 0, sizeof(int), c->stream));
    return VV_OK;
}

int vv_nodepool_upload(vv_ctx* c, int32_t tree, const uint32_t* words, int32_t dx, int32_t dy, int32_t dz) {
    if (!c || !words || tree < 0 || tree >= VV_MAX_TREES) return fail(c, VV_ERR_ARG, "bad node pool arguments");
    if (dx <= 0 || dy <= 0 || dz <= 0 || (dx & 1) || (dy & 1) || (dz & 1) || dx > 1024 || dy > 1024 || dz > 1024)
        return fail(c, VV_ERR_ARG, "node pool dims must be even and <= 1024");
    cudaSetDevice(c->device);
    DeviceTree& t = c->trees[tree];
    const size_t cells = (size_t)dx * dy * dz;
    if (t.nodes && t.cells != cells) {
        cudaFree(t.nodes);
        t.nodes = nullptr;
    }
    if (!t.nodes) {
        cudaError_t e = cudaMalloc(&t.nodes, cells * sizeof(uint2));
        if (e != cudaSuccess) {
            t.nodes = nullptr;
            return fail(c, VV_ERR_OOM, "cudaMalloc node pool");
        }
    }
    t.cells = cells;
    t.dim[0] = dx;
    t.dim[1] = dy;
    t.dim[2] = dz;
    int rc = ensure(c, (void**)&c->d_grid_words, &c->grid_words_cap, cells * sizeof(uint2), "node staging");
    if (rc) return rc;
    VV_CUDA(c, cudaMemcpyAsync(c->d_grid_words, words, cells * sizeof(uint2), cudaMemcpyHostToDevice, c->stream));
    VV_CUDA(c, launch_node_upload(c->d_grid_words, t.nodes, t.dim, c->stream));
    VV_CUDA(c, cudaStreamSynchronize(c->stream));
    return VV_OK;
}

int vv_nodepool_patch(vv_ctx* c, int32_t tree, const vv_node_patch* patches, int32_t n) {
    if (!c || tree < 0 || tree >= VV_MAX_TREES || n < 0 || (n > 0 && !patches))
        return fail(c, VV_ERR_ARG, "bad patch arguments");
    DeviceTree& t = c->trees[tree];
    if (!t.nodes) return fail(c, VV_ERR_STATE, "node pool not uploaded");
    if (n == 0) return VV_OK;
    cudaSetDevice(c->device);
    const size_t bytes = (size_t)n * sizeof(vv_node_patch);
    int rc = ensure(c, (void**)&c->d_patches, &c->patches_cap, bytes, "patch staging");
    if (rc) return rc;
    rc = ensure_host(c, &c->h_stage, &c->h_stage_cap, bytes);
    if (rc) return rc;
    VV_CUDA(c, cudaStreamSynchronize(c->stream));  // staging buffer reuse
    std::memcpy(c->h_stage, patches, bytes);
    VV_CUDA(c, cudaMemcpyAsync(c->d_patches, c->h_stage, bytes, cudaMemcpyHostToDevice, c->stream));
    VV_CUDA(c, launch_node_patch(c->d_patches, n, t.nodes, t.dim, c->d_status, c->stream));
    return VV_OK;
}

int vv_nodepool_download(vv_ctx* c, int32_t tree, uint32_t* words) {
    if (!c || !words || tree < 0 || tree >= VV_MAX_TREES) return fail(c, VV_ERR_ARG, "bad arguments");
    DeviceTree& t = c->trees[tree];
    if (!t.nodes) return fail(c, VV_ERR_STATE, "node pool not uploaded");
    cudaSetDevice(c->device);
    int rc = ensure(c, (void**)&c->d_grid_words, &c->grid_words_cap, t.cells * sizeof(uint2), "node staging");
    if (rc) return rc;
    VV_CUDA(c, launch_node_download(t.nodes, c->d_grid_words, t.dim, c->stream));
    VV_CUDA(c, cudaMemcpyAsync(words, c->d_grid_words, t.cells * sizeof(uint2), cudaMemcpyDeviceToHost, c->stream));
    VV_CUDA(c, cudaStreamSynchronize(c->stream));
    return VV_OK;
}

int vv_brickpool_create(vv_ctx* c, int32_t sx, int32_t sy, int32_t sz, int32_t fmt) {
    if (!c) return VV_ERR_ARG;
    if (sx <= 0 || sy <= 0 || sz <= 0 || sx * 10 > 1023 || sy * 10 > 1023 || sz * 10 > 1023)
        return fail(c, VV_ERR_ARG, "brick pool slots per axis must be in [1,102]");
    const size_t bb = fmt_brick_bytes(fmt, false);
    if (!bb) return fail(c, VV_ERR_ARG, "unknown brick format");
    cudaSetDevice(c->device);
    if (c->bricks) {
        VV_CUDA(c, cudaStreamSynchronize(c->stream));
        if (!c->bricks_external) cudaFree(c->bricks);
        c->bricks = nullptr;
    }
    if (c->grads) {  // its slots were those of the old pool
        cudaFree(c->grads);
        c->grads = nullptr;
    }
    c->bricks_external = false;
    const long long total = (long long)sx * sy * sz;
    const size_t bytes = (size_t)total * bb;
    cudaError_t e = cudaMalloc(&c->bricks, bytes);
    if (e != cudaSuccess) {
        c->bricks = nullptr;
        return fail(c, VV_ERR_OOM, "cudaMalloc brick pool");
    }
    VV_CUDA(c, cudaMemsetAsync(c->bricks, 0, bytes, c->stream));
    c->slots[0] = sx;
    c->slots[1] = sy;
    c->slots[2] = sz;
    c->total_slots = total;
    c->fmt = fmt;
    c->brick_bytes = bb;
    c->pool_bytes = bytes;
    return rebuild_cell_masks(c);  // of the zeroed pool
}

int vv_brickpool_update_cell_masks(vv_ctx* c) {
    if (!c) return VV_ERR_ARG;
    if (!c->bricks) return fail(c, VV_ERR_STATE, "brick pool not created");
    cudaSetDevice(c->device);
    return rebuild_cell_masks(c);
}

int vv_brickpool_download_cell_masks(vv_ctx* c, uint32_t* words) {
    if (!c || !words) return VV_ERR_ARG;
    if (!c->bricks || !c->cell_mask_valid) return fail(c, VV_ERR_STATE, "cell masks not valid");
    cudaSetDevice(c->device);
    VV_CUDA(c, cudaMemcpyAsync(words, c->cell_mask, (size_t)c->total_slots * kCellMaskWords * sizeof(uint32_t),
                               cudaMemcpyDeviceToHost, c->stream));
    VV_CUDA(c, cudaStreamSynchronize(c->stream));
    return VV_OK;
}

int vv_upload_bricks_device(vv_ctx* c, const uint32_t* slots_dev, int32_t n, const void* texels_dev) {
    if (!c || n < 0 || (n > 0 && (!slots_dev || !texels_dev))) return fail(c, VV_ERR_ARG, "bad upload arguments");
    if (!c->bricks) return fail(c, VV_ERR_STATE, "brick pool not created");
    cudaSetDevice(c->device);
    VV_CUDA(c, launch_brick_scatter(slots_dev, n, texels_dev, c->bricks, c->brick_bytes, c->total_slots,
                                    c->d_status, c->stream));
    if (c->cell_mask_valid)
        VV_CUDA(c, launch_cell_masks(slots_dev, n, c->bricks, c->fmt, c->total_slots, c->cell_mask, c->stream));
    return VV_OK;
}

int vv_upload_bricks(vv_ctx* c, const uint32_t* slots, int32_t n, const void* texels) {
    if (!c || n < 0 || (n > 0 && (!slots || !texels))) return fail(c, VV_ERR_ARG, "bad upload arguments");
    if (!c->bricks) return fail(c, VV_ERR_STATE, "brick pool not created");
    if (n == 0) return VV_OK;
    cudaSetDevice(c->device);
    const size_t bb = (size_t)n * c->brick_bytes, sb = (size_t)n * sizeof(uint32_t);
    int rc = ensure(c, &c->d_up_bricks, &c->up_bricks_cap, bb, "brick staging");
    if (rc) return rc;
    rc = ensure(c, (void**)&c->d_up_slots, &c->up_slots_cap, sb, "slot staging");
    if (rc) return rc;
    VV_CUDA(c, cudaMemcpyAsync(c->d_up_bricks, texels, bb, cudaMemcpyHostToDevice, c->stream));
    VV_CUDA(c, cudaMemcpyAsync(c->d_up_slots, slots, sb, cudaMemcpyHostToDevice, c->stream));
    VV_CUDA(c, launch_brick_scatter(c->d_up_slots, n, c->d_up_bricks, c->bricks, c->brick_bytes, c->total_slots,
                                    c->d_status, c->stream));
    if (c->cell_mask_valid)
        VV_CUDA(c, launch_cell_masks(c->d_up_slots, n, c->bricks, c->fmt, c->total_slots, c->cell_mask, c->stream));
    // The caller's host buffers may be pageable and reused right after return.
    VV_CUDA(c, cudaStreamSynchronize(c->stream));
    return VV_OK;
}

int vv_gradpool_create(vv_ctx* c, int32_t fmt) {
    if (!c) return VV_ERR_ARG;
    if (!fmt_brick_bytes(fmt, true)) return fail(c, VV_ERR_ARG, "gradient pool format: FP32, RGBA8 or DXT1");
    if (!c->bricks) return fail(c, VV_ERR_STATE, "create the brick pool first");
    cudaSetDevice(c->device);
    if (c->grads) {
        VV_CUDA(c, cudaStreamSynchronize(c->stream));
        cudaFree(c->grads);
        c->grads = nullptr;
    }
    const size_t gb = fmt_brick_bytes(fmt, true);
    const size_t bytes = (size_t)c->total_slots * gb;
    cudaError_t e = cudaMalloc(&c->grads, bytes);
    if (e != cudaSuccess) {
        c->grads = nullptr;
        return fail(c, VV_ERR_OOM, "cudaMalloc gradient pool");
    }
    VV_CUDA(c, cudaMemsetAsync(c->grads, 0, bytes, c->stream));
    c->grad_fmt = fmt;
    c->grad_brick_bytes = gb;
    c->grad_pool_bytes = bytes;
    return VV_OK;
}

int vv_upload_gradients(vv_ctx* c, const uint32_t* slots, int32_t n, const void* texels) {
    if (!c || n < 0 || (n > 0 && (!slots || !texels))) return fail(c, VV_ERR_ARG, "bad upload arguments");
    if (!c->grads) return fail(c, VV_ERR_STATE, "gradient pool not created");
    if (n == 0) return VV_OK;
    cudaSetDevice(c->device);
    const size_t bb = (size_t)n * c->grad_brick_bytes, sb = (size_t)n * sizeof(uint32_t);
    int rc = ensure(c, &c->d_up_bricks, &c->up_bricks_cap, bb, "gradient staging");
    if (rc) return rc;
    rc = ensure(c, (void**)&c->d_up_slots, &c->up_slots_cap, sb, "slot staging");
    if (rc) return rc;
    VV_CUDA(c, cudaMemcpyAsync(c->d_up_bricks, texels, bb, cudaMemcpyHostToDevice, c->stream));
    VV_CUDA(c, cudaMemcpyAsync(c->d_up_slots, slots, sb, cudaMemcpyHostToDevice, c->stream));
    VV_CUDA(c, launch_brick_scatter(c->d_up_slots, n, c->d_up_bricks, c->grads, c->grad_brick_bytes, c->total_slots,
                                    c->d_status, c->stream));
    VV_CUDA(c, cudaStreamSynchronize(c->stream));
    return VV_OK;
}

int vv_gradpool_download(vv_ctx* c, void* texels) {
    if (!c || !texels) return VV_ERR_ARG;
    if (!c->grads) return fail(c, VV_ERR_STATE, "gradient pool not created");
    cudaSetDevice(c->device);
    VV_CUDA(c, cudaMemcpyAsync(texels, c->grads, c->grad_pool_bytes, cudaMemcpyDeviceToHost, c->stream));
    VV_CUDA(c, cudaStreamSynchronize(c->stream));
    return VV_OK;
}

int vv_brickpool_download(vv_ctx* c, void* texels) {
    if (!c || !texels) return VV_ERR_ARG;
    if (!c->bricks) return fail(c, VV_ERR_STATE, "brick pool not created");
    cudaSetDevice(c->device);
    VV_CUDA(c, cudaMemcpyAsync(texels, c->bricks, c->pool_bytes, cudaMemcpyDeviceToHost, c->stream));
    VV_CUDA(c, cudaStreamSynchronize(c->stream));
    return VV_OK;
}

int vv_brickpool_attach(vv_ctx* c, void* texels, int32_t sx, int32_t sy, int32_t sz, int32_t fmt) {
    if (!c || !texels) return fail(c, VV_ERR_ARG, "bad attach arguments");
    if (sx <= 0 || sy <= 0 || sz <= 0 || sx * 10 > 1023 || sy * 10 > 1023 || sz * 10 > 1023)
        return fail(c, VV_ERR_ARG, "brick pool slots per axis must be in [1,102]");
    const size_t bb = fmt_brick_bytes(fmt, false);
    if (!bb) return fail(c, VV_ERR_ARG, "unknown brick format");
    if (((uintptr_t)texels & 15u) != 0) return fail(c, VV_ERR_ARG, "attached pool must be 16-byte aligned");
    cudaSetDevice(c->device);
    // Launches already queued hold the old pointer by value; only an owned
    // pool has to outlive them before it is freed.
    if (c->bricks && !c->bricks_external) {
        VV_CUDA(c, cudaStreamSynchronize(c->stream));
        cudaFree(c->bricks);
    }
    c->bricks = texels;
    c->bricks_external = true;
    c->slots[0] = sx;
    c->slots[1] = sy;
    c->slots[2] = sz;
    c->total_slots = (long long)sx * sy * sz;
    c->fmt = fmt;
    c->brick_bytes = bb;
    c->pool_bytes = (size_t)c->total_slots * bb;
    // the caller writes this memory: no empty-cell skipping until
    // vv_brickpool_update_cell_masks
    return alloc_cell_masks(c);
}

size_t vv_ckpt_bytes(int32_t width, int32_t height, int32_t per_ray) {
    if (width <= 0 || height <= 0 || per_ray <= 0) return 0;
    return ckpt_bytes(width, height, per_ray);
}

// Shared set-up of the differentiable passes.
static int diff_params(vv_ctx* c, int32_t tree, const vv_uniforms* u, RaycastParams& p) {
    if (!c || !u || tree < 0 || tree >= VV_MAX_TREES) return fail(c, VV_ERR_ARG, "bad arguments");
    const DeviceTree& t = c->trees[tree];
    if (!t.nodes || !c->bricks) return fail(c, VV_ERR_STATE, "pools not ready");
    if (u->width <= 0 || u->height <= 0) return fail(c, VV_ERR_ARG, "bad viewport");
    if (u->jitter_tex_size != c->jitter_size) return fail(c, VV_ERR_ARG, "jitter_tex_size does not match the table");
    for (int a = 0; a < 3; ++a)
        if (u->brick_pool_dimension[a] != (float)(c->slots[a] * 10))
            return fail(c, VV_ERR_ARG, "brick_pool_dimension does not match the brick pool");
    if (u->compute_lighting) return fail(c, VV_ERR_ARG, "the adjoint covers the unlit ray cast only");
    if (c->fmt == VV_FMT_DXT5) return fail(c, VV_ERR_ARG, "the adjoint needs an uncompressed brick pool");
    std::memset(&p, 0, sizeof(p));
    p.u = *u;
    set_divisors(p);
    p.nodes = t.nodes;
    for (int a = 0; a < 3; ++a) {
        p.node_dim[a] = t.dim[a];
        p.slots[a] = c->slots[a];
    }
    p.bricks = c->bricks;
    p.cell_mask = ctx_cell_mask(c);
    p.jitter = c->d_jitter;
    p.status = c->d_status;
    p.max_iter = vv_max_iterations(u);
    return VV_OK;
}

int vv_render_forward_ckpt(vv_ctx* c, int32_t tree, const vv_uniforms* u, float* color, void* ckpt,
                           int32_t per_ray) {
    RaycastParams p;
    int rc = diff_params(c, tree, u, p);
    if (rc) return rc;
    if (!ckpt || per_ray <= 0) return fail(c, VV_ERR_ARG, "checkpoint buffer required");
    cudaSetDevice(c->device);
    p.color = (float4*)color;
    VV_CUDA(c, launch_forward_ckpt(c->fmt, p, ckpt, per_ray, c->stream));
    return VV_OK;
}

int vv_backward(vv_ctx* c, int32_t tree, const vv_uniforms* u, const float* dl_dcolor, const void* ckpt,
                int32_t per_ray, float* grad_texels) {
    vv_grad_desc g;
    std::memset(&g, 0, sizeof(g));
    g.grad = grad_texels;
    return vv_backward_ex(c, tree, u, dl_dcolor, ckpt, per_ray, &g);
}

int vv_backward_ex(vv_ctx* c, int32_t tree, const vv_uniforms* u, const float* dl_dcolor, const void* ckpt,
                   int32_t per_ray, const vv_grad_desc* g) {
    RaycastParams p;
    int rc = diff_params(c, tree, u, p);
    if (rc) return rc;
    if (!ckpt || per_ray <= 0 || !dl_dcolor || !g || !g->grad) return fail(c, VV_ERR_ARG, "bad backward buffers");
    if ((g->flags & ~(VV_GRAD_F64 | VV_GRAD_WARP_SUM | VV_GRAD_SPREAD | VV_GRAD_SPREAD_KEEP)) != 0)
        return fail(c, VV_ERR_ARG, "unknown gradient flags");
    const bool spread = (g->flags & VV_GRAD_SPREAD) != 0;
    const bool keep = (g->flags & VV_GRAD_SPREAD_KEEP) != 0;
    if ((spread && (g->flags & VV_GRAD_F64)) || (keep && !spread))
        return fail(c, VV_ERR_ARG, "VV_GRAD_SPREAD needs binary32 rows; VV_GRAD_SPREAD_KEEP needs VV_GRAD_SPREAD");
    const uintptr_t align = (g->flags & VV_GRAD_F64) ? 32u : 16u;
    if (((uintptr_t)g->grad & (align - 1)) != 0 || ((uintptr_t)dl_dcolor & 15u) != 0)
        return fail(c, VV_ERR_ARG, "gradient buffers must be aligned to a texel (16 bytes, 32 for binary64)");
    if (g->slot_map && (!g->rows_used || g->rows_cap <= 0))
        return fail(c, VV_ERR_ARG, "a slot map needs a row counter and a row capacity");
    cudaSetDevice(c->device);
    GradTarget gt;
    gt.grad = g->grad;
    gt.f64 = (g->flags & VV_GRAD_F64) ? 1 : 0;
    gt.warp_sum = (g->flags & VV_GRAD_WARP_SUM) ? 1 : 0;
    gt.slot_map = g->slot_map;
    gt.rows_used = g->rows_used;
    gt.rows_cap = g->slot_map ? g->rows_cap : 0;
    gt.copies = 1;
    gt.spread = nullptr;
    gt.spread_rows = 0;
    if (spread) {
        const long long rows = g->slot_map ? (long long)g->rows_cap : c->total_slots;
        if (rows <= 0 || rows > INT32_MAX) return fail(c, VV_ERR_ARG, "no rows to spread over");
        if (c->spread_rows_kept && c->spread_rows_kept != rows)
            return fail(c, VV_ERR_ARG, "kept gradient copies have another row count");
        const size_t need = (size_t)(VV_GRAD_SPREAD_COPIES - 1) * (size_t)rows * 1000u;
        if (c->spread_elems < need) {
            // grown by half again at least, so that row capacities that vary
            // from call to call settle after a few calls
            const size_t want = std::max(need, c->spread_elems + c->spread_elems / 2);
            if (c->d_spread) cudaFree(c->d_spread);
            c->d_spread = nullptr;
            c->spread_elems = 0;
            if (cudaMalloc((void**)&c->d_spread, want * sizeof(float4)) != cudaSuccess) {
                c->d_spread = nullptr;
                return fail(c, VV_ERR_OOM, "cudaMalloc gradient copies");
            }
            // zero once: the reduction re-zeroes what the adjoint wrote
            VV_CUDA(c, cudaMemsetAsync(c->d_spread, 0, want * sizeof(float4), c->stream));
            c->spread_elems = want;
        }
        gt.copies = VV_GRAD_SPREAD_COPIES;
        gt.spread = c->d_spread;
        gt.spread_rows = (int)rows;
    }
    VV_CUDA(c, launch_backward(c->fmt, p, ckpt, per_ray, (const float4*)dl_dcolor, gt, c->stream));
    if (keep) {
        c->spread_rows_kept = gt.spread_rows;
    } else {
        c->spread_rows_kept = 0;
        VV_CUDA(c, launch_spread_reduce(gt, c->stream));
    }
    return VV_OK;
}

int vv_brickpool_info(const vv_ctx* c, int32_t slots[3], int32_t* fmt) {
    if (!c || !slots) return VV_ERR_ARG;
    for (int a = 0; a < 3; ++a) slots[a] = c->bricks ? c->slots[a] : 0;
    if (fmt) *fmt = c->fmt;
    return VV_OK;
}

int vv_nodepool_info(const vv_ctx* c, int32_t tree, int32_t dims[3]) {
    if (!c || !dims || tree < 0 || tree >= VV_MAX_TREES) return VV_ERR_ARG;
    for (int a = 0; a < 3; ++a) dims[a] = c->trees[tree].nodes ? c->trees[tree].dim[a] : 0;
    return VV_OK;
}

int vv_brickpool_device_ptr(vv_ctx* c, void** ptr, size_t* bytes) {
    if (!c || !ptr) return VV_ERR_ARG;
    *ptr = c->bricks;
    if (bytes) *bytes = c->pool_bytes;
    return VV_OK;
}

int vv_set_jitter(vv_ctx* c, const uint8_t* table, int32_t size) {
    if (!c || !table || size <= 0 || size > 256) return fail(c, VV_ERR_ARG, "bad jitter table");
    cudaSetDevice(c->device);
    VV_CUDA(c, cudaStreamSynchronize(c->stream));
    if (c->d_jitter) cudaFree(c->d_jitter);
    c->d_jitter = nullptr;
    VV_CUDA(c, cudaMalloc(&c->d_jitter, (size_t)size * size));
    VV_CUDA(c, cudaMemcpy(c->d_jitter, table, (size_t)size * size, cudaMemcpyHostToDevice));
    c->jitter_size = size;
    return VV_OK;
}

int vv_render(vv_ctx* c, int32_t tree, const vv_uniforms* u, const vv_frame_out* out) {
    if (!c || !u || !out || tree < 0 || tree >= VV_MAX_TREES) return fail(c, VV_ERR_ARG, "bad render arguments");
    const DeviceTree& t = c->trees[tree];
    if (!t.nodes) return fail(c, VV_ERR_STATE, "node pool not uploaded");
    if (!c->bricks) return fail(c, VV_ERR_STATE, "brick pool not created");
    const int W = u->width, H = u->height;
    if (W <= 0 || H <= 0 || W > 16384 || H > 16384) return fail(c, VV_ERR_ARG, "bad viewport");
    if (u->jitter_tex_size != c->jitter_size) return fail(c, VV_ERR_ARG, "jitter_tex_size does not match the table");
    if (!(u->ray_step_size > 0.0f)) return fail(c, VV_ERR_ARG, "ray_step_size must be > 0");
    for (int a = 0; a < 3; ++a)
        if (u->brick_pool_dimension[a] != (float)(c->slots[a] * 10))
            return fail(c, VV_ERR_ARG, "brick_pool_dimension does not match the brick pool");
    cudaSetDevice(c->device);
    const size_t npix = (size_t)W * H;
    const int passes = out->passes ? out->passes : VV_PASS_ALL;

    uint4* usage = (uint4*)out->usage;
    if (!usage && (passes & (VV_PASS_SELECT | VV_PASS_COMPACT))) {
        int rc = ensure(c, (void**)&c->d_usage, &c->usage_cap, npix * 48, "usage scratch");
        if (rc) return rc;
        usage = (uint4*)c->d_usage;
    }
    c->timed = c->profiling;
    if (c->profiling) VV_CUDA(c, cudaEventRecord(c->ev[0], c->stream));
    if (passes & VV_PASS_RAYCAST) {
        RaycastParams p;
        std::memset(&p, 0, sizeof(p));
        p.u = *u;
        set_divisors(p);
        p.nodes = t.nodes;
        p.node_dim[0] = t.dim[0];
        p.node_dim[1] = t.dim[1];
        p.node_dim[2] = t.dim[2];
        p.bricks = c->bricks;
        p.cell_mask = ctx_cell_mask(c);
        p.slots[0] = c->slots[0];
        p.slots[1] = c->slots[1];
        p.slots[2] = c->slots[2];
        p.jitter = c->d_jitter;
        p.color = (float4*)out->color;
        p.color8 = (out->passes & VV_PASS_COLOR_RGBA8) ? 1 : 0;
        p.usage = usage;
        p.status = c->d_status;
        p.max_iter = vv_max_iterations(u);
        if (u->compute_lighting) {
            if (!c->grads) return fail(c, VV_ERR_STATE, "lighting needs a gradient pool (vv_gradpool_create)");
            p.grads = c->grads;
            p.grad_fmt = c->grad_fmt;
        }
        if (c->raycast_mode == VV_RAYCAST_REFILL && !u->compute_lighting) {
            if (!c->d_refill_counter) VV_CUDA(c, cudaMalloc(&c->d_refill_counter, sizeof(unsigned int)));
            VV_CUDA(c, launch_raycast_refill(c->fmt, p, c->d_refill_counter, c->stream));
        } else if (c->raycast_mode == VV_RAYCAST_STAGED && !u->compute_lighting && c->fmt == VV_FMT_RGBA8) {
            VV_CUDA(c, launch_raycast_staged(c->fmt, p, c->stream));
        } else {
            VV_CUDA(c, launch_raycast_any(c, p));
        }
    }
    if (c->profiling) VV_CUDA(c, cudaEventRecord(c->ev[1], c->stream));
    if (!(passes & (VV_PASS_SELECT | VV_PASS_COMPACT))) {
        if (c->profiling) VV_CUDA(c, cudaEventRecord(c->ev[2], c->stream));
        return VV_OK;
    }

    // level dims of the histopyramid (GigaVoxelsRenderer.cpp:1967-2046)
    CompactParams cp;
    std::memset(&cp, 0, sizeof(cp));
    cp.width = W;
    cp.height = H;
    {
        int w = W, h = H, l = 0;
        long long off = 0;
        while (true) {
            if (l >= 24) return fail(c, VV_ERR_ARG, "viewport too large for the pyramid");
            cp.level_w[l] = w;
            cp.level_h[l] = h;
            cp.level_off[l] = off;
            off += (long long)w * h;
            ++l;
            if (w == 1 && h == 1) break;
            if (w != 1) w >>= 1;
            if (h != 1) h >>= 1;
        }
        cp.levels = l;
        int rc = ensure(c, (void**)&c->d_counts, &c->counts_cap, (size_t)off * 4, "pyramid counts");
        if (rc) return rc;
        rc = ensure(c, (void**)&c->d_offsets, &c->offsets_cap, (size_t)off * 4, "pyramid offsets");
        if (rc) return rc;
    }
    uint32_t* mask = out->mask;
    if (!mask) {
        int rc = ensure(c, (void**)&c->d_mask, &c->mask_cap, npix * 4, "mask scratch");
        if (rc) return rc;
        mask = c->d_mask;
    }
    if (!(passes & VV_PASS_COMPACT)) {
        VV_CUDA(c, launch_select(usage, mask, c->d_counts, W, H, c->stream));
        if (c->profiling) VV_CUDA(c, cudaEventRecord(c->ev[2], c->stream));
        return VV_OK;
    }
    cp.counts = c->d_counts;
    cp.offsets = c->d_offsets;
    cp.usage = usage;
    cp.mask = mask;
    cp.requests = out->requests;
    cp.request_count = out->request_count;
    cp.cap = out->requests ? out->request_cap : 0;
    cp.max_push = out->compress_max_push > 0 ? out->compress_max_push : 4;
    // three launches where the frame allows (compact.cu), else one per level
    const cudaError_t fe = c->per_level_compaction ? cudaErrorNotSupported : launch_compact_fused(cp, mask, c->stream);
    if (fe == cudaErrorNotSupported) {
        VV_CUDA(c, launch_select(usage, mask, c->d_counts, W, H, c->stream));
        VV_CUDA(c, launch_compact(cp, c->stream));
    } else {
        VV_CUDA(c, fe);
    }
    if (c->profiling) VV_CUDA(c, cudaEventRecord(c->ev[2], c->stream));
    return VV_OK;
}

int vv_ctx_set_compaction(vv_ctx* c, int32_t mode) {
    if (!c || (mode != VV_COMPACT_FUSED && mode != VV_COMPACT_PER_LEVEL))
        return fail(c, VV_ERR_ARG, "unknown compaction mode");
    c->per_level_compaction = mode == VV_COMPACT_PER_LEVEL;
    return VV_OK;
}

int vv_ctx_set_raycast_mode(vv_ctx* c, int32_t mode) {
    if (!c || (mode != VV_RAYCAST_TILES && mode != VV_RAYCAST_REFILL && mode != VV_RAYCAST_STAGED))
        return fail(c, VV_ERR_ARG, "unknown ray-cast mode");
    if (mode == VV_RAYCAST_STAGED && c->fmt != VV_FMT_RGBA8)
        return fail(c, VV_ERR_ARG, "brick staging needs an RGBA8 brick pool");
    c->raycast_mode = mode;
    return VV_OK;
}

int vv_ctx_set_profiling(vv_ctx* c, int32_t on) {
    if (!c) return VV_ERR_ARG;
    cudaSetDevice(c->device);
    if (on && !c->ev[0])
        for (auto& e : c->ev) VV_CUDA(c, cudaEventCreate(&e));
    c->profiling = on != 0;
    c->timed = false;
    return VV_OK;
}

int vv_ctx_last_times(vv_ctx* c, float* raycast_ms, float* compact_ms) {
    if (!c) return VV_ERR_ARG;
    if (!c->timed) return fail(c, VV_ERR_STATE, "no profiled draw");
    cudaSetDevice(c->device);
    VV_CUDA(c, cudaEventSynchronize(c->ev[2]));
    float a = 0.f, b = 0.f;
    VV_CUDA(c, cudaEventElapsedTime(&a, c->ev[0], c->ev[1]));
    VV_CUDA(c, cudaEventElapsedTime(&b, c->ev[1], c->ev[2]));
    if (raycast_ms) *raycast_ms = a;
    if (compact_ms) *compact_ms = b;
    return VV_OK;
}

int vv_measure_footprint_views(vv_ctx* c, int32_t tree, const vv_uniforms* us, int32_t n, int64_t* nodes,
                               int64_t* bricks) {
    if (!c || !us || n <= 0 || tree < 0 || tree >= VV_MAX_TREES) return fail(c, VV_ERR_ARG, "bad footprint arguments");
    const DeviceTree& t = c->trees[tree];
    if (!t.nodes || !c->bricks) return fail(c, VV_ERR_STATE, "pools not ready");
    for (int32_t i = 0; i < n; ++i)
        if (us[i].jitter_tex_size != c->jitter_size)
            return fail(c, VV_ERR_ARG, "jitter_tex_size does not match the table");
    cudaSetDevice(c->device);
    const size_t nwords = (t.cells + 31) / 32, bwords = ((size_t)c->total_slots + 31) / 32;
    uint32_t* bits = nullptr;
    VV_CUDA(c, cudaMalloc(&bits, (nwords + bwords) * 4));
    cudaError_t e = cudaMemsetAsync(bits, 0, (nwords + bwords) * 4, c->stream);
    // one counting ray cast per view into the same touch bitmaps: the union
    for (int32_t i = 0; i < n && e == cudaSuccess; ++i) {
        RaycastParams p;
        std::memset(&p, 0, sizeof(p));
        p.u = us[i];
        set_divisors(p);
        p.nodes = t.nodes;
        for (int a = 0; a < 3; ++a) {
            p.node_dim[a] = t.dim[a];
            p.slots[a] = c->slots[a];
        }
        p.bricks = c->bricks;
        p.jitter = c->d_jitter;
        p.status = c->d_status;
        p.max_iter = vv_max_iterations(&us[i]);
        p.u.compute_lighting = 0;  // lighting reads the same slots of the gradient pool
        p.node_touch = bits;
        p.brick_touch = bits + nwords;
        e = launch_raycast_any(c, p);
    }
    std::vector<uint32_t> h(nwords + bwords);
    if (e == cudaSuccess) e = cudaMemcpyAsync(h.data(), bits, h.size() * 4, cudaMemcpyDeviceToHost, c->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    cudaFree(bits);
    if (e != cudaSuccess) return cuda_fail(c, e, "footprint");
    int64_t nn = 0, b = 0;
    for (size_t i = 0; i < nwords; ++i) nn += __builtin_popcount(h[i]);
    for (size_t i = 0; i < bwords; ++i) b += __builtin_popcount(h[nwords + i]);
    if (nodes) *nodes = nn;
    if (bricks) *bricks = b;
    return VV_OK;
}

int vv_measure_footprint(vv_ctx* c, int32_t tree, const vv_uniforms* u, int64_t* nodes, int64_t* bricks) {
    if (!u) return fail(c, VV_ERR_ARG, "bad footprint arguments");
    return vv_measure_footprint_views(c, tree, u, 1, nodes, bricks);
}

}  // extern "C"

namespace vv {

void set_thread_error(const std::string& msg) { g_global_error = msg; }

int vv_max_iterations(const vv_uniforms* u) {
    // Every leaf segment advances the ray by at least one half-voxel step of
    // the leaf level and a descent has at most depth+1 fetches, so a ray
    // entering anywhere needs fewer than (sqrt(3) / step + 2) * (depth + 2)
    // iterations.  The bound has a factor 2 of margin.
    double segs = 1.7320508 / (double)u->ray_step_size + 2.0;
    double it = 2.0 * segs * (double)(u->oct_tree_depth_minus_one + 2) + 64.0;
    if (u->max_segments > 0) it = (double)u->max_segments;
    if (it > 2.0e9) it = 2.0e9;
    return (int)it;
}

}  // namespace vv
