// adjoint.cu - differentiable ray cast: checkpointing forward and adjoint.
//
// The forward composites  dst_{k+1} = dst_k + T_k * src_k,  T_k = 1 - dst_k.a
// (GigaVoxelsNoLighting.frag:280,354).  Its adjoint with g = dL/d dst is
//   dL/d src_k = g_{k+1} * T_k
//   g_k.rgb    = g_{k+1}.rgb,   g_k.a = g_{k+1}.a - dot(g_{k+1}, src_k)
// and a brick sample is the trilinear blend of 8 texels, so each texel gets
// its blend weight times dL/d src_k.  Walking the samples backwards needs
// T_k, which is not recoverable from the final colour once a sample is
// opaque, so the forward stores a checkpoint at the start of a leaf segment
// whenever 32 or more samples were composited since the last one; there the
// walk restarts from the root, so a checkpoint is only the ray position,
// dst, the iteration count, the sample index and the node pointer.  The
// adjoint replays each chunk from its checkpoint (in pieces of at most 64
// samples, the last piece first), keeps the samples of the piece in local
// memory and back-propagates through them in reverse.  The control flow
// (descent, step counts, early termination) is that of the forward and is
// held fixed, as any reverse-mode derivative of this shader does.
#include "raycast_common.cuh"

namespace vv {

using namespace rc;

namespace {

constexpr int kCkptEvery = 32;
constexpr int kPiece = 64;

struct Ckpt {
    float4 a;  // pos.xyz, dst.x
    float4 b;  // dst.yzw, iter (bits)
    uint4 c;   // nsamples, nptr xyz
};

struct CkptVisitor {
    Ckpt* out;
    int cap, count, last;
    int* status;
    __device__ __forceinline__ bool segment_begin(const RayState& s) {
        if ((count == 0 || s.nsamples - last >= kCkptEvery) && count < cap) {
            Ckpt c;
            c.a = make_float4(s.pos.x, s.pos.y, s.pos.z, s.dst.x);
            c.b = make_float4(s.dst.y, s.dst.z, s.dst.w, __int_as_float(s.iter));
            c.c = make_uint4((uint32_t)s.nsamples, s.nptr_x, s.nptr_y, s.nptr_z);
            out[count++] = c;
            last = s.nsamples;
        }
        return true;
    }
    __device__ __forceinline__ bool sample(int, const float4&, F3, float, int) { return true; }
    __device__ __forceinline__ void segment_end(const RayState&, bool, bool) {}
    __device__ __forceinline__ void fail(int code) { set_status(status, code); }
};

// The samples of one piece, compactly: T (the transmittance before the
// sample, negated for a constant-node sample: T > 0 or +0 for brick samples),
// the sample's alpha, r = dot(dL/dc.rgb, src.rgb) (dL/dc.rgb is constant
// along the ray) and the brick position.  24 bytes a sample.
struct ReplayVisitor {
    int first, last, n;
    float gx, gy, gz;  // dL/dc.rgb
    float T[kPiece];
    float a[kPiece];
    float r[kPiece];
    F3 bpos[kPiece];
    __device__ __forceinline__ bool segment_begin(const RayState& s) { return s.nsamples < last; }
    __device__ __forceinline__ bool sample(int kind, const float4& v, F3 b, float t, int index) {
        if (index >= first && n < kPiece) {
            T[n] = kind == kSampleBrick ? t : -t;
            a[n] = v.w;
            // the first three products of the g.a update, in its order
            r[n] = gx * v.x + gy * v.y + gz * v.z;
            bpos[n] = b;
            ++n;
        }
        return index + 1 < last;
    }
    __device__ __forceinline__ void segment_end(const RayState&, bool, bool) {}
    __device__ __forceinline__ void fail(int) {}
};

// The row of the gradient that holds `slot`: the slot itself (dense), or,
// with a slot map, the row claimed by the first sample that reaches the
// slot (-1 in the map: unclaimed; -2: being claimed; -3: no row left).
// The claiming thread never waits, so a waiting thread's bound is never
// reached on valid data; reaching it, or running out of rows, sets the
// device status and drops the contribution.
__device__ __forceinline__ int grad_row(const GradTarget& gt, uint32_t slot, int* status) {
    if (!gt.slot_map) return (int)slot;
    int* m = gt.slot_map + slot;
    int r = *(volatile int*)m;
    if (r >= 0) return r;
    if (r == -1 && atomicCAS(m, -1, -2) == -1) {
        const int nr = atomicAdd(gt.rows_used, 1);
        if (nr >= gt.rows_cap) {
            atomicExch(m, -3);
            set_status(status, VV_ERR_OOM);
            return -1;
        }
        __threadfence();
        atomicExch(m, nr);
        return nr;
    }
    for (int i = 0; i < (1 << 22); ++i) {
        r = *(volatile int*)m;
        if (r >= 0) return r;
        if (r == -3) return -1;
        __nanosleep(64);
    }
    set_status(status, VV_ERR_TIMEOUT);
    return -1;
}

// gradient element i += v (binary32 rows: one vector reduction, red.v4.f32,
// which returns nothing - atomicAdd(float4*) returns the old value and so
// holds four registers until the L2 answers - into the warp's copy of the
// rows; binary64 rows: four double atomics).
template <bool F64>
__device__ __forceinline__ void texel_atomic(const GradTarget& gt, size_t i, float4 v) {
    if (F64) {
        double* g = (double*)gt.grad + 4 * i;
        atomicAdd(g + 0, (double)v.x);
        atomicAdd(g + 1, (double)v.y);
        atomicAdd(g + 2, (double)v.z);
        atomicAdd(g + 3, (double)v.w);
    } else {
        float4* g = (float4*)gt.grad + i;
        // the warp's copy: its index in the CTA, then the CTA's column parity
        const unsigned c = ((threadIdx.x >> 5) | ((blockIdx.x & 1u) << 2)) & (unsigned)(gt.copies - 1);
        if (c) g = gt.spread + (size_t)(c - 1u) * (size_t)gt.spread_rows * 1000u + i;
        asm volatile("red.global.add.v4.f32 [%0], {%1, %2, %3, %4};" ::"l"(g), "f"(v.x), "f"(v.y), "f"(v.z),
                     "f"(v.w)
                     : "memory");
    }
}

// dL/d texel += w_j * d for the 8 taps of the sample at uvw (the addressing
// of sample_brick, clamps included: clamped taps share a texel).  The slot
// map is read once per slot change: (c_slot, c_row) is the thread's last
// slot and its row.  Taps in one slot (the usual case): WSUM groups the
// lanes whose samples lie in the same cell (one __match_any_sync a sample:
// the same 8 texels), sums each tap over the group by shuffles in lane order
// and lets the group's first lane issue the atomics; without WSUM each lane
// starts its 8 taps at a different one (fewer lanes of one instruction on
// one texel).
template <bool F64, bool WSUM>
__device__ __forceinline__ void scatter_texels(const RaycastParams& p, F3 uvw, float4 d, const GradTarget& gt,
                                               uint32_t& c_slot, int& c_row) {
    const float* N = p.u.brick_pool_dimension;
    const Axis ax = axis_taps(uvw.x, N[0], p.slots[0] * 10);
    const Axis ay = axis_taps(uvw.y, N[1], p.slots[1] * 10);
    const Axis az = axis_taps(uvw.z, N[2], p.slots[2] * 10);
    const uint32_t SX = (uint32_t)p.slots[0], SY = (uint32_t)p.slots[1];
    const int lane = (int)(threadIdx.x & 31u);
    if (ax.s0 == ax.s1 && ay.s0 == ay.s1 && az.s0 == az.s1) {
        const uint32_t slot = ((uint32_t)az.s0 * SY + (uint32_t)ay.s0) * SX + (uint32_t)ax.s0;
        if (slot != c_slot) {
            c_row = grad_row(gt, slot, p.status);
            c_slot = slot;
        }
        if (c_row < 0) return;
        const uint32_t t0 = (uint32_t)((az.l0 * 10 + ay.l0) * 10 + ax.l0);
        const uint32_t dx = (uint32_t)(ax.l1 - ax.l0), dy = (uint32_t)(10 * (ay.l1 - ay.l0)),
                       dz = (uint32_t)(100 * (az.l1 - az.l0));
        const size_t base = (size_t)c_row * 1000u + t0;
        if (WSUM) {
            const uint64_t key = ((uint64_t)(uint32_t)c_row << 16) | (t0 << 3) | (dx << 2) | ((dy ? 1u : 0u) << 1) |
                                 (dz ? 1u : 0u);
            const unsigned peers = __match_any_sync(__activemask(), key);
            const bool group = __popc(peers) > 1;
            const bool lead = lane == __ffs(peers) - 1;
#pragma unroll
            for (int t = 0; t < 8; ++t) {
                const int bx = t & 1, by = (t >> 1) & 1, bz = t >> 2;
                const float w = (bx ? ax.f : 1.0f - ax.f) * (by ? ay.f : 1.0f - ay.f) * (bz ? az.f : 1.0f - az.f);
                float4 v = make_float4(w * d.x, w * d.y, w * d.z, w * d.w);
                if (group) {
                    float4 s = make_float4(0.f, 0.f, 0.f, 0.f);
                    for (unsigned m = peers; m; m &= m - 1) {
                        const int src = __ffs(m) - 1;
                        s.x += __shfl_sync(peers, v.x, src);
                        s.y += __shfl_sync(peers, v.y, src);
                        s.z += __shfl_sync(peers, v.z, src);
                        s.w += __shfl_sync(peers, v.w, src);
                    }
                    v = s;
                }
                if (lead && (v.x != 0.f || v.y != 0.f || v.z != 0.f || v.w != 0.f))
                    texel_atomic<F64>(gt, base + (bx ? dx : 0u) + (by ? dy : 0u) + (bz ? dz : 0u), v);
            }
        } else {
#pragma unroll
            for (int q = 0; q < 8; ++q) {
                const int t = (q + lane) & 7;
                const int bx = t & 1, by = (t >> 1) & 1, bz = t >> 2;
                const float w = (bx ? ax.f : 1.0f - ax.f) * (by ? ay.f : 1.0f - ay.f) * (bz ? az.f : 1.0f - az.f);
                if (w == 0.0f) continue;
                texel_atomic<F64>(gt, base + (bx ? dx : 0u) + (by ? dy : 0u) + (bz ? dz : 0u),
                                  make_float4(w * d.x, w * d.y, w * d.z, w * d.w));
            }
        }
        return;
    }
    // taps in two or more slots
#pragma unroll 1
    for (int t = 0; t < 8; ++t) {
        const int bx = t & 1, by = (t >> 1) & 1, bz = t >> 2;
        const float w = (bx ? ax.f : 1.0f - ax.f) * (by ? ay.f : 1.0f - ay.f) * (bz ? az.f : 1.0f - az.f);
        if (w == 0.0f) continue;
        const int sx = bx ? ax.s1 : ax.s0, lx = bx ? ax.l1 : ax.l0;
        const int sy = by ? ay.s1 : ay.s0, ly = by ? ay.l1 : ay.l0;
        const int sz = bz ? az.s1 : az.s0, lz = bz ? az.l1 : az.l0;
        const uint32_t slot = ((uint32_t)sz * SY + (uint32_t)sy) * SX + (uint32_t)sx;
        if (slot != c_slot) {
            c_row = grad_row(gt, slot, p.status);
            c_slot = slot;
        }
        if (c_row < 0) continue;
        texel_atomic<F64>(gt, (size_t)c_row * 1000u + (uint32_t)((lz * 10 + ly) * 10 + lx),
                          make_float4(w * d.x, w * d.y, w * d.z, w * d.w));
    }
}

__device__ __forceinline__ void pixel_of(int& px, int& py) {
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    px = blockIdx.x * 16 + (warp & 1) * 8 + (lane & 7);
    py = blockIdx.y * 8 + (warp >> 1) * 4 + (lane >> 3);
}
// The adjoint's pixels: a CTA covers the same 16x8 pixels, each warp every
// second pixel of them in x and y, so that a warp's lanes sample fewer
// common texels at once (fewer lanes of one atomic on one address).
__device__ __forceinline__ void pixel_of_strided(int& px, int& py) {
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    px = blockIdx.x * 16 + 2 * (lane & 7) + (warp & 1);
    py = blockIdx.y * 8 + 2 * (lane >> 3) + (warp >> 1);
}

}  // namespace

// 7 resident CTAs (28 warps) per SM, at most 72 registers per thread (no
// spills): the occupancy that measured fastest for the plain ray cast
template <int FMT>
__global__ void __launch_bounds__(128, 7) forward_ckpt_kernel(const __grid_constant__ RaycastParams p, int2* hdr,
                                                           Ckpt* ckpt, int per_ray) {
    int px, py;
    pixel_of(px, py);
    const vv_uniforms& u = p.u;
    if (px >= u.width || py >= u.height) return;
    const size_t pix = (size_t)py * u.width + px;
    bool ok = true;
    const WalkConsts k = walk_consts(p, fetch_node<false>(p, 0, 0, 0, ok));
    CkptVisitor vis;
    vis.out = ckpt + pix * (size_t)per_ray;
    vis.cap = per_ray;
    vis.count = 0;
    vis.last = 0;
    vis.status = p.status;
    RayState s;
    s.dst = make_float4(0.f, 0.f, 0.f, 0.f);
    s.nsamples = 0;
    F3 pos;
    __shared__ uint2 path_w[kPathLevels][128];
    __shared__ uint32_t path_p[kPathLevels][128];
    if (ray_origin(u, k, px, py, pos) && ray_start(p, k, px, py, pos, s))
        walk<FMT, false, CkptVisitor, 1, true>(p, k, s, vis,
                                               PathSlots{&path_w[0][threadIdx.x], &path_p[0][threadIdx.x], 128, nullptr});
    if (p.color) p.color[pix] = s.dst;
    hdr[pix] = make_int2(vis.count, s.nsamples);
}

// 6 resident CTAs per SM (80 registers, fewer spills): on the paged 1080p
// frames 5.73-5.78 ms against 5.83-6.02 at 7 CTAs and 6.18-6.21 at 8 (the
// atomics' contention, not the walk's latency, bounds it).  F64: binary64
// gradient rows; WSUM: the lanes of a cell summed before the atomics
// (scatter_texels).
template <int FMT, bool F64, bool WSUM>
__global__ void __launch_bounds__(128, 6) backward_kernel(const __grid_constant__ RaycastParams p, const int2* hdr,
                                                       const Ckpt* ckpt, int per_ray, const float4* dl_dcolor,
                                                       const GradTarget gt) {
    int px, py;
    pixel_of_strided(px, py);
    const vv_uniforms& u = p.u;
    if (px >= u.width || py >= u.height) return;
    const size_t pix = (size_t)py * u.width + px;
    const int2 h = hdr[pix];
    const int C = h.x, total = h.y;
    if (C == 0 || total == 0) return;
    float4 g = dl_dcolor[pix];
    if (g.x == 0.f && g.y == 0.f && g.z == 0.f && g.w == 0.f) return;
    bool ok = true;
    const WalkConsts k = walk_consts(p, fetch_node<false>(p, 0, 0, 0, ok));
    RayState s0;
    F3 pos;
    if (!ray_origin(u, k, px, py, pos)) return;
    ray_start(p, k, px, py, pos, s0);  // direction and brick step of this ray
    const Ckpt* ck = ckpt + pix * (size_t)per_ray;
    __shared__ uint2 path_w[kPathLevels][128];
    __shared__ uint32_t path_p[kPathLevels][128];
    uint32_t c_slot = 0xFFFFFFFFu;  // the last slot scattered into and its gradient row
    int c_row = -1;
    ReplayVisitor rv;
    rv.gx = g.x;
    rv.gy = g.y;
    rv.gz = g.z;
    for (int c = C - 1; c >= 0; --c) {
        const Ckpt cc = ck[c];
        const int a = (int)cc.c.x, b = c + 1 < C ? (int)ck[c + 1].c.x : total;
        for (int m = (b - a - 1) / kPiece; m >= 0; --m) {
            RayState s = s0;
            s.pos = f3(cc.a.x, cc.a.y, cc.a.z);
            s.dst = make_float4(cc.a.w, cc.b.x, cc.b.y, cc.b.z);
            s.iter = __float_as_int(cc.b.w);
            s.nsamples = a;
            s.nptr_x = cc.c.y;
            s.nptr_y = cc.c.z;
            s.nptr_z = cc.c.w;
            rv.first = a + m * kPiece;
            rv.last = min(b, rv.first + kPiece);
            rv.n = 0;
            walk<FMT, false, ReplayVisitor, 1, true>(
                p, k, s, rv, PathSlots{&path_w[0][threadIdx.x], &path_p[0][threadIdx.x], 128, nullptr});
            for (int j = rv.n - 1; j >= 0; --j) {
                const float tj = rv.T[j];
                const float t = fabsf(tj);
                if (!(__float_as_uint(tj) >> 31))
                    scatter_texels<F64, WSUM>(p, rv.bpos[j], make_float4(g.x * t, g.y * t, g.z * t, g.w * t), gt,
                                              c_slot, c_row);
                // g.a -= dot(g, src), the products summed in the order x, y, z, w
                g.w = g.w - (rv.r[j] + g.w * rv.a[j]);
            }
        }
    }
}

// grad[e] += copy_k[e] for the extra copies k of the rows in use (all rows
// without a row counter), each copy element zeroed after it is read (the
// copies are all zero between reductions).  All loads of an element are
// issued before its stores (streaming: the copies are not read again soon).
template <int EXTRA>
__global__ void spread_reduce_kernel(float4* __restrict__ grad, float4* __restrict__ spread,
                                     const int* __restrict__ rows_used, int rows) {
    const size_t n = (size_t)(rows_used ? min(*rows_used, rows) : rows) * 1000u;
    const size_t stride = (size_t)rows * 1000u;
    const float4 zero = make_float4(0.f, 0.f, 0.f, 0.f);
    for (size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (size_t)gridDim.x * blockDim.x) {
        float4 v[EXTRA];
#pragma unroll
        for (int k = 0; k < EXTRA; ++k) v[k] = __ldcs(spread + (size_t)k * stride + e);
        float4 s = grad[e];
#pragma unroll
        for (int k = 0; k < EXTRA; ++k) s = make_float4(s.x + v[k].x, s.y + v[k].y, s.z + v[k].z, s.w + v[k].w);
        grad[e] = s;
#pragma unroll
        for (int k = 0; k < EXTRA; ++k) __stcs(spread + (size_t)k * stride + e, zero);
    }
}

cudaError_t launch_spread_reduce(const GradTarget& grad, cudaStream_t s) {
    if (grad.copies <= 1) return cudaSuccess;
    int dev = 0, sms = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (e != cudaSuccess) return e;
    const dim3 blocks((unsigned)(sms * 16)), threads(256);
    switch (grad.copies) {
        case 2: spread_reduce_kernel<1><<<blocks, threads, 0, s>>>((float4*)grad.grad, grad.spread, grad.rows_used,
                                                                   grad.spread_rows); break;
        case 4: spread_reduce_kernel<3><<<blocks, threads, 0, s>>>((float4*)grad.grad, grad.spread, grad.rows_used,
                                                                   grad.spread_rows); break;
        case 8: spread_reduce_kernel<7><<<blocks, threads, 0, s>>>((float4*)grad.grad, grad.spread, grad.rows_used,
                                                                   grad.spread_rows); break;
        default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

size_t ckpt_bytes(int w, int h, int per_ray) {
    return (size_t)w * h * (sizeof(int2) + (size_t)per_ray * sizeof(Ckpt));
}

cudaError_t launch_forward_ckpt(int fmt, const RaycastParams& p, void* ckpt, int per_ray, cudaStream_t s) {
    const int W = p.u.width, H = p.u.height;
    int2* hdr = (int2*)ckpt;
    Ckpt* ck = (Ckpt*)((char*)ckpt + (size_t)W * H * sizeof(int2));
    dim3 block(128), grid((unsigned)((W + 15) / 16), (unsigned)((H + 7) / 8));
    switch (fmt) {
        case VV_FMT_RGBA8: forward_ckpt_kernel<VV_FMT_RGBA8><<<grid, block, 0, s>>>(p, hdr, ck, per_ray); break;
        case VV_FMT_FP16: forward_ckpt_kernel<VV_FMT_FP16><<<grid, block, 0, s>>>(p, hdr, ck, per_ray); break;
        case VV_FMT_BF16: forward_ckpt_kernel<VV_FMT_BF16><<<grid, block, 0, s>>>(p, hdr, ck, per_ray); break;
        case VV_FMT_FP32: forward_ckpt_kernel<VV_FMT_FP32><<<grid, block, 0, s>>>(p, hdr, ck, per_ray); break;
        default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

cudaError_t launch_backward(int fmt, const RaycastParams& p, const void* ckpt, int per_ray, const float4* dl_dcolor,
                            const GradTarget& grad, cudaStream_t s) {
    const int W = p.u.width, H = p.u.height;
    const int2* hdr = (const int2*)ckpt;
    const Ckpt* ck = (const Ckpt*)((const char*)ckpt + (size_t)W * H * sizeof(int2));
    dim3 block(128), grid((unsigned)((W + 15) / 16), (unsigned)((H + 7) / 8));
#define VV_BWD(F)                                                                                    \
    if (grad.f64 && grad.warp_sum)                                                                   \
        backward_kernel<F, true, true><<<grid, block, 0, s>>>(p, hdr, ck, per_ray, dl_dcolor, grad);   \
    else if (grad.f64)                                                                               \
        backward_kernel<F, true, false><<<grid, block, 0, s>>>(p, hdr, ck, per_ray, dl_dcolor, grad);  \
    else if (grad.warp_sum)                                                                          \
        backward_kernel<F, false, true><<<grid, block, 0, s>>>(p, hdr, ck, per_ray, dl_dcolor, grad);  \
    else                                                                                             \
        backward_kernel<F, false, false><<<grid, block, 0, s>>>(p, hdr, ck, per_ray, dl_dcolor, grad);
    switch (fmt) {
        case VV_FMT_RGBA8: VV_BWD(VV_FMT_RGBA8) break;
        case VV_FMT_FP16: VV_BWD(VV_FMT_FP16) break;
        case VV_FMT_BF16: VV_BWD(VV_FMT_BF16) break;
        case VV_FMT_FP32: VV_BWD(VV_FMT_FP32) break;
        default: return cudaErrorInvalidValue;
    }
#undef VV_BWD
    return cudaGetLastError();
}

}  // namespace vv
