// raycast_common.cuh - device side of the GigaVoxels ray walk, shared by the
// forward ray cast, the checkpointing forward and the adjoint replay.
//
// Floating point: every translation unit that includes this header is
// compiled with -fmad=false -prec-div=true -prec-sqrt=true and without
// fast-math, so each +,-,*,/ and sqrt below is one IEEE binary32 operation in
// the written order; the only fused operation is the explicit fmaf() of
// lerpf().  The host oracle performs the same sequence, which makes descent
// decisions, step counts, LOD choices and node-usage lists bit-identical.
#pragma once

#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include "cellmask.cuh"
#include "dxt.h"
#include "fixed_div.h"
#include "kernels.cuh"
#include "lod_bound.h"

namespace vv {
namespace rc {

constexpr uint32_t kResident = 0x80000000u;
constexpr uint32_t kConstant = 0x40000000u;

struct F3 {
    float x, y, z;
};
__device__ __forceinline__ F3 f3(float x, float y, float z) { return F3{x, y, z}; }
__device__ __forceinline__ F3 ld3(const float* a) { return F3{a[0], a[1], a[2]}; }
__device__ __forceinline__ F3 add(F3 a, F3 b) { return F3{a.x + b.x, a.y + b.y, a.z + b.z}; }
__device__ __forceinline__ F3 sub(F3 a, F3 b) { return F3{a.x - b.x, a.y - b.y, a.z - b.z}; }
__device__ __forceinline__ F3 mul(F3 a, F3 b) { return F3{a.x * b.x, a.y * b.y, a.z * b.z}; }
__device__ __forceinline__ F3 muls(F3 a, float s) { return F3{a.x * s, a.y * s, a.z * s}; }
__device__ __forceinline__ F3 divv(F3 a, F3 b) { return F3{a.x / b.x, a.y / b.y, a.z / b.z}; }
__device__ __forceinline__ float dot3(F3 a, F3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
// normalize(v) = v * (1 / sqrt(dot(v,v))), correctly rounded sqrt and divide.
__device__ __forceinline__ F3 normalize3(F3 v) {
    float r = 1.0f / sqrtf(dot3(v, v));
    return muls(v, r);
}
__device__ __forceinline__ float lerpf(float a, float b, float t) { return fmaf(t, b - a, a); }

__device__ __forceinline__ void set_status(int* status, int code) {
    if (status) atomicCAS(status, 0, code);
}

// 2^e for e in [-126, 127], exactly: the normal power of two built from its
// exponent bits (ldexpf covers every case and costs more instructions).  Every
// use below scales by a tree level, well inside that range.
__device__ __forceinline__ float pow2i(int e) { return __int_as_float((e + 127) << 23); }

// pow(x, 2^k) as k squarings (the sample-ratio powers of the shader).
__device__ __forceinline__ float pow_pow2(float x, int k) {
    for (int i = 0; i < k; ++i) x = x * x;
    return x;
}

// Texel loads per storage format: 4 channels as float (RGBA8 as 0..255).
template <int FMT>
struct Texel;
// Byte k of v as a float, exactly: the bit pattern 0x4B0000bb is 2^23 + b.
// (A byte-select and an add instead of an integer-to-float conversion, which
// runs at a quarter of the add rate.)
__device__ __forceinline__ float byte_as_float(uint32_t v, uint32_t sel) {
    return __uint_as_float(__byte_perm(v, 0x4B000000u, sel)) - 8388608.0f;
}
template <>
struct Texel<VV_FMT_RGBA8> {
    static constexpr float kScale = 1.0f / 255.0f;
    __device__ __forceinline__ static float4 unpack(uint32_t v) {
        // selectors: result bytes (low to high) = byte k of v, 0, 0, 0x4B
        return make_float4(byte_as_float(v, 0x7440u), byte_as_float(v, 0x7441u), byte_as_float(v, 0x7442u),
                           byte_as_float(v, 0x7443u));
    }
    __device__ __forceinline__ static float4 load(const void* pool, uint32_t i) {
        return unpack(__ldg((const uint32_t*)pool + i));
    }
};
template <>
struct Texel<VV_FMT_FP16> {
    static constexpr float kScale = 1.0f;
    __device__ __forceinline__ static float4 load(const void* pool, uint32_t i) {
        uint2 v = __ldg((const uint2*)pool + i);
        __half2 a = *reinterpret_cast<__half2*>(&v.x), b = *reinterpret_cast<__half2*>(&v.y);
        float2 fa = __half22float2(a), fb = __half22float2(b);
        return make_float4(fa.x, fa.y, fb.x, fb.y);
    }
};
template <>
struct Texel<VV_FMT_BF16> {
    static constexpr float kScale = 1.0f;
    __device__ __forceinline__ static float4 load(const void* pool, uint32_t i) {
        uint2 v = __ldg((const uint2*)pool + i);
        return make_float4(__uint_as_float(v.x << 16), __uint_as_float(v.x & 0xFFFF0000u),
                           __uint_as_float(v.y << 16), __uint_as_float(v.y & 0xFFFF0000u));
    }
};
template <>
struct Texel<VV_FMT_FP32> {
    static constexpr float kScale = 1.0f;
    __device__ __forceinline__ static float4 load(const void* pool, uint32_t i) {
        return __ldg((const float4*)pool + i);
    }
};

// Block-compressed pools (dxt.h): texel i = slot * 1000 + (z*10 + y)*10 + x
// decoded from its 4x4 block of slice z, as RGBA8 values.
__device__ __forceinline__ void dxt_address(uint32_t i, uint32_t& block, int& t) {
    const uint32_t slot = i / 1000u, r = i - slot * 1000u;
    const uint32_t z = r / 100u, yx = r - z * 100u, y = yx / 10u, x = yx - y * 10u;
    block = slot * (uint32_t)dxt::kBlocksPerSlot + (uint32_t)dxt::block_of((int)x, (int)y, (int)z);
    t = dxt::texel_of((int)x, (int)y);
}
template <>
struct Texel<VV_FMT_DXT5> {
    static constexpr float kScale = 1.0f / 255.0f;
    __device__ __forceinline__ static float4 load(const void* pool, uint32_t i) {
        uint32_t b;
        int t;
        dxt_address(i, b, t);
        const uint4 v = __ldg((const uint4*)pool + b);
        const uint32_t w[4] = {v.x, v.y, v.z, v.w};
        const uint32_t c = dxt::decode_dxt5(w, t);
        return make_float4(byte_as_float(c, 0x7440u), byte_as_float(c, 0x7441u), byte_as_float(c, 0x7442u),
                           byte_as_float(c, 0x7443u));
    }
};
template <>
struct Texel<VV_FMT_DXT1> {
    static constexpr float kScale = 1.0f / 255.0f;
    __device__ __forceinline__ static float4 load(const void* pool, uint32_t i) {
        uint32_t b;
        int t;
        dxt_address(i, b, t);
        const uint2 v = __ldg((const uint2*)pool + b);
        const uint32_t w[2] = {v.x, v.y};
        const uint32_t c = dxt::decode_dxt1(w, t);
        return make_float4(byte_as_float(c, 0x7440u), byte_as_float(c, 0x7441u), byte_as_float(c, 0x7442u), 0.0f);
    }
};

__device__ __forceinline__ float4 lerp4(float4 a, float4 b, float t) {
    return make_float4(lerpf(a.x, b.x, t), lerpf(a.y, b.y, t), lerpf(a.z, b.z, t), lerpf(a.w, b.w, t));
}

// One axis of GL_LINEAR + CLAMP_TO_EDGE (GL 3.3 spec 3.8.8): texel centres at
// i+0.5, i0 = floor(u*N - 0.5), weight = frac.  Returns brick-linear
// coordinates (slot, local) of both taps.
struct Axis {
    int s0, l0, s1, l1;
    float f;
};
__device__ __forceinline__ Axis axis_taps(float u, float N, int n) {
    float t = u * N - 0.5f;
    t = fminf(fmaxf(t, -1.0f), N);
    float fi = floorf(t);
    Axis a;
    a.f = t - fi;
    int i0 = (int)fi, i1 = i0 + 1;
    i0 = min(max(i0, 0), n - 1);
    i1 = min(max(i1, 0), n - 1);
    a.s0 = i0 / 10;
    a.l0 = i0 - 10 * a.s0;
    a.s1 = i1 / 10;
    a.l1 = i1 - 10 * a.s1;
    return a;
}

__device__ __forceinline__ void touch(uint32_t* bits, uint32_t i) { atomicOr(bits + (i >> 5), 1u << (i & 31u)); }

template <int FMT, bool COUNT>
__device__ __forceinline__ float4 sample_brick(const RaycastParams& p, F3 uvw) {
    const float* N = p.u.brick_pool_dimension;
    const int nx = p.slots[0] * 10, ny = p.slots[1] * 10, nz = p.slots[2] * 10;
    Axis ax = axis_taps(uvw.x, N[0], nx);
    Axis ay = axis_taps(uvw.y, N[1], ny);
    Axis az = axis_taps(uvw.z, N[2], nz);
    const uint32_t SX = (uint32_t)p.slots[0], SY = (uint32_t)p.slots[1];
    auto idx = [&](int sx, int lx, int sy, int ly, int sz, int lz) -> uint32_t {
        uint32_t slot = ((uint32_t)sz * SY + (uint32_t)sy) * SX + (uint32_t)sx;
        return slot * 1000u + (uint32_t)((lz * 10 + ly) * 10 + lx);
    };
    const void* pool = p.bricks;
    float4 v000 = Texel<FMT>::load(pool, idx(ax.s0, ax.l0, ay.s0, ay.l0, az.s0, az.l0));
    float4 v100 = Texel<FMT>::load(pool, idx(ax.s1, ax.l1, ay.s0, ay.l0, az.s0, az.l0));
    float4 v010 = Texel<FMT>::load(pool, idx(ax.s0, ax.l0, ay.s1, ay.l1, az.s0, az.l0));
    float4 v110 = Texel<FMT>::load(pool, idx(ax.s1, ax.l1, ay.s1, ay.l1, az.s0, az.l0));
    float4 v001 = Texel<FMT>::load(pool, idx(ax.s0, ax.l0, ay.s0, ay.l0, az.s1, az.l1));
    float4 v101 = Texel<FMT>::load(pool, idx(ax.s1, ax.l1, ay.s0, ay.l0, az.s1, az.l1));
    float4 v011 = Texel<FMT>::load(pool, idx(ax.s0, ax.l0, ay.s1, ay.l1, az.s1, az.l1));
    float4 v111 = Texel<FMT>::load(pool, idx(ax.s1, ax.l1, ay.s1, ay.l1, az.s1, az.l1));
    if (COUNT) {
        for (int k = 0; k < 8; ++k) {
            const uint32_t sx = (uint32_t)((k & 1) ? ax.s1 : ax.s0), sy = (uint32_t)((k & 2) ? ay.s1 : ay.s0),
                           sz = (uint32_t)((k & 4) ? az.s1 : az.s0);
            touch(p.brick_touch, (sz * SY + sy) * SX + sx);
        }
    }
    float4 c00 = lerp4(v000, v100, ax.f);
    float4 c10 = lerp4(v010, v110, ax.f);
    float4 c01 = lerp4(v001, v101, ax.f);
    float4 c11 = lerp4(v011, v111, ax.f);
    float4 c0 = lerp4(c00, c10, ay.f);
    float4 c1 = lerp4(c01, c11, ay.f);
    float4 c = lerp4(c0, c1, az.f);
    if (Texel<FMT>::kScale != 1.0f) {
        const float k = Texel<FMT>::kScale;
        c = make_float4(c.x * k, c.y * k, c.z * k, c.w * k);
    }
    return c;
}

// Trilinear sample when all 8 taps lie in the brick-pool slot whose first
// texel per axis is base[]: kInSlot (out = the sample, same arithmetic as
// sample_brick, only the texel addressing is shorter) or, when the slot's
// cell mask `cmask` (or nullptr) marks the taps' cell all zero, kEmptyCell
// (out = 0, exactly what the taps give); kOutside (and nothing) otherwise.
// With STAGED and `stex` (the slot's RGBA8 texels in shared memory) the taps
// are read from there.
enum { kOutside = 0, kInSlot = 1, kEmptyCell = 2 };
template <int FMT, bool STAGED = false>
__device__ __forceinline__ int sample_in_slot(const RaycastParams& p, F3 uvw, const int base[3], uint32_t slot_texel0,
                                              const uint32_t* cmask, float4& out, const uint32_t* stex = nullptr) {
    const float* N = p.u.brick_pool_dimension;
    const float ta[3] = {uvw.x * N[0] - 0.5f, uvw.y * N[1] - 0.5f, uvw.z * N[2] - 0.5f};
    // the first tap per axis, floor(t) as an integer in one conversion (the
    // weights below are only formed for a sample that is filtered)
    int l[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) l[a] = __float2int_rd(ta[a]) - base[a];
    if ((unsigned)l[0] > 8u || (unsigned)l[1] > 8u || (unsigned)l[2] > 8u) return kOutside;
    if (cmask) {
        const uint32_t c = (uint32_t)((l[2] * kCellsPerAxis + l[1]) * kCellsPerAxis + l[0]);
        if ((__ldg(cmask + (c >> 5)) >> (c & 31u)) & 1u) {
            out = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
            return kEmptyCell;
        }
    }
    float f[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) f[a] = ta[a] - floorf(ta[a]);
    const uint32_t l000 = (uint32_t)((l[2] * 10 + l[1]) * 10 + l[0]);
    const uint32_t i000 = slot_texel0 + l000;
    const void* pool = p.bricks;
    float4 v000, v100, v010, v110, v001, v101, v011, v111;
    if (STAGED && stex) {
        static_assert(!STAGED || FMT == VV_FMT_RGBA8, "staging holds RGBA8 slots");
        const uint32_t* t = stex + l000;
        v000 = Texel<VV_FMT_RGBA8>::unpack(t[0]);
        v100 = Texel<VV_FMT_RGBA8>::unpack(t[1]);
        v010 = Texel<VV_FMT_RGBA8>::unpack(t[10]);
        v110 = Texel<VV_FMT_RGBA8>::unpack(t[11]);
        v001 = Texel<VV_FMT_RGBA8>::unpack(t[100]);
        v101 = Texel<VV_FMT_RGBA8>::unpack(t[101]);
        v011 = Texel<VV_FMT_RGBA8>::unpack(t[110]);
        v111 = Texel<VV_FMT_RGBA8>::unpack(t[111]);
    } else {
        v000 = Texel<FMT>::load(pool, i000);
        v100 = Texel<FMT>::load(pool, i000 + 1u);
        v010 = Texel<FMT>::load(pool, i000 + 10u);
        v110 = Texel<FMT>::load(pool, i000 + 11u);
        v001 = Texel<FMT>::load(pool, i000 + 100u);
        v101 = Texel<FMT>::load(pool, i000 + 101u);
        v011 = Texel<FMT>::load(pool, i000 + 110u);
        v111 = Texel<FMT>::load(pool, i000 + 111u);
    }
    const float4 c0 = lerp4(lerp4(v000, v100, f[0]), lerp4(v010, v110, f[0]), f[1]);
    const float4 c1 = lerp4(lerp4(v001, v101, f[0]), lerp4(v011, v111, f[0]), f[1]);
    float4 c = lerp4(c0, c1, f[2]);
    if (Texel<FMT>::kScale != 1.0f) {
        const float k = Texel<FMT>::kScale;
        c = make_float4(c.x * k, c.y * k, c.z * k, c.w * k);
    }
    out = c;
    return kInSlot;
}


// A colour as RGBA8 unorm: round(clamp(c, 0, 1) * 255) per channel, to the
// nearest (ties to even); NaN stores 0.
__device__ __forceinline__ uint32_t unorm8(float c) {
    return __float2uint_rn(__fmul_rn(fminf(fmaxf(c, 0.0f), 1.0f), 255.0f));
}
__device__ __forceinline__ uint32_t pack_unorm8(float4 c) {
    return unorm8(c.x) | (unorm8(c.y) << 8) | (unorm8(c.z) << 16) | (unorm8(c.w) << 24);
}

// t / step for step = RS * 2^e.  With RS a power of two (rstep = 1 / RS)
// the quotient is t times a power of two: the same real number, so the same
// rounded result, as the division.
__device__ __forceinline__ float div_step(const RaycastParams& p, float t, float step, int e) {
    return p.rstep != 0.0f ? t * (p.rstep * pow2i(-e)) : t / step;
}

// ComputeMinRayBoxIntersection (GigaVoxelsNoLighting.frag:124-180): exit
// time over the planes facing away from the ray, 4.0 if none, t == 0 ignored.
__device__ __forceinline__ float min_exit(F3 p, F3 d, F3 mn, F3 mx) {
    float tmin = 4.0f;
    // planes 0..2: min faces with normals -x,-y,-z
    const float pa[3] = {p.x, p.y, p.z}, da[3] = {d.x, d.y, d.z};
    const float mna[3] = {mn.x, mn.y, mn.z}, mxa[3] = {mx.x, mx.y, mx.z};
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        float dn = -da[a];
        if (dn > 0.0f) {
            float t = (pa[a] - mna[a]) / dn;
            if (t < tmin && fabsf(t) > 0.0f) tmin = t;
        }
    }
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        float dn = da[a];
        if (dn > 0.0f) {
            float t = -(pa[a] - mxa[a]) / dn;
            if (t < tmin && fabsf(t) > 0.0f) tmin = t;
        }
    }
    return tmin;
}

__device__ __forceinline__ bool inside_box(F3 p, F3 mn, F3 mx) {
    return p.x > mn.x && p.y > mn.y && p.z > mn.z && mx.x > p.x && mx.y > p.y && mx.z > p.z;
}

template <bool COUNT>
__device__ __forceinline__ uint2 fetch_node(const RaycastParams& p, uint32_t x, uint32_t y, uint32_t z,
                                            bool& ok) {
    if (x >= (uint32_t)p.node_dim[0] || y >= (uint32_t)p.node_dim[1] || z >= (uint32_t)p.node_dim[2]) {
        ok = false;
        return make_uint2(0u, 0u);
    }
    const uint32_t bx = (uint32_t)p.node_dim[0] >> 1, by = (uint32_t)p.node_dim[1] >> 1;
    uint32_t blk = ((z >> 1) * by + (y >> 1)) * bx + (x >> 1);
    uint32_t idx = blk * 8u + ((x & 1u) | ((y & 1u) << 1) | ((z & 1u) << 2));
    if (COUNT) touch(p.node_touch, idx);
    return __ldg(p.nodes + idx);
}

// ---------------------------------------------------------------------------
// The ray walk of GigaVoxelsNoLighting.frag main (:490-751) after the ray
// set-up: leaf segments, each a descent from the root to the node that stops
// it (:563-622, :722-746) followed by TraverseConstant (:230-282) or
// TraverseBrick (:311-359) and the break test (:673-679).  The descent is its
// own loop, so the lanes of a warp descend together and march together.
// A visitor observes the walk:
//   bool segment_begin(const RayState&)   false ends the walk
//   bool sample(int kind, float4 src, F3 bpos, float T, int index)
//                                          before a sample is composited;
//                                          false ends the walk after it
//   void segment_end(const RayState&, bool is_const, bool loaded)
//   void fail(int code)
// STEPS unrolls the two march loops (samples issued per loop trip); the
// results do not depend on it.

struct WalkConsts {
    F3 C, vmin, vmax, up, left, bdim, pdim;
    float RS, astop, lod, pixel_size, rvh;
    int L, max_iter;
    uint2 root;
    lodb::Consts lodk;  // certificate constants of the LOD test (lod_bound.h)
    bool unit_box;      // volume extent [0,1]^3 (as compute_uniforms derives it)
};

struct RayState {
    F3 pos, dir, brick_step;
    float4 dst;
    int iter;
    int nsamples;                        // samples composited so far
    uint32_t nptr_x, nptr_y, nptr_z;     // octTreeNodePtr (not reset between segments)
};

enum { kSampleConst = 0, kSampleBrick = 1 };

__device__ __forceinline__ WalkConsts walk_consts(const RaycastParams& p, uint2 root) {
    const vv_uniforms& u = p.u;
    WalkConsts k;
    k.C = ld3(u.camera_position);
    k.vmin = ld3(u.vol_extent_min);
    k.vmax = ld3(u.vol_extent_max);
    k.up = ld3(u.camera_up);
    k.left = ld3(u.camera_left);
    k.bdim = ld3(u.brick_dimension);
    k.pdim = ld3(u.brick_pool_dimension);
    k.RS = u.ray_step_size;
    k.astop = u.alpha_stop;
    k.lod = u.lod_scalar;
    k.pixel_size = u.pixel_size;
    k.rvh = u.root_voxel_half_size;
    k.L = u.oct_tree_depth_minus_one;
    k.max_iter = p.max_iter;
    k.root = root;
    k.unit_box = k.vmin.x == 0.0f && k.vmin.y == 0.0f && k.vmin.z == 0.0f && k.vmax.x == 1.0f &&
                 k.vmax.y == 1.0f && k.vmax.z == 1.0f;
    k.lodk = lodb::make_consts(lodb::V3{k.C.x, k.C.y, k.C.z}, lodb::V3{k.up.x, k.up.y, k.up.z},
                               lodb::V3{k.left.x, k.left.y, k.left.z}, k.rvh, k.lod, k.pixel_size, k.L,
                               k.unit_box);
    return k;
}

// The fragment's RayPosition: the box entry point of pixel (px,py)'s ray
// (GigaVoxels.vert) or its near-plane point (NearPlaneQuad.vert); false when
// the pixel has no fragment.
__device__ __forceinline__ bool ray_origin(const vv_uniforms& u, const WalkConsts& k, int px, int py, F3& pos) {
    const float fx = (float)px + 0.5f, fy = (float)py + 0.5f;
    const F3 d = f3(u.near_origin[0] + fx * u.near_dx[0] + fy * u.near_dy[0],
                    u.near_origin[1] + fx * u.near_dx[1] + fy * u.near_dy[1],
                    u.near_origin[2] + fx * u.near_dx[2] + fy * u.near_dy[2]);
    if (u.camera_inside) {
        pos = add(k.C, d);
        return true;
    }
    const float da[3] = {d.x, d.y, d.z}, ca[3] = {k.C.x, k.C.y, k.C.z};
    const float mn[3] = {k.vmin.x, k.vmin.y, k.vmin.z}, mx[3] = {k.vmax.x, k.vmax.y, k.vmax.z};
    float tenter = -INFINITY, texit = INFINITY;
    int axis = -1;
    bool frag = true;
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        if (da[a] != 0.0f) {
            float t0 = (mn[a] - ca[a]) / da[a];
            float t1 = (mx[a] - ca[a]) / da[a];
            float tn = t0 < t1 ? t0 : t1, tf = t0 < t1 ? t1 : t0;
            if (tn > tenter) {
                tenter = tn;
                axis = a;
            }
            if (tf < texit) texit = tf;
        } else if (!(ca[a] > mn[a] && ca[a] < mx[a])) {
            frag = false;
        }
    }
    if (axis < 0 || !(tenter <= texit) || !(tenter > 0.0f)) frag = false;
    if (!frag) return false;
    float pa[3] = {ca[0] + da[0] * tenter, ca[1] + da[1] * tenter, ca[2] + da[2] * tenter};
#pragma unroll
    for (int a = 0; a < 3; ++a)
        if (a == axis) pa[a] = da[a] > 0.0f ? mn[a] : mx[a];
    pos = f3(pa[0], pa[1], pa[2]);
    return true;
}

// Ray set-up after the origin (:500-510): direction, jitter, inside test.
__device__ __forceinline__ bool ray_start(const RaycastParams& p, const WalkConsts& k, int px, int py, F3 pos,
                                          RayState& s) {
    const vv_uniforms& u = p.u;
    s.dir = normalize3(sub(pos, k.C));
    const int J = u.jitter_tex_size;
    const float jitter = (float)p.jitter[(py % J) * J + (px % J)] / 255.0f;
    s.pos = add(pos, muls(muls(s.dir, k.RS), jitter));
    s.brick_step = mul(s.dir, ld3(u.brick_step_vector));
    s.dst = make_float4(0.f, 0.f, 0.f, 0.f);
    s.iter = 0;
    s.nsamples = 0;
    s.nptr_x = s.nptr_y = s.nptr_z = 0u;
    return inside_box(s.pos, k.vmin, k.vmax);
}

// The path of the ray's last descent, per thread in shared memory: node word
// and packed grid position (x<<20 | y<<10 | z) of each level, `stride`
// elements apart per level.  A later descent whose position lies in the same
// level-r node, and whose LOD test lodb::clear_range shows to continue at
// every level above r, starts at that node instead of the root: the levels
// it skips would take exactly the recorded path (same nodes, same words,
// every stop condition false), so the walk is unchanged.
constexpr int kPathLevels = 11;  // levels 0..10
struct StageBuf;
struct PathSlots {
    uint2* w;
    uint32_t* p;
    int stride;
    StageBuf* stage;  // the warp's staged brick (VV_RAYCAST_STAGED), else nullptr
};

// ---- brick staging (VV_RAYCAST_STAGED, RGBA8 pools) ------------------------
//
// Each warp owns one 10^3-texel RGBA8 slot copy in shared memory.  When the
// lanes that reach a brick segment together share a slot (__match_any_sync),
// the largest such group copies that slot's 4000 bytes with one
// cp.async.bulk (global -> this CTA's own shared memory) and
// samples it from shared memory; other lanes read the pool as usual.
//   state = tag << 32 | mask: tag = the slot the buffer holds (kNoSlot while
//   a copy is in flight), mask = the lanes reading it.  A group joins a
//   buffer that holds its slot, or refills an unread one; both by one
//   atomicCAS of its leader, so a copy never overwrites texels being read.
// The only wait is the copy's own mbarrier (bounded: on timeout the status
// is set, the buffer stays claimed and the lanes read the pool).
constexpr uint32_t kNoSlot = 0xFFFFFFFFu;
constexpr int kStageMinLanes = 4;  // smallest group worth a copy
struct __align__(16) StageBuf {
    uint32_t texels[1000];
    unsigned long long state;
    unsigned long long bar;
    uint32_t phase;  // completed copies (the mbarrier's phase parity)
};

// Lane 0 of the warp, before any lane returns.
__device__ __forceinline__ void stage_init(StageBuf* sb) {
    sb->state = (unsigned long long)kNoSlot << 32;
    sb->phase = 0u;
    const uint32_t bar = (uint32_t)__cvta_generic_to_shared(&sb->bar);
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// Called by the converged lanes entering a brick segment; `slot` is the
// lane's slot or kNoSlot.  True: the lane reads its slot from sb->texels
// until stage_release.
__device__ __forceinline__ bool stage_acquire(StageBuf* sb, const void* pool, uint32_t slot, int* status) {
    const unsigned am = __activemask();
    const unsigned peers = __match_any_sync(am, slot);
    const int lane = (int)(threadIdx.x & 31u);
    const int leader = __ffs(peers) - 1;
    // 1: joined a buffer holding the slot, 2: claimed it for a copy
    int act = 0;
    if (lane == leader && slot != kNoSlot) {
        unsigned long long st = *(volatile unsigned long long*)&sb->state;
        for (int tries = 0; tries < 4; ++tries) {
            unsigned long long want;
            int a;
            if ((uint32_t)(st >> 32) == slot) {
                want = st | peers;
                a = 1;
            } else if ((uint32_t)st == 0u && __popc(peers) >= kStageMinLanes) {
                want = ((unsigned long long)kNoSlot << 32) | peers;
                a = 2;
            } else {
                break;
            }
            const unsigned long long old = atomicCAS(&sb->state, st, want);
            if (old == st) {
                act = a;
                break;
            }
            st = old;
        }
        __threadfence_block();
    }
    act = __shfl_sync(peers, act, leader);
    if (act == 2) {
        const uint32_t bar = (uint32_t)__cvta_generic_to_shared(&sb->bar);
        const uint32_t parity = sb->phase & 1u;
        if (lane == leader) {
            const uint32_t dst = (uint32_t)__cvta_generic_to_shared(sb->texels);
            const uint32_t* src = (const uint32_t*)pool + (size_t)slot * 1000u;
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], 4000;" ::"r"(bar) : "memory");
            asm volatile(
                "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], 4000, [%2];" ::"r"(dst),
                "l"(src), "r"(bar)
                : "memory");
        }
        uint32_t done = 0u;
        for (int i = 0; i < (1 << 20) && !done; ++i) {
            asm volatile(
                "{\n\t.reg .pred p;\n\t"
                "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
                "selp.u32 %0, 1, 0, p;\n\t}"
                : "=r"(done)
                : "r"(bar), "r"(parity)
                : "memory");
        }
        done = __all_sync(peers, done != 0u);
        if (!done) {
            set_status(status, VV_ERR_TIMEOUT);
            return false;
        }
        __syncwarp(peers);
        if (lane == leader) {
            sb->phase = sb->phase + 1u;
            __threadfence_block();
            atomicExch(&sb->state, ((unsigned long long)slot << 32) | peers);
        }
        __syncwarp(peers);
        return true;
    }
    return act == 1;
}

// The lane stops reading the staged slot.
__device__ __forceinline__ void stage_release(StageBuf* sb) {
    __threadfence_block();
    atomicAnd(&sb->state, ~(1ull << (threadIdx.x & 31u)));
}

// ---- lighting (GigaVoxels.frag with ComputeLighting) ----------------------

// texture(BrickGradientsSampler, p).rgb (:316): the trilinear filter of
// sample_brick over the gradient pool (FP32 gradients, or RGBA8 / 255).
template <int GFMT>
__device__ __forceinline__ F3 sample_gradient(const RaycastParams& p, F3 uvw) {
    const float* N = p.u.brick_pool_dimension;
    const Axis ax = axis_taps(uvw.x, N[0], p.slots[0] * 10);
    const Axis ay = axis_taps(uvw.y, N[1], p.slots[1] * 10);
    const Axis az = axis_taps(uvw.z, N[2], p.slots[2] * 10);
    const uint32_t SX = (uint32_t)p.slots[0], SY = (uint32_t)p.slots[1];
    auto idx = [&](int sx, int lx, int sy, int ly, int sz, int lz) -> uint32_t {
        const uint32_t slot = ((uint32_t)sz * SY + (uint32_t)sy) * SX + (uint32_t)sx;
        return slot * 1000u + (uint32_t)((lz * 10 + ly) * 10 + lx);
    };
    const void* g = p.grads;
    const float4 v000 = Texel<GFMT>::load(g, idx(ax.s0, ax.l0, ay.s0, ay.l0, az.s0, az.l0));
    const float4 v100 = Texel<GFMT>::load(g, idx(ax.s1, ax.l1, ay.s0, ay.l0, az.s0, az.l0));
    const float4 v010 = Texel<GFMT>::load(g, idx(ax.s0, ax.l0, ay.s1, ay.l1, az.s0, az.l0));
    const float4 v110 = Texel<GFMT>::load(g, idx(ax.s1, ax.l1, ay.s1, ay.l1, az.s0, az.l0));
    const float4 v001 = Texel<GFMT>::load(g, idx(ax.s0, ax.l0, ay.s0, ay.l0, az.s1, az.l1));
    const float4 v101 = Texel<GFMT>::load(g, idx(ax.s1, ax.l1, ay.s0, ay.l0, az.s1, az.l1));
    const float4 v011 = Texel<GFMT>::load(g, idx(ax.s0, ax.l0, ay.s1, ay.l1, az.s1, az.l1));
    const float4 v111 = Texel<GFMT>::load(g, idx(ax.s1, ax.l1, ay.s1, ay.l1, az.s1, az.l1));
    const float4 c0 = lerp4(lerp4(v000, v100, ax.f), lerp4(v010, v110, ax.f), ay.f);
    const float4 c1 = lerp4(lerp4(v001, v101, ax.f), lerp4(v011, v111, ax.f), ay.f);
    float4 c = lerp4(c0, c1, az.f);
    if (Texel<GFMT>::kScale != 1.0f) {
        const float kk = Texel<GFMT>::kScale;
        c = make_float4(c.x * kk, c.y * kk, c.z * kk, c.w * kk);
    }
    return f3(c.x, c.y, c.z);
}

// pow(x, 100) as x^64 * x^32 * x^4 by squarings (the shininess power).
__device__ __forceinline__ float pow100(float x) {
    const float x2 = x * x, x4 = x2 * x2, x8 = x4 * x4, x16 = x8 * x8, x32 = x16 * x16, x64 = x32 * x32;
    return (x64 * x32) * x4;
}

// shading (:293-312) with k_Ambient 0.05, k_Diffuse = k_Specular = 1,
// k_Shininess 100, added to src.rgb when the gradient normalizes (:370-384).
__device__ __forceinline__ void light_sample(const RaycastParams& p, F3 bpos, F3 dir, F3 light_dir, float4& src) {
    F3 n = p.grad_fmt == VV_FMT_RGBA8  ? sample_gradient<VV_FMT_RGBA8>(p, bpos)
           : p.grad_fmt == VV_FMT_DXT1 ? sample_gradient<VV_FMT_DXT1>(p, bpos)
                                       : sample_gradient<VV_FMT_FP32>(p, bpos);
    if (p.u.gradients_unsigned) n = sub(muls(n, 2.0f), f3(1.0f, 1.0f, 1.0f));  // LookupGradient :318-322
    n = normalize3(n);
    if (isnan(n.x) || isnan(n.y) || isnan(n.z)) return;  // homogeneous region: no lighting
    const F3 rgb = f3(src.x, src.y, src.z);
    const F3 to_camera = muls(dir, -1.0f);
    const F3 halfway = normalize3(add(light_dir, to_camera));
    const float diffuse_light = fmaxf(dot3(light_dir, n), 0.0f);
    F3 diffuse = f3(0.0f, 0.0f, 0.0f), specular = f3(0.0f, 0.0f, 0.0f);
    if (diffuse_light > 0.0f) {
        diffuse = muls(rgb, diffuse_light);
        specular = muls(rgb, pow100(fmaxf(dot3(halfway, n), 0.0f)));
    }
    const F3 ambient = muls(rgb, 0.05f);
    const F3 sh = add(add(ambient, diffuse), specular);
    src.x = src.x + sh.x;
    src.y = src.y + sh.y;
    src.z = src.z + sh.z;
}

// Where a ray's last descent stopped (RESUME): its depth and its node's
// cell there, packed 10:10:10.
struct WalkResume {
    int prev_depth = -1;
    uint32_t prev_cell = 0u;
};

// One leaf segment of the walk (a descent and its march); false when the
// walk has ended.  walk() runs it until then.
template <int FMT, bool COUNT, class V, int STEPS = 1, bool RESUME = false, bool LIT = false, bool STAGED = false>
__device__ __forceinline__ bool walk_segment(const RaycastParams& p, const WalkConsts& k, RayState& s, V& vis,
                                             PathSlots path, WalkResume& wr) {
    bool ok = true;
    int& prev_depth = wr.prev_depth;
    uint32_t& prev_cell = wr.prev_cell;
    {
        if (!vis.segment_begin(s)) return false;
        int skip_lo, skip_hi;
        lodb::clear_range(k.lodk, lodb::V3{s.pos.x, s.pos.y, s.pos.z}, skip_lo, skip_hi);
        uint2 node = k.root;
        F3 ext_min = k.vmin, ext_max = k.vmax;
        float node_size = 1.0f, vhalf = k.rvh;
        // In the unit box the node's extent is its integer cell times 2^-depth
        // exactly (the sums below add distinct powers of two), so the cell is
        // tracked instead and the extent formed once after the descent.
        uint32_t ccx = 0u, ccy = 0u, ccz = 0u;
        F3 rbp = s.pos, cur_brp = s.pos;
        uint32_t cur_bw = k.root.y;
        int depth = 0, brick_depth = 0;
        bool is_const, loaded;
        if (RESUME && !COUNT && k.unit_box && prev_depth > 0 && prev_depth < kPathLevels && skip_lo == 0) {
            // the deepest level whose node holds both this and the last position
            const float sc = pow2i(prev_depth);
            const uint32_t nx = (uint32_t)(s.pos.x * sc), ny = (uint32_t)(s.pos.y * sc),
                           nz = (uint32_t)(s.pos.z * sc);
            const uint32_t diff = (nx ^ (prev_cell >> 20)) | (ny ^ ((prev_cell >> 10) & 0x3FFu)) |
                                  (nz ^ (prev_cell & 0x3FFu));
            int r = prev_depth - (diff ? 32 - __clz(diff) : 0);
            r = min(r, skip_hi + 1);
            if (r >= 1 && s.iter + r <= k.max_iter) {
                node = path.w[r * path.stride];
                const uint32_t pp = path.p[r * path.stride];
                s.nptr_x = pp >> 20;
                s.nptr_y = (pp >> 10) & 0x3FFu;
                s.nptr_z = pp & 0x3FFu;
                depth = r;
                vhalf = k.rvh * pow2i(-r);
                // cell and position in the cell at level r: exact (power-of-two scaling)
                const float sr = pow2i(r);
                const F3 pr = f3(s.pos.x * sr, s.pos.y * sr, s.pos.z * sr);
                ccx = (uint32_t)pr.x;
                ccy = (uint32_t)pr.y;
                ccz = (uint32_t)pr.z;
                rbp = f3(pr.x - (float)ccx, pr.y - (float)ccy, pr.z - (float)ccz);
                // the deepest resident node above r holds the brick state
#pragma unroll 1
                for (int l = r - 1; l >= 0; --l) {
                    const uint2 wl = path.w[l * path.stride];
                    if (wl.x & kResident) {
                        cur_bw = wl.y;
                        brick_depth = l;
                        const float sl = pow2i(l);
                        const F3 pl = f3(s.pos.x * sl, s.pos.y * sl, s.pos.z * sl);
                        cur_brp = f3(pl.x - floorf(pl.x), pl.y - floorf(pl.y), pl.z - floorf(pl.z));
                        break;
                    }
                }
                s.iter += r;
            }
        }
        // ---- descent to the node that stops it
        for (;;) {
            if (++s.iter > k.max_iter) {
                vis.fail(VV_ERR_TIMEOUT);
                return false;
            }
            if (RESUME && depth < kPathLevels) {
                path.w[depth * path.stride] = node;
                path.p[depth * path.stride] = (s.nptr_x << 20) | (s.nptr_y << 10) | s.nptr_z;
            }
            is_const = (node.x & kConstant) != 0u;
            loaded = (node.x & kResident) != 0u;
            if (loaded) {
                cur_bw = node.y;
                cur_brp = rbp;
                brick_depth = depth;
            }
            const uint32_t cx = (node.x >> 20) & 0x3FFu, cy = (node.x >> 10) & 0x3FFu, cz = node.x & 0x3FFu;
            if ((!is_const && !loaded) || (cx == 0u && cy == 0u && cz == 0u)) break;
            // ComputeVoxelSize (:429-441) * LodScalar, only when the other two
            // stop conditions do not decide (it has no side effects), and not
            // at the levels lodb::clear_range has shown to continue
            if (depth < skip_lo || depth > skip_hi) {
                const F3 uh = muls(k.up, vhalf), lh = muls(k.left, vhalf);
                const F3 ll = normalize3(sub(add(sub(s.pos, uh), lh), k.C));
                const F3 ur = normalize3(sub(sub(add(s.pos, uh), lh), k.C));
                const float proj = (1.0f - dot3(ll, ur)) * k.lod;
                if (k.pixel_size > proj) break;
            }
            const F3 boff = muls(rbp, 2.0f);
            const uint32_t ox = boff.x >= 1.0f ? 1u : 0u;
            const uint32_t oy = boff.y >= 1.0f ? 1u : 0u;
            const uint32_t oz = boff.z >= 1.0f ? 1u : 0u;
            rbp = sub(boff, f3((float)ox, (float)oy, (float)oz));
            s.nptr_x = cx + ox;
            s.nptr_y = cy + oy;
            s.nptr_z = cz + oz;
            ++depth;
            if (k.unit_box) {
                ccx = 2u * ccx + ox;
                ccy = 2u * ccy + oy;
                ccz = 2u * ccz + oz;
            } else {
                node_size = node_size * 0.5f;
                ext_min = add(ext_min, muls(f3((float)ox, (float)oy, (float)oz), node_size));
                ext_max = sub(ext_max, muls(f3(1.0f - (float)ox, 1.0f - (float)oy, 1.0f - (float)oz), node_size));
            }
            vhalf = vhalf * 0.5f;
            node = fetch_node<COUNT>(p, s.nptr_x, s.nptr_y, s.nptr_z, ok);
            if (!ok) {
                vis.fail(VV_ERR_BOUNDS);
                return false;
            }
        }
        if (k.unit_box) {
            const float sc = pow2i(-depth);
            ext_min = f3((float)ccx * sc, (float)ccy * sc, (float)ccz * sc);
            ext_max = f3((float)(ccx + 1u) * sc, (float)(ccy + 1u) * sc, (float)(ccz + 1u) * sc);
            if (RESUME) {
                prev_depth = depth;
                prev_cell = (ccx << 20) | (ccy << 10) | ccz;
            }
        }
        // ---- the leaf segment
        if (is_const) {
            const float ratio = pow2i(k.L - depth);
            const float step = k.RS * ratio;
            const float aw = (float)(node.y >> 24) / 255.0f;
            const float t = min_exit(s.pos, s.dir, ext_min, ext_max);
            const int n = (int)div_step(p, t, step, k.L - depth) + 1;
            if (aw < 0.005f) {
                s.pos = add(s.pos, muls(s.dir, (float)n * step));
            } else {
                const F3 wstep = muls(s.dir, step);
                const float sa = 1.0f - pow_pow2(1.0f - aw, k.L - depth);
                const float4 src = make_float4((float)(node.y & 255u) / 255.0f * ratio,
                                               (float)((node.y >> 8) & 255u) / 255.0f * ratio,
                                               (float)((node.y >> 16) & 255u) / 255.0f * ratio, sa);
#pragma unroll(STEPS)
                for (int i = 0; i < n; ++i) {
                    s.pos = add(s.pos, wstep);
                    if (s.dst.w > k.astop) {
                        const int rem = n - (i + 1);
                        s.pos = add(s.pos, muls(s.dir, (float)rem * step));
                        break;
                    }
                    const float T = 1.0f - s.dst.w;
                    const bool go = vis.sample(kSampleConst, src, s.pos, T, s.nsamples);
                    s.dst = make_float4(T * src.x + s.dst.x, T * src.y + s.dst.y, T * src.z + s.dst.z,
                                        T * src.w + s.dst.w);
                    ++s.nsamples;
                    if (!go) return false;
                }
            }
        } else {
            // lightDir = normalize(LightPosition - rayWorldPosition) at entry (:337)
            const F3 light_dir = LIT ? normalize3(sub(ld3(p.u.light_position), s.pos)) : f3(0.0f, 0.0f, 0.0f);
            // the six quotients by the pool dimensions from their reciprocals (fixed_div.h)
            const F3 bptr = f3(fixed_div((float)((cur_bw >> 20) & 0x3FFu), k.pdim.x, p.rpdim[0]),
                               fixed_div((float)((cur_bw >> 10) & 0x3FFu), k.pdim.y, p.rpdim[1]),
                               fixed_div((float)(cur_bw & 0x3FFu), k.pdim.z, p.rpdim[2]));
            const F3 brb = mul(cur_brp, k.bdim);
            F3 bpos = add(bptr, f3(fixed_div(brb.x, k.pdim.x, p.rpdim[0]), fixed_div(brb.y, k.pdim.y, p.rpdim[1]),
                                   fixed_div(brb.z, k.pdim.z, p.rpdim[2])));
            const float ratio = pow2i(k.L - brick_depth);
            const F3 wstep = muls(muls(s.dir, k.RS), ratio);
            const float t = min_exit(s.pos, s.dir, ext_min, ext_max);
            const float step = k.RS * ratio;
            const int n = (int)div_step(p, t, step, k.L - brick_depth) + 1;
            // taps inside this brick's slot skip the general texel addressing
            int base[3] = {(int)((cur_bw >> 20) & 0x3FFu) - 1, (int)((cur_bw >> 10) & 0x3FFu) - 1,
                           (int)(cur_bw & 0x3FFu) - 1};
            uint32_t slot_texel0 = 0u, slot_id = kNoSlot;
            const uint32_t* cmask = nullptr;  // the slot's empty-cell mask (not in footprint counts)
            if (base[0] >= 0 && base[1] >= 0 && base[2] >= 0 && base[0] % 10 == 0 && base[1] % 10 == 0 &&
                base[2] % 10 == 0 && base[0] < p.slots[0] * 10 && base[1] < p.slots[1] * 10 &&
                base[2] < p.slots[2] * 10) {
                const uint32_t slot = ((uint32_t)base[2] / 10u * (uint32_t)p.slots[1] + (uint32_t)base[1] / 10u) *
                                          (uint32_t)p.slots[0] + (uint32_t)base[0] / 10u;
                slot_texel0 = slot * 1000u;
                slot_id = slot;
                if (!COUNT && p.cell_mask) cmask = p.cell_mask + (size_t)slot * kCellMaskWords;
            } else {
                base[0] = base[1] = base[2] = -100000;
            }
            const bool staged = STAGED && stage_acquire(path.stage, p.bricks, slot_id, p.status);
            const uint32_t* stex = staged ? path.stage->texels : nullptr;
#pragma unroll(STEPS)
            for (int i = 0; i < n; ++i) {
                s.pos = add(s.pos, wstep);
                if (s.dst.w > k.astop) {
                    const int rem = n - (i + 1);
                    s.pos = add(s.pos, muls(s.dir, (float)rem * step));
                    break;
                }
                float4 src;
                const int in = COUNT ? kOutside : sample_in_slot<FMT, STAGED>(p, bpos, base, slot_texel0, cmask, src, stex);
                if (in == kOutside) src = sample_brick<FMT, COUNT>(p, bpos);
                src.w = 1.0f - (1.0f - src.w);
                // shading adds rgb times finite factors: nothing to a zero sample
                if (LIT && in != kEmptyCell) light_sample(p, bpos, s.dir, light_dir, src);
                const float T = 1.0f - s.dst.w;
                const bool go = vis.sample(kSampleBrick, src, bpos, T, s.nsamples);
                // a zero sample leaves dst as it is (T * 0 + dst == dst)
                if (in != kEmptyCell)
                    s.dst = make_float4(T * src.x + s.dst.x, T * src.y + s.dst.y, T * src.z + s.dst.z,
                                        T * src.w + s.dst.w);
                ++s.nsamples;
                if (!go) {
                    if (staged) stage_release(path.stage);
                    return false;
                }
                bpos = add(bpos, s.brick_step);
            }
            if (staged) stage_release(path.stage);
        }
        vis.segment_end(s, is_const, loaded);
        if (s.dst.w > k.astop && (is_const || loaded)) return false;
        // restart from the root (:688-720); the node pointer keeps its value
        return inside_box(s.pos, k.vmin, k.vmax);
    }
}

template <int FMT, bool COUNT, class V, int STEPS = 1, bool RESUME = false, bool LIT = false, bool STAGED = false>
__device__ __forceinline__ void walk(const RaycastParams& p, const WalkConsts& k, RayState& s, V& vis,
                                     PathSlots path = PathSlots{nullptr, nullptr, 0, nullptr}) {
    WalkResume wr;
    while (walk_segment<FMT, COUNT, V, STEPS, RESUME, LIT, STAGED>(p, k, s, vis, path, wr)) {
    }
}

// Visitor of the forward draw: AddToNodeUsageList (:454-488) for the leaf
// segments whose traversal index falls in this pixel's window (:663-671).
// Entries go straight to the pixel's 12 usage words in memory (zeroed
// before the walk), which keeps 12 registers free during the walk.
struct UsageVisitor {
    uint32_t* out;  // this pixel's usage words, or nullptr
    int list_slot, nl_count, pushed, start_push, max_push;
    int* status;
    __device__ __forceinline__ bool segment_begin(const RayState&) { return true; }
    __device__ __forceinline__ bool sample(int, const float4&, F3, float, int) { return true; }
    __device__ __forceinline__ void segment_end(const RayState& s, bool, bool) {
        if (nl_count >= start_push && nl_count < start_push + 12 && pushed < max_push) {
            ++pushed;
            const uint32_t bits = ((s.nptr_x + 1u) << 20) | ((s.nptr_y + 1u) << 10) | (s.nptr_z + 1u);
            if (out) out[list_slot] = bits;
            list_slot = list_slot == 11 ? 0 : list_slot + 1;
        }
        if (++nl_count >= 48) nl_count = 0;
    }
    __device__ __forceinline__ void fail(int code) { set_status(status, code); }
};

// The set-up of pixel (px,py)'s draw: its usage-list record zeroed and the
// visitor pointed at it, dst cleared, and the fragment's ray started; false
// when the pixel has no fragment or its ray starts outside the volume (its
// walk is then empty).
__device__ __forceinline__ bool start_pixel(const RaycastParams& p, const WalkConsts& k, int px, int py,
                                            RayState& s, UsageVisitor& vis) {
    const vv_uniforms& u = p.u;
    const size_t pix = (size_t)py * u.width + px;
    vis.out = nullptr;
    if (p.usage) {
        uint4* o = p.usage + pix * 3;
        o[0] = o[1] = o[2] = make_uint4(0u, 0u, 0u, 0u);
        vis.out = reinterpret_cast<uint32_t*>(o);
    }
    vis.list_slot = 0;
    vis.nl_count = 0;
    vis.pushed = 0;
    vis.start_push = (px % 2) * 12 + (py % 2) * 24;
    vis.max_push = u.max_nodes_to_push;
    vis.status = p.status;
    s.dst = make_float4(0.f, 0.f, 0.f, 0.f);
    F3 pos;
    return ray_origin(u, k, px, py, pos) && ray_start(p, k, px, py, pos, s);
}

// FragColor of pixel `pix` (:751): float4, or RGBA8 unorm.
__device__ __forceinline__ void finish_pixel(const RaycastParams& p, size_t pix, const RayState& s) {
    if (p.color) {
        if (p.color8) ((uint32_t*)p.color)[pix] = pack_unorm8(s.dst);
        else p.color[pix] = s.dst;
    }
}

// One pixel of the forward draw: the fragment's ray walk, FragColor and the
// three RGBA32UI usage-list layers (:490-751).
template <int FMT, bool COUNT, int STEPS, bool RESUME = false, bool LIT = false, bool STAGED = false>
__device__ __forceinline__ void render_pixel(const RaycastParams& p, int px, int py,
                                             PathSlots path = PathSlots{nullptr, nullptr, 0, nullptr}) {
    bool ok = true;
    const WalkConsts k = walk_consts(p, fetch_node<COUNT>(p, 0, 0, 0, ok));
    UsageVisitor vis;
    RayState s;
    if (start_pixel(p, k, px, py, s, vis))
        walk<FMT, COUNT, UsageVisitor, STEPS, RESUME, LIT, STAGED>(p, k, s, vis, path);
    finish_pixel(p, (size_t)py * p.u.width + px, s);
}

// Persistent ray cast that keeps the lanes of a warp busy: each warp takes
// 8x4 pixel tiles from a device counter and runs its rays one leaf segment
// at a time (walk_segment); a lane whose ray has ended takes the next pixel
// of the warp's tile (ballot + popc rank) before the next segment, instead
// of idling until the warp's slowest ray ends.  Same pixels, same walk, same
// results as render_pixel.
template <int FMT>
__device__ __forceinline__ void render_refill(const RaycastParams& p, unsigned int* counter, PathSlots path) {
    const vv_uniforms& u = p.u;
    const int W = u.width, H = u.height;
    const int tiles_x = (W + 7) >> 3;
    const int tiles = tiles_x * ((H + 3) >> 2);
    const unsigned lane = threadIdx.x & 31u;
    const unsigned below = (1u << lane) - 1u;
    bool ok = true;
    const WalkConsts k = walk_consts(p, fetch_node<false>(p, 0, 0, 0, ok));
    int tile = 0, taken = 32;  // the warp's tile and how many of its pixels are handed out
    bool more = true;          // tiles left
    bool active = false;
    size_t pix = 0;
    RayState s;
    UsageVisitor vis;
    WalkResume wr;
    for (;;) {
        unsigned idle = __ballot_sync(0xFFFFFFFFu, !active);
        while (idle && more) {
            if (taken == 32) {
                unsigned t = 0u;
                if (lane == 0u) t = atomicAdd(counter, 1u);
                tile = (int)__shfl_sync(0xFFFFFFFFu, t, 0);
                taken = 0;
                if (tile >= tiles) {
                    more = false;
                    break;
                }
            }
            const int n = min(__popc(idle), 32 - taken);
            const int rank = __popc(idle & below);
            if (!active && rank < n) {
                const int q = taken + rank;
                const int px = (tile % tiles_x) * 8 + (q & 7), py = (tile / tiles_x) * 4 + (q >> 3);
                if (px < W && py < H) {
                    pix = (size_t)py * W + px;
                    wr = WalkResume{};
                    active = start_pixel(p, k, px, py, s, vis);
                    if (!active) finish_pixel(p, pix, s);
                }
            }
            taken += n;
            idle = __ballot_sync(0xFFFFFFFFu, !active);
        }
        if (__ballot_sync(0xFFFFFFFFu, active) == 0u) return;
        if (active && !walk_segment<FMT, false, UsageVisitor, 1, true, false>(p, k, s, vis, path, wr)) {
            finish_pixel(p, pix, s);
            active = false;
        }
    }
}

}  // namespace rc
}  // namespace vv
