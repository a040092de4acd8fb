// kernels.cu - sm_100a kernels of the GigaVoxels hot path.
//
// raycast_kernel      GigaVoxelsNoLighting.frag main (:490-751) per pixel
// select_kernel       GenerateSelectionMask.frag + ComputeActiveTexels.frag
// pyramid_up_kernel   GenerateHistoPyramid.frag (one launch per level)
// pyramid_down_kernel the key walk of CompressNodeUsageList.frag (:55-105),
//                     run top-down as exclusive offsets instead of per key
// compact_kernel      CompressNodeUsageList.frag (:107-149), scattered by rank
//
// Floating point: this file is compiled with -fmad=false -prec-div=true
// -prec-sqrt=true and without fast-math, so every +,-,*,/ and sqrt below is
// one IEEE binary32 operation in the written order.  The only fused
// operation is the explicit fmaf() of lerp().  The host oracle performs the
// same sequence, which makes descent decisions, step counts, LOD choices and
// node-usage lists bit-identical.
#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include "kernels.cuh"

namespace vv {

namespace {

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

// pow(x, 2^k) as k squarings (the sample-ratio powers of the shader).
__device__ __forceinline__ float pow_pow2(float x, int k) {
    for (int i = 0; i < k; ++i) x = x * x;
    return x;
}

// Texel loads per storage format: 4 channels as float (RGBA8 as 0..255).
template <int FMT>
struct Texel;
template <>
struct Texel<VV_FMT_RGBA8> {
    static constexpr float kScale = 1.0f / 255.0f;
    __device__ __forceinline__ static float4 load(const void* pool, uint32_t i) {
        uint32_t v = __ldg((const uint32_t*)pool + i);
        return make_float4((float)(v & 255u), (float)((v >> 8) & 255u), (float)((v >> 16) & 255u),
                           (float)(v >> 24));
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
// texel per axis is base[]; returns false (and nothing) otherwise.  Same
// arithmetic as sample_brick: only the texel addressing is shorter.
template <int FMT>
__device__ __forceinline__ bool sample_in_slot(const RaycastParams& p, F3 uvw, const int base[3], uint32_t slot_texel0,
                                               float4& out) {
    const float* N = p.u.brick_pool_dimension;
    const float ta[3] = {uvw.x * N[0] - 0.5f, uvw.y * N[1] - 0.5f, uvw.z * N[2] - 0.5f};
    float f[3];
    int l[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        const float fi = floorf(ta[a]);
        f[a] = ta[a] - fi;
        l[a] = (int)fi - base[a];
    }
    if ((unsigned)l[0] > 8u || (unsigned)l[1] > 8u || (unsigned)l[2] > 8u) return false;
    const uint32_t i000 = slot_texel0 + (uint32_t)((l[2] * 10 + l[1]) * 10 + l[0]);
    const void* pool = p.bricks;
    const float4 v000 = Texel<FMT>::load(pool, i000), v100 = Texel<FMT>::load(pool, i000 + 1u);
    const float4 v010 = Texel<FMT>::load(pool, i000 + 10u), v110 = Texel<FMT>::load(pool, i000 + 11u);
    const float4 v001 = Texel<FMT>::load(pool, i000 + 100u), v101 = Texel<FMT>::load(pool, i000 + 101u);
    const float4 v011 = Texel<FMT>::load(pool, i000 + 110u), v111 = Texel<FMT>::load(pool, i000 + 111u);
    const float4 c0 = lerp4(lerp4(v000, v100, f[0]), lerp4(v010, v110, f[0]), f[1]);
    const float4 c1 = lerp4(lerp4(v001, v101, f[0]), lerp4(v011, v111, f[0]), f[1]);
    float4 c = lerp4(c0, c1, f[2]);
    if (Texel<FMT>::kScale != 1.0f) {
        const float k = Texel<FMT>::kScale;
        c = make_float4(c.x * k, c.y * k, c.z * k, c.w * k);
    }
    out = c;
    return true;
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

}  // namespace

template <int FMT, bool COUNT>
__global__ void __launch_bounds__(128) raycast_kernel(const __grid_constant__ RaycastParams p) {
    const vv_uniforms& u = p.u;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int px = blockIdx.x * 16 + (warp & 1) * 8 + (lane & 7);
    const int py = blockIdx.y * 8 + (warp >> 1) * 4 + (lane >> 3);
    if (px >= u.width || py >= u.height) return;
    const size_t pix = (size_t)py * u.width + px;

    uint32_t usage[12];
#pragma unroll
    for (int i = 0; i < 12; ++i) usage[i] = 0u;
    float4 dst = make_float4(0.f, 0.f, 0.f, 0.f);

    const F3 C = ld3(u.camera_position);
    const F3 vmin = ld3(u.vol_extent_min), vmax = ld3(u.vol_extent_max);

    // Ray origin: the fragment's RayPosition (box entry or near-plane point).
    bool frag = true;
    F3 pos;
    {
        const float fx = (float)px + 0.5f, fy = (float)py + 0.5f;
        const F3 d = f3(u.near_origin[0] + fx * u.near_dx[0] + fy * u.near_dy[0],
                        u.near_origin[1] + fx * u.near_dx[1] + fy * u.near_dy[1],
                        u.near_origin[2] + fx * u.near_dx[2] + fy * u.near_dy[2]);
        if (u.camera_inside) {
            pos = add(C, d);
        } else {
            const float da[3] = {d.x, d.y, d.z}, ca[3] = {C.x, C.y, C.z};
            const float mn[3] = {vmin.x, vmin.y, vmin.z}, mx[3] = {vmax.x, vmax.y, vmax.z};
            float tenter = -INFINITY, texit = INFINITY;
            int axis = -1;
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
            if (frag) {
                float pa[3] = {ca[0] + da[0] * tenter, ca[1] + da[1] * tenter, ca[2] + da[2] * tenter};
#pragma unroll
                for (int a = 0; a < 3; ++a)
                    if (a == axis) pa[a] = da[a] > 0.0f ? mn[a] : mx[a];
                pos = f3(pa[0], pa[1], pa[2]);
            }
        }
    }

    if (frag) {
        const float RS = u.ray_step_size;
        const int L = u.oct_tree_depth_minus_one;
        const float astop = u.alpha_stop;
        const F3 dir = normalize3(sub(pos, C));
        const int J = u.jitter_tex_size;
        const float jitter = (float)p.jitter[(py % J) * J + (px % J)] / 255.0f;
        pos = add(pos, muls(muls(dir, RS), jitter));
        bool inside = inside_box(pos, vmin, vmax);
        if (inside) {
            int list_slot = 0;  // curListIndex*4 + curComponentIndex
            const int start_push = (px % 2) * 12 + (py % 2) * 24;
            const int stop_push = start_push + 12;
            const F3 brick_step = mul(dir, ld3(u.brick_step_vector));
            const F3 bdim = ld3(u.brick_dimension), pdim = ld3(u.brick_pool_dimension);
            const F3 up = ld3(u.camera_up), left = ld3(u.camera_left);

            bool ok = true;
            uint32_t nptr_x = 0, nptr_y = 0, nptr_z = 0;
            const uint2 root = fetch_node<COUNT>(p, 0, 0, 0, ok);
            uint2 node = root;
            F3 ext_min = vmin, ext_max = vmax;
            float node_size = 1.0f;
            float vhalf = u.root_voxel_half_size;
            F3 rbp = pos;       // rayBrickPosition
            F3 cur_brp = pos;   // curBrickRayPosition
            uint2 cur_brick = root;
            int depth = 0, brick_depth = 0;
            int nl_count = 0, pushed = 0;
            int iter = 0;
            // Segment-synchronous ("while-while") form: the descent to the
            // stopping node is its own loop, then the segment is marched.  Lanes of
            // a warp descend together and march together, which keeps far more of
            // them converged than alternating single levels with whole segments.
            bool failed = false;
            while (inside) {
                // ---- descent from the root to the node that stops it (:563-622, :722-746)
                bool is_const, loaded;
                for (;;) {
                    if (++iter > p.max_iter) {
                        set_status(p.status, VV_ERR_TIMEOUT);
                        failed = true;
                        break;
                    }
                    is_const = (node.x & kConstant) != 0u;
                    loaded = (node.x & kResident) != 0u;
                    if (loaded) {
                        cur_brick = node;
                        cur_brp = rbp;
                        brick_depth = depth;
                    }
                    const uint32_t cx = (node.x >> 20) & 0x3FFu, cy = (node.x >> 10) & 0x3FFu, cz = node.x & 0x3FFu;
                    if ((!is_const && !loaded) || (cx == 0u && cy == 0u && cz == 0u)) break;
                    // ComputeVoxelSize (:429-441) * LodScalar, only when the other
                    // two stop conditions do not decide (it has no side effects)
                    {
                        const F3 uh = muls(up, vhalf), lh = muls(left, vhalf);
                        const F3 ll = normalize3(sub(add(sub(pos, uh), lh), C));
                        const F3 ur = normalize3(sub(sub(add(pos, uh), lh), C));
                        const float proj = (1.0f - dot3(ll, ur)) * u.lod_scalar;
                        if (u.pixel_size > proj) break;
                    }
                    const F3 boff = muls(rbp, 2.0f);
                    const uint32_t ox = boff.x >= 1.0f ? 1u : 0u;
                    const uint32_t oy = boff.y >= 1.0f ? 1u : 0u;
                    const uint32_t oz = boff.z >= 1.0f ? 1u : 0u;
                    rbp = sub(boff, f3((float)ox, (float)oy, (float)oz));
                    nptr_x = cx + ox;
                    nptr_y = cy + oy;
                    nptr_z = cz + oz;
                    ++depth;
                    node_size = node_size * 0.5f;
                    ext_min = add(ext_min, muls(f3((float)ox, (float)oy, (float)oz), node_size));
                    ext_max = sub(ext_max, muls(f3(1.0f - (float)ox, 1.0f - (float)oy, 1.0f - (float)oz), node_size));
                    vhalf = vhalf * 0.5f;
                    node = fetch_node<COUNT>(p, nptr_x, nptr_y, nptr_z, ok);
                    if (!ok) {
                        set_status(p.status, VV_ERR_BOUNDS);
                        failed = true;
                        break;
                    }
                }
                if (failed) break;
                // ---- the leaf segment
                if (is_const) {
                    // TraverseConstant (:230-282)
                    const float ratio = ldexpf(1.0f, L - depth);
                    const float step = RS * ratio;
                    const float aw = (float)(node.y >> 24) / 255.0f;
                    const float t = min_exit(pos, dir, ext_min, ext_max);
                    const int n = (int)(t / step) + 1;
                    if (aw < 0.005f) {
                        pos = add(pos, muls(dir, (float)n * step));
                    } else {
                        const F3 wstep = muls(dir, step);
                        const float sa = 1.0f - pow_pow2(1.0f - aw, L - depth);
                        const float4 src = make_float4((float)(node.y & 255u) / 255.0f * ratio,
                                                       (float)((node.y >> 8) & 255u) / 255.0f * ratio,
                                                       (float)((node.y >> 16) & 255u) / 255.0f * ratio, sa);
                        for (int i = 0; i < n; ++i) {
                            pos = add(pos, wstep);
                            if (dst.w > astop) {
                                const int rem = n - (i + 1);
                                pos = add(pos, muls(dir, (float)rem * step));
                                break;
                            }
                            const float k = 1.0f - dst.w;
                            dst = make_float4(k * src.x + dst.x, k * src.y + dst.y, k * src.z + dst.z,
                                              k * src.w + dst.w);
                        }
                    }
                } else {
                    // TraverseBrick (:311-359) over the most recently found brick
                    const uint32_t bw = cur_brick.y;
                    const F3 bptr = f3((float)((bw >> 20) & 0x3FFu) / pdim.x, (float)((bw >> 10) & 0x3FFu) / pdim.y,
                                       (float)(bw & 0x3FFu) / pdim.z);
                    F3 bpos = add(bptr, divv(mul(cur_brp, bdim), pdim));
                    const float ratio = ldexpf(1.0f, L - brick_depth);
                    const F3 wstep = muls(muls(dir, RS), ratio);
                    const float t = min_exit(pos, dir, ext_min, ext_max);
                    const float step = RS * ratio;
                    const int n = (int)(t / step) + 1;
                    // taps inside this brick's slot skip the general texel addressing
                    int base[3] = {(int)((bw >> 20) & 0x3FFu) - 1, (int)((bw >> 10) & 0x3FFu) - 1,
                                   (int)(bw & 0x3FFu) - 1};
                    uint32_t slot_texel0 = 0u;
                    if (base[0] >= 0 && base[1] >= 0 && base[2] >= 0 && base[0] % 10 == 0 && base[1] % 10 == 0 &&
                        base[2] % 10 == 0 && base[0] < p.slots[0] * 10 && base[1] < p.slots[1] * 10 &&
                        base[2] < p.slots[2] * 10) {
                        slot_texel0 = (((uint32_t)base[2] / 10u * (uint32_t)p.slots[1] + (uint32_t)base[1] / 10u) *
                                           (uint32_t)p.slots[0] + (uint32_t)base[0] / 10u) * 1000u;
                    } else {
                        base[0] = base[1] = base[2] = -100000;
                    }
                    for (int i = 0; i < n; ++i) {
                        pos = add(pos, wstep);
                        if (dst.w > astop) {
                            const int rem = n - (i + 1);
                            pos = add(pos, muls(dir, (float)rem * step));
                            break;
                        }
                        float4 src;
                        if (COUNT || !sample_in_slot<FMT>(p, bpos, base, slot_texel0, src))
                            src = sample_brick<FMT, COUNT>(p, bpos);
                        src.w = 1.0f - (1.0f - src.w);
                        const float k = 1.0f - dst.w;
                        dst = make_float4(k * src.x + dst.x, k * src.y + dst.y, k * src.z + dst.z, k * src.w + dst.w);
                        bpos = add(bpos, brick_step);
                    }
                }
                // AddToNodeUsageList (:454-488)
                if (nl_count >= start_push && nl_count < stop_push && pushed < u.max_nodes_to_push) {
                    ++pushed;
                    const uint32_t bits = ((nptr_x + 1u) << 20) | ((nptr_y + 1u) << 10) | (nptr_z + 1u);
#pragma unroll
                    for (int i = 0; i < 12; ++i)
                        if (i == list_slot) usage[i] = bits;
                    list_slot = list_slot == 11 ? 0 : list_slot + 1;
                }
                if (dst.w > astop && (is_const || loaded)) break;
                // restart from the root (:688-720); the node pointer keeps its value
                node = root;
                ext_min = vmin;
                ext_max = vmax;
                node_size = 1.0f;
                vhalf = u.root_voxel_half_size;
                rbp = pos;
                cur_brp = pos;
                cur_brick = root;
                depth = 0;
                brick_depth = 0;
                inside = inside_box(pos, vmin, vmax);
                ++nl_count;
                if (nl_count >= 48) nl_count = 0;
            }
        }
    }
    if (p.color) p.color[pix] = dst;
    if (p.usage) {
        uint4* o = p.usage + pix * 3;
        o[0] = make_uint4(usage[0], usage[1], usage[2], usage[3]);
        o[1] = make_uint4(usage[4], usage[5], usage[6], usage[7]);
        o[2] = make_uint4(usage[8], usage[9], usage[10], usage[11]);
    }
}

cudaError_t launch_raycast(int fmt, const RaycastParams& p, cudaStream_t s) {
    dim3 block(128);
    dim3 grid((unsigned)((p.u.width + 15) / 16), (unsigned)((p.u.height + 7) / 8));
    const bool count = p.node_touch && p.brick_touch;
#define VV_LAUNCH(F)                                                           \
    if (count) raycast_kernel<F, true><<<grid, block, 0, s>>>(p);              \
    else raycast_kernel<F, false><<<grid, block, 0, s>>>(p);
    switch (fmt) {
        case VV_FMT_RGBA8: VV_LAUNCH(VV_FMT_RGBA8) break;
        case VV_FMT_FP16: VV_LAUNCH(VV_FMT_FP16) break;
        case VV_FMT_BF16: VV_LAUNCH(VV_FMT_BF16) break;
        case VV_FMT_FP32: VV_LAUNCH(VV_FMT_FP32) break;
        default: return cudaErrorInvalidValue;
    }
#undef VV_LAUNCH
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// GenerateSelectionMask.frag (:15-187) + ComputeActiveTexels.frag (:9-25)

__global__ void select_kernel(const uint4* __restrict__ usage, uint32_t* __restrict__ mask,
                              uint32_t* __restrict__ level0, int w, int h) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= w || y >= h) return;
    const size_t pix = (size_t)y * w + x;
    uint32_t own[12];
    {
        const uint4* o = usage + pix * 3;
        uint4 a = o[0], b = o[1], c = o[2];
        own[0] = a.x; own[1] = a.y; own[2] = a.z; own[3] = a.w;
        own[4] = b.x; own[5] = b.y; own[6] = b.z; own[7] = b.w;
        own[8] = c.x; own[9] = c.y; own[10] = c.z; own[11] = c.w;
    }
    uint32_t bits = 0u;
    if (own[0] != 0u) {
        uint32_t top[12], tr[12], rt[12];
        const bool has_top = y < h - 2, has_right = x < w - 2;
        auto load = [&](uint32_t* dstl, bool cond, int nx, int ny) {
            if (cond) {
                const uint4* o = usage + ((size_t)ny * w + nx) * 3;
                uint4 a = o[0], b = o[1], c = o[2];
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
    }
    if (mask) mask[pix] = bits;
    level0[pix] = bits != 0u ? 1u : 0u;
}

cudaError_t launch_select(const uint4* usage, uint32_t* mask, uint32_t* level0, int w, int h,
                          cudaStream_t s) {
    dim3 block(32, 4);
    dim3 grid((unsigned)((w + 31) / 32), (unsigned)((h + 3) / 4));
    select_kernel<<<grid, block, 0, s>>>(usage, mask, level0, w, h);
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Histopyramid.  Children of parent (X,Y) at the finer level (w,h), in the
// order CompressNodeUsageList walks them: the 2x2 block, then for an odd last
// row (x,y+2),(x+1,y+2) and for an odd last column the (x+2,*) cells.

__device__ __forceinline__ int child_list(int X, int Y, int w, int h, int* cx, int* cy) {
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

__device__ __forceinline__ uint32_t cell(const uint32_t* lvl, int x, int y, int w, int h) {
    return (x < w && y < h) ? lvl[(size_t)y * w + x] : 0u;
}

__global__ void pyramid_up_kernel(const uint32_t* __restrict__ fine, uint32_t* __restrict__ coarse, int w,
                                  int h, int cw, int ch) {
    const int X = blockIdx.x * blockDim.x + threadIdx.x;
    const int Y = blockIdx.y * blockDim.y + threadIdx.y;
    if (X >= cw || Y >= ch) return;
    int cx[9], cy[9];
    const int n = child_list(X, Y, w, h, cx, cy);
    uint32_t sum = 0u;
    for (int i = 0; i < n; ++i) sum += cell(fine, cx[i], cy[i], w, h);
    coarse[(size_t)Y * cw + X] = sum;
}

// Offsets at the finer level from the coarser level's offsets: each child
// finds its parent and adds the counts of the siblings walked before it.
__global__ void pyramid_down_kernel(const uint32_t* __restrict__ fine_cnt, uint32_t* __restrict__ fine_off,
                                    const uint32_t* __restrict__ coarse_off, int w, int h, int cw, int ch) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= w || y >= h) return;
    const int X = min(x >> 1, cw - 1), Y = min(y >> 1, ch - 1);
    int cx[9], cy[9];
    const int n = child_list(X, Y, w, h, cx, cy);
    uint32_t off = coarse_off[(size_t)Y * cw + X];
    for (int i = 0; i < n; ++i) {
        if (cx[i] == x && cy[i] == y) break;
        off += cell(fine_cnt, cx[i], cy[i], w, h);
    }
    fine_off[(size_t)y * w + x] = off;
}

__global__ void compact_kernel(const __grid_constant__ CompactParams p) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= p.width || y >= p.height) return;
    const size_t pix = (size_t)y * p.width + x;
    uint32_t bits = p.mask[pix];
    if (bits == 0u) return;
    const uint32_t rank = p.offsets[pix];
    if (rank >= (uint32_t)p.cap) return;
    const uint4* o = p.usage + pix * 3;
    uint4 a = o[0], b = o[1], c = o[2];
    const uint32_t list[12] = {a.x, a.y, a.z, a.w, b.x, b.y, b.z, b.w, c.x, c.y, c.z, c.w};
    uint32_t out[4] = {0u, 0u, 0u, 0u};
    int pushed = 0;
    for (int item = 0; item < 12 && bits != 0u && pushed < p.max_push; ++item, bits >>= 1) {
        if (bits & 1u) {
            out[pushed & 3] = list[item];
            ++pushed;
        }
    }
    reinterpret_cast<uint4*>(p.requests)[rank] = make_uint4(out[0], out[1], out[2], out[3]);
}

__global__ void copy_total_kernel(const uint32_t* top, uint32_t* dst) {
    if (threadIdx.x == 0 && blockIdx.x == 0) *dst = *top;
}

cudaError_t launch_pyramid_levels(uint32_t* counts, uint32_t* offsets, const int* lw, const int* lh,
                                  const long long* loff, int first, int levels, cudaStream_t s) {
    dim3 block(32, 4);
    for (int l = first; l + 1 < levels; ++l) {
        const int cw = lw[l + 1], ch = lh[l + 1];
        dim3 grid((unsigned)((cw + 31) / 32), (unsigned)((ch + 3) / 4));
        pyramid_up_kernel<<<grid, block, 0, s>>>(counts + loff[l], counts + loff[l + 1], lw[l], lh[l], cw, ch);
    }
    cudaError_t e = cudaMemsetAsync(offsets + loff[levels - 1], 0, sizeof(uint32_t), s);
    if (e != cudaSuccess) return e;
    for (int l = levels - 2; l >= first; --l) {
        dim3 grid((unsigned)((lw[l] + 31) / 32), (unsigned)((lh[l] + 3) / 4));
        pyramid_down_kernel<<<grid, block, 0, s>>>(counts + loff[l], offsets + loff[l], offsets + loff[l + 1], lw[l],
                                                   lh[l], lw[l + 1], lh[l + 1]);
    }
    return cudaGetLastError();
}

cudaError_t launch_compact(const CompactParams& p, cudaStream_t s) {
    dim3 block(32, 4);
    for (int l = 0; l + 1 < p.levels; ++l) {
        const int cw = p.level_w[l + 1], ch = p.level_h[l + 1];
        dim3 grid((unsigned)((cw + 31) / 32), (unsigned)((ch + 3) / 4));
        pyramid_up_kernel<<<grid, block, 0, s>>>(p.counts + p.level_off[l], p.counts + p.level_off[l + 1],
                                                 p.level_w[l], p.level_h[l], cw, ch);
    }
    const int top = p.levels - 1;
    cudaMemsetAsync(p.offsets + p.level_off[top], 0, sizeof(uint32_t), s);
    for (int l = top - 1; l >= 0; --l) {
        const int w = p.level_w[l], h = p.level_h[l];
        dim3 grid((unsigned)((w + 31) / 32), (unsigned)((h + 3) / 4));
        pyramid_down_kernel<<<grid, block, 0, s>>>(p.counts + p.level_off[l], p.offsets + p.level_off[l],
                                                   p.offsets + p.level_off[l + 1], w, h, p.level_w[l + 1],
                                                   p.level_h[l + 1]);
    }
    if (p.request_count) copy_total_kernel<<<1, 32, 0, s>>>(p.counts + p.level_off[top], p.request_count);
    if (p.requests && p.cap > 0) {
        dim3 grid((unsigned)((p.width + 31) / 32), (unsigned)((p.height + 3) / 4));
        compact_kernel<<<grid, block, 0, s>>>(p);
    }
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Node pool: reference texture order <-> block-linear device layout.

__device__ __forceinline__ size_t block_linear(uint32_t x, uint32_t y, uint32_t z, int dx, int dy) {
    const uint32_t bx = (uint32_t)dx >> 1, by = (uint32_t)dy >> 1;
    size_t blk = ((size_t)(z >> 1) * by + (y >> 1)) * bx + (x >> 1);
    return blk * 8u + ((x & 1u) | ((y & 1u) << 1) | ((z & 1u) << 2));
}

__global__ void node_upload_kernel(const uint2* __restrict__ grid, uint2* __restrict__ nodes, int dx, int dy,
                                   int dz) {
    const size_t total = (size_t)dx * dy * dz;
    for (size_t g = blockIdx.x * (size_t)blockDim.x + threadIdx.x; g < total; g += (size_t)gridDim.x * blockDim.x) {
        uint32_t x = (uint32_t)(g % dx), y = (uint32_t)((g / dx) % dy), z = (uint32_t)(g / ((size_t)dx * dy));
        nodes[block_linear(x, y, z, dx, dy)] = grid[g];
    }
}

__global__ void node_download_kernel(const uint2* __restrict__ nodes, uint2* __restrict__ grid, int dx, int dy,
                                     int dz) {
    const size_t total = (size_t)dx * dy * dz;
    for (size_t g = blockIdx.x * (size_t)blockDim.x + threadIdx.x; g < total; g += (size_t)gridDim.x * blockDim.x) {
        uint32_t x = (uint32_t)(g % dx), y = (uint32_t)((g / dx) % dy), z = (uint32_t)(g / ((size_t)dx * dy));
        grid[g] = nodes[block_linear(x, y, z, dx, dy)];
    }
}

__global__ void node_patch_kernel(const vv_node_patch* __restrict__ patches, int n, uint2* __restrict__ nodes,
                                  int dx, int dy, int dz, int* status) {
    // The host hands over at most one patch per node (the last one it made),
    // so the parallel writes are order-independent.
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const vv_node_patch q = patches[i];
    if (q.x >= (uint32_t)dx || q.y >= (uint32_t)dy || q.z >= (uint32_t)dz) {
        set_status(status, VV_ERR_BOUNDS);
        return;
    }
    nodes[block_linear(q.x, q.y, q.z, dx, dy)] = make_uint2(q.word0, q.word1);
}

cudaError_t launch_node_upload(const uint32_t* grid_words, uint2* nodes, const int dim[3], cudaStream_t s) {
    node_upload_kernel<<<592, 256, 0, s>>>((const uint2*)grid_words, nodes, dim[0], dim[1], dim[2]);
    return cudaGetLastError();
}

cudaError_t launch_node_download(const uint2* nodes, uint32_t* grid_words, const int dim[3], cudaStream_t s) {
    node_download_kernel<<<592, 256, 0, s>>>(nodes, (uint2*)grid_words, dim[0], dim[1], dim[2]);
    return cudaGetLastError();
}

cudaError_t launch_node_patch(const vv_node_patch* patches, int n, uint2* nodes, const int dim[3], int* status,
                              cudaStream_t s) {
    if (n <= 0) return cudaSuccess;
    node_patch_kernel<<<(n + 255) / 256, 256, 0, s>>>(patches, n, nodes, dim[0], dim[1], dim[2], status);
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Brick upload: scatter n staged bricks into their pool slots, 16-byte
// vectors, one CTA per brick.

__global__ void brick_scatter_kernel(const uint32_t* __restrict__ slots, const uint4* __restrict__ src,
                                     uint4* __restrict__ pool, int vec_per_brick, long long total_slots,
                                     int* status) {
    const int b = blockIdx.x;
    const uint32_t slot = slots[b];
    if ((long long)slot >= total_slots) {
        if (threadIdx.x == 0) set_status(status, VV_ERR_BOUNDS);
        return;
    }
    const uint4* s = src + (size_t)b * vec_per_brick;
    uint4* d = pool + (size_t)slot * vec_per_brick;
    for (int i = threadIdx.x; i < vec_per_brick; i += blockDim.x) d[i] = __ldg(s + i);
}

cudaError_t launch_brick_scatter(const uint32_t* slots, int n, const void* src, void* pool, size_t brick_bytes,
                                 long long total_slots, int* status, cudaStream_t s) {
    if (n <= 0) return cudaSuccess;
    brick_scatter_kernel<<<n, 256, 0, s>>>(slots, (const uint4*)src, (uint4*)pool, (int)(brick_bytes / 16),
                                           total_slots, status);
    return cudaGetLastError();
}

}  // namespace vv
