// gv_oracle.cpp - CPU oracle of the GigaVoxels hot path.  TEST INFRASTRUCTURE.
//
// This file is the checker, not the product: only tests/, the smoke check in
// __graft_entry__.py and the cpu_baseline leg of bench.py load it.  It is a
// C++ transcription of the reference's GLSL passes, written the way
// GigaVoxelsShaderCodeTester.cpp:14-18 runs shader code on the host (shader
// bodies over a small vector shim), but following the CURRENT shaders:
//
//   raycast     VoxViz/Shaders/GigaVoxelsNoLighting.frag main (:490-751)
//               (= GigaVoxels.frag:544-805 without lighting)
//   select      VoxViz/Shaders/GenerateSelectionMask.frag (:15-187)
//   pyramid     VoxViz/Shaders/ComputeActiveTexels.frag (:9-25) and
//               VoxViz/Shaders/GenerateHistoPyramid.frag (:9-55), level sizes
//               as GigaVoxelsRenderer::generateSelectionMaskHistoPyramid
//               (VoxViz/GigaVoxels/GigaVoxelsRenderer.cpp:1967-2046)
//   compress    VoxViz/Shaders/CompressNodeUsageList.frag (:44-150), one key
//               at a time by walking the pyramid as the shader does
//
// Decisions the GLSL leaves open, fixed identically in the CUDA kernels:
//   * every vector op is per-component IEEE arithmetic in source order, no
//     contraction (built with -ffp-contract=off); normalize(v) = v*(1/sqrt(dot))
//   * texture() is GL_LINEAR + CLAMP_TO_EDGE from the GL 3.3 specification
//     (section 3.8.8) with exact weights; lerp(a,b,t) = fma(t, b-a, a) and the
//     lerps run x, then y, then z; RGBA8 texels are filtered as 0..255 and the
//     result is scaled by 1/255
//   * pow(x, 2^k) is k squarings; pow(2, k) is exact
//   * float -> uint conversion of a negative value gives 0
//   * the early-termination literal 0.995 is the parameter alpha_stop
//   * a ray runs at most max_iter outer iterations (never reached on valid data)
//
// The FP64 instantiation runs the same algorithm in double from the same
// uniforms; it is the colour-error reference, not a bit-exact target.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

#ifdef _OPENMP
#include <omp.h>
#endif

#include "../include/voxviz_b200.h"
#include "gv_oracle.h"

namespace {

template <typename T>
struct vec3 {
    T x, y, z;
    vec3() : x(0), y(0), z(0) {}
    vec3(T a, T b, T c) : x(a), y(b), z(c) {}
    vec3 operator+(const vec3& o) const { return vec3(x + o.x, y + o.y, z + o.z); }
    vec3 operator-(const vec3& o) const { return vec3(x - o.x, y - o.y, z - o.z); }
    vec3 operator*(const vec3& o) const { return vec3(x * o.x, y * o.y, z * o.z); }
    vec3 operator/(const vec3& o) const { return vec3(x / o.x, y / o.y, z / o.z); }
    vec3 operator*(T s) const { return vec3(x * s, y * s, z * s); }
    vec3& operator+=(const vec3& o) { return *this = *this + o; }
    vec3& operator-=(const vec3& o) { return *this = *this - o; }
    vec3& operator*=(T s) { return *this = *this * s; }
    vec3& operator*=(const vec3& o) { return *this = *this * o; }
};
template <typename T>
struct vec4 {
    T r, g, b, a;
};
template <typename T>
T dot(const vec3<T>& a, const vec3<T>& b) {
    return a.x * b.x + a.y * b.y + a.z * b.z;
}
template <typename T>
vec3<T> normalize(const vec3<T>& v) {
    T inv = T(1) / std::sqrt(dot(v, v));
    return v * inv;
}
template <typename T>
vec3<T> from(const float* f) {
    return vec3<T>((T)f[0], (T)f[1], (T)f[2]);
}
template <typename T>
T glsl_lerp(T a, T b, T t) {
    return std::fma(t, b - a, a);
}
template <typename T>
T pow_pow2(T x, int k) {
    for (int i = 0; i < k; ++i) x = x * x;
    return x;
}
inline uint32_t to_uint(float f) { return f > 0.0f ? (uint32_t)f : 0u; }
inline uint32_t to_uint(double f) { return f > 0.0 ? (uint32_t)f : 0u; }

uint16_t rd16(const void* p, size_t i) {
    uint16_t v;
    std::memcpy(&v, (const unsigned char*)p + 2 * i, 2);
    return v;
}
float half_to_float(uint16_t h) {
    const uint32_t s = (uint32_t)(h & 0x8000u) << 16;
    uint32_t e = (h >> 10) & 0x1Fu, m = h & 0x3FFu;
    uint32_t bits;
    if (e == 0) {
        if (m == 0) {
            bits = s;
        } else {  // subnormal
            int sh = 0;
            while (!(m & 0x400u)) {
                m <<= 1;
                ++sh;
            }
            m &= 0x3FFu;
            bits = s | ((uint32_t)(127 - 15 + 1 - sh) << 23) | (m << 13);
        }
    } else if (e == 31) {
        bits = s | 0x7F800000u | (m << 13);
    } else {
        bits = s | ((e + 112u) << 23) | (m << 13);
    }
    float f;
    std::memcpy(&f, &bits, 4);
    return f;
}
float bf16_to_float(uint16_t h) {
    uint32_t bits = (uint32_t)h << 16;
    float f;
    std::memcpy(&f, &bits, 4);
    return f;
}

// S3TC decode (EXT_texture_compression_s3tc) of one texel, with the
// expansion and rounding the library fixes: 5/6-bit channels widened by bit
// replication, interpolated colours (2a+b+1)/3 and (a+2b+1)/3 (or (a+b+1)/2
// and black in DXT1's three-colour mode), interpolated alphas
// ((8-k)a0+(k-1)a1+3)/7, or ((6-k)a0+(k-1)a1+2)/5 with codes 6, 7 = 0, 255.
// The block's bytes are read one by one (little endian).
void s3tc_colour(const unsigned char* blk, int texel, bool force_four, int rgb[3]) {
    const unsigned c0 = (unsigned)blk[0] | ((unsigned)blk[1] << 8), c1 = (unsigned)blk[2] | ((unsigned)blk[3] << 8);
    const unsigned code = ((unsigned)blk[4 + texel / 4] >> (2 * (texel % 4))) & 3u;
    const int e0[3] = {(int)(((c0 >> 11) << 3) | ((c0 >> 11) >> 2)), (int)((((c0 >> 5) & 63u) << 2) | (((c0 >> 5) & 63u) >> 4)),
                       (int)(((c0 & 31u) << 3) | ((c0 & 31u) >> 2))};
    const int e1[3] = {(int)(((c1 >> 11) << 3) | ((c1 >> 11) >> 2)), (int)((((c1 >> 5) & 63u) << 2) | (((c1 >> 5) & 63u) >> 4)),
                       (int)(((c1 & 31u) << 3) | ((c1 & 31u) >> 2))};
    for (int ch = 0; ch < 3; ++ch) {
        int v;
        if (code == 0) v = e0[ch];
        else if (code == 1) v = e1[ch];
        else if (force_four || c0 > c1) v = code == 2 ? (2 * e0[ch] + e1[ch] + 1) / 3 : (e0[ch] + 2 * e1[ch] + 1) / 3;
        else v = code == 2 ? (e0[ch] + e1[ch] + 1) / 2 : 0;
        rgb[ch] = v;
    }
}
int s3tc_alpha(const unsigned char* blk, int texel) {
    const int a0 = blk[0], a1 = blk[1];
    uint64_t bits = 0;
    for (int b = 0; b < 6; ++b) bits |= (uint64_t)blk[2 + b] << (8 * b);
    const int k = (int)((bits >> (3 * texel)) & 7u);
    if (k == 0) return a0;
    if (k == 1) return a1;
    if (a0 > a1) return ((8 - k) * a0 + (k - 1) * a1 + 3) / 7;
    if (k == 6) return 0;
    if (k == 7) return 255;
    return ((6 - k) * a0 + (k - 1) * a1 + 2) / 5;
}

// The brick pool as the reference's 3D texture: texelFetch at global texel
// (i,j,k) of a (10*slots) per-axis grid, read from the brick-linear slots.
template <typename T>
struct BrickTexture {
    const void* data;
    int fmt;
    int sx, sy, sz;
    vec4<T> fetch(int i, int j, int k) const {
        const size_t slot = ((size_t)(k / 10) * sy + (size_t)(j / 10)) * sx + (size_t)(i / 10);
        const size_t t = slot * 1000 + (size_t)((k % 10) * 100 + (j % 10) * 10 + (i % 10));
        vec4<T> v;
        if (fmt == VV_FMT_DXT5 || fmt == VV_FMT_DXT1) {
            // a slot's 10 slices of 3x3 blocks of 4x4 texels
            const int x = i % 10, y = j % 10, z = k % 10;
            const size_t blk = slot * 90 + (size_t)(z * 9 + (y / 4) * 3 + x / 4);
            const int texel = (y % 4) * 4 + x % 4;
            int rgb[3], a = 0;
            if (fmt == VV_FMT_DXT5) {
                const unsigned char* b = (const unsigned char*)data + 16 * blk;
                a = s3tc_alpha(b, texel);
                s3tc_colour(b + 8, texel, true, rgb);
            } else {
                s3tc_colour((const unsigned char*)data + 8 * blk, texel, false, rgb);
            }
            v.r = (T)rgb[0];
            v.g = (T)rgb[1];
            v.b = (T)rgb[2];
            v.a = (T)a;
            return v;
        }
        switch (fmt) {
            case VV_FMT_RGBA8: {
                uint32_t w;
                std::memcpy(&w, (const unsigned char*)data + 4 * t, 4);
                v.r = (T)(w & 255u);
                v.g = (T)((w >> 8) & 255u);
                v.b = (T)((w >> 16) & 255u);
                v.a = (T)(w >> 24);
                break;
            }
            case VV_FMT_FP16:
                v.r = (T)half_to_float(rd16(data, 4 * t));
                v.g = (T)half_to_float(rd16(data, 4 * t + 1));
                v.b = (T)half_to_float(rd16(data, 4 * t + 2));
                v.a = (T)half_to_float(rd16(data, 4 * t + 3));
                break;
            case VV_FMT_BF16:
                v.r = (T)bf16_to_float(rd16(data, 4 * t));
                v.g = (T)bf16_to_float(rd16(data, 4 * t + 1));
                v.b = (T)bf16_to_float(rd16(data, 4 * t + 2));
                v.a = (T)bf16_to_float(rd16(data, 4 * t + 3));
                break;
            default: {
                float f[4];
                std::memcpy(f, (const unsigned char*)data + 16 * t, 16);
                v.r = (T)f[0];
                v.g = (T)f[1];
                v.b = (T)f[2];
                v.a = (T)f[3];
            }
        }
        return v;
    }
};

template <typename T>
vec4<T> lerp4(const vec4<T>& a, const vec4<T>& b, T t) {
    return vec4<T>{glsl_lerp(a.r, b.r, t), glsl_lerp(a.g, b.g, t), glsl_lerp(a.b, b.b, t), glsl_lerp(a.a, b.a, t)};
}

struct SampleRec {
    bool brick;
    double src[4];
    double T;
    float bpos[3];
};

// Per-pixel shader state and body.
template <typename T>
struct Shader {
    // uniforms
    const vv_uniforms* U;
    T RayStepSize;
    vec3<T> BrickStepVector, CameraPosition, CameraUp, CameraLeft, VolExtentMin, VolExtentMax;
    vec3<T> BrickDimension, BrickPoolDimension;
    T RootVoxelHalfSize, PixelSize, LodScalar, AlphaStop;
    int OctTreeDepthMinusOne, MaxNodesToPushThisFrame, JitterTexSize;
    bool RootNodeIsConstant;
    bool ComputeLighting = false, GradientsAreUnsigned = false;
    vec3<T> LightPosition;
    // samplers
    const uint32_t* nodes;  // texture order, 2 words per texel
    int ndim[3];
    BrickTexture<T> brick;
    BrickTexture<T> grads;  // BrickGradientsSampler (lighting); data NULL when absent
    const uint8_t* jitter;
    int max_iter;
    int* status;
    std::vector<SampleRec>* tape = nullptr;

    void init(const vv_uniforms* u) {
        U = u;
        RayStepSize = (T)u->ray_step_size;
        BrickStepVector = from<T>(u->brick_step_vector);
        CameraPosition = from<T>(u->camera_position);
        CameraUp = from<T>(u->camera_up);
        CameraLeft = from<T>(u->camera_left);
        VolExtentMin = from<T>(u->vol_extent_min);
        VolExtentMax = from<T>(u->vol_extent_max);
        BrickDimension = from<T>(u->brick_dimension);
        BrickPoolDimension = from<T>(u->brick_pool_dimension);
        RootVoxelHalfSize = (T)u->root_voxel_half_size;
        PixelSize = (T)u->pixel_size;
        LodScalar = (T)u->lod_scalar;
        AlphaStop = (T)u->alpha_stop;
        OctTreeDepthMinusOne = u->oct_tree_depth_minus_one;
        MaxNodesToPushThisFrame = u->max_nodes_to_push;
        JitterTexSize = u->jitter_tex_size;
        RootNodeIsConstant = u->root_node_is_constant != 0;
        ComputeLighting = u->compute_lighting != 0;
        GradientsAreUnsigned = u->gradients_unsigned != 0;
        LightPosition = from<T>(u->light_position);
    }

    bool texelFetchNode(int x, int y, int z, uint32_t& r, uint32_t& g) const {
        if (x < 0 || y < 0 || z < 0 || x >= ndim[0] || y >= ndim[1] || z >= ndim[2]) return false;
        const size_t i = ((size_t)z * ndim[1] + y) * ndim[0] + x;
        r = nodes[2 * i];
        g = nodes[2 * i + 1];
        return true;
    }

    // texture(BrickSampler, p): GL_LINEAR, CLAMP_TO_EDGE.
    vec4<T> texture(const vec3<T>& p) const { return texture_of(brick, p); }
    vec4<T> texture_of(const BrickTexture<T>& brick, const vec3<T>& p) const {
        const T uv[3] = {p.x, p.y, p.z};
        const T N[3] = {BrickPoolDimension.x, BrickPoolDimension.y, BrickPoolDimension.z};
        const int n[3] = {brick.sx * 10, brick.sy * 10, brick.sz * 10};
        int i0[3], i1[3];
        T w[3];
        for (int a = 0; a < 3; ++a) {
            T t = uv[a] * N[a] - (T)0.5;
            t = std::fmin(std::fmax(t, (T)-1), N[a]);
            T fl = std::floor(t);
            w[a] = t - fl;
            int k = (int)fl;
            i0[a] = std::min(std::max(k, 0), n[a] - 1);
            i1[a] = std::min(std::max(k + 1, 0), n[a] - 1);
        }
        vec4<T> c000 = brick.fetch(i0[0], i0[1], i0[2]), c100 = brick.fetch(i1[0], i0[1], i0[2]);
        vec4<T> c010 = brick.fetch(i0[0], i1[1], i0[2]), c110 = brick.fetch(i1[0], i1[1], i0[2]);
        vec4<T> c001 = brick.fetch(i0[0], i0[1], i1[2]), c101 = brick.fetch(i1[0], i0[1], i1[2]);
        vec4<T> c011 = brick.fetch(i0[0], i1[1], i1[2]), c111 = brick.fetch(i1[0], i1[1], i1[2]);
        vec4<T> x00 = lerp4(c000, c100, w[0]), x10 = lerp4(c010, c110, w[0]);
        vec4<T> x01 = lerp4(c001, c101, w[0]), x11 = lerp4(c011, c111, w[0]);
        vec4<T> y0 = lerp4(x00, x10, w[1]), y1 = lerp4(x01, x11, w[1]);
        vec4<T> c = lerp4(y0, y1, w[2]);
        if (brick.fmt == VV_FMT_RGBA8 || brick.fmt == VV_FMT_DXT5 || brick.fmt == VV_FMT_DXT1) {
            const T k = sizeof(T) == 4 ? (T)(1.0f / 255.0f) : (T)1 / (T)255;
            c.r = c.r * k;
            c.g = c.g * k;
            c.b = c.b * k;
            c.a = c.a * k;
        }
        return c;
    }

    // GigaVoxelsNoLighting.frag:124-150
    void ComputeMinRayPlaneIntersection(const vec3<T>& rayPos, const vec3<T>& rayDir, const vec3<T>& pointOnPlane,
                                        const T plane[4], T& tMin) const {
        vec3<T> n(plane[0], plane[1], plane[2]);
        // dot(rayDir, n) with n an axis vector: the non-axis products are +-0
        T dirDotN = axis_dot(rayDir, n);
        if (dirDotN > 0) {
            vec3<T> v = rayPos - pointOnPlane;
            T tIsect = -(axis_dot(v, n)) / dirDotN;
            if (tIsect < tMin) {
                if (std::fabs(tIsect) > (T)0) tMin = tIsect;
            }
        }
    }
    static T axis_dot(const vec3<T>& a, const vec3<T>& n) {
        // n is (+-1,0,0), (0,+-1,0) or (0,0,+-1): the dot is exactly the one product
        if (n.x != 0) return a.x * n.x;
        if (n.y != 0) return a.y * n.y;
        return a.z * n.z;
    }
    // :152-180
    T ComputeMinRayBoxIntersection(const vec3<T>& rayPos, const vec3<T>& rayDir, const vec3<T>& mn,
                                   const vec3<T>& mx) const {
        const T planes[6][4] = {{-1, 0, 0, mn.x}, {0, -1, 0, mn.y}, {0, 0, -1, mn.z},
                                {1, 0, 0, -mx.x}, {0, 1, 0, -mx.y}, {0, 0, 1, -mx.z}};
        T tMin = (T)4.0;
        for (int i = 0; i < 6; ++i) ComputeMinRayPlaneIntersection(rayPos, rayDir, i < 3 ? mn : mx, planes[i], tMin);
        return tMin;
    }
    // :190-197
    void AdvanceRay(vec3<T>& pos, const vec3<T>& dir, T dist, T step) const {
        int numSteps = (int)(dist / step) + 1;
        pos += dir * ((T)numSteps * step);
    }
    // :230-282
    // Returns the step count and the samples composited (the control flow of
    // the segment, for the trace): (numSteps << 32) | composited.
    uint64_t TraverseConstant(vec4<T> constValue, vec3<T>& pos, const vec3<T>& dir, T rayStepSize, T sampleRatio,
                              int ratioLog2, const vec3<T>& mn, const vec3<T>& mx, vec4<T>& dst) const {
        T timeToExit = ComputeMinRayBoxIntersection(pos, dir, mn, mx);
        if (constValue.a < (T)0.005f) {
            AdvanceRay(pos, dir, timeToExit, rayStepSize);
            return ((uint64_t)(uint32_t)((int)(timeToExit / rayStepSize) + 1) << 32) | 0xFFFFFFFFu;
        }
        int numSteps = (int)(timeToExit / rayStepSize) + 1;
        const uint64_t steps0 = (uint64_t)(uint32_t)numSteps << 32;
        vec3<T> worldRayStep = dir * rayStepSize;
        for (int i = 0; i < numSteps; ++i) {
            pos += worldRayStep;
            if (dst.a > AlphaStop) {
                numSteps -= (i + 1);
                pos += dir * ((T)numSteps * rayStepSize);
                return steps0 | (uint32_t)i;
            }
            vec4<T> src = constValue;
            src.a = (T)1 - pow_pow2((T)1 - src.a, ratioLog2);
            src.r *= sampleRatio;
            src.g *= sampleRatio;
            src.b *= sampleRatio;
            record(false, src, dst, pos);
            composite(dst, src);
        }
        return steps0 | (uint32_t)numSteps;
    }
    // The adjoint's tape: every composited sample with the transmittance
    // before it (and for brick samples the brick-pool coordinate).
    void record(bool brick, const vec4<T>& src, const vec4<T>& dst, const vec3<T>& bpos) const {
        if (!tape) return;
        SampleRec r;
        r.brick = brick;
        r.src[0] = (double)src.r;
        r.src[1] = (double)src.g;
        r.src[2] = (double)src.b;
        r.src[3] = (double)src.a;
        r.T = (double)((T)1 - dst.a);
        r.bpos[0] = (float)bpos.x;
        r.bpos[1] = (float)bpos.y;
        r.bpos[2] = (float)bpos.z;
        tape->push_back(r);
    }
    static void composite(vec4<T>& dst, const vec4<T>& src) {
        T k = (T)1 - dst.a;
        dst.r = k * src.r + dst.r;
        dst.g = k * src.g + dst.g;
        dst.b = k * src.b + dst.b;
        dst.a = k * src.a + dst.a;
    }
    // :311-359 (no lighting: sampleRatio is reset to 1 before the loop)
    uint64_t TraverseBrick(vec3<T>& pos, const vec3<T>& dir, const vec3<T>& worldRayStep, vec3<T> curBrickRayPos,
                           const vec3<T>& brickRayStep, T sampleRatio, const vec3<T>& mn, const vec3<T>& mx,
                           vec4<T>& dst) const {
        // GigaVoxels.frag :337: lightDir at entry (lighting only)
        const vec3<T> lightDir = ComputeLighting ? normalize(LightPosition - pos) : vec3<T>{0, 0, 0};
        T timeToExit = ComputeMinRayBoxIntersection(pos, dir, mn, mx);
        T rayStepSize = RayStepSize * sampleRatio;
        int numSteps = (int)(timeToExit / rayStepSize) + 1;
        const uint64_t steps0 = (uint64_t)(uint32_t)numSteps << 32;
        for (int i = 0; i < numSteps; ++i) {
            pos += worldRayStep;
            if (dst.a > AlphaStop) {
                numSteps -= (i + 1);
                pos += dir * ((T)numSteps * rayStepSize);
                return steps0 | (uint32_t)i;
            }
            vec4<T> src = texture(curBrickRayPos);
            src.a = (T)1 - pow_pow2((T)1 - src.a, 0);
            if (ComputeLighting) Light(curBrickRayPos, dir, lightDir, src);
            record(true, src, dst, curBrickRayPos);
            composite(dst, src);
            curBrickRayPos += brickRayStep;
        }
        return steps0 | (uint32_t)numSteps;
    }
    // GigaVoxels.frag shading (:293-312): k_Ambient 0.05, k_Diffuse =
    // k_Specular = 1, k_Shininess 100 with pow(x, 100) restated as
    // x^64 * x^32 * x^4 by squarings.
    static T pow100(T x) {
        const T x2 = x * x, x4 = x2 * x2, x8 = x4 * x4, x16 = x8 * x8, x32 = x16 * x16, x64 = x32 * x32;
        return (x64 * x32) * x4;
    }
    vec3<T> shading(const vec3<T>& rgb, const vec3<T>& normal, const vec3<T>& toCamera,
                    const vec3<T>& toLight) const {
        const vec3<T> halfway = normalize(toLight + toCamera);
        const T diffuseLight = std::fmax(dot(toLight, normal), (T)0);
        vec3<T> diffuse{0, 0, 0}, specular{0, 0, 0};
        if (diffuseLight > (T)0) {
            diffuse = rgb * diffuseLight;
            specular = rgb * pow100(std::fmax(dot(halfway, normal), (T)0));
        }
        const T ka = sizeof(T) == 4 ? (T)0.05f : (T)0.05;
        const vec3<T> ambient = rgb * ka;
        return (ambient + diffuse) + specular;
    }
    // LookupGradient (:314-325) and the lighting of TraverseBrick (:370-384).
    void Light(const vec3<T>& curBrickRayPos, const vec3<T>& rayDir, const vec3<T>& lightDir, vec4<T>& src) const {
        const vec4<T> g = texture_of(grads, curBrickRayPos);
        vec3<T> normal{g.r, g.g, g.b};
        if (GradientsAreUnsigned) {
            normal = normal * (T)2;
            normal = normal - vec3<T>{(T)1, (T)1, (T)1};
        }
        normal = normalize(normal);
        if (std::isnan(normal.x) || std::isnan(normal.y) || std::isnan(normal.z)) return;
        const vec3<T> rgb{src.r, src.g, src.b};
        const vec3<T> sh = shading(rgb, normal, rayDir * (T)-1, lightDir);
        src.r = src.r + sh.x;
        src.g = src.g + sh.y;
        src.b = src.b + sh.z;
    }

    // :429-441
    T ComputeVoxelSize(const vec3<T>& p, T h) const {
        vec3<T> camToLL = normalize(((p - (CameraUp * h)) + (CameraLeft * h)) - CameraPosition);
        vec3<T> camToUR = normalize(((p + (CameraUp * h)) - (CameraLeft * h)) - CameraPosition);
        return (T)1 - dot(camToLL, camToUR);
    }

    static bool inside(const vec3<T>& p, const vec3<T>& mn, const vec3<T>& mx) {
        // dot(sign(p - mn), sign(mx - p)) >= 3
        auto sgn = [](T v) { return v > 0 ? (T)1 : (v < 0 ? (T)-1 : (T)0); };
        T d = sgn(p.x - mn.x) * sgn(mx.x - p.x) + sgn(p.y - mn.y) * sgn(mx.y - p.y) + sgn(p.z - mn.z) * sgn(mx.z - p.z);
        return d >= (T)3;
    }

    // The fragment's RayPosition: the volume-box entry point of the pixel's
    // ray (GigaVoxels.vert) or the near-plane point (NearPlaneQuad.vert).
    bool RayPosition(int px, int py, vec3<T>& out) const {
        const T fx = (T)px + (T)0.5, fy = (T)py + (T)0.5;
        // camera-to-near-plane vector of this pixel
        vec3<T> d;
        const float* o = U->near_origin;
        const float* dx = U->near_dx;
        const float* dy = U->near_dy;
        d.x = (T)o[0] + fx * (T)dx[0] + fy * (T)dy[0];
        d.y = (T)o[1] + fx * (T)dx[1] + fy * (T)dy[1];
        d.z = (T)o[2] + fx * (T)dx[2] + fy * (T)dy[2];
        const vec3<T> C = CameraPosition;
        if (U->camera_inside) {
            out = C + d;
            return true;
        }
        const T da[3] = {d.x, d.y, d.z}, ca[3] = {C.x, C.y, C.z};
        const T mn[3] = {VolExtentMin.x, VolExtentMin.y, VolExtentMin.z};
        const T mx[3] = {VolExtentMax.x, VolExtentMax.y, VolExtentMax.z};
        T tenter = -INFINITY, texit = INFINITY;
        int axis = -1;
        for (int a = 0; a < 3; ++a) {
            if (da[a] != 0) {
                T t0 = (mn[a] - ca[a]) / da[a];
                T t1 = (mx[a] - ca[a]) / da[a];
                T tn = t0 < t1 ? t0 : t1, tf = t0 < t1 ? t1 : t0;
                if (tn > tenter) {
                    tenter = tn;
                    axis = a;
                }
                if (tf < texit) texit = tf;
            } else if (!(ca[a] > mn[a] && ca[a] < mx[a])) {
                return false;
            }
        }
        if (axis < 0 || !(tenter <= texit) || !(tenter > 0)) return false;
        T pa[3] = {ca[0] + da[0] * tenter, ca[1] + da[1] * tenter, ca[2] + da[2] * tenter};
        pa[axis] = da[axis] > 0 ? mn[axis] : mx[axis];
        out = vec3<T>(pa[0], pa[1], pa[2]);
        return true;
    }

    // main (:490-751)
    // FNV-1a over 64-bit words: the trace of a pixel's control flow.
    static void mix(uint64_t& h, uint64_t v) {
        for (int b = 0; b < 8; ++b) {
            h ^= (v >> (8 * b)) & 0xFFu;
            h *= 1099511628211ull;
        }
    }

    // `trace` (may be NULL) receives a hash of the pixel's control flow:
    // whether it has a fragment and starts inside, and per leaf segment the
    // node, its depth and flags, the brick's depth, the step count and the
    // samples composited, then the loop's iteration count.  Two runs with
    // equal traces took the same decisions (descent, LOD, step counts, early
    // termination); the colour then differs only by the arithmetic.
    void main(int px, int py, vec4<T>& FragColor, uint32_t NodeUsageList[12], uint64_t* trace = nullptr) const {
        for (int i = 0; i < 12; ++i) NodeUsageList[i] = 0u;
        vec4<T> dst{0, 0, 0, 0};
        FragColor = dst;
        uint64_t th = 1469598103934665603ull;
        if (trace) *trace = th;
        vec3<T> rayWorldPosition;
        if (!RayPosition(px, py, rayWorldPosition)) return;
        vec3<T> rayDir = normalize(rayWorldPosition - CameraPosition);
        const int jx = px % JitterTexSize, jy = py % JitterTexSize;
        T jitterOffset = (T)jitter[jy * JitterTexSize + jx] / (T)255;
        rayWorldPosition += (rayDir * RayStepSize) * jitterOffset;
        bool in = inside(rayWorldPosition, VolExtentMin, VolExtentMax);
        mix(th, in ? 3u : 2u);
        int iterations = 0;
        if (in) {
            int curListIndex = 0, curComponentIndex = 0;
            const int pcx = px % 2, pcy = py % 2;
            const int startPushingNodes = (pcx * 12) + (pcy * 12 * 2);
            const int stopPushingNodes = startPushingNodes + 12;
            const int maxNodesPerPixelBlock = 12 * 2 * 2;
            vec3<T> brickRayStep = rayDir;
            brickRayStep *= BrickStepVector;
            int octTreeNodePtr[3] = {0, 0, 0};
            uint32_t root_r = 0, root_g = 0;
            if (!texelFetchNode(0, 0, 0, root_r, root_g)) {
                flag(VV_ERR_BOUNDS);
                return;
            }
            uint32_t node_r = root_r, node_g = root_g;
            vec3<T> nodeExtentMin = VolExtentMin, nodeExtentMax = VolExtentMax;
            T nodeSize = 1, voxelHalfSize = RootVoxelHalfSize;
            vec3<T> rayBrickPosition = rayWorldPosition, curBrickRayPosition = rayWorldPosition;
            uint32_t curBrickPtr_g = root_g;
            bool brickIsLoaded = false, curNodeIsConstant = RootNodeIsConstant;
            T projVoxelSize = 0;
            int curDepth = 0, curBrickDepth = 0;
            uint32_t childNodePtr[3] = {0, 0, 0};
            int nodeListTraversalCount = 0, pushedNodeCount = 0;
            while (in) {
                if (++iterations > max_iter) {
                    flag(VV_ERR_TIMEOUT);
                    break;
                }
                curNodeIsConstant = (node_r & 0x40000000u) != 0u;
                brickIsLoaded = (node_r & 0x80000000u) != 0u;
                if (brickIsLoaded) {
                    curBrickPtr_g = node_g;
                    curBrickRayPosition = rayBrickPosition;
                    curBrickDepth = curDepth;
                }
                projVoxelSize = ComputeVoxelSize(rayWorldPosition, voxelHalfSize) * LodScalar;
                childNodePtr[0] = (node_r >> 20u) & 0x3FFu;
                childNodePtr[1] = (node_r >> 10u) & 0x3FFu;
                childNodePtr[2] = node_r & 0x3FFu;
                const bool leaf = childNodePtr[0] == 0u && childNodePtr[1] == 0u && childNodePtr[2] == 0u;
                if ((!curNodeIsConstant && !brickIsLoaded) || PixelSize > projVoxelSize || leaf) {
                    const uint32_t nodeUsage[3] = {(uint32_t)octTreeNodePtr[0], (uint32_t)octTreeNodePtr[1],
                                                   (uint32_t)octTreeNodePtr[2]};
                    if (curNodeIsConstant) {
                        const int k = OctTreeDepthMinusOne - curDepth;
                        T sampleRatio = std::ldexp((T)1, k);
                        vec4<T> cv{(T)(node_g & 255u) / (T)255, (T)((node_g >> 8) & 255u) / (T)255,
                                   (T)((node_g >> 16) & 255u) / (T)255, (T)(node_g >> 24) / (T)255};
                        const uint64_t seg = TraverseConstant(cv, rayWorldPosition, rayDir, RayStepSize * sampleRatio,
                                                              sampleRatio, k, nodeExtentMin, nodeExtentMax, dst);
                        mix(th, ((uint64_t)nodeUsage[0] << 40) | ((uint64_t)nodeUsage[1] << 20) | nodeUsage[2]);
                        mix(th, (uint64_t)curDepth | (1u << 8) | ((uint64_t)brickIsLoaded << 9));
                        mix(th, seg);
                    } else {
                        vec3<T> ptr((T)((curBrickPtr_g >> 20u) & 0x3FFu) / BrickPoolDimension.x,
                                    (T)((curBrickPtr_g >> 10u) & 0x3FFu) / BrickPoolDimension.y,
                                    (T)(curBrickPtr_g & 0x3FFu) / BrickPoolDimension.z);
                        vec3<T> curBrickRayPos = ptr + ((curBrickRayPosition * BrickDimension) / BrickPoolDimension);
                        T sampleRatio = std::ldexp((T)1, OctTreeDepthMinusOne - curBrickDepth);
                        vec3<T> worldRayStep = rayDir;
                        worldRayStep *= RayStepSize;
                        worldRayStep *= sampleRatio;
                        const uint64_t seg = TraverseBrick(rayWorldPosition, rayDir, worldRayStep, curBrickRayPos,
                                                           brickRayStep, sampleRatio, nodeExtentMin, nodeExtentMax, dst);
                        mix(th, ((uint64_t)nodeUsage[0] << 40) | ((uint64_t)nodeUsage[1] << 20) | nodeUsage[2]);
                        mix(th, (uint64_t)curDepth | ((uint64_t)brickIsLoaded << 9) | ((uint64_t)curBrickDepth << 16));
                        mix(th, seg);
                    }
                    if (nodeListTraversalCount >= startPushingNodes && nodeListTraversalCount < stopPushingNodes &&
                        pushedNodeCount < MaxNodesToPushThisFrame) {
                        ++pushedNodeCount;
                        // AddToNodeUsageList (:454-488)
                        uint32_t bits = 0u;
                        bits |= ((nodeUsage[0] + 1u) << 20u);
                        bits |= ((nodeUsage[1] + 1u) << 10u);
                        bits |= (nodeUsage[2] + 1u);
                        NodeUsageList[curListIndex * 4 + curComponentIndex] = bits;
                        ++curComponentIndex;
                        if (curComponentIndex == 4) {
                            curComponentIndex = 0;
                            ++curListIndex;
                            if (curListIndex == 3) curListIndex = 0;
                        }
                    }
                    if (dst.a > AlphaStop && (curNodeIsConstant || brickIsLoaded)) break;
                    node_r = root_r;
                    node_g = root_g;
                    nodeExtentMin = VolExtentMin;
                    nodeExtentMax = VolExtentMax;
                    nodeSize = 1;
                    voxelHalfSize = RootVoxelHalfSize;
                    rayBrickPosition = rayWorldPosition;
                    curBrickRayPosition = rayWorldPosition;
                    curBrickPtr_g = root_g;
                    brickIsLoaded = false;
                    curNodeIsConstant = RootNodeIsConstant;
                    projVoxelSize = 0;
                    curDepth = 0;
                    curBrickDepth = 0;
                    in = inside(rayWorldPosition, VolExtentMin, VolExtentMax);
                    ++nodeListTraversalCount;
                    if (nodeListTraversalCount >= maxNodesPerPixelBlock) nodeListTraversalCount = 0;
                } else {
                    vec3<T> brickOffset = rayBrickPosition * (T)2;
                    uint32_t childOffset[3] = {std::min(to_uint(brickOffset.x), 1u), std::min(to_uint(brickOffset.y), 1u),
                                               std::min(to_uint(brickOffset.z), 1u)};
                    vec3<T> off((T)childOffset[0], (T)childOffset[1], (T)childOffset[2]);
                    rayBrickPosition = brickOffset - off;
                    for (int a = 0; a < 3; ++a) octTreeNodePtr[a] = (int)(childNodePtr[a] + childOffset[a]);
                    ++curDepth;
                    nodeSize *= (T)0.5;
                    nodeExtentMin += off * nodeSize;
                    nodeExtentMax -= (vec3<T>(1, 1, 1) - off) * nodeSize;
                    voxelHalfSize *= (T)0.5;
                    if (!texelFetchNode(octTreeNodePtr[0], octTreeNodePtr[1], octTreeNodePtr[2], node_r, node_g)) {
                        flag(VV_ERR_BOUNDS);
                        break;
                    }
                }
            }
        }
        mix(th, (uint64_t)iterations);
        if (trace) *trace = th;
        FragColor = dst;
    }

    void flag(int code) const {
        if (status && *status == 0) {
#pragma omp critical(gv_oracle_status)
            if (*status == 0) *status = code;
        }
    }
};

int max_iterations(const vv_uniforms* u) {
    double segs = 1.7320508 / (double)u->ray_step_size + 2.0;
    double it = 2.0 * segs * (double)(u->oct_tree_depth_minus_one + 2) + 64.0;
    if (u->max_segments > 0) it = (double)u->max_segments;
    if (it > 2.0e9) it = 2.0e9;
    return (int)it;
}

template <typename T>
int run_raycast(const vv_uniforms* u, const oracle_scene* s, int row0, int row1, void* color, uint32_t* usage,
                int threads, int32_t* status, uint64_t* trace = nullptr) {
    Shader<T> sh;
    sh.init(u);
    sh.nodes = s->nodes;
    for (int a = 0; a < 3; ++a) sh.ndim[a] = s->node_dim[a];
    sh.brick.data = s->bricks;
    sh.brick.fmt = s->fmt;
    sh.brick.sx = s->slots[0];
    sh.brick.sy = s->slots[1];
    sh.brick.sz = s->slots[2];
    sh.jitter = s->jitter;
    sh.grads.data = s->grads;
    sh.grads.fmt = s->grad_fmt;
    sh.grads.sx = s->slots[0];
    sh.grads.sy = s->slots[1];
    sh.grads.sz = s->slots[2];
    if (sh.ComputeLighting && !s->grads) return VV_ERR_STATE;  // lighting needs the gradient pool
    sh.max_iter = max_iterations(u);
    int st = 0;
    sh.status = &st;
    const int W = u->width;
#ifdef _OPENMP
    const int nt = threads > 0 ? threads : omp_get_max_threads();
#pragma omp parallel for schedule(dynamic, 1) num_threads(nt)
#endif
    for (int y = row0; y < row1; ++y) {
        for (int x = 0; x < W; ++x) {
            vec4<T> c;
            uint32_t lst[12];
            const size_t pix = (size_t)y * W + x;
            sh.main(x, y, c, lst, trace ? trace + pix : nullptr);
            if (color) {
                T* o = (T*)color + 4 * pix;
                o[0] = c.r;
                o[1] = c.g;
                o[2] = c.b;
                o[3] = c.a;
            }
            if (usage) std::memcpy(usage + 12 * pix, lst, sizeof(lst));
        }
    }
    if (status) *status = st;
    return 0;
}

// GenerateHistoPyramid.frag (:9-55) for one output texel at (x,y) reading a
// level of size (w,h); out-of-range fetches read 0.
uint32_t histo_texel(const std::vector<uint32_t>& in, int w, int h, int fx, int fy) {
    auto fetch = [&](int x, int y) -> uint32_t {
        if (x < 0 || y < 0 || x >= w || y >= h) return 0u;
        return in[(size_t)y * w + x];
    };
    int tx = fx * 2, ty = fy * 2;
    uint32_t v = fetch(tx, ty);
    tx += 1;
    v += fetch(tx, ty);
    ty += 1;
    v += fetch(tx, ty);
    tx -= 1;
    v += fetch(tx, ty);
    ty += 1;
    if (ty == h - 1) {
        v += fetch(tx, ty);
        tx += 1;
        v += fetch(tx, ty);
        tx += 1;
        if (tx == w - 1) {
            v += fetch(tx, ty);
            ty -= 1;
            v += fetch(tx, ty);
            ty -= 1;
            v += fetch(tx, ty);
        }
    } else if ((tx += 2) == w - 1) {
        ty -= 1;
        v += fetch(tx, ty);
        ty -= 1;
        v += fetch(tx, ty);
    }
    return v;
}

}  // namespace

extern "C" {

int oracle_raycast(const vv_uniforms* u, const oracle_scene* s, int precision, int row0, int row1, void* color,
                   uint32_t* usage, int threads, int32_t* status) {
    if (!u || !s || row0 < 0 || row1 > u->height || row0 > row1) return VV_ERR_ARG;
    if (precision == 64) return run_raycast<double>(u, s, row0, row1, color, usage, threads, status);
    return run_raycast<float>(u, s, row0, row1, color, usage, threads, status);
}

int oracle_max_iterations(const vv_uniforms* u) { return max_iterations(u); }

int oracle_dxt_decode(const void* blocks, int fmt, long long bricks, uint32_t* rgba8) {
    if (!blocks || !rgba8 || bricks < 0 || (fmt != VV_FMT_DXT5 && fmt != VV_FMT_DXT1)) return VV_ERR_ARG;
    for (long long s = 0; s < bricks; ++s)
        for (int t = 0; t < 1000; ++t) {
            const int x = t % 10, y = (t / 10) % 10, z = t / 100;
            const size_t blk = (size_t)s * 90 + (size_t)(z * 9 + (y / 4) * 3 + x / 4);
            const int texel = (y % 4) * 4 + x % 4;
            int rgb[3], a = 0;
            if (fmt == VV_FMT_DXT5) {
                const unsigned char* b = (const unsigned char*)blocks + 16 * blk;
                a = s3tc_alpha(b, texel);
                s3tc_colour(b + 8, texel, true, rgb);
            } else {
                s3tc_colour((const unsigned char*)blocks + 8 * blk, texel, false, rgb);
            }
            rgba8[(size_t)s * 1000 + (size_t)t] =
                (uint32_t)rgb[0] | ((uint32_t)rgb[1] << 8) | ((uint32_t)rgb[2] << 16) | ((uint32_t)a << 24);
        }
    return VV_OK;
}

int oracle_raycast_trace(const vv_uniforms* u, const oracle_scene* s, int precision, int row0, int row1,
                         void* color, uint32_t* usage, uint64_t* trace, int threads, int32_t* status) {
    if (!u || !s || row0 < 0 || row1 > u->height || row0 > row1) return VV_ERR_ARG;
    if (precision == 64) return run_raycast<double>(u, s, row0, row1, color, usage, threads, status, trace);
    return run_raycast<float>(u, s, row0, row1, color, usage, threads, status, trace);
}

namespace {

// binary64 GL_LINEAR + CLAMP_TO_EDGE sample of `vals` at the binary32
// texture coordinate bpos (the taps and weights of texture(), in double).
void sample64(const BrickTexture<double>& bt, const float N[3], const float bpos[3], double out[4]) {
    const int n[3] = {bt.sx * 10, bt.sy * 10, bt.sz * 10};
    int i0[3], i1[3];
    double w[3];
    for (int a = 0; a < 3; ++a) {
        double t = (double)bpos[a] * (double)N[a] - 0.5;
        t = std::fmin(std::fmax(t, -1.0), (double)N[a]);
        const double fl = std::floor(t);
        w[a] = t - fl;
        const int k = (int)fl;
        i0[a] = std::min(std::max(k, 0), n[a] - 1);
        i1[a] = std::min(std::max(k + 1, 0), n[a] - 1);
    }
    double acc[4] = {0, 0, 0, 0};
    for (int t8 = 0; t8 < 8; ++t8) {
        const int bx = t8 & 1, by = (t8 >> 1) & 1, bz = t8 >> 2;
        const double wt = (bx ? w[0] : 1.0 - w[0]) * (by ? w[1] : 1.0 - w[1]) * (bz ? w[2] : 1.0 - w[2]);
        const vec4<double> v = bt.fetch(bx ? i1[0] : i0[0], by ? i1[1] : i0[1], bz ? i1[2] : i0[2]);
        acc[0] += wt * v.r;
        acc[1] += wt * v.g;
        acc[2] += wt * v.b;
        acc[3] += wt * v.a;
    }
    const double k = (bt.fmt == VV_FMT_RGBA8 || bt.fmt == VV_FMT_DXT5 || bt.fmt == VV_FMT_DXT1) ? 1.0 / 255.0 : 1.0;
    for (int c = 0; c < 4; ++c) out[c] = acc[c] * k;
}

}  // namespace

// The binary32 ray cast's sample sequence (descent, LOD choices, step
// counts, sample positions, early termination: all taken from `traj`)
// re-evaluated in binary64: brick samples are filtered in double from the
// texels of `vals` (same pool layout) and every sample is composited in
// double.  With vals == traj this isolates the arithmetic error of the
// binary32 sampler and compositing; with vals a perturbed copy it is a
// smooth function of the texels (the control flow is fixed), which is what
// finite differences of the adjoint need.
int oracle_fixed_path(const vv_uniforms* u, const oracle_scene* traj, const oracle_scene* vals, int row0, int row1,
                      double* color, int threads) {
    if (!u || !traj || !vals || !color || row0 < 0 || row1 > u->height || row0 > row1) return VV_ERR_ARG;
    if (vals->slots[0] != traj->slots[0] || vals->slots[1] != traj->slots[1] || vals->slots[2] != traj->slots[2])
        return VV_ERR_ARG;
    Shader<float> base;
    base.init(u);
    base.nodes = traj->nodes;
    for (int a = 0; a < 3; ++a) base.ndim[a] = traj->node_dim[a];
    base.brick.data = traj->bricks;
    base.brick.fmt = traj->fmt;
    base.brick.sx = traj->slots[0];
    base.brick.sy = traj->slots[1];
    base.brick.sz = traj->slots[2];
    base.jitter = traj->jitter;
    if (base.ComputeLighting) return VV_ERR_ARG;  // unlit sample sequences only
    base.max_iter = max_iterations(u);
    int st = 0;
    base.status = &st;
    BrickTexture<double> bt;
    bt.data = vals->bricks;
    bt.fmt = vals->fmt;
    bt.sx = vals->slots[0];
    bt.sy = vals->slots[1];
    bt.sz = vals->slots[2];
    const float N[3] = {u->brick_pool_dimension[0], u->brick_pool_dimension[1], u->brick_pool_dimension[2]};
    const int W = u->width;
#ifdef _OPENMP
    const int nt = threads > 0 ? threads : omp_get_max_threads();
#pragma omp parallel num_threads(nt)
#endif
    {
        Shader<float> sh = base;
        std::vector<SampleRec> tape;
        sh.tape = &tape;
#ifdef _OPENMP
#pragma omp for schedule(dynamic, 1)
#endif
        for (int y = row0; y < row1; ++y)
            for (int x = 0; x < W; ++x) {
                tape.clear();
                vec4<float> c;
                uint32_t lst[12];
                sh.main(x, y, c, lst);
                double d[4] = {0, 0, 0, 0};
                for (const SampleRec& r : tape) {
                    double s[4];
                    if (r.brick) sample64(bt, N, r.bpos, s);
                    else
                        for (int k = 0; k < 4; ++k) s[k] = r.src[k];
                    const double T = 1.0 - d[3];
                    for (int k = 0; k < 4; ++k) d[k] = T * s[k] + d[k];
                }
                double* o = color + 4 * ((size_t)y * W + x);
                for (int k = 0; k < 4; ++k) o[k] = d[k];
            }
    }
    return st;
}

// Adjoint of the binary32 ray cast in binary64: the forward runs exactly as
// oracle_raycast(precision 32) and records its samples; the backward walks
// them in reverse, g_k.a = g_{k+1}.a - dot(g_{k+1}, src_k), dL/dsrc_k =
// g_{k+1} * T_k, and adds w_j * dL/dsrc_k to the 8 texels of each brick
// sample (weights from the forward's float tap fractions).  grad holds 4
// doubles per pool texel (slot-major, brick-linear), added to.
int oracle_backward(const vv_uniforms* u, const oracle_scene* s, const float* dl_dcolor, double* grad, int row0,
                    int row1) {
    return oracle_backward_bound(u, s, dl_dcolor, grad, nullptr, row0, row1);
}

int oracle_backward_bound(const vv_uniforms* u, const oracle_scene* s, const float* dl_dcolor, double* grad,
                          double* grad_abs, int row0, int row1) {
    if (!u || !s || !dl_dcolor || !grad || row0 < 0 || row1 > u->height || row0 > row1) return VV_ERR_ARG;
    Shader<float> sh;
    sh.init(u);
    sh.nodes = s->nodes;
    for (int a = 0; a < 3; ++a) sh.ndim[a] = s->node_dim[a];
    sh.brick.data = s->bricks;
    sh.brick.fmt = s->fmt;
    sh.brick.sx = s->slots[0];
    sh.brick.sy = s->slots[1];
    sh.brick.sz = s->slots[2];
    sh.jitter = s->jitter;
    if (sh.ComputeLighting) return VV_ERR_ARG;  // the adjoint covers the unlit ray cast
    sh.max_iter = max_iterations(u);
    int st = 0;
    sh.status = &st;
    std::vector<SampleRec> tape;
    sh.tape = &tape;
    const int W = u->width;
    const float N[3] = {u->brick_pool_dimension[0], u->brick_pool_dimension[1], u->brick_pool_dimension[2]};
    const int n[3] = {s->slots[0] * 10, s->slots[1] * 10, s->slots[2] * 10};
    for (int y = row0; y < row1; ++y)
        for (int x = 0; x < W; ++x) {
            tape.clear();
            vec4<float> c;
            uint32_t lst[12];
            sh.main(x, y, c, lst);
            const float* gp = dl_dcolor + 4 * ((size_t)y * W + x);
            double g[4] = {gp[0], gp[1], gp[2], gp[3]};
            // the same recurrence over absolute values: the magnitude that the
            // terms summed into g and into each texel carry (a running bound
            // for the rounding of an implementation in lower precision)
            double ga[4] = {std::fabs(g[0]), std::fabs(g[1]), std::fabs(g[2]), std::fabs(g[3])};
            for (size_t k = tape.size(); k-- > 0;) {
                const SampleRec& r = tape[k];
                if (r.brick) {
                    const double d[4] = {g[0] * r.T, g[1] * r.T, g[2] * r.T, g[3] * r.T};
                    const double da[4] = {ga[0] * std::fabs(r.T), ga[1] * std::fabs(r.T), ga[2] * std::fabs(r.T),
                                          ga[3] * std::fabs(r.T)};
                    int i0[3], i1[3];
                    double f[3];
                    for (int a = 0; a < 3; ++a) {
                        float t = r.bpos[a] * N[a] - 0.5f;
                        t = std::fmin(std::fmax(t, -1.0f), N[a]);
                        const float fl = std::floor(t);
                        f[a] = (double)(t - fl);
                        const int kk = (int)fl;
                        i0[a] = std::min(std::max(kk, 0), n[a] - 1);
                        i1[a] = std::min(std::max(kk + 1, 0), n[a] - 1);
                    }
                    for (int t8 = 0; t8 < 8; ++t8) {
                        const int bx = t8 & 1, by = (t8 >> 1) & 1, bz = t8 >> 2;
                        const double w = (bx ? f[0] : 1.0 - f[0]) * (by ? f[1] : 1.0 - f[1]) * (bz ? f[2] : 1.0 - f[2]);
                        const int ix = bx ? i1[0] : i0[0], iy = by ? i1[1] : i0[1], iz = bz ? i1[2] : i0[2];
                        const size_t slot = ((size_t)(iz / 10) * s->slots[1] + (size_t)(iy / 10)) * s->slots[0] + (size_t)(ix / 10);
                        const size_t ti = slot * 1000 + (size_t)((iz % 10) * 100 + (iy % 10) * 10 + (ix % 10));
                        for (int ch = 0; ch < 4; ++ch) grad[4 * ti + ch] += w * d[ch];
                        if (grad_abs)
                            for (int ch = 0; ch < 4; ++ch) grad_abs[4 * ti + ch] += std::fabs(w) * da[ch];
                    }
                }
                g[3] = g[3] - (g[0] * r.src[0] + g[1] * r.src[1] + g[2] * r.src[2] + g[3] * r.src[3]);
                ga[3] = ga[3] + (ga[0] * std::fabs(r.src[0]) + ga[1] * std::fabs(r.src[1]) +
                                 ga[2] * std::fabs(r.src[2]) + ga[3] * std::fabs(r.src[3]));
            }
        }
    return st;
}

// GenerateSelectionMask.frag (:15-187): the red channel per pixel.
int oracle_select(const uint32_t* usage, int w, int h, uint32_t* mask) {
    const float dimMinusTwoX = (float)(w - 2), dimMinusTwoY = (float)(h - 2);
    for (int y = 0; y < h; ++y)
        for (int x = 0; x < w; ++x) {
            const uint32_t* L = usage + 12 * ((size_t)y * w + x);
            uint32_t out = 0u;
            mask[(size_t)y * w + x] = 0u;
            if (L[0] == 0u) continue;
            uint32_t top[12] = {0}, topRight[12] = {0}, right[12] = {0};
            auto get = [&](uint32_t* d, int nx, int ny) { std::memcpy(d, usage + 12 * ((size_t)ny * w + nx), 48); };
            if ((float)y < dimMinusTwoY) {
                get(top, x, y + 2);
                if ((float)x < dimMinusTwoX) {
                    get(topRight, x + 2, y + 2);
                    get(right, x + 2, y);
                }
            } else if ((float)x < dimMinusTwoX) {
                get(right, x + 2, y);
            }
            int curList = 2, curComp = 3, nextList = 0, nextComp = 0;
            for (int i = 0; i < 12; ++i) {
                const int prevList = curList, prevComp = curComp;
                curList = nextList;
                curComp = nextComp;
                ++nextComp;
                if (nextComp == 4) {
                    nextComp = 0;
                    ++nextList;
                    if (nextList == 3) nextList = 0;
                }
                const uint32_t nodeUsage = L[curList * 4 + curComp];
                if (nodeUsage == 0u) break;
                const int c = curList * 4 + curComp, p = prevList * 4 + prevComp, n = nextList * 4 + nextComp;
                if (nodeUsage == top[c] || nodeUsage == top[p] || nodeUsage == top[n]) continue;
                if (nodeUsage == topRight[c] || nodeUsage == topRight[p] || nodeUsage == topRight[n]) continue;
                if (nodeUsage == right[c] || nodeUsage == right[p] || nodeUsage == right[n]) continue;
                out |= (1u << (uint32_t)i);
            }
            mask[(size_t)y * w + x] = out;
        }
    return 0;
}

// ComputeActiveTexels + GenerateHistoPyramid passes, then CompressNodeUsageList
// for keys 0..min(total,cap)-1.  out: cap x 4 words; *total: active pixels.
int oracle_compress(const uint32_t* usage, const uint32_t* mask, int w, int h, int max_push, int cap, uint32_t* out,
                    uint32_t* total) {
    std::vector<std::vector<uint32_t>> lv;
    std::vector<int> lw, lh;
    {
        std::vector<uint32_t> l0((size_t)w * h);
        for (size_t i = 0; i < l0.size(); ++i) l0[i] = mask[i] == 0u ? 0u : 1u;
        lv.push_back(std::move(l0));
        lw.push_back(w);
        lh.push_back(h);
        int cw = w, ch = h;
        while (!(cw == 1 && ch == 1)) {
            const int pw = cw, ph = ch;
            if (cw != 1) cw >>= 1;
            if (ch != 1) ch >>= 1;
            std::vector<uint32_t> nxt((size_t)cw * ch);
            for (int y = 0; y < ch; ++y)
                for (int x = 0; x < cw; ++x) nxt[(size_t)y * cw + x] = histo_texel(lv.back(), pw, ph, x, y);
            lv.push_back(std::move(nxt));
            lw.push_back(cw);
            lh.push_back(ch);
        }
    }
    const int levels = (int)lv.size();
    const uint32_t count = lv.back()[0];
    if (total) *total = count;
    const uint32_t n = std::min<uint32_t>(count, (uint32_t)std::max(cap, 0));
    static const int incr[9][2] = {{1, 0}, {-1, 1}, {1, 0}, {-1, 1}, {1, 0}, {1, 0}, {0, -1}, {0, -1}, {0, 0}};
    for (uint32_t key = 0; key < n; ++key) {
        uint32_t start = 0, end = 0;
        int tx = 0, ty = 0, sw = 1, sh = 1;
        int level = levels - 1, loop = 0;
        bool bad = false;
        auto fetch = [&](int l, int x, int y) -> uint32_t {
            if (x < 0 || y < 0 || x >= lw[(size_t)l] || y >= lh[(size_t)l]) return 0u;
            return lv[(size_t)l][(size_t)y * lw[(size_t)l] + x];
        };
        while (level >= 0) {
            end = start + fetch(level, tx, ty);
            if (key >= start && key < end) {
                --level;
                loop = 0;
                tx <<= 1;
                ty <<= 1;
                if (level >= 0) {
                    sw = lw[(size_t)level];
                    sh = lh[(size_t)level];
                }
            } else {
                tx += incr[loop][0];
                ty += incr[loop][1];
                ++loop;
                if (loop == 4 && ty != sh - 1) {
                    loop = 7;
                    tx += 2;
                    ty -= 1;
                }
                if (loop >= 6 && tx != sw - 1) loop = 9;
                start = end;
                if (loop == 9) {
                    bad = true;
                    break;
                }
            }
        }
        uint32_t* o = out + 4 * (size_t)key;
        if (bad) {  // the shader's escape value (:97-103)
            o[0] = start;
            o[1] = end;
            o[2] = key;
            o[3] = (uint32_t)level;
            continue;
        }
        tx >>= 1;
        ty >>= 1;
        uint32_t bits = mask[(size_t)ty * w + tx];
        const uint32_t* L = usage + 12 * ((size_t)ty * w + tx);
        uint32_t items[4] = {0u, 0u, 0u, 0u};
        int pushed = 0;
        for (int item = 0; item < 12 && bits != 0u && pushed < max_push; ++item, bits >>= 1u) {
            if (bits & 1u) {
                items[pushed % 4] = L[item];
                ++pushed;
            }
        }
        std::memcpy(o, items, 16);
    }
    return 0;
}

}  // extern "C"
