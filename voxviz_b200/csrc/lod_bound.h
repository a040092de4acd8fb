// lod_bound.h - a certificate that the descent's LOD test continues.
//
// The descent of GigaVoxelsNoLighting.frag (:563-622) stops at a node when
// PixelSize > ComputeVoxelSize (:429-441) * LodScalar, evaluated here in
// binary32 as
//     uh = up*vh, lh = left*vh                     (vh = rvh * 2^-level)
//     ll = normalize(pos - uh + lh - C), ur = normalize(pos + uh - lh - C)
//     stop iff pixel_size > (1 - dot(ll, ur)) * lod
// with normalize(v) = v * (1/sqrt(dot(v,v))), no contraction.
//
// lod_bound_clears() shows, for a ray position, that this test is FALSE
// (the descent continues) at every level j in [j0, m], without evaluating
// it.  With a = pos - C, d = vh*(up - left) (exact: vh is a power of two),
// the test measures R = 1 - cos(theta), theta the angle between a - d and
// a + d, and
//     R >= sin^2(theta)/2 >= 2 vh^2 |a x w|^2 / (|a|^2 + vh^2 |w|^2)^2 = Rlow
// (w = up - left).  For levels with vh |w| <= |a|/4 the binary32 sequence
// returns at least lod * (R - theta * Dmax - 11.2 u)(1 - u) (u = 2^-24):
// Dmax bounds the angle error of its two directions (rounding of
// pos - uh + lh - C per component <= u (2 max|pos| + max|a| + 5 vh) with
// pos in the unit box, plus 1.8 u from normalising) and 11.2 u the length
// and dot-product rounding.  Rlow is evaluated with approximate reciprocal
// square root and division (<= 2 ulp each on the device; exact on the
// host); the (1 - 1e-4) factors cover that.  If the bound clears
// pixel_size at level m and theta >= 5 Dmax there, it clears it at every
// shallower level down to j0, the first level with vh |w| <= |a|/4, since
// R grows faster with theta than theta * Dmax.
//
// Shared by the kernels and by the host check in tests/ (which compares it
// with the exact binary32 sequence on random and adversarial inputs).
#pragma once

#include <stdint.h>

#include <cmath>
#include <cstring>

#ifdef __CUDACC__
#define VV_HD __host__ __device__ __forceinline__
#else
#define VV_HD inline
#endif

namespace vv {
namespace lodb {

struct V3 {
    float x, y, z;
};

VV_HD V3 sub3(V3 a, V3 b) { return V3{a.x - b.x, a.y - b.y, a.z - b.z}; }
VV_HD float dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
VV_HD V3 cross(V3 a, V3 b) { return V3{a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }

VV_HD float fast_rsqrt(float x) {
#ifdef __CUDA_ARCH__
    return rsqrtf(x);
#else
    return 1.0f / std::sqrt(x);
#endif
}
VV_HD float fast_div(float a, float b) {
#ifdef __CUDA_ARCH__
    return __fdividef(a, b);
#else
    return a / b;
#endif
}
VV_HD float fast_log2(float x) {
#ifdef __CUDA_ARCH__
    return __log2f(x);
#else
    return std::log2(x);
#endif
}
VV_HD float vabs(float x) { return x < 0.0f ? -x : x; }
VV_HD float vmax(float a, float b) { return a > b ? a : b; }
VV_HD uint32_t float_bits(float f) {
#ifdef __CUDA_ARCH__
    return __float_as_uint(f);
#else
    uint32_t b;
    std::memcpy(&b, &f, 4);
    return b;
#endif
}
// x * 2^e for a normal power-of-two scale (exact); on the device 2^e is built
// from its exponent bits (e in [-126, 127])
VV_HD float scale2(float x, int e) {
#ifdef __CUDA_ARCH__
    return x * __int_as_float((e + 127) << 23);
#else
    return std::ldexp(x, e);
#endif
}

// Per-ray constants.
struct Consts {
    V3 C, w;       // camera position, w = up - left
    float W, wn;   // |w|^2, |w| rounded up
    float cmax;    // max |C| component
    float rvh, lod, pixel_size;
    int max_level;
    bool ok;
};

VV_HD Consts make_consts(V3 C, V3 up, V3 left, float rvh, float lod, float pixel_size, int max_level, bool unit_box) {
    Consts k;
    k.C = C;
    k.w = sub3(up, left);
    k.W = dot(k.w, k.w);
    k.wn = (k.W > 0.0f ? 1.0f / fast_rsqrt(k.W) : 0.0f) * 1.0001f;
    k.cmax = vmax(vabs(C.x), vmax(vabs(C.y), vabs(C.z)));
    k.rvh = rvh;
    k.lod = lod;
    k.pixel_size = pixel_size;
    k.max_level = max_level;
    k.ok = unit_box && lod > 0.0f && lod < 1e30f && pixel_size < 1e30f && rvh > 0.0f && k.W > 0.5f && k.W < 8.0f &&
           k.cmax < 1e6f;
    return k;
}

// Levels [lo, hi] at which the LOD test surely continues for position pos
// (inside the unit box); lo > hi when nothing is shown.  `guess` picks the
// deepest level tried first (the level where Rlow is ~4x the threshold);
// two levels are tried.
VV_HD void clear_range(const Consts& k, V3 pos, int& lo, int& hi) {
    lo = 1;
    hi = 0;
    if (!k.ok) return;
    const float u = 5.9604645e-8f;  // 2^-24
    const V3 a = sub3(pos, k.C);
    const float A = dot(a, a);
    if (!(A > 1e-12f)) return;
    const float ra = fast_rsqrt(A);
    // a lower bound on |a| (the 1e-4 covers the approximate reciprocal square
    // root and division, <= 2 ulp each on the device)
    const float alen_lo = fast_div(1.0f, ra * 1.0001f);
    // j0: the smallest j with 2^j >= t = 4 rvh |w| / |a|
    const float t = 4.0f * k.rvh * k.wn * ra * 1.001f;
    int j0 = 0;
    if (t > 1.0f) {
        const uint32_t b = float_bits(t);
        const int e = (int)((b >> 23) & 255u) - 127;  // t in [2^e, 2^(e+1))
        j0 = (b & 0x7FFFFFu) ? e + 1 : e;
    }
    const V3 c = cross(a, k.w);
    const float S = dot(c, c);
    if (!(S >= 0.1001f * A * k.W)) return;  // sin(angle(a, w)) >= 0.316: a x w is well conditioned
    const float amax = vmax(vabs(a.x), vmax(vabs(a.y), vabs(a.z)));
    // Levels below j0 (vh |w| > |a|/4): sin(theta) = 2|a||d| sin(phi) /
    // (|a - d||a + d|) >= 2 * 0.25 * 0.316 / 1.25^2 at vh |w| = |a|/4 and theta
    // grows with vh, so R >= 1 - cos(0.101) > 0.0051.  |a -+ d| >= |a| sin(phi),
    // so each direction of the binary32 sequence is off by at most
    // 1.01 sqrt(3) eps_c / (0.316 |a|) + 1.8 u (eps_c: per-component rounding
    // with vh <= rvh), which moves 1 - cos by at most that angle.
    int lo_level = j0;
    if (j0 > 0) {
        const float eps_c = u * (3.0f + 8.0f * k.rvh + amax + 2.0f * k.cmax) * 1.01f;
        // upper bounds below: approximate quotients are raised by 1e-6 (> 2 ulp)
        const float dsh = 2.0f * (fast_div(1.01f * 1.7321f * eps_c, 0.316f * alen_lo) * 1.000001f + 1.8f * u);
        if ((0.0051f - dsh - 13.2f * u) * k.lod * (1.0f - 2.0f * u) >= k.pixel_size * (1.0f + 1e-4f)) lo_level = 0;
    }
    const float eps = 1.7321f * u * (2.0f + amax + fast_div(1.25f * alen_lo, k.wn) * 1.000001f + 2.0f * k.cmax) * 1.01f;
    const float dmax = 2.0f * (fast_div(1.34f * eps, alen_lo) * 1.000001f + 1.8f * u) * 1.01f;
    if (lo_level == 0) {  // whatever the deeper levels give, [0, j0) is shown
        lo = 0;
        hi = j0 - 1;
    }
    const float r0 = fast_div(2.0f * k.rvh * k.rvh * S, A * A);
    const float q = fast_div(r0 * k.lod, 4.0f * vmax(k.pixel_size, 1e-30f));
    if (!(q > 1.0f)) return;
    int m = (int)(0.5f * fast_log2(q));
    m = m < k.max_level ? m : k.max_level;
    for (int tries = 0; tries < 2 && m >= j0; ++tries, --m) {
        const float vh = scale2(k.rvh, -m);
        const float vh2 = vh * vh;
        const float den = A + vh2 * k.W;
        const float Rlow = fast_div(2.0f * vh2 * S, den * den) * (1.0f - 1e-4f);
        const float theta_up = fast_div(2.7f * vh * k.wn, alen_lo) * 1.000001f;
        const float x = 2.0f * Rlow;
        const float theta_lo = x * fast_rsqrt(x) * (1.0f - 1e-4f);
        if (!(theta_lo >= 5.0f * dmax)) continue;
        const float margin = (Rlow - theta_up * dmax - 11.2f * u) * (1.0f - 1e-5f);
        if (margin * k.lod * (1.0f - 4.0f * u) >= k.pixel_size * (1.0f + 1e-4f)) {
            lo = lo_level;
            hi = m;
            return;
        }
    }
}

}  // namespace lodb
}  // namespace vv
