// Host check of voxviz_b200/csrc/lod_bound.h against the exact binary32 LOD
// test of the descent.  Built and run by tests/test_lod_bound.py.
//   random:      random cameras, positions, pixel sizes and LOD scalars; every
//                level the certificate clears must continue exactly
//   adversarial: the pixel size is set one ulp (or 1e-6 relative) above the
//                exact projection at a level j, so the exact test stops at j;
//                the certificate must never clear j
// Prints "<checks> <violations>" and exits non-zero on a violation.
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <random>

#include "../voxviz_b200/csrc/lod_bound.h"

using vv::lodb::V3;

static V3 add(V3 a, V3 b) { return V3{a.x + b.x, a.y + b.y, a.z + b.z}; }
static V3 sub(V3 a, V3 b) { return V3{a.x - b.x, a.y - b.y, a.z - b.z}; }
static V3 muls(V3 a, float s) { return V3{a.x * s, a.y * s, a.z * s}; }
static float dot3(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
static V3 normalize3(V3 v) {
    float r = 1.0f / std::sqrt(dot3(v, v));
    return muls(v, r);
}
static V3 cross3(V3 a, V3 b) { return V3{a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }

// the descent's test (GigaVoxelsNoLighting.frag:429-441 * LodScalar), binary32
static float exact_proj(V3 pos, V3 C, V3 up, V3 left, float vhalf, float lod) {
    V3 uh = muls(up, vhalf), lh = muls(left, vhalf);
    V3 ll = normalize3(sub(add(sub(pos, uh), lh), C));
    V3 ur = normalize3(sub(sub(add(pos, uh), lh), C));
    return (1.0f - dot3(ll, ur)) * lod;
}

int main(int argc, char** argv) {
    const long n = argc > 1 ? atol(argv[1]) : 200000;
    std::mt19937_64 rng(argc > 2 ? atol(argv[2]) : 1);
    std::uniform_real_distribution<float> U(0.f, 1.f);
    const float rvh = 1.0f / 16.0f;
    const int L = 12;
    long checks = 0, violations = 0;
    for (long it = 0; it < n; ++it) {
        V3 C{U(rng) * 3.f - 1.f, U(rng) * 3.f - 1.f, U(rng) * 1.6f - 0.2f};
        V3 pos{U(rng), U(rng), U(rng)};
        if (pos.x <= 0.f || pos.y <= 0.f || pos.z <= 0.f) continue;
        V3 look = sub(pos, C);
        const float ln = std::sqrt(dot3(look, look));
        if (ln < 1e-4f) continue;
        V3 jit{U(rng) - 0.5f, U(rng) - 0.5f, U(rng) - 0.5f};
        look = normalize3(add(muls(look, 1.0f / ln), muls(jit, 0.8f)));
        V3 left = cross3(V3{0.f, 0.f, 1.f}, look);
        if (dot3(left, left) < 1e-6f) continue;
        left = normalize3(left);
        V3 up = normalize3(cross3(look, left));
        const float lod = (U(rng) < 0.8f) ? 1.0f : 0.25f + 2.f * U(rng);
        float pix;
        int stop_level = -1;
        if (it & 1) {
            pix = std::pow(10.f, -7.5f + 3.5f * U(rng));
        } else {
            stop_level = (int)(U(rng) * (L + 1));
            const float proj = exact_proj(pos, C, up, left, std::ldexp(rvh, -stop_level), lod);
            pix = (U(rng) < 0.7f) ? std::nextafter(proj, 1e30f) : proj * (1.0f + 1e-6f * U(rng));
            if (!(pix > proj)) continue;
        }
        const vv::lodb::Consts k = vv::lodb::make_consts(C, up, left, rvh, lod, pix, L, true);
        int lo, hi;
        vv::lodb::clear_range(k, pos, lo, hi);
        for (int j = lo; j <= hi; ++j) {
            ++checks;
            const float proj = exact_proj(pos, C, up, left, std::ldexp(rvh, -j), lod);
            if (pix > proj || j == stop_level) {
                ++violations;
                if (violations <= 5) fprintf(stderr, "violation: it=%ld level=%d range=[%d,%d]\n", it, j, lo, hi);
            }
        }
    }
    printf("%ld %ld\n", checks, violations);
    return violations ? 1 : 0;
}
