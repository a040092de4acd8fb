// Exhaustive host check of voxviz_b200/csrc/fixed_div.h: for every divisor
// b = 10*s (s = 1..102, the brick-pool texel dimensions) and every float
// significand of a in [1, 2) (plus the binades [2^-99, 2^-98) and
// [2^10, 2^11), which must agree by exact scaling), fixed_div(a, b, 1/b)
// equals a / b bit for bit.  Built and run by tests/test_fixed_div.py.
// Prints "<checks> <mismatches>" and exits non-zero on a mismatch.
#include <cstdint>
#include <cstdio>
#include <cstring>

#include "../voxviz_b200/csrc/fixed_div.h"

static uint32_t bits(float f) {
    uint32_t u;
    std::memcpy(&u, &f, 4);
    return u;
}

int main() {
    unsigned long long checks = 0, bad = 0;
    const float scales[3] = {1.0f, 0x1p-99f, 0x1p10f};
#pragma omp parallel for schedule(dynamic, 1) reduction(+ : checks, bad)
    for (int s = 1; s <= 102; ++s) {
        const float b = (float)(10 * s);
        const float y = 1.0f / b;
        for (int k = 0; k < 3; ++k)
            for (uint32_t m = 0; m < (1u << 23); ++m) {
                uint32_t ab = 0x3F800000u | m;
                float a;
                std::memcpy(&a, &ab, 4);
                a *= scales[k];
                const float q = vv::fixed_div(a, b, y), e = a / b;
                ++checks;
                if (bits(q) != bits(e)) {
#pragma omp critical
                    std::printf("mismatch b=%g a=%a: %a vs %a\n", (double)b, (double)a, (double)q, (double)e);
                    ++bad;
                }
            }
    }
    std::printf("%llu %llu\n", checks, bad);
    return bad ? 1 : 0;
}
