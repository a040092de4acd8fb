// fixed_div.h - quotients by a divisor that is fixed for a frame (the brick
// pool's texel dimensions), from its correctly rounded reciprocal.
//
// Markstein's correction (P. W. Markstein, "Computation of elementary
// functions on the IBM RISC System/6000 processor", IBM J. Res. Dev. 34(1),
// 1990): with y = RN(1/b), q0 = RN(a*y), r = a - b*q0 (exact through one
// fused multiply-add) and q = RN(q0 + r*y).  For the divisors the kernels
// pass here (b = 10*s, s = 1..102) q equals RN(a/b), the IEEE quotient, for
// every significand of a (checked exhaustively by tests/test_fixed_div.py);
// every step scales exactly with a's exponent, so that holds for all a
// whose quotient and intermediates are normal numbers.  Smaller |a| takes
// the division itself.
#pragma once

#include <cmath>

namespace vv {

#if defined(__CUDACC__)
#define VV_FIXED_DIV_HD __host__ __device__ __forceinline__
#else
#define VV_FIXED_DIV_HD inline
#endif

// |a| below this takes the IEEE division (intermediates near the subnormal range)
constexpr float kFixedDivSmall = 7.8886090522101181e-31f;  // 2^-100

VV_FIXED_DIV_HD float fixed_div(float a, float b, float y) {
#if defined(__CUDA_ARCH__)
    if (fabsf(a) < kFixedDivSmall) return __fdiv_rn(a, b);
    const float q0 = __fmul_rn(a, y);
    const float r = __fmaf_rn(-b, q0, a);
    return __fmaf_rn(r, y, q0);
#else
    if (std::fabs(a) < kFixedDivSmall) return a / b;
    const float q0 = a * y;
    const float r = std::fma(-b, q0, a);
    return std::fma(r, y, q0);
#endif
}

}  // namespace vv
