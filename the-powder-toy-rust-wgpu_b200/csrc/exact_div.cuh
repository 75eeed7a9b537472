// exact_div.cuh -- correctly rounded division by a constant without a
// division instruction sequence.
//
// Markstein's correction step (P. Markstein, "Computation of elementary
// functions on the IBM RISC System/6000 processor", IBM J. Res. Dev. 34(1),
// 1990; also Brisebarre, Muller and Raina, "Accelerating correctly rounded
// floating-point division when the divisor is known in advance", IEEE Trans.
// Computers 53(8), 2004): with r = RN(1/c),
//     q  = RN(x * r)            a first quotient
//     e  = x - q * c            exact, as one fused multiply-add
//     q' = RN(q + e * r)        one fused multiply-add
// The remainder e is exact only while it is a normal number, i.e. for |x|
// above about 2^-102 (and the step gives NaN for infinite x), so the shortcut
// is taken for 2^-100 <= |x| <= FLT_MAX; zeros return x * r (keeping the
// sign) and everything else takes the IEEE division. For the divisors this
// build uses, tests/test_gpu_exact_div.py checks all 2^32 inputs against IEEE
// division on the device: the function is bit-identical to `x / c`.
#pragma once

namespace tpt {

__device__ __forceinline__ float div_by_const(float x, float c, float rc) {
    const float q = __fmul_rn(x, rc);
    const float ax = fabsf(x);
    if (ax >= 0x1p-100f && ax <= 3.40282347e+38f) {
        const float e = __fmaf_rn(-q, c, x);
        return __fmaf_rn(e, rc, q);
    }
    return x == 0.0f ? q : __fdiv_rn(x, c);
}

// The smoothing weights' sum in the order the 3x3 loops add them (advect.rs
// 205-253 and heat.rs 60-104 add all nine weights, blocked taps included):
// rows dy = -1, 0, 1, columns dx = -1, 0, 1; e^-4 at the corners, e^-2 at the
// edges, 1 at the centre; every addition rounded to f32.
constexpr float smooth_wsum() {
    float s = 0.0f;
    for (int dy = 0; dy < 3; ++dy)
        for (int dx = 0; dx < 3; ++dx) {
            float w = 0.01831564f;
            if (dx == 1) w = 0.13533528f;
            if (dy == 1) w = 0.13533528f;
            if (dx == 1 && dy == 1) w = 1.0f;
            s += w;
        }
    return s;
}
constexpr float kSmoothWsum = smooth_wsum();
constexpr float kSmoothWsumRcp = 1.0f / kSmoothWsum;
constexpr float kConvLegacy = 5000.0f, kConvLegacyRcp = 1.0f / kConvLegacy;   // heat.rs legacy convection
constexpr float kConvBouss = 10000.0f, kConvBoussRcp = 1.0f / kConvBouss;     // heat.rs Boussinesq convection

}  // namespace tpt
