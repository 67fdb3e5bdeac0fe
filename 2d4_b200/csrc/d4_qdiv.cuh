// d4_qdiv.cuh: correctly rounded quotients a / b from a precomputed
// correctly rounded reciprocal y = RN(1/b), for division chains whose divisor
// is known before the chain runs (the LU's rows below a factorised diagonal
// block, the substitutions' diagonal).
//
// Method (Markstein, "Computation of elementary functions on the IBM RISC
// System/6000 processor", IBM J. Res. Develop. 34(1), 1990; Muller et al.,
// Handbook of Floating-Point Arithmetic, ch. "Newton-Raphson-based division"):
// if y = RN(1/b) and q is a faithful approximation of a / b (within one ulp),
// the residual r = a - b q is exact in one FMA and RN(q + r y) = RN(a / b).
// q0 = RN(a y) is within 1.5 ulp, so one correction first makes it faithful
// and a second gives the correctly rounded quotient: five dependent
// operations instead of a full division.  The exponent window keeps every
// intermediate (q, the residual's bit grid, r y) normal; outside it, and for
// zero numerators (sign of zero), the helpers divide.  The result is the IEEE
// quotient bit for bit, so the exact-order factorisation keeps its rounding.
#pragma once

namespace d4 {
namespace qdiv {

// |v| in [2^-400, 2^401) (double) or [2^-38, 2^39) (float)
__device__ __forceinline__ bool in_range(double v) {
    const unsigned e = ((unsigned)__double2hiint(v) >> 20) & 0x7ffu;
    return e - 623u <= 800u;
}
__device__ __forceinline__ bool in_range(float v) {
    const unsigned e = ((unsigned)__float_as_uint(v) >> 23) & 0xffu;
    return e - 89u <= 76u;
}

// RN(1/b), or 0 when b is outside the window (the quotient then divides)
template <typename T>
__device__ __forceinline__ T recip(T b) {
    return in_range(b) ? T(1) / b : T(0);
}

// A zero numerator over an in-window divisor gives a y: the zero with the
// quotient's sign, as the division would (whose zero case is a slow path).
__device__ __forceinline__ double div(double a, double b, double y) {
    if (y != 0.0) {
        if (a == 0.0) return __dmul_rn(a, y);
        if (in_range(a)) {
            const double q0 = __dmul_rn(a, y);
            const double q1 = __fma_rn(__fma_rn(-b, q0, a), y, q0);
            return __fma_rn(__fma_rn(-b, q1, a), y, q1);
        }
    }
    return a / b;
}
__device__ __forceinline__ float div(float a, float b, float y) {
    if (y != 0.0f) {
        if (a == 0.0f) return __fmul_rn(a, y);
        if (in_range(a)) {
            const float q0 = __fmul_rn(a, y);
            const float q1 = __fmaf_rn(__fmaf_rn(-b, q0, a), y, q0);
            return __fmaf_rn(__fmaf_rn(-b, q1, a), y, q1);
        }
    }
    return a / b;
}

}  // namespace qdiv
}  // namespace d4
