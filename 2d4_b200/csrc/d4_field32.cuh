// d4_field32.cuh: FP32 form of the periodic wall field for the mixed form.
//
// The function is the reference's non-IEEE image sum (src/Fields/Field.cpp:
// 172-346): images dx+m for m = -3..3 summed, images +-4 and -+5 blended
// linearly in dx, and sinh taken equal to cosh for |m| >= 3.  Evaluated in FP32
// as follows (mathematically the same quantities):
//  - central image (m = 0): cosh(a) - cos(b) and cosh(a) cos(b) - 1, which
//    cancel catastrophically for close pairs, are formed from half angles,
//        cosh a - cos b     = 2 (sinh^2(a/2) + sin^2(b/2)),
//        cosh a cos b - 1   = 2 sinh^2(a/2) cos b - 2 sin^2(b/2),
//    which removes the cancellation (the reference switches to a Taylor
//    series below r^2 = 1e-6 for the same reason);
//  - other images: e_m = exp(2 pi dx) * exp(2 pi m), cosh = (e_m + 1/e_m)/2 and
//    sinh = (e_m - 1/e_m)/2 (no cancellation for |dx + m| >= 1/2); for |m| >= 3
//    the reference's cosh(2 pi m) e^(2 pi dx) differs from this by a relative
//    e^(-4 pi |dx+m|) < 2e-14, far below FP32 resolution;
//  - the per-image terms are summed with Neumaier compensation.
// Derivative terms are arranged as (1/q^2)(n1 + am (S c - 2 n1 S / q)) so no
// q^3 overflows FP32 for the outer images.
#pragma once

namespace d4 {
namespace f32 {

constexpr float kPi = 3.14159265358979f;
constexpr float k2Pi = 6.28318530717959f;
constexpr float kPi2Ln2Inv = 9.06472028365439f;  // 2 pi / ln 2

struct Neumaier {
    float s = 0.f, c = 0.f;
    __device__ __forceinline__ void add(float x) {
        const float t = s + x;
        c += fabsf(s) >= fabsf(x) ? (s - t) + x : (x - t) + s;
        s = t;
    }
    __device__ __forceinline__ float value() const { return s + c; }
};

// One image wall at offset am = 2 pi (dx + m) with cosh C, sinh S, cos c:
// stress term and its x-derivative (f_l / f_dx_l of the reference).
__device__ __forceinline__ void image(float am, float C, float S, float c, float &f, float &fd) {
    const float q = C - c;
    const float n1 = C * c - 1.f;
    const float iq = __frcp_rn(q);
    const float iq2 = iq * iq;
    f = am * n1 * iq2 * kPi;
    fd = iq2 * (n1 + am * (S * c - 2.f * n1 * S * iq)) * (2.f * kPi * kPi);
}

__device__ __forceinline__ void image_m(float dx, float e, float Em, float m, float c, bool sh_eq_ch,
                                        float &f, float &fd) {
    const float em = e * Em;
    const float im = __frcp_rn(em);
    const float C = 0.5f * (em + im);
    const float S = sh_eq_ch ? C : 0.5f * (em - im);
    image(k2Pi * (dx + m), C, S, c, f, fd);
}

// sigma_xy and d sigma_xy / dx at (dx, dy) in [-0.5, 0.5)^2.  want_grad = false
// skips the derivative.
template <bool kGrad>
__device__ __forceinline__ void field(float dx, float dy, float &sxy, float &sxyd) {
    // exp(2 pi m) for m = 1..5 and their inverses
    constexpr float E1 = 535.491655524764f, E2 = 286751.313136653f, E3 = 153552935.395f,
                    E4 = 82226315585.59f, E5 = 4.40315050606e13f;
    const float e = exp2f(kPi2Ln2Inv * dx);
    float sb2, c;
    sincospif(dy, &sb2, &c);  // sin(pi dy), cos(pi dy)
    c = 1.f - 2.f * sb2 * sb2;  // cos(2 pi dy), without cancellation issues for the wall sum
    Neumaier sf, sd;
    // central image
    {
        const float a = k2Pi * dx;
        const float sha = sinhf(0.5f * a);
        const float D = 2.f * (sha * sha + sb2 * sb2);
        const float N0 = 2.f * sha * sha * c - 2.f * sb2 * sb2;
        const float iD = __frcp_rn(D);
        const float iD2 = iD * iD;
        sf.add(a * N0 * iD2 * kPi);
        if (kGrad) {
            const float Sa = sinhf(a);
            sd.add(iD2 * (N0 + a * (Sa * c - 2.f * N0 * Sa * iD)) * (2.f * kPi * kPi));
        }
    }
    float f, fd;
    image_m(dx, e, E1, 1.f, c, false, f, fd);
    sf.add(f);
    if (kGrad) sd.add(fd);
    image_m(dx, e, 1.f / E1, -1.f, c, false, f, fd);
    sf.add(f);
    if (kGrad) sd.add(fd);
    image_m(dx, e, E2, 2.f, c, false, f, fd);
    sf.add(f);
    if (kGrad) sd.add(fd);
    image_m(dx, e, 1.f / E2, -2.f, c, false, f, fd);
    sf.add(f);
    if (kGrad) sd.add(fd);
    image_m(dx, e, E3, 3.f, c, true, f, fd);
    sf.add(f);
    if (kGrad) sd.add(fd);
    image_m(dx, e, 1.f / E3, -3.f, c, true, f, fd);
    sf.add(f);
    if (kGrad) sd.add(fd);
    // blended outer images (src/Fields/Field.cpp:297-310, 316-329)
    float f4p, fd4p, f4m, fd4m, f5, fd5;
    image_m(dx, e, E4, 4.f, c, true, f4p, fd4p);
    image_m(dx, e, 1.f / E4, -4.f, c, true, f4m, fd4m);
    if (dx < 0) {
        image_m(dx, e, E5, 5.f, c, true, f5, fd5);
        sf.add(f5 * (-dx));
        sf.add(f4m * (1.f + dx));
        sf.add(f4p);
        if (kGrad) {
            sd.add(fd5 * (-dx));
            sd.add(-f5);
            sd.add(fd4m * (1.f + dx));
            sd.add(f4m);
            sd.add(fd4p);
        }
    } else {
        image_m(dx, e, 1.f / E5, -5.f, c, true, f5, fd5);
        sf.add(f5 * dx);
        sf.add(f4p * (1.f - dx));
        sf.add(f4m);
        if (kGrad) {
            sd.add(fd5 * dx);
            sd.add(f5);
            sd.add(fd4p * (1.f - dx));
            sd.add(-f4p);
            sd.add(fd4m);
        }
    }
    sxy = sf.value();
    sxyd = kGrad ? sd.value() : 0.f;
}

}  // namespace f32
}  // namespace d4
