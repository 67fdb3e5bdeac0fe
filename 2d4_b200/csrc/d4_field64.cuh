// d4_field64.cuh: FP64 device form of the periodic edge-dislocation wall field.
//
// Shear stress sigma_xy of a periodic wall array and its x-derivative, as
// src/Fields/Field.cpp:172-346 (non-IEEE path, USE_IEEE_HYPERBOLIC 0,
// include/constants.h:40-80) defines them: images -3..3 summed exactly, the
// images +-4 and -+5 blended linearly in dx, cosh/sinh of 2*pi*(dx+-i) built from
// one e = exp(2*pi*dx) with the addition theorems, and cosh = sinh taken for
// |i| >= 3.  The expressions keep the reference's operation order; the
// translation unit that includes this file is compiled with --fmad=false, so no
// product-add is contracted and every operation rounds as in the reference's
// IEEE build.  The only deviations are the transcendental calls (exp2, cos,
// pow for cubes, sinh), which CUDA rounds to within an ulp or two of glibc.
#pragma once

namespace d4 {
namespace f64 {

constexpr double kPi = 3.14159265358979323846;
// 2*pi/ln(2) and cosh/sinh(k*pi), as the decimal literals of include/constants.h.
constexpr double kPi2Ln2Inv = 9.0647202836543876192553658914333336203437229354476;
constexpr double kCosh2Pi = 267.746761483748222245931879901;
constexpr double kCosh4Pi = 143375.656570070321051450310133;
constexpr double kCosh6Pi = 7.67764676977233502175191858009e7;
constexpr double kCosh8Pi = 4.11131577927974976374895337541e10;
constexpr double kCoshTPi = 2.20157529303160145057002722946e13;
constexpr double kSinh2Pi = 267.744894041016514257117449688;
constexpr double kSinh4Pi = 143375.656566582978695241314640;

// x^3 rounded once: x*x split exactly into p + e (TwoProduct via fma), then
// p*x + e*x with a single rounding.  The reference calls pow(q, 3).
__device__ __forceinline__ double cube(double x) {
    double p = x * x;
    double e = fma(x, x, -p);
    return fma(p, x, e * x);
}

// Hyperbolic values of 2*pi*(dx +- i) from e = exp(2*pi*dx).
struct Hyp {
    double ch0, sh0, chp1, chm1, shp1, shm1, chp2, chm2, shp2, shm2;
    double chp3, chm3, chp4, chm4, chp5, chm5;
    __device__ __forceinline__ explicit Hyp(double e) {
        double inv = 1 / e;
        double s = e + inv, d = e - inv;
        ch0 = s / 2;
        sh0 = d / 2;
        chp1 = (s * kCosh2Pi + d * kSinh2Pi) / 2;
        chm1 = (s * kCosh2Pi - d * kSinh2Pi) / 2;
        shp1 = (d * kCosh2Pi + s * kSinh2Pi) / 2;
        shm1 = (d * kCosh2Pi - s * kSinh2Pi) / 2;
        chp2 = (s * kCosh4Pi + d * kSinh4Pi) / 2;
        chm2 = (s * kCosh4Pi - d * kSinh4Pi) / 2;
        shp2 = (d * kCosh4Pi + s * kSinh4Pi) / 2;
        shm2 = (d * kCosh4Pi - s * kSinh4Pi) / 2;
        chp3 = kCosh6Pi * e;
        chm3 = kCosh6Pi / e;
        chp4 = kCosh8Pi * e;
        chm4 = kCosh8Pi / e;
        chp5 = kCoshTPi * e;
        chm5 = kCoshTPi / e;
    }
};

// f_l, src/Fields/Field.cpp:191-196.
__device__ __forceinline__ double f_l(double dx, double c, double ch) {
    double dx2pi = kPi * 2 * dx;
    double q = ch - c;
    return dx2pi * (ch * c - 1) / (q * q) * kPi;
}

// Taylor branch of f_0 for dx^2 + dy^2 <= 1e-6, src/Fields/Field.cpp:183-187.
static __device__ __noinline__ double f0_taylor(double dx2pi, double dy2pi) {
    double x2 = dx2pi * dx2pi, y2 = dy2pi * dy2pi;
    double x4 = pow(dx2pi, 4.0), y4 = pow(dy2pi, 4.0);
    double x6 = pow(dx2pi, 6.0), y6 = pow(dy2pi, 6.0);
    double chm1 = x6 / 720 + x4 / 24 + x2 * 0.5;
    double cm1 = -y6 / 720 + y4 / 24 - y2 * 0.5;
    double cmc = (y6 + x6) / 720 + (x4 - y4) / 24 + (x2 + y2) * 0.5;
    return ((chm1 * cm1 + cm1 + chm1) * dx2pi) / (cmc * cmc) * kPi;
}

// f_0, src/Fields/Field.cpp:172-188.
__device__ __forceinline__ double f_0(double dx, double c, double dy, double ch) {
    double dx2pi = kPi * 2 * dx;
    if (dx * dx + dy * dy > 1e-6) {
        double q = ch - c;
        return dx2pi * (ch * c - 1) / (q * q) * kPi;
    }
    return f0_taylor(dx2pi, kPi * 2 * dy);
}

// f_dx_l / f_dx_h, src/Fields/Field.cpp:253-282 (f_dx_h passes sh = ch).
__device__ __forceinline__ double f_dx_l(double dx, double c, double ch, double sh) {
    double dx2pi = dx * 2 * kPi;
    double q = ch - c;
    double n1 = ch * c - 1;
    double q2 = q * q;
    return (n1 / q2 + dx2pi * (sh * c / q2 - n1 / cube(q) * 2 * sh)) * kPi * 2 * kPi;
}

// Taylor branch of f_dx_0, src/Fields/Field.cpp:224-249.
static __device__ __noinline__ double fdx0_taylor(double dx, double dy) {
    double dx2pi = dx * 2 * kPi;
    double dy2pi = dy * kPi * 2;
    double x2 = dx2pi * dx2pi, y2 = dy2pi * dy2pi;
    double x3 = cube(dx2pi), x4 = pow(dx2pi, 4.0), x5 = pow(dx2pi, 5.0);
    double x6 = pow(dx2pi, 6.0), x7 = pow(dx2pi, 7.0);
    double y4 = pow(dy2pi, 4.0), y6 = pow(dy2pi, 6.0);
    double chm1 = x6 / 720 + x4 / 24 + x2 * 0.5;
    double cm1 = -y6 / 720 + y4 / 24 - y2 * 0.5;
    double cmc = (y6 + x6) / 720 + (x4 - y4) / 24 + (x2 + y2) * 0.5;
    double cs = -(x7 * y6) / 3628800 - (x5 * y6) / 86400 - (x3 * y6) / 4320 - (y6 * dx2pi) / 720 +
                (x7 * y4) / 120960 + (x5 * y4) / 2880 + (x3 * y4) / 144 + (y4 * dx2pi) / 24 -
                (x7 * y2) / 1080 - (x5 * y2) / 240 - (x3 * y2) / 12 - (y2 * dx2pi) * 0.5 +
                x7 / 5040 + x5 / 120 + x3 / 6 + dx2pi;
    double num = chm1 * cm1 + cm1 + chm1;
    return (num / (cmc * cmc) +
            ((cs * dx) / (cmc * cmc) - num / cube(cmc) * dx * sinh(dx2pi) * 2) * 2 * kPi) *
           kPi * 2 * kPi;
}

// f_dx_0, src/Fields/Field.cpp:209-250.
__device__ __forceinline__ double f_dx_0(double dx, double c, double dy, double ch, double sh) {
    if (dx * dx + dy * dy > 1e-6) {
        double dx2pi = dx * 2 * kPi;
        double q = ch - c;
        double q2 = q * q;
        return ((ch * c - 1) / q2 + dx2pi * (sh * c / q2 - (ch * c - 1) / cube(q) * 2 * sh)) *
               kPi * 2 * kPi;
    }
    return fdx0_taylor(dx, dy);
}

// Field::xy (4-arg), src/Fields/Field.cpp:295-311 with g3 (:199-206) inlined in
// the reference's summation order.
__device__ __forceinline__ double xy(double dx, double dy, const Hyp &h, double c) {
    double g3 = f_l(dx + 3, c, h.chp3) + f_l(dx - 3, c, h.chm3) + f_l(dx + 2, c, h.chp2) +
                f_l(dx - 2, c, h.chm2) + f_l(dx + 1, c, h.chp1) + f_l(dx - 1, c, h.chm1) +
                f_0(dx + 0, c, dy, h.ch0);
    if (dx < 0)
        return f_l(dx + 5, c, h.chp5) * (0 - dx) + f_l(dx - 4, c, h.chm4) * (1 + dx) +
               f_l(dx + 4, c, h.chp4) + g3;
    return f_l(dx - 5, c, h.chm5) * (0 + dx) + f_l(dx + 4, c, h.chp4) * (1 - dx) +
           f_l(dx - 4, c, h.chm4) + g3;
}

// Field::xy_diff_x (4-arg), src/Fields/Field.cpp:314-330 with g3_dx (:285-292).
__device__ __forceinline__ double xy_diff_x(double dx, double dy, const Hyp &h, double c) {
    double g3 = f_dx_0(dx + 0, c, dy, h.ch0, h.sh0) + f_dx_l(dx + 1, c, h.chp1, h.shp1) +
                f_dx_l(dx - 1, c, h.chm1, h.shm1) + f_dx_l(dx + 2, c, h.chp2, h.shp2) +
                f_dx_l(dx - 2, c, h.chm2, h.shm2) + f_dx_l(dx + 3, c, h.chp3, h.chp3) +
                f_dx_l(dx - 3, c, h.chm3, h.chm3);
    if (dx < 0)
        return f_dx_l(dx + 5, c, h.chp5, h.chp5) * (0 - dx) + f_l(dx + 5, c, h.chp5) * (-1) +
               f_dx_l(dx - 4, c, h.chm4, h.chm4) * (1 + dx) + f_l(dx - 4, c, h.chm4) * (+1) +
               f_dx_l(dx + 4, c, h.chp4, h.chp4) + g3;
    return f_dx_l(dx - 5, c, h.chm5, h.chm5) * (0 + dx) + f_l(dx - 5, c, h.chm5) * (+1) +
           f_dx_l(dx + 4, c, h.chp4, h.chp4) * (1 - dx) + f_l(dx + 4, c, h.chp4) * (-1) +
           f_dx_l(dx - 4, c, h.chm4, h.chm4) + g3;
}

// normalize, src/sim_utils.cpp:6-13 (while-loop wrap into [-0.5, 0.5)).  The
// loops take at most a few turns for the differences of positions in the cell;
// a value that is not finite, or so large that n -+ 1 == n, would keep them
// turning forever (the reference's loops too), so such values skip the loops:
// infinities and NaN give NaN, the large finite values wrap by rounding.
__device__ __forceinline__ double normalize(double n) {
    if (!(fabs(n) < 1048576.0)) return n - rint(n);  // inf - inf and NaN give NaN
    while (n < -0.5) n += 1;
    while (n >= 0.5) n -= 1;
    return n;
}

// e = exp(2*pi*dx) computed as the reference does: exp2((2*pi/ln 2) * dx).
__device__ __forceinline__ double exp2pix(double dx) { return exp2(kPi2Ln2Inv * dx); }
__device__ __forceinline__ double cos2piy(double dy) { return cos(kPi * 2 * dy); }

// weight, src/sim_utils.cpp:36-55.
__device__ __forceinline__ double weight(double s, char t) {
    if (s > 0) {
        if (t == 'c') {
            double r = s / (s + 1);
            return r * r;
        }
        if (t == 'p') return s / (s + 1);
        if (t == 'm') {
            double c = 0.412073;
            return 1 / (1 + 1.5 / (s + c * s * s));
        }
    }
    return 0;
}

// weightInv, src/sim_utils.cpp:57-75.
__device__ __forceinline__ double weight_inv(double w, char t) {
    if (w > 0) {
        if (t == 'c') return sqrt(w) / (1 - sqrt(w));
        if (t == 'p') return w / (1 - w);
        if (t == 'm') {
            double c = 0.412073;
            return (1 - w - sqrt(1 - 2 * w + 6 * c * w + w * w - 6 * c * w * w)) /
                   (2 * (-c + c * w));
        }
    }
    return 0;
}

}  // namespace f64
}  // namespace d4
