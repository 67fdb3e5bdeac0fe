// d4_field_dual.cuh: Field::xy and Field::xy_diff_x with their x-derivatives in
// one pass, by forward-mode differentiation (dual numbers) of the same
// expressions as d4_field64.cuh (src/Fields/Field.cpp:172-330).
//
// The derivative code needs both, and they differ.  Field::xy_diff_x is not the
// exact x-derivative of Field::xy: for the images |i| >= 3 it takes
// sinh = cosh (f_dx_h, Field.cpp:253-282), whose sign is wrong for the images
// at negative argument, so it departs from d xy / dx by up to ~2e-5 relative
// and is not even in (dx, dy).  The engine's velocities come from xy, so their
// Jacobian is d xy / dx (dual of xy); the engine's implicit-step matrix and
// its row weights are built from xy_diff_x, so their dependence on positions
// is d xy_diff_x / dx (dual of xy_diff_x).
#pragma once
#include "d4_field64.cuh"

namespace d4 {
namespace dual {

struct D {
    double v, d;  // value and derivative with respect to dx
};

__device__ __forceinline__ D mk(double v, double d = 0) { return D{v, d}; }
__device__ __forceinline__ D operator+(D a, D b) { return D{a.v + b.v, a.d + b.d}; }
__device__ __forceinline__ D operator-(D a, D b) { return D{a.v - b.v, a.d - b.d}; }
__device__ __forceinline__ D operator-(D a) { return D{-a.v, -a.d}; }
__device__ __forceinline__ D operator*(D a, D b) { return D{a.v * b.v, a.d * b.v + a.v * b.d}; }
__device__ __forceinline__ D operator/(D a, D b) {
    const double q = a.v / b.v;
    return D{q, (a.d - q * b.d) / b.v};
}
__device__ __forceinline__ D operator+(D a, double b) { return D{a.v + b, a.d}; }
__device__ __forceinline__ D operator-(D a, double b) { return D{a.v - b, a.d}; }
__device__ __forceinline__ D operator-(double a, D b) { return D{a - b.v, -b.d}; }
__device__ __forceinline__ D operator+(double a, D b) { return D{a + b.v, b.d}; }
__device__ __forceinline__ D operator*(D a, double b) { return D{a.v * b, a.d * b}; }
__device__ __forceinline__ D operator*(double a, D b) { return D{a * b.v, a * b.d}; }
__device__ __forceinline__ D operator/(D a, double b) { return D{a.v / b, a.d / b}; }
__device__ __forceinline__ D operator/(double a, D b) {
    const double q = a / b.v;
    return D{q, -q * b.d / b.v};
}
__device__ __forceinline__ D ipow(D x, int k) {
    D r = mk(1.0);
    for (int i = 0; i < k; ++i) r = r * x;
    return r;
}
__device__ __forceinline__ D dsinh(D x) { return D{sinh(x.v), cosh(x.v) * x.d}; }

using f64::kPi;

// Hyperbolic values of 2 pi (dx +- i) from e = exp(2 pi dx), as f64::Hyp.
struct Hyp {
    D ch0, sh0, chp1, chm1, shp1, shm1, chp2, chm2, shp2, shm2;
    D chp3, chm3, chp4, chm4, chp5, chm5;
    __device__ __forceinline__ explicit Hyp(D e) {
        const D inv = 1.0 / e;
        const D s = e + inv, d = e - inv;
        ch0 = s / 2;
        sh0 = d / 2;
        chp1 = (s * f64::kCosh2Pi + d * f64::kSinh2Pi) / 2;
        chm1 = (s * f64::kCosh2Pi - d * f64::kSinh2Pi) / 2;
        shp1 = (d * f64::kCosh2Pi + s * f64::kSinh2Pi) / 2;
        shm1 = (d * f64::kCosh2Pi - s * f64::kSinh2Pi) / 2;
        chp2 = (s * f64::kCosh4Pi + d * f64::kSinh4Pi) / 2;
        chm2 = (s * f64::kCosh4Pi - d * f64::kSinh4Pi) / 2;
        shp2 = (d * f64::kCosh4Pi + s * f64::kSinh4Pi) / 2;
        shm2 = (d * f64::kCosh4Pi - s * f64::kSinh4Pi) / 2;
        chp3 = e * f64::kCosh6Pi;
        chm3 = f64::kCosh6Pi / e;
        chp4 = e * f64::kCosh8Pi;
        chm4 = f64::kCosh8Pi / e;
        chp5 = e * f64::kCoshTPi;
        chm5 = f64::kCoshTPi / e;
    }
};

__device__ __forceinline__ D f_l(D dx, double c, D ch) {
    const D q = ch - c;
    return dx * (2 * kPi) * (ch * c - 1) / (q * q) * kPi;
}

__device__ __forceinline__ D f_dx_l(D dx, double c, D ch, D sh) {
    const D dx2pi = dx * (2 * kPi);
    const D q = ch - c;
    const D n1 = ch * c - 1;
    const D q2 = q * q;
    return (n1 / q2 + dx2pi * (sh * c / q2 - n1 / (q2 * q) * 2 * sh)) * (2 * kPi * kPi);
}

// Taylor branch of f_dx_0 (dx^2 + dy^2 <= 1e-6), Field.cpp:224-249.
__device__ __noinline__ D fdx0_taylor(D dx, double dy) {
    const D X = dx * (2 * kPi);
    const double Y = dy * kPi * 2;
    const D x2 = X * X, x3 = ipow(X, 3), x4 = ipow(X, 4), x5 = ipow(X, 5), x6 = ipow(X, 6),
            x7 = ipow(X, 7);
    const double y2 = Y * Y, y4 = y2 * y2, y6 = y4 * y2;
    const D chm1 = x6 / 720 + x4 / 24 + x2 * 0.5;
    const double cm1 = -y6 / 720 + y4 / 24 - y2 * 0.5;
    const D cmc = (x6 + y6) / 720 + (x4 - y4) / 24 + (x2 + y2) * 0.5;
    const D cs = -(x7 * y6) / 3628800 - (x5 * y6) / 86400 - (x3 * y6) / 4320 - (X * y6) / 720 +
                 (x7 * y4) / 120960 + (x5 * y4) / 2880 + (x3 * y4) / 144 + (X * y4) / 24 -
                 (x7 * y2) / 1080 - (x5 * y2) / 240 - (x3 * y2) / 12 - (X * y2) * 0.5 +
                 x7 / 5040 + x5 / 120 + x3 / 6 + X;
    const D num = chm1 * cm1 + cm1 + chm1;
    const D cmc2 = cmc * cmc;
    return (num / cmc2 + ((cs * dx) / cmc2 - num / (cmc2 * cmc) * dx * dsinh(X) * 2) * 2 * kPi) *
           (kPi * 2 * kPi);
}

__device__ __forceinline__ D f_dx_0(D dx, double c, double dy, D ch, D sh) {
    if (dx.v * dx.v + dy * dy > 1e-6) return f_dx_l(dx, c, ch, sh);
    return fdx0_taylor(dx, dy);
}

// Taylor branch of f_0 (dx^2 + dy^2 <= 1e-6), Field.cpp:183-187.
__device__ __noinline__ D f0_taylor(D dx, double dy) {
    const D X = dx * (2 * kPi);
    const double Y = dy * (2 * kPi);
    const D x2 = X * X, x4 = x2 * x2, x6 = x4 * x2;
    const double y2 = Y * Y, y4 = y2 * y2, y6 = y4 * y2;
    const D chm1 = x6 / 720 + x4 / 24 + x2 * 0.5;
    const double cm1 = -y6 / 720 + y4 / 24 - y2 * 0.5;
    const D cmc = (x6 + y6) / 720 + (x4 - y4) / 24 + (x2 + y2) * 0.5;
    return ((chm1 * cm1 + cm1 + chm1) * X) / (cmc * cmc) * kPi;
}

__device__ __forceinline__ D f_0(D dx, double c, double dy, D ch) {
    if (dx.v * dx.v + dy * dy > 1e-6) return f_l(dx, c, ch);
    return f0_taylor(dx, dy);
}

__device__ __forceinline__ Hyp hyp_of(double dxv) {
    const double ev = exp(2 * kPi * dxv);
    return Hyp(D{ev, 2 * kPi * ev});
}

// {Field::xy(dx, dy), its derivative in dx} (Field.cpp:295-311).
__device__ __forceinline__ D xy(double dxv, double dy) {
    const D dx = mk(dxv, 1.0);
    const Hyp h = hyp_of(dxv);
    const double c = cos(kPi * 2 * dy);
    const D g3 = f_l(dx + 3, c, h.chp3) + f_l(dx - 3, c, h.chm3) + f_l(dx + 2, c, h.chp2) +
                 f_l(dx - 2, c, h.chm2) + f_l(dx + 1, c, h.chp1) + f_l(dx - 1, c, h.chm1) +
                 f_0(dx, c, dy, h.ch0);
    if (dxv < 0)
        return f_l(dx + 5, c, h.chp5) * (0 - dx) + f_l(dx - 4, c, h.chm4) * (1 + dx) +
               f_l(dx + 4, c, h.chp4) + g3;
    return f_l(dx - 5, c, h.chm5) * dx + f_l(dx + 4, c, h.chp4) * (1 - dx) +
           f_l(dx - 4, c, h.chm4) + g3;
}

// {Field::xy_diff_x(dx, dy), its derivative in dx}.
__device__ __forceinline__ D xy_diff_x(double dxv, double dy) {
    const D dx = mk(dxv, 1.0);
    const Hyp h = hyp_of(dxv);
    const double c = cos(kPi * 2 * dy);
    const D g3 = f_dx_0(dx, c, dy, h.ch0, h.sh0) + f_dx_l(dx + 1, c, h.chp1, h.shp1) +
                 f_dx_l(dx - 1, c, h.chm1, h.shm1) + f_dx_l(dx + 2, c, h.chp2, h.shp2) +
                 f_dx_l(dx - 2, c, h.chm2, h.shm2) + f_dx_l(dx + 3, c, h.chp3, h.chp3) +
                 f_dx_l(dx - 3, c, h.chm3, h.chm3);
    if (dxv < 0)
        return f_dx_l(dx + 5, c, h.chp5, h.chp5) * (0 - dx) - f_l(dx + 5, c, h.chp5) +
               f_dx_l(dx - 4, c, h.chm4, h.chm4) * (1 + dx) + f_l(dx - 4, c, h.chm4) +
               f_dx_l(dx + 4, c, h.chp4, h.chp4) + g3;
    return f_dx_l(dx - 5, c, h.chm5, h.chm5) * dx + f_l(dx - 5, c, h.chm5) +
           f_dx_l(dx + 4, c, h.chp4, h.chp4) * (1 - dx) - f_l(dx + 4, c, h.chp4) +
           f_dx_l(dx - 4, c, h.chm4, h.chm4) + g3;
}

}  // namespace dual
}  // namespace d4
