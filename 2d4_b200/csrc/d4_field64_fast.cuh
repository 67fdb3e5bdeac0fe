// d4_field64_fast.cuh: the wall field of d4_field64.cuh for the mixed form's
// FP64 sweeps, without the reference's operation order.
//
// Same images, blends and branches as d4::f64 (src/Fields/Field.cpp:172-346):
// images -3..3 summed exactly, the images +-4 and -+5 blended linearly in dx,
// the hyperbolic values of 2*pi*(dx +- i) from one e = exp(2*pi*dx) with the
// addition theorems.  Each image's quotients are formed from one reciprocal
// r = 1 / (ch - c) (f_l = dx2pi (ch c - 1) r^2 pi and its x-derivative from r^2
// and r^3), the field and its derivative share those reciprocals, and the
// translation unit that includes this file contracts product-adds.  The result
// is within a few ulps of the exact-order form: the mixed form's accuracy bar
// (positions per step against the FP64 form) has room for it, the plain form's
// bit parity does not, so only the mixed form's sweeps use it.  The Taylor
// branches near the pair's own origin stay those of d4::f64.
#pragma once

#include "d4_field64.cuh"

namespace d4 {
namespace f64fast {

using f64::cos2piy;
using f64::exp2pix;
using f64::kPi;
using f64::normalize;
using f64::weight;
using f64::weight_inv;

constexpr double k2Pi2 = 2 * f64::kPi * f64::kPi;

// cosh/sinh of 2*pi*(dx +- i) from e = exp(2*pi*dx) and one reciprocal.
struct Hyp {
    double ch0, sh0, chp1, chm1, shp1, shm1, chp2, chm2, shp2, shm2;
    double chp3, chm3, chp4, chm4, chp5, chm5;
    __device__ __forceinline__ explicit Hyp(double e) {
        const double inv = 1 / e;
        const double s = (e + inv) * 0.5, d = (e - inv) * 0.5;
        ch0 = s;
        sh0 = d;
        chp1 = s * f64::kCosh2Pi + d * f64::kSinh2Pi;
        chm1 = s * f64::kCosh2Pi - d * f64::kSinh2Pi;
        shp1 = d * f64::kCosh2Pi + s * f64::kSinh2Pi;
        shm1 = d * f64::kCosh2Pi - s * f64::kSinh2Pi;
        chp2 = s * f64::kCosh4Pi + d * f64::kSinh4Pi;
        chm2 = s * f64::kCosh4Pi - d * f64::kSinh4Pi;
        shp2 = d * f64::kCosh4Pi + s * f64::kSinh4Pi;
        shm2 = d * f64::kCosh4Pi - s * f64::kSinh4Pi;
        chp3 = f64::kCosh6Pi * e;
        chm3 = f64::kCosh6Pi * inv;
        chp4 = f64::kCosh8Pi * e;
        chm4 = f64::kCosh8Pi * inv;
        chp5 = f64::kCoshTPi * e;
        chm5 = f64::kCoshTPi * inv;
    }
};

// One image: f_l and, when wanted, f_dx_l (sh = ch for |i| >= 3), from r = 1/q.
__device__ __forceinline__ double f_l(double dx, double c, double ch) {
    const double r = 1 / (ch - c);
    return (2 * kPi * kPi) * dx * (ch * c - 1) * (r * r);
}

__device__ __forceinline__ double f_dx_l(double dx, double c, double ch, double sh) {
    const double r = 1 / (ch - c);
    const double r2 = r * r;
    const double n1 = ch * c - 1;
    return (n1 * r2 + (2 * kPi) * dx * (sh * c * r2 - 2 * n1 * sh * (r2 * r))) * k2Pi2;
}

__device__ __forceinline__ double f_0(double dx, double c, double dy, double ch) {
    if (dx * dx + dy * dy > 1e-6) return f_l(dx, c, ch);
    return f64::f_0(dx, c, dy, ch);
}

__device__ __forceinline__ double f_dx_0(double dx, double c, double dy, double ch, double sh) {
    if (dx * dx + dy * dy > 1e-6) return f_dx_l(dx, c, ch, sh);
    return f64::f_dx_0(dx, c, dy, ch, sh);
}

// Field::xy and Field::xy_diff_x (4-arg) over the same images and blends as
// d4::f64::xy / xy_diff_x.
__device__ __forceinline__ double xy(double dx, double dy, const Hyp &h, double c) {
    const double g3 = f_l(dx + 3, c, h.chp3) + f_l(dx - 3, c, h.chm3) + f_l(dx + 2, c, h.chp2) +
                      f_l(dx - 2, c, h.chm2) + f_l(dx + 1, c, h.chp1) + f_l(dx - 1, c, h.chm1) +
                      f_0(dx, c, dy, h.ch0);
    if (dx < 0)
        return f_l(dx + 5, c, h.chp5) * (0 - dx) + f_l(dx - 4, c, h.chm4) * (1 + dx) +
               f_l(dx + 4, c, h.chp4) + g3;
    return f_l(dx - 5, c, h.chm5) * dx + f_l(dx + 4, c, h.chp4) * (1 - dx) +
           f_l(dx - 4, c, h.chm4) + g3;
}

__device__ __forceinline__ double xy_diff_x(double dx, double dy, const Hyp &h, double c) {
    const double g3 = f_dx_0(dx, c, dy, h.ch0, h.sh0) + f_dx_l(dx + 1, c, h.chp1, h.shp1) +
                      f_dx_l(dx - 1, c, h.chm1, h.shm1) + f_dx_l(dx + 2, c, h.chp2, h.shp2) +
                      f_dx_l(dx - 2, c, h.chm2, h.shm2) + f_dx_l(dx + 3, c, h.chp3, h.chp3) +
                      f_dx_l(dx - 3, c, h.chm3, h.chm3);
    if (dx < 0)
        return f_dx_l(dx + 5, c, h.chp5, h.chp5) * (0 - dx) - f_l(dx + 5, c, h.chp5) +
               f_dx_l(dx - 4, c, h.chm4, h.chm4) * (1 + dx) + f_l(dx - 4, c, h.chm4) +
               f_dx_l(dx + 4, c, h.chp4, h.chp4) + g3;
    return f_dx_l(dx - 5, c, h.chm5, h.chm5) * dx + f_l(dx - 5, c, h.chm5) +
           f_dx_l(dx + 4, c, h.chp4, h.chp4) * (1 - dx) - f_l(dx + 4, c, h.chp4) +
           f_dx_l(dx - 4, c, h.chm4, h.chm4) + g3;
}

}  // namespace f64fast
}  // namespace d4
