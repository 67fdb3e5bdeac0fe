// d4_table.cuh: the tabulated field, device evaluation.
//
// The reference's Python binding loads a tabulated periodic field
// (PeriodicShearStressELTE: loadStress(pwd, "xy", 1024) and
// loadStress(pwd, "xy_diff_x", 1024), python/src/periodic_shear_stress_ELTE_wrapper.cpp:43-44)
// whose generator and file format are not part of the reference.  This engine
// builds its own tables, on the device, from the FP64 field of
// src/Fields/Field.cpp:172-346.  Interpolating that field directly would fail
// next to the pair singularity (sigma ~ 1/r at the origin), so each node holds
// the smooth remainder after the free-space core of one edge dislocation,
//     sigma_0(x, y)   = x (x^2 - y^2) / (x^2 + y^2)^2
//     sigma_0,x(x, y) = (-x^4 + 6 x^2 y^2 - y^4) / (x^2 + y^2)^3,
// (the r -> 0 limit of f_0 and f_dx_0, Field.cpp:172-250), i.e.
//     R(x, y) = Field::xy(x, y) - sigma_0,   R_x(x, y) = Field::xy_diff_x(x, y) - sigma_0,x,
// interleaved as double2 {R, R_x}.  The grid spans [-0.5, 0.5] in both
// coordinates with T intervals (spacing 1/T) plus kGuard nodes beyond each edge,
// row-major in y: node (ix, iy) at (-0.5 + (ix - kGuard)/T, -0.5 + (iy - kGuard)/T).
// Evaluation is tensor-product four-point Lagrange (bicubic) interpolation of
// R and R_x over the 4 x 4 nodes around the point, plus the analytic core.
// The Lagrange cubic's error is (h^4 / 24) |d^4 R| times a node factor <= 9/16
// per direction; R's nearest singularities (the periodic images) are >= 0.5
// away, so at T = 1024 the interpolation error is ~1e-11 of the field scale.
#pragma once

namespace d4 {
namespace tab {

constexpr int kGuard = 2;

struct Table {
    const double2 *t;  // W x W nodes {R, R_x}, W = T + 1 + 2 kGuard
    int T;
    int W;
};

// Four-point Lagrange weights for nodes -1, 0, 1, 2 at offset s in [0, 1).
__device__ __forceinline__ void lagrange4(double s, double w[4]) {
    const double sm1 = s - 1, sm2 = s - 2, sp1 = s + 1;
    w[0] = -s * sm1 * sm2 / 6;
    w[1] = sp1 * sm1 * sm2 / 2;
    w[2] = -sp1 * s * sm2 / 2;
    w[3] = sp1 * s * sm1 / 6;
}

// {Field::xy, Field::xy_diff_x} at (dx, dy) in [-0.5, 0.5)^2 from the table.
// With kDiff false only the first component is formed.
template <bool kDiff>
__device__ __forceinline__ double2 eval(const Table &tb, double dx, double dy) {
    const double u = (dx + 0.5) * tb.T + kGuard;
    const double v = (dy + 0.5) * tb.T + kGuard;
    int iu = (int)floor(u), iv = (int)floor(v);
    // dx, dy in [-0.5, 0.5) give iu, iv in [kGuard, kGuard + T - 1]; clamp anyway
    iu = min(max(iu, 1), tb.W - 3);
    iv = min(max(iv, 1), tb.W - 3);
    double wu[4], wv[4];
    lagrange4(u - iu, wu);
    lagrange4(v - iv, wv);
    double r = 0, rx = 0;
    const double2 *row = tb.t + (size_t)(iv - 1) * tb.W + (iu - 1);
#pragma unroll
    for (int b = 0; b < 4; ++b) {
        double sr = 0, sx = 0;
#pragma unroll
        for (int a = 0; a < 4; ++a) {
            const double2 e = __ldg(row + a);
            sr += wu[a] * e.x;
            if (kDiff) sx += wu[a] * e.y;
        }
        r += wv[b] * sr;
        if (kDiff) rx += wv[b] * sx;
        row += tb.W;
    }
    const double x2 = dx * dx, y2 = dy * dy, r2 = x2 + y2;
    const double inv = 1 / r2;
    double2 out;
    out.x = r + dx * (x2 - y2) * inv * inv;
    out.y = kDiff ? rx + (6 * x2 * y2 - x2 * x2 - y2 * y2) * inv * inv * inv : 0.0;
    return out;
}

}  // namespace tab
}  // namespace d4
