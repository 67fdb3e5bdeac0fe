// d4_table.cu: construction of the tabulated field (d4_table.cuh) on the device.
//
// One thread per node.  The remainder after the free-space core is formed
// without cancellation in the near field: the central wall term f_0 / f_dx_0
// (src/Fields/Field.cpp:172-250) is evaluated from half-angle forms,
//     cosh X - cos Y  = 2 (sinh^2(X/2) + sin^2(Y/2)),
//     cosh X cos Y - 1 = 2 (sinh^2(X/2) - sin^2(Y/2) - 2 sinh^2(X/2) sin^2(Y/2)),
// (X = 2 pi dx, Y = 2 pi dy) before the core is subtracted, and the other
// images and the blended outer images are the reference's terms
// (Field.cpp:191-206,253-330).  The wall sum f_0 equals the sum over k of the
// free-space field at (dx, dy + k), so at the origin node the remainder of f_0
// is 0 and that of f_dx_0 is sum_{k != 0} (-k^4 / k^6) = -pi^2 / 3.
#include "d4_field64.cuh"
#include "d4_internal.h"
#include "d4_table.cuh"

namespace d4 {
namespace {

using namespace f64;

__global__ void k_table_build(int T, int W, double2 *t) {
    const int ix = blockIdx.x * blockDim.x + threadIdx.x;
    const int iy = blockIdx.y;
    if (ix >= W || iy >= W) return;
    const double dx = -0.5 + (double)(ix - tab::kGuard) / T;
    const double dy = -0.5 + (double)(iy - tab::kGuard) / T;
    // the images i != 0 and the blends, in the reference's expressions
    const Hyp h(exp2pix(dx));
    const double c = cos2piy(dy);
    double rxy = f_l(dx + 3, c, h.chp3) + f_l(dx - 3, c, h.chm3) + f_l(dx + 2, c, h.chp2) +
                 f_l(dx - 2, c, h.chm2) + f_l(dx + 1, c, h.chp1) + f_l(dx - 1, c, h.chm1);
    double rdx = f_dx_l(dx + 1, c, h.chp1, h.shp1) + f_dx_l(dx - 1, c, h.chm1, h.shm1) +
                 f_dx_l(dx + 2, c, h.chp2, h.shp2) + f_dx_l(dx - 2, c, h.chm2, h.shm2) +
                 f_dx_l(dx + 3, c, h.chp3, h.chp3) + f_dx_l(dx - 3, c, h.chm3, h.chm3);
    if (dx < 0) {
        rxy += f_l(dx + 5, c, h.chp5) * (0 - dx) + f_l(dx - 4, c, h.chm4) * (1 + dx) +
               f_l(dx + 4, c, h.chp4);
        rdx += f_dx_l(dx + 5, c, h.chp5, h.chp5) * (0 - dx) - f_l(dx + 5, c, h.chp5) +
               f_dx_l(dx - 4, c, h.chm4, h.chm4) * (1 + dx) + f_l(dx - 4, c, h.chm4) +
               f_dx_l(dx + 4, c, h.chp4, h.chp4);
    } else {
        rxy += f_l(dx - 5, c, h.chm5) * dx + f_l(dx + 4, c, h.chp4) * (1 - dx) +
               f_l(dx - 4, c, h.chm4);
        rdx += f_dx_l(dx - 5, c, h.chm5, h.chm5) * dx + f_l(dx - 5, c, h.chm5) +
               f_dx_l(dx + 4, c, h.chp4, h.chp4) * (1 - dx) - f_l(dx + 4, c, h.chp4) +
               f_dx_l(dx - 4, c, h.chm4, h.chm4);
    }
    // central wall minus the free-space core
    double w0 = 0, w0x = -kPi * kPi / 3;
    if (dx != 0 || dy != 0) {
        const double X = 2 * kPi * dx, Y = 2 * kPi * dy;
        const double sh2 = sinh(X / 2), sn2 = sin(Y / 2);
        const double s2 = sh2 * sh2, t2 = sn2 * sn2;
        const double q = 2 * (s2 + t2);
        const double n1 = 2 * (s2 - t2 - 2 * s2 * t2);
        const double cy = 1 - 2 * t2;
        const double shx = 2 * sh2 * cosh(X / 2);
        const double q2 = q * q;
        const double f0 = kPi * X * n1 / q2;
        const double f0x = (n1 / q2 + X * (shx * cy / q2 - 2 * n1 * shx / (q2 * q))) * 2 * kPi * kPi;
        const double x2 = dx * dx, y2 = dy * dy, r2 = x2 + y2;
        w0 = f0 - dx * (x2 - y2) / (r2 * r2);
        w0x = f0x - (6 * x2 * y2 - x2 * x2 - y2 * y2) / (r2 * r2 * r2);
    }
    t[(size_t)iy * W + ix] = make_double2(rxy + w0, rdx + w0x);
}

}  // namespace

void table_build(Ctx &c) {
    const int T = c.tab_T, W = T + 1 + 2 * tab::kGuard;
    D4_CUDA_OK(d4::dmalloc((void **)&c.tab, sizeof(double2) * (size_t)W * W));
    k_table_build<<<dim3((W + 127) / 128, W), 128, 0, c.stream>>>(T, W, c.tab);
    check_launch("k_table_build");
}

}  // namespace d4
