/*
 * d4_oracle.c: plain-C restatement of the 2D4_sim implicit-step hot path.
 *
 * TEST INFRASTRUCTURE ONLY (see d4_oracle.h).  It is the checker the CUDA
 * product is compared with; nothing in the product calls it.
 *
 * The expressions keep the reference's floating-point operation order (the
 * order C evaluates the reference's source in), because the tests pin this
 * file bit for bit against the reference core built with the same flags.
 */
#define _GNU_SOURCE
#include "d4_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#ifndef M_PI
#define M_PI 3.14159265358979323846
#endif

/* Constants of include/constants.h:40-65 (cosh/sinh of multiples of pi and
 * 2*pi/ln 2), written as the same decimal literals so they round to the same
 * doubles. */
#define D4O_PI2LN2INV 9.0647202836543876192553658914333336203437229354476
#define D4O_COSH2PI 267.746761483748222245931879901
#define D4O_COSH4PI 143375.656570070321051450310133
#define D4O_COSH6PI 7.67764676977233502175191858009e7
#define D4O_COSH8PI 4.11131577927974976374895337541e10
#define D4O_COSHTPI 2.20157529303160145057002722946e13
#define D4O_SINH2PI 267.744894041016514257117449688
#define D4O_SINH4PI 143375.656566582978695241314640

/* ---------------------------------------------------------------- field -- */

/* Taylor branch shared by f_0 (src/Fields/Field.cpp:183-187). */
static double taylor_f0(double dx2pi, double dy2pi) {
    double cosh2pixminus1 = pow(dx2pi, 6) / 720 + pow(dx2pi, 4) / 24 + pow(dx2pi, 2) * 0.5;
    double cos2piyminus1 = -pow(dy2pi, 6) / 720 + pow(dy2pi, 4) / 24 - pow(dy2pi, 2) * 0.5;
    double coshminuscos = (pow(dy2pi, 6) + pow(dx2pi, 6)) / 720 +
                          (pow(dx2pi, 4) - pow(dy2pi, 4)) / 24 +
                          (pow(dx2pi, 2) + pow(dy2pi, 2)) * 0.5;
    return ((cosh2pixminus1 * cos2piyminus1 + cos2piyminus1 + cosh2pixminus1) * dx2pi) /
           pow(coshminuscos, 2) * M_PI;
}

/* f_0, src/Fields/Field.cpp:172-188: wall through the own cell. */
static double f_0(double dx, double cos2piy, double dy, double cosh2pix) {
    double dx2pi = M_PI * 2 * dx;
    if (dx * dx + dy * dy > 1e-6) {
        double coshpixyd = cosh2pix - cos2piy;
        return dx2pi * (cosh2pix * cos2piy - 1) / pow(coshpixyd, 2) * M_PI;
    }
    double dy2pi = M_PI * 2 * dy;
    return taylor_f0(dx2pi, dy2pi);
}

/* f_l, src/Fields/Field.cpp:191-196: image wall at distance >= 1. */
static double f_l(double dx, double cos2piy, double cosh2pix) {
    double dx2pi = M_PI * 2 * dx;
    double coshpixyd = cosh2pix - cos2piy;
    return dx2pi * (cosh2pix * cos2piy - 1) / pow(coshpixyd, 2) * M_PI;
}

/* Hyperbolic values of 2*pi*(dx +- i) from e = exp(2*pi*dx)
 * (include/constants.h:67-79). */
#define CH_X(e) (((e) + 1 / (e)) / 2)
#define CH_XP1(e) ((((e) + 1 / (e)) * D4O_COSH2PI + ((e) - 1 / (e)) * D4O_SINH2PI) / 2)
#define CH_XM1(e) ((((e) + 1 / (e)) * D4O_COSH2PI - ((e) - 1 / (e)) * D4O_SINH2PI) / 2)
#define CH_XP2(e) ((((e) + 1 / (e)) * D4O_COSH4PI + ((e) - 1 / (e)) * D4O_SINH4PI) / 2)
#define CH_XM2(e) ((((e) + 1 / (e)) * D4O_COSH4PI - ((e) - 1 / (e)) * D4O_SINH4PI) / 2)
#define CH_XP3(e) (D4O_COSH6PI * (e))
#define CH_XM3(e) (D4O_COSH6PI / (e))
#define CH_XP4(e) (D4O_COSH8PI * (e))
#define CH_XM4(e) (D4O_COSH8PI / (e))
#define CH_XP5(e) (D4O_COSHTPI * (e))
#define CH_XM5(e) (D4O_COSHTPI / (e))
#define SH_X(e) (((e) - 1 / (e)) / 2)
#define SH_XP1(e) ((((e) - 1 / (e)) * D4O_COSH2PI + ((e) + 1 / (e)) * D4O_SINH2PI) / 2)
#define SH_XM1(e) ((((e) - 1 / (e)) * D4O_COSH2PI - ((e) + 1 / (e)) * D4O_SINH2PI) / 2)
#define SH_XP2(e) ((((e) - 1 / (e)) * D4O_COSH4PI + ((e) + 1 / (e)) * D4O_SINH4PI) / 2)
#define SH_XM2(e) ((((e) - 1 / (e)) * D4O_COSH4PI - ((e) + 1 / (e)) * D4O_SINH4PI) / 2)

/* g3, src/Fields/Field.cpp:199-206: images -3..3. */
static double g3(double dx, double cos2piy, double dy, double e) {
    return f_l(dx + 3, cos2piy, CH_XP3(e)) + f_l(dx - 3, cos2piy, CH_XM3(e)) +
           f_l(dx + 2, cos2piy, CH_XP2(e)) + f_l(dx - 2, cos2piy, CH_XM2(e)) +
           f_l(dx + 1, cos2piy, CH_XP1(e)) + f_l(dx - 1, cos2piy, CH_XM1(e)) +
           f_0(dx + 0, cos2piy, dy, CH_X(e));
}

/* f_dx_0, src/Fields/Field.cpp:209-250. */
static double f_dx_0(double dx, double cos2piy, double dy, double cosh2pix, double sinh2pix) {
    double dx2pi = dx * 2 * M_PI;
    if (dx * dx + dy * dy > 1e-6) {
        double coshpixyd = cosh2pix - cos2piy;
        return ((cosh2pix * cos2piy - 1) / pow(coshpixyd, 2) +
                dx2pi * (sinh2pix * cos2piy / pow(coshpixyd, 2) -
                         (cosh2pix * cos2piy - 1) / pow(coshpixyd, 3) * 2 * sinh2pix)) *
               M_PI * 2 * M_PI;
    }
    double dy2pi = dy * M_PI * 2;
    double cosh2pixminus1 = pow(dx2pi, 6) / 720 + pow(dx2pi, 4) / 24 + pow(dx2pi, 2) * 0.5;
    double cos2piyminus1 = -pow(dy2pi, 6) / 720 + pow(dy2pi, 4) / 24 - pow(dy2pi, 2) * 0.5;
    double coshminuscos = (pow(dy2pi, 6) + pow(dx2pi, 6)) / 720 +
                          (pow(dx2pi, 4) - pow(dy2pi, 4)) / 24 +
                          (pow(dx2pi, 2) + pow(dy2pi, 2)) * 0.5;
    double cosysinhx = -(pow(dx2pi, 7) * pow(dy2pi, 6)) / 3628800 -
                       (pow(dx2pi, 5) * pow(dy2pi, 6)) / 86400 -
                       (pow(dx2pi, 3) * pow(dy2pi, 6)) / 4320 - (pow(dy2pi, 6) * dx2pi) / 720 +
                       (pow(dx2pi, 7) * pow(dy2pi, 4)) / 120960 +
                       (pow(dx2pi, 5) * pow(dy2pi, 4)) / 2880 +
                       (pow(dx2pi, 3) * pow(dy2pi, 4)) / 144 + (pow(dy2pi, 4) * dx2pi) / 24 -
                       (pow(dx2pi, 7) * pow(dy2pi, 2)) / 1080 -
                       (pow(dx2pi, 5) * pow(dy2pi, 2)) / 240 -
                       (pow(dx2pi, 3) * pow(dy2pi, 2)) / 12 - (pow(dy2pi, 2) * dx2pi) * 0.5 +
                       pow(dx2pi, 7) / 5040 + pow(dx2pi, 5) / 120 + pow(dx2pi, 3) / 6 + dx2pi;
    return ((cosh2pixminus1 * cos2piyminus1 + cos2piyminus1 + cosh2pixminus1) /
                pow(coshminuscos, 2) +
            ((cosysinhx * dx) / pow(coshminuscos, 2) -
             (cosh2pixminus1 * cos2piyminus1 + cos2piyminus1 + cosh2pixminus1) /
                 pow(coshminuscos, 3) * dx * sinh(dx2pi) * 2) *
                2 * M_PI) *
           M_PI * 2 * M_PI;
}

/* f_dx_l, src/Fields/Field.cpp:253-266. */
static double f_dx_l(double dx, double cos2piy, double cosh2pix, double sinh2pix) {
    double dx2pi = dx * 2 * M_PI;
    double chx_cy = cosh2pix - cos2piy;
    double chxcy_1 = cosh2pix * cos2piy - 1;
    return (chxcy_1 / pow(chx_cy, 2) +
            dx2pi * (sinh2pix * cos2piy / pow(chx_cy, 2) - chxcy_1 / pow(chx_cy, 3) * 2 * sinh2pix)) *
           M_PI * 2 * M_PI;
}

/* f_dx_h, src/Fields/Field.cpp:269-282: sinh taken equal to cosh. */
static double f_dx_h(double dx, double cos2piy, double coshsinh2pix) {
    double dx2pi = dx * 2 * M_PI;
    double chx_cy = coshsinh2pix - cos2piy;
    double chxcy_1 = coshsinh2pix * cos2piy - 1;
    return (chxcy_1 / pow(chx_cy, 2) +
            dx2pi * (coshsinh2pix * cos2piy / pow(chx_cy, 2) -
                     chxcy_1 / pow(chx_cy, 3) * 2 * coshsinh2pix)) *
           M_PI * 2 * M_PI;
}

/* g3_dx, src/Fields/Field.cpp:285-292. */
static double g3_dx(double dx, double cos2piy, double dy, double e) {
    return f_dx_0(dx + 0, cos2piy, dy, CH_X(e), SH_X(e)) +
           f_dx_l(dx + 1, cos2piy, CH_XP1(e), SH_XP1(e)) +
           f_dx_l(dx - 1, cos2piy, CH_XM1(e), SH_XM1(e)) +
           f_dx_l(dx + 2, cos2piy, CH_XP2(e), SH_XP2(e)) +
           f_dx_l(dx - 2, cos2piy, CH_XM2(e), SH_XM2(e)) + f_dx_h(dx + 3, cos2piy, CH_XP3(e)) +
           f_dx_h(dx - 3, cos2piy, CH_XM3(e));
}

/* Field::xy (4-arg), src/Fields/Field.cpp:295-311. */
double d4o_xy4(double dx, double dy, double e, double c) {
    if (dx < 0)
        return f_l(dx + 5, c, CH_XP5(e)) * (0 - dx) + f_l(dx - 4, c, CH_XM4(e)) * (1 + dx) +
               f_l(dx + 4, c, CH_XP4(e)) + g3(dx, c, dy, e);
    return f_l(dx - 5, c, CH_XM5(e)) * (0 + dx) + f_l(dx + 4, c, CH_XP4(e)) * (1 - dx) +
           f_l(dx - 4, c, CH_XM4(e)) + g3(dx, c, dy, e);
}

/* Field::xy_diff_x (4-arg), src/Fields/Field.cpp:314-330. */
double d4o_xy_diff_x4(double dx, double dy, double e, double c) {
    if (dx < 0)
        return f_dx_h(dx + 5, c, CH_XP5(e)) * (0 - dx) + f_l(dx + 5, c, CH_XP5(e)) * (-1) +
               f_dx_h(dx - 4, c, CH_XM4(e)) * (1 + dx) + f_l(dx - 4, c, CH_XM4(e)) * (+1) +
               f_dx_h(dx + 4, c, CH_XP4(e)) + g3_dx(dx, c, dy, e);
    return f_dx_h(dx - 5, c, CH_XM5(e)) * (0 + dx) + f_l(dx - 5, c, CH_XM5(e)) * (+1) +
           f_dx_h(dx + 4, c, CH_XP4(e)) * (1 - dx) + f_l(dx + 4, c, CH_XP4(e)) * (-1) +
           f_dx_h(dx - 4, c, CH_XM4(e)) + g3_dx(dx, c, dy, e);
}

/* Field::xy (2-arg), src/Fields/Field.cpp:333-338. */
double d4o_xy(double dx, double dy) {
    double e = exp2(D4O_PI2LN2INV * dx);
    double c = cos(M_PI * 2 * dy);
    return d4o_xy4(dx, dy, e, c);
}

/* Field::xy_diff_x (2-arg), src/Fields/Field.cpp:341-346 (uses exp, not exp2). */
double d4o_xy_diff_x(double dx, double dy) {
    double e = exp(M_PI * 2 * dx);
    double c = cos(M_PI * 2 * dy);
    return d4o_xy_diff_x4(dx, dy, e, c);
}

/* ------------------------------------------- IEEE variant of the field -- */
/* The reference's exact truncated image sum with cosh and sinh, compiled when
 * USE_IEEE_HYPERBOLIC is 1 (src/Fields/Field.cpp:26-168; the same expressions
 * as sandbox/ieee_hyperbolic/ieee_hyperbolic.cpp:11-140, which the tests
 * build as the pin).  Not on the reference's default path: the secondary
 * oracle of the field, against which the FP32 gradient's error is measured.
 * Every expression keeps the reference's operation order (pow for the integer
 * powers, as std::pow(double, int) does). */

/* f, src/Fields/Field.cpp:28-44: one wall image. */
static double ieee_f(double dx, double cos2piy, double dy) {
    if (dx * dx + dy * dy > 1e-6) {
        double cosh2pix = cosh(dx * 2 * M_PI);
        double coshpixyd = cosh2pix - cos2piy;
        return dx * (cosh2pix * cos2piy - 1) / pow(coshpixyd, 2) * 2 * M_PI * M_PI;
    }
    double dx2pi = dx * 2 * M_PI;
    double dy2pi = dy * 2 * M_PI;
    double cosh2pixminus1 = pow(dx2pi, 6) / 720 + pow(dx2pi, 4) / 24 + pow(dx2pi, 2) * 0.5;
    double cos2piyminus1 = -pow(dy2pi, 6) / 720 + pow(dy2pi, 4) / 24 - pow(dy2pi, 2) * 0.5;
    double coshminuscos = (pow(dy2pi, 6) + pow(dx2pi, 6)) / 720 +
                          (pow(dx2pi, 4) - pow(dy2pi, 4)) / 24 +
                          (pow(dx2pi, 2) + pow(dy2pi, 2)) * 0.5;
    return ((cosh2pixminus1 * cos2piyminus1 + cos2piyminus1 + cosh2pixminus1) * dx) /
           pow(coshminuscos, 2) * 2 * M_PI * M_PI;
}

/* g<images>, src/Fields/Field.cpp:47-58: g<0> = f(dx), then
 * g<k> = g<k-1> + f(dx - k) + f(dx + k). */
static double ieee_g(int images, double dx, double cos2piy, double dy) {
    double s = ieee_f(dx, cos2piy, dy);
    for (int k = 1; k <= images; ++k) {
        s = s + ieee_f(dx - k, cos2piy, dy);
        s = s + ieee_f(dx + k, cos2piy, dy);
    }
    return s;
}

/* f_dx, src/Fields/Field.cpp:61-105: x-derivative of one wall image. */
static double ieee_f_dx(double dx, double cos2piy, double dy) {
    double dx2pi = dx * 2 * M_PI;
    if (dx * dx + dy * dy > 1e-6) {
        double cosh2pix = cosh(dx2pi);
        double sinh2pix = sinh(dx2pi);
        double coshpixyd = cosh2pix - cos2piy;
        return ((cosh2pix * cos2piy - 1) / pow(coshpixyd, 2) +
                dx * (sinh2pix * cos2piy * 2 * M_PI / pow(coshpixyd, 2) -
                      (cosh2pix * cos2piy - 1) / pow(coshpixyd, 3) * 4 * M_PI * sinh2pix)) *
               M_PI * 2 * M_PI;
    }
    double dy2pi = dy * M_PI * 2;
    double cosh2pixminus1 = pow(dx2pi, 6) / 720 + pow(dx2pi, 4) / 24 + pow(dx2pi, 2) * 0.5;
    double cos2piyminus1 = -pow(dy2pi, 6) / 720 + pow(dy2pi, 4) / 24 - pow(dy2pi, 2) * 0.5;
    double coshminuscos = (pow(dy2pi, 6) + pow(dx2pi, 6)) / 720 +
                          (pow(dx2pi, 4) - pow(dy2pi, 4)) / 24 +
                          (pow(dx2pi, 2) + pow(dy2pi, 2)) * 0.5;
    double cosysinhx = -(pow(dx2pi, 7) * pow(dy2pi, 6)) / 3628800
                       - (pow(dx2pi, 5) * pow(dy2pi, 6)) / 86400
                       - (pow(dx2pi, 3) * pow(dy2pi, 6)) / 4320
                       - (pow(dy2pi, 6) * dx2pi) / 720
                       + (pow(dx2pi, 7) * pow(dy2pi, 4)) / 120960
                       + (pow(dx2pi, 5) * pow(dy2pi, 4)) / 2880
                       + (pow(dx2pi, 3) * pow(dy2pi, 4)) / 144
                       + (pow(dy2pi, 4) * dx2pi) / 24
                       - (pow(dx2pi, 7) * pow(dy2pi, 2)) / 1080
                       - (pow(dx2pi, 5) * pow(dy2pi, 2)) / 240
                       - (pow(dx2pi, 3) * pow(dy2pi, 2)) / 12
                       - (pow(dy2pi, 2) * dx2pi) * 0.5
                       + pow(dx2pi, 7) / 5040
                       + pow(dx2pi, 5) / 120
                       + pow(dx2pi, 3) / 6
                       + dx2pi;
    return ((cosh2pixminus1 * cos2piyminus1 + cos2piyminus1 + cosh2pixminus1) /
                pow(coshminuscos, 2) +
            ((cosysinhx * dx) / pow(coshminuscos, 2) -
             (cosh2pixminus1 * cos2piyminus1 + cos2piyminus1 + cosh2pixminus1) /
                 pow(coshminuscos, 3) * dx * sinh(dx2pi) * 2) *
                2 * M_PI) *
           M_PI * 2 * M_PI;
}

/* g_dx<images>, src/Fields/Field.cpp:108-119. */
static double ieee_g_dx(int images, double dx, double cos2piy, double dy) {
    double s = ieee_f_dx(dx, cos2piy, dy);
    for (int k = 1; k <= images; ++k) {
        s = s + ieee_f_dx(dx - k, cos2piy, dy);
        s = s + ieee_f_dx(dx + k, cos2piy, dy);
    }
    return s;
}

#define D4O_FIELD_N 4 /* ANALYTIC_FIELD_N, include/constants.h */

/* Field::xy (IEEE), src/Fields/Field.cpp:122-137. */
double d4o_ieee_xy(double dx, double dy) {
    double cos2piy = cos(M_PI * 2 * dy);
    if (dx < 0)
        return -dx * ieee_f(dx + D4O_FIELD_N + 1, cos2piy, dy) +
               (1 + dx) * ieee_f(dx - D4O_FIELD_N, cos2piy, dy) +
               ieee_f(dx + D4O_FIELD_N, cos2piy, dy) +
               ieee_g(D4O_FIELD_N - 1, dx, cos2piy, dy);
    return dx * ieee_f(dx - D4O_FIELD_N - 1, cos2piy, dy) +
           (1 - dx) * ieee_f(dx + D4O_FIELD_N, cos2piy, dy) +
           ieee_f(dx - D4O_FIELD_N, cos2piy, dy) + ieee_g(D4O_FIELD_N - 1, dx, cos2piy, dy);
}

/* Field::xy_diff_x (IEEE), src/Fields/Field.cpp:146-164. */
double d4o_ieee_xy_diff_x(double dx, double dy) {
    double cos2piy = cos(M_PI * 2 * dy);
    if (dx < 0)
        return -ieee_f(dx + D4O_FIELD_N + 1, cos2piy, dy) -
               dx * ieee_f_dx(dx + D4O_FIELD_N + 1, cos2piy, dy) +
               ieee_f_dx(dx - D4O_FIELD_N, cos2piy, dy) * (1 + dx) +
               ieee_f(dx - D4O_FIELD_N, cos2piy, dy) +
               ieee_f_dx(dx + D4O_FIELD_N, cos2piy, dy) +
               ieee_g_dx(D4O_FIELD_N - 1, dx, cos2piy, dy);
    return ieee_f(dx - D4O_FIELD_N - 1, cos2piy, dy) +
           dx * ieee_f_dx(dx - D4O_FIELD_N - 1, cos2piy, dy) +
           ieee_f_dx(dx + D4O_FIELD_N, cos2piy, dy) * (1 - dx) -
           ieee_f(dx + D4O_FIELD_N, cos2piy, dy) +
           ieee_f_dx(dx - D4O_FIELD_N, cos2piy, dy) +
           ieee_g_dx(D4O_FIELD_N - 1, dx, cos2piy, dy);
}

/* ------------------------------------------------------------ utilities -- */

/* normalize, src/sim_utils.cpp:6-13. */
double d4o_normalize(double n) {
    while (n < -0.5) n += 1;
    while (n >= 0.5) n -= 1;
    return n;
}

/* weight, src/sim_utils.cpp:36-55. */
double d4o_weight(double s, char t) {
    if (s > 0) {
        if (t == 'c') return pow(s / (s + 1), 2);
        if (t == 'p') return s / (s + 1);
        if (t == 'm') {
            double c = 0.412073;
            return 1 / (1 + 1.5 / (s + c * s * s));
        }
    }
    return 0;
}

/* weightInv, src/sim_utils.cpp:57-75. */
double d4o_weight_inv(double w, char t) {
    if (w > 0) {
        if (t == 'c') return sqrt(w) / (1 - sqrt(w));
        if (t == 'p') return w / (1 - w);
        if (t == 'm') {
            double c = 0.412073;
            return (1 - w - sqrt(1 - 2 * w + 6 * c * w + w * w - 6 * c * w * w)) / (2 * (-c + c * w));
        }
    }
    return 0;
}

/* StressProtocol family, src/stress_protocol.cpp:13-73. */
double d4o_ext_stress(const d4o_protocol *p, double t) {
    switch (p->kind) {
    case 1:
        return t * p->rate + p->tau0;
    case 2:
    case 3: {
        double periodic = t - floor((t / p->period + 1. / 4)) * p->period;
        double stress = p->rate * periodic + p->tau0;
        if (periodic > p->period / 4) stress = p->rate * p->period / 2 - stress + p->tau0;
        if (p->kind == 3) return stress * p->amp_rate * t;
        return stress;
    }
    default:
        return 0;
    }
}

static int b_of(int i, int n) { return i < n / 2 ? 1 : -1; } /* simulation_data.cpp:265-270 */

static void update_tol(double *tol, double min_prec_sq, double d, int id) {
    /* PrecisionHandler::updateTolerance, src/precision_handler.cpp:34-38 */
    if (tol && d < min_prec_sq && d < tol[id]) tol[id] = d;
}

typedef struct {
    double key;
    int id;
} sort_item;

static int cmp_desc(const void *a, const void *b) {
    const sort_item *l = (const sort_item *)a, *r = (const sort_item *)b;
    if (l->key > r->key) return -1;
    if (l->key < r->key) return 1;
    return (l->id > r->id) - (l->id < r->id);
}

/* readDislocationDataFromFile ordering, src/simulation_data.cpp:86-123. */
int d4o_sort(int n, const double *x, const double *y, const double *b, double *xs, double *ys,
             int *order) {
    double sum_b = 0;
    sort_item *it = (sort_item *)malloc(sizeof(sort_item) * (size_t)(n > 0 ? n : 1));
    for (int i = 0; i < n; ++i) {
        if (fabs(b[i] - rint(b[i])) > 1e-5) {
            free(it);
            return -1;
        }
        sum_b += b[i];
        it[i].key = y[i] + b[i];
        it[i].id = i;
    }
    if (sum_b != 0) {
        free(it);
        return -1;
    }
    qsort(it, (size_t)n, sizeof(sort_item), cmp_desc);
    for (int i = 0; i < n; ++i) {
        xs[i] = x[it[i].id];
        ys[i] = y[it[i].id];
        order[it[i].id] = i;
    }
    free(it);
    return 0;
}

/* --------------------------------------------------------------- sweeps -- */

/* Simulation::calculateSpeedsAtTime, src/simulation.cpp:287-333. */
void d4o_speeds(int n, const double *x, const double *y, double ext, double *v, double *tol,
                double min_prec_sq) {
    for (int i = 0; i < n; ++i) v[i] = 0;
    for (int i = 0; i < n; ++i) {
        for (int j = i + 1; j < n; ++j) {
            double dx = d4o_normalize(x[i] - x[j]);
            double dy = d4o_normalize(y[i] - y[j]);
            double dist_sq = dx * dx + dy * dy;
            update_tol(tol, min_prec_sq, dist_sq, i);
            update_tol(tol, min_prec_sq, dist_sq, j);
            double force = d4o_xy(dx, dy) * b_of(i, n) * b_of(j, n);
            v[i] += force;
            v[j] -= force;
        }
        v[i] += ext * b_of(i, n);
    }
}

/* Simulation::calcJacobianAndSpeedsAtTimes, src/simulation.cpp:345-527, with
 * the CSC matrix expanded to dense row-major a (entries outside the cutoff
 * range are 0, as they are absent from the CSC pattern). */
void d4o_jacobian(int n, const double *x, const double *y, double stepsize, double ext_a,
                  double ext_b, double cutoff_sq, double cutoff, int heaviside, char weight_fn,
                  double *v_a, double *v_b, double *a, double *dvec, double *tol,
                  double min_prec_sq) {
    const double range_sq = heaviside ? 1 : 49;
    /* present[i*n+j]: the (i,j) entry is in the sparse pattern */
    unsigned char *present = (unsigned char *)calloc((size_t)n * n + 1, 1);
    memset(a, 0, sizeof(double) * (size_t)n * n);
    for (int i = 0; i < n; ++i) {
        v_a[i] = 0;
        v_b[i] = 0;
    }
    for (int i = 0; i < n; ++i) {
        double sub_sum = 0;
        /* previously computed part: column j < i holds row i (mirror copy) */
        for (int j = 0; j < i; ++j) {
            double v = present[(size_t)i * n + j] ? a[(size_t)i * n + j] : 0;
            if (v != 0) sub_sum -= v;
        }
        for (int j = i + 1; j < n; ++j) {
            double dx = d4o_normalize(x[i] - x[j]);
            double dy = d4o_normalize(y[i] - y[j]);
            double dist_sq = dx * dx + dy * dy;
            update_tol(tol, min_prec_sq, dist_sq, i);
            update_tol(tol, min_prec_sq, dist_sq, j);
            double e = exp2(D4O_PI2LN2INV * dx);
            double c = cos(2 * M_PI * dy);
            double force = d4o_xy4(dx, dy, e, c) * b_of(i, n) * b_of(j, n);
            if (dist_sq < range_sq * cutoff_sq) {
                double v = stepsize * b_of(j, n) * b_of(i, n) * d4o_xy_diff_x4(dx, dy, e, c);
                if (!heaviside && dist_sq > cutoff_sq)
                    v *= exp(-pow(sqrt(dist_sq) - cutoff, 2) * (1 / cutoff_sq));
                /* stored in column i, row j; the mirror (column j, row i) is
                 * read back when column j is built */
                a[(size_t)j * n + i] = v;
                a[(size_t)i * n + j] = v;
                present[(size_t)j * n + i] = 1;
                present[(size_t)i * n + j] = 1;
                sub_sum -= v;
            }
            v_a[i] += force;
            v_a[j] -= force;
        }
        v_b[i] = v_a[i] + ext_b * b_of(i, n);
        v_a[i] += ext_a * b_of(i, n);
        a[(size_t)i * n + i] = sub_sum;
        dvec[i] = d4o_weight(sub_sum, weight_fn);
    }
    for (int c = 0; c < n; ++c)
        for (int r = 0; r < n; ++r) {
            if (r == c || present[(size_t)r * n + c]) a[(size_t)r * n + c] *= (1 + dvec[r]) / 2;
            if (r == c) a[(size_t)r * n + c] += 1;
        }
    free(present);
}

/* Simulation::calcJacobianAndSpeedsFromPrev (matrix part),
 * src/simulation.cpp:552-595.  factor = (t_new - t_base) / (t_old - t_base). */
void d4o_jacobian_from_prev(int n, double *a, double *dvec, double factor, char weight_fn) {
    double *new_w = (double *)malloc(sizeof(double) * (size_t)(n > 0 ? n : 1));
    double *fac = (double *)malloc(sizeof(double) * (size_t)(n > 0 ? n : 1));
    for (int i = 0; i < n; ++i) {
        if (dvec[i] == 0)
            new_w[i] = 0.;
        else
            new_w[i] = d4o_weight(d4o_weight_inv(dvec[i], weight_fn) * factor, weight_fn);
    }
    for (int i = 0; i < n; ++i) fac[i] = (1 + new_w[i]) / (1 + dvec[i]);
    for (int r = 0; r < n; ++r) {
        double f = fac[r];
        for (int c = 0; c < n; ++c) {
            double *e = &a[(size_t)r * n + c];
            if (r == c)
                *e = 1 + (*e - 1) / 2 * f;
            else
                *e = *e / 2 * f;
        }
    }
    for (int i = 0; i < n; ++i) dvec[i] = new_w[i];
    free(new_w);
    free(fac);
}

/* ------------------------------------------------------------------- LU -- */

/* Same loops as the shim's native backend (oracle/shim/umfpack_shim.cpp). */
int d4o_lu(int n, double *a, int *piv) {
    int singular = 0;
    for (int k = 0; k < n; ++k) {
        int p = k;
        double amax = fabs(a[k + (size_t)k * n]);
        for (int i = k + 1; i < n; ++i) {
            double v = fabs(a[i + (size_t)k * n]);
            if (v > amax) {
                amax = v;
                p = i;
            }
        }
        piv[k] = p;
        if (a[p + (size_t)k * n] == 0.0) {
            singular = 1;
            continue;
        }
        if (p != k) {
            for (int j = 0; j < n; ++j) {
                double t = a[k + (size_t)j * n];
                a[k + (size_t)j * n] = a[p + (size_t)j * n];
                a[p + (size_t)j * n] = t;
            }
        }
        double d = a[k + (size_t)k * n];
        for (int i = k + 1; i < n; ++i) a[i + (size_t)k * n] /= d;
        for (int j = k + 1; j < n; ++j) {
            double t = a[k + (size_t)j * n];
            if (t != 0.0) {
                double *cj = a + (size_t)j * n;
                const double *ck = a + (size_t)k * n;
                for (int i = k + 1; i < n; ++i) cj[i] -= ck[i] * t;
            }
        }
    }
    return singular;
}

void d4o_lu_solve(int n, const double *a, const int *piv, double *x) {
    for (int k = 0; k < n; ++k) {
        int p = piv[k];
        if (p != k) {
            double t = x[k];
            x[k] = x[p];
            x[p] = t;
        }
    }
    for (int k = 0; k < n; ++k) {
        double t = x[k];
        if (t != 0.0) {
            const double *ck = a + (size_t)k * n;
            for (int i = k + 1; i < n; ++i) x[i] -= ck[i] * t;
        }
    }
    for (int k = n - 1; k >= 0; --k) {
        x[k] /= a[k + (size_t)k * n];
        double t = x[k];
        if (t != 0.0) {
            const double *ck = a + (size_t)k * n;
            for (int i = 0; i < k; ++i) x[i] -= ck[i] * t;
        }
    }
}

/* ----------------------------------------------------------- step / run -- */

typedef struct {
    int n;
    double *a, *lu, *g, *dx;
    int *piv;
    int singular;
} solver_t;

static void factor(solver_t *s) {
    int n = s->n;
    /* row-major a -> column-major lu */
    for (int r = 0; r < n; ++r)
        for (int c = 0; c < n; ++c) s->lu[r + (size_t)c * n] = s->a[(size_t)r * n + c];
    s->singular = d4o_lu(n, s->lu, s->piv);
}

/* Simulation::solveEQSys, src/simulation.cpp:643-659. */
static void solve(solver_t *s) {
    memcpy(s->dx, s->g, sizeof(double) * (size_t)s->n);
    d4o_lu_solve(s->n, s->lu, s->piv, s->dx);
    if (s->singular)
        for (int i = 0; i < s->n; ++i)
            if (!((-1 < s->dx[i]) && (s->dx[i] < 1))) s->dx[i] = 0;
}

typedef struct {
    const d4o_params *p;
    int n;
    int use_dipole;
    double min_prec_sq, dipole_prec_sq;
    double cutoff, cutoff_sq;
    double *tol;
    int selected_id; /* PrecisionHandler::selectedID: kept across reset() */
    double *init_speed, *init_speed2, *speed, *speed2, *dvec;
    solver_t s;
} ctx_t;

/* Simulation::calcGSolveAndUpdate, src/simulation.cpp:618-627. */
static void g_solve_update(ctx_t *c, double *new_x, const double *old_x, double h,
                           const double *end_speed, const double *init_speed) {
    for (int i = 0; i < c->n; ++i)
        c->s.g[i] = new_x[i] - old_x[i] -
                    h * ((1 + c->dvec[i]) * end_speed[i] + (1 - c->dvec[i]) * init_speed[i]) / 2;
    solve(&c->s);
    for (int i = 0; i < c->n; ++i) new_x[i] -= c->s.dx[i];
}

static void jac(ctx_t *c, const double *x, const double *y, double h, double *va, double *vb,
                double ta, double tb) {
    double ea = d4o_ext_stress(&c->p->protocol, ta);
    double eb = d4o_ext_stress(&c->p->protocol, tb);
    d4o_jacobian(c->n, x, y, h, ea, eb, c->cutoff_sq, c->cutoff, c->p->heaviside_cutoff,
                 c->p->weight_function, va, vb, c->s.a, c->dvec,
                 c->use_dipole ? c->tol : NULL, c->min_prec_sq);
    factor(&c->s);
}

static void speeds(ctx_t *c, const double *x, const double *y, double *v, double t) {
    d4o_speeds(c->n, x, y, d4o_ext_stress(&c->p->protocol, t), v, c->use_dipole ? c->tol : NULL,
               c->min_prec_sq);
}

/* Stages I-III of src/simulation.cpp:90-156 and calculateXError (:692-700). */
static void attempt(ctx_t *c, const double *x0, const double *y, double t0, double h,
                    double *xb, double *xh, double *x2, double *ratio, int *max_id) {
    const int n = c->n;
    double t_1__ = t0 + h;
    double t_1p2 = t0 + h / 2;
    /* stage I */
    jac(c, x0, y, h, c->init_speed, c->speed, t0, t_1__);
    for (int i = 0; i < n; ++i)
        c->s.g[i] = -h * ((1 + c->dvec[i]) * c->speed[i] + (1 - c->dvec[i]) * c->init_speed[i]) / 2;
    solve(&c->s);
    for (int i = 0; i < n; ++i) xb[i] = x0[i] - c->s.dx[i];
    speeds(c, xb, y, c->speed2, t_1__);
    g_solve_update(c, xb, x0, h, c->speed2, c->init_speed);
    /* stage II: calcJacobianAndSpeedsFromPrev(t0, t_1p2, t_1__) */
    {
        double factor_t = (t_1p2 - t0) / (t_1__ - t0);
        d4o_jacobian_from_prev(n, c->s.a, c->dvec, factor_t, c->p->weight_function);
        factor(&c->s);
        double dif = d4o_ext_stress(&c->p->protocol, t_1p2) - d4o_ext_stress(&c->p->protocol, t_1__);
        for (int i = 0; i < n; ++i) c->speed[i] += dif * b_of(i, n);
    }
    for (int i = 0; i < n; ++i)
        c->s.g[i] =
            -h / 2 * ((1 + c->dvec[i]) * c->speed[i] + (1 - c->dvec[i]) * c->init_speed[i]) / 2;
    solve(&c->s);
    for (int i = 0; i < n; ++i) xh[i] = x0[i] - c->s.dx[i];
    speeds(c, xh, y, c->speed2, t_1p2);
    g_solve_update(c, xh, x0, h / 2, c->speed2, c->init_speed);
    /* stage III */
    jac(c, xh, y, h / 2, c->init_speed2, c->speed2, t_1p2, t_1__);
    for (int i = 0; i < n; ++i)
        c->s.g[i] =
            -h / 2 * ((1 + c->dvec[i]) * c->speed2[i] + (1 - c->dvec[i]) * c->init_speed2[i]) / 2;
    solve(&c->s);
    for (int i = 0; i < n; ++i) x2[i] = xh[i] - c->s.dx[i];
    speeds(c, x2, y, c->speed2, t_1__);
    g_solve_update(c, x2, xh, h / 2, c->speed2, c->init_speed2);
    /* stage IV: calculateXError + PrecisionHandler::updateMaxErrorToleranceRatioSq */
    double max_r = 0;
    int sel = c->selected_id;
    for (int i = 0; i < n; ++i) {
        double e = fabs(xb[i] - x2[i]);
        double tmp = c->use_dipole ? e * e / c->tol[i] : e * e / c->min_prec_sq;
        if (tmp > max_r) {
            max_r = tmp;
            sel = i;
        }
    }
    *ratio = max_r / c->dipole_prec_sq;
    *max_id = sel;
    c->selected_id = sel;
}

static void ctx_init(ctx_t *c, int n, const d4o_params *p) {
    memset(c, 0, sizeof(*c));
    c->p = p;
    c->n = n;
    /* PrecisionHandler::setMinPrecisity then setDipolePrecisity
     * (src/precision_handler.cpp:65-89, called at src/simulation.cpp:24-26) */
    c->min_prec_sq = p->position_precision * p->position_precision;
    if (p->dipole_precision == 0) {
        c->use_dipole = 0;
        c->dipole_prec_sq = 1;
    } else {
        c->use_dipole = 1;
        c->dipole_prec_sq = p->dipole_precision * p->dipole_precision;
        c->min_prec_sq /= p->dipole_precision * p->dipole_precision;
    }
    /* SimulationData::updateCutOff, src/simulation_data.cpp:253-262 */
    double mult = p->cutoff_multiplier;
    if (!p->heaviside_cutoff && p->cutoff_multiplier >= sqrt(2 * (double)n) / 12) mult = 1e20;
    c->cutoff = mult / sqrt((double)n);
    c->cutoff_sq = c->cutoff * c->cutoff;
    size_t nn = (size_t)n > 0 ? (size_t)n : 1;
    c->tol = (double *)malloc(sizeof(double) * nn);
    for (int i = 0; i < n; ++i) c->tol[i] = c->min_prec_sq;
    c->init_speed = (double *)calloc(nn, sizeof(double));
    c->init_speed2 = (double *)calloc(nn, sizeof(double));
    c->speed = (double *)calloc(nn, sizeof(double));
    c->speed2 = (double *)calloc(nn, sizeof(double));
    c->dvec = (double *)calloc(nn, sizeof(double));
    c->s.n = n;
    c->s.a = (double *)calloc(nn * nn, sizeof(double));
    c->s.lu = (double *)calloc(nn * nn, sizeof(double));
    c->s.g = (double *)calloc(nn, sizeof(double));
    c->s.dx = (double *)calloc(nn, sizeof(double));
    c->s.piv = (int *)calloc(nn, sizeof(int));
}

static void ctx_free(ctx_t *c) {
    free(c->tol);
    free(c->init_speed);
    free(c->init_speed2);
    free(c->speed);
    free(c->speed2);
    free(c->dvec);
    free(c->s.a);
    free(c->s.lu);
    free(c->s.g);
    free(c->s.dx);
    free(c->s.piv);
}

void d4o_attempt_step(int n, const double *x0, const double *y, double t0, double h,
                      const d4o_params *p, double *x_big, double *x_half, double *x_two,
                      double *tol, double *ratio, int *max_id) {
    ctx_t c;
    ctx_init(&c, n, p);
    for (int i = 0; i < n; ++i) c.tol[i] = tol[i];
    attempt(&c, x0, y, t0, h, x_big, x_half, x_two, ratio, max_id);
    for (int i = 0; i < n; ++i) tol[i] = c.tol[i];
    ctx_free(&c);
}

void d4o_default_params(d4o_params *p) {
    memset(p, 0, sizeof(*p));
    p->position_precision = 1e-5;
    p->dipole_precision = 0.05;
    p->cutoff_multiplier = 1e20;
    p->initial_stepsize = 1e-6;
    p->max_stepsize = -1;
    p->weight_function = 'c';
    p->time_limit = -1;
    p->step_count_limit = -1;
    p->strain_increase_limit = -1;
    p->avalanche_limit = -1;
    p->avalanche_speed_threshold = 1e-3;
    p->sub_config_delay = 5;
    p->sub_config_delay_during_avalanche = 1;
    p->sub_config_times_type = 'a';
}

/* SimulationData::getNextWriteOutTime, src/simulation_data.cpp:231-246. */
static double next_write_out(const d4o_params *p, double sim_time) {
    if (p->sub_config_times == 0) return INFINITY;
    if (p->sub_config_times_type == 'a')
        return (double)((size_t)(sim_time / p->sub_config_times) + 1) * p->sub_config_times;
    if (p->sub_config_times_type == 'b') {
        double exponent =
            nextafter(log(sim_time / p->initial_stepsize) / log(p->sub_config_times), INFINITY);
        int next_exp = (int)exponent + 1;
        if (next_exp < 1) next_exp = 1;
        return p->initial_stepsize * pow(p->sub_config_times, next_exp);
    }
    return INFINITY;
}

static double absvalsq(const double *v, int n) {
    double s = 0;
    for (int i = 0; i < n; ++i) s = s + v[i] * v[i];
    return s;
}

/* Simulation::run, src/simulation.cpp:30-281 (log output and file writes
 * omitted; every quantity that feeds back into the state is kept). */
long long d4o_run(int n, double *x, double *y, const d4o_params *p, d4o_result *res,
                  d4o_attempt *rec, long long rec_cap) {
    ctx_t c;
    ctx_init(&c, n, p);
    size_t nn = (size_t)(n > 0 ? n : 1);
    double *xb = (double *)malloc(sizeof(double) * nn);
    double *xh = (double *)malloc(sizeof(double) * nn);
    double *x2 = (double *)malloc(sizeof(double) * nn);
    double sim_time = 0, h = p->initial_stepsize, strain = 0, energy = 0;
    double h_before_writeout = 0;
    long long ok = 0, failed = 0, attempts = 0;
    long long aval_count = 0;
    int in_aval = 0;
    unsigned sub_counter = 0;
    double next_wo = p->save_sub_configs ? next_write_out(p, 0) : INFINITY;

    speeds(&c, x, y, c.init_speed, sim_time); /* src/simulation.cpp:46 */
    for (;;) {
        /* interrupt(), src/simulation.cpp:722-750 */
        if (p->time_limit >= 0 && sim_time > p->time_limit) break;
        if (p->strain_increase_limit >= 0 && strain > p->strain_increase_limit) break;
        if (p->step_count_limit >= 0 && ok > p->step_count_limit) break;
        if (p->avalanche_limit >= 0 && aval_count > p->avalanche_limit) break;

        double ratio;
        int max_id;
        attempt(&c, x, y, sim_time, h, xb, xh, x2, &ratio, &max_id);
        if (rec && attempts < rec_cap) {
            rec[attempts].sim_time = sim_time;
            rec[attempts].step_size = h;
            rec[attempts].ratio = ratio;
            rec[attempts].max_id = max_id;
            rec[attempts].accepted = ratio < 1;
        }
        attempts++;
        if (ratio < 1) {
            sim_time += h;
            ok++;
            if (p->calculate_strain) {
                double r = 0;
                for (int i = 0; i < n; ++i) r += b_of(i, n) * (xh[i] - x[i]);
                strain += r;
                r = 0;
                for (int i = 0; i < n; ++i) r += b_of(i, n) * (x2[i] - xh[i]);
                strain += r;
            }
            for (int i = 0; i < n; ++i) x[i] = d4o_normalize(x2[i]);
            double sum_avg_sp = 0;
            for (int i = 0; i < n; ++i) sum_avg_sp = sum_avg_sp + fabs(c.init_speed2[i]);
            sum_avg_sp /= n;
            double vsq_end = absvalsq(c.speed2, n);
            energy += (absvalsq(c.init_speed, n) + 2 * absvalsq(c.init_speed2, n) + vsq_end) * h / 4;
            if (p->avalanche_limit >= 0) {
                if (in_aval && sum_avg_sp < p->avalanche_speed_threshold) {
                    aval_count++;
                    in_aval = 0;
                } else if (sum_avg_sp > p->avalanche_speed_threshold)
                    in_aval = 1;
            }
            if (p->save_sub_configs) {
                if ((!in_aval && p->sub_config_delay <= sub_counter) ||
                    (in_aval && p->sub_config_delay_during_avalanche <= sub_counter) ||
                    next_wo <= sim_time) {
                    sub_counter = 0;
                    next_wo = next_write_out(p, sim_time);
                } else
                    sub_counter++;
            }
        } else
            failed++;

        /* getNewStepSize, src/precision_handler.cpp:57-62 */
        double fct = fmin(2., pow(ratio, -1. / 6));
        h = 0.9 * h * fct;
        if (h_before_writeout != 0) {
            if (ratio < 1) h = fmax(h, h_before_writeout);
            h_before_writeout = 0;
        }
        double rem = nextafter(next_wo, INFINITY) - sim_time;
        if (rem < h) {
            h_before_writeout = h;
            h = rem;
        }
        for (int i = 0; i < n; ++i) c.tol[i] = c.min_prec_sq; /* PrecisionHandler::reset */
        if (p->max_stepsize > 0 && p->max_stepsize < h) h = p->max_stepsize;
    }
    if (res) {
        res->sim_time = sim_time;
        res->step_size = h;
        res->strain = strain;
        res->successful_steps = ok;
        res->failed_steps = failed;
        res->energy = energy;
    }
    free(xb);
    free(xh);
    free(x2);
    ctx_free(&c);
    return attempts;
}
