"""CPU check of the algebra of the mixed form's fast field (d4_field64_fast.cuh).

The fast field forms each image's quotients from one reciprocal r = 1/(ch - c)
(f_l = 2 pi^2 dx (ch c - 1) r^2, its x-derivative from r^2 and r^3) and builds
the hyperbolic values from one reciprocal of e.  Restated here in numpy and
compared with the oracle's exact-order field (Field::xy / Field::xy_diff_x,
oracle/d4_oracle.c) over points of the cell away from the Taylor branch: the
difference stays within a few ulps of the magnitudes that are summed (the
largest image term for the field; for the derivative, the products inside
each image's term, which cancel strongly near a pair), not of the result.
The CUDA form itself is checked on the GPU
(tests/test_gpu_mixed.py::test_mixed_fast_sweeps).
"""
from decimal import Decimal, getcontext

import numpy as np

PI = np.pi


def _hyperbolic_constants():
    """cosh(k pi) and sinh(k pi), correctly rounded to float64: computed in
    50-digit decimal arithmetic (pi by Machin's formula).  The image sums
    subtract products of these constants, so an ulp off in one of them shows
    as hundreds of ulps in a term."""
    getcontext().prec = 60

    def atan_inv(m):  # atan(1/m) by its Taylor series
        x, x2, total, k, term = Decimal(1) / m, Decimal(1) / (m * m), Decimal(0), 0, None
        power = x
        while term is None or abs(term) > Decimal(10) ** -58:
            term = power / (2 * k + 1) * (1 if k % 2 == 0 else -1)
            total += term
            power *= x2
            k += 1
        return total

    pi = 16 * atan_inv(5) - 4 * atan_inv(239)
    ch = {k: float(((k * pi).exp() + (-k * pi).exp()) / 2) for k in (2, 4, 6, 8, 10)}
    sh = {k: float(((k * pi).exp() - (-k * pi).exp()) / 2) for k in (2, 4)}
    return ch, sh


_CH, _SH = _hyperbolic_constants()
COSH2PI, COSH4PI, COSH6PI, COSH8PI, COSHTPI = (_CH[k] for k in (2, 4, 6, 8, 10))
SINH2PI, SINH4PI = _SH[2], _SH[4]


def hyp(e):
    inv = 1 / e
    s, d = (e + inv) * 0.5, (e - inv) * 0.5
    return dict(ch0=s, sh0=d,
                chp1=s * COSH2PI + d * SINH2PI, chm1=s * COSH2PI - d * SINH2PI,
                shp1=d * COSH2PI + s * SINH2PI, shm1=d * COSH2PI - s * SINH2PI,
                chp2=s * COSH4PI + d * SINH4PI, chm2=s * COSH4PI - d * SINH4PI,
                shp2=d * COSH4PI + s * SINH4PI, shm2=d * COSH4PI - s * SINH4PI,
                chp3=COSH6PI * e, chm3=COSH6PI * inv, chp4=COSH8PI * e, chm4=COSH8PI * inv,
                chp5=COSHTPI * e, chm5=COSHTPI * inv)


def f_l(dx, c, ch):
    r = 1 / (ch - c)
    return (2 * PI * PI) * dx * (ch * c - 1) * (r * r)


def f_dx_l(dx, c, ch, sh):
    r = 1 / (ch - c)
    r2 = r * r
    n1 = ch * c - 1
    return (n1 * r2 + (2 * PI) * dx * (sh * c * r2 - 2 * n1 * sh * (r2 * r))) * (2 * PI * PI)


def xy_terms(dx, c, h):
    """The image terms of Field::xy as the fast form weights them."""
    g3 = [f_l(dx + 3, c, h["chp3"]), f_l(dx - 3, c, h["chm3"]), f_l(dx + 2, c, h["chp2"]),
          f_l(dx - 2, c, h["chm2"]), f_l(dx + 1, c, h["chp1"]), f_l(dx - 1, c, h["chm1"]),
          f_l(dx, c, h["ch0"])]
    if dx < 0:
        return [f_l(dx + 5, c, h["chp5"]) * (0 - dx), f_l(dx - 4, c, h["chm4"]) * (1 + dx),
                f_l(dx + 4, c, h["chp4"])] + g3
    return [f_l(dx - 5, c, h["chm5"]) * dx, f_l(dx + 4, c, h["chp4"]) * (1 - dx),
            f_l(dx - 4, c, h["chm4"])] + g3


def xy_diff_x_terms(dx, c, h):
    g3 = [f_dx_l(dx, c, h["ch0"], h["sh0"]), f_dx_l(dx + 1, c, h["chp1"], h["shp1"]),
          f_dx_l(dx - 1, c, h["chm1"], h["shm1"]), f_dx_l(dx + 2, c, h["chp2"], h["shp2"]),
          f_dx_l(dx - 2, c, h["chm2"], h["shm2"]), f_dx_l(dx + 3, c, h["chp3"], h["chp3"]),
          f_dx_l(dx - 3, c, h["chm3"], h["chm3"])]
    if dx < 0:
        return [f_dx_l(dx + 5, c, h["chp5"], h["chp5"]) * (0 - dx), -f_l(dx + 5, c, h["chp5"]),
                f_dx_l(dx - 4, c, h["chm4"], h["chm4"]) * (1 + dx), f_l(dx - 4, c, h["chm4"]),
                f_dx_l(dx + 4, c, h["chp4"], h["chp4"])] + g3
    return [f_dx_l(dx - 5, c, h["chm5"], h["chm5"]) * dx, f_l(dx - 5, c, h["chm5"]),
            f_dx_l(dx + 4, c, h["chp4"], h["chp4"]) * (1 - dx), -f_l(dx + 4, c, h["chp4"]),
            f_dx_l(dx - 4, c, h["chm4"], h["chm4"])] + g3


def dx_scale(dx, c, h):
    """Sum over the images -3..3 of the magnitudes inside each derivative term
    (its three products cancel strongly near a pair, so rounding is relative
    to them)."""
    def one(d, ch, sh):
        r = 1 / (ch - c)
        n1 = ch * c - 1
        return (abs(n1 * r * r) + abs(2 * PI * d * sh * c * r * r) +
                abs(4 * PI * d * n1 * sh * r ** 3)) * (2 * PI * PI)
    return (one(dx, h["ch0"], h["sh0"]) + one(dx + 1, h["chp1"], h["shp1"]) +
            one(dx - 1, h["chm1"], h["shm1"]) + one(dx + 2, h["chp2"], h["shp2"]) +
            one(dx - 2, h["chm2"], h["shm2"]) + one(dx + 3, h["chp3"], h["chp3"]) +
            one(dx - 3, h["chm3"], h["chm3"]))


def test_fast_field_matches_exact_order_field(restated):
    rng = np.random.default_rng(11)
    pts = rng.uniform(-0.5, 0.5, size=(4000, 2))
    # close pairs too (the cancellation case), outside the Taylor branch
    close = rng.uniform(-0.02, 0.02, size=(1000, 2))
    pts = np.vstack([pts, close])
    worst_xy = worst_dx = 0.0
    checked = 0
    for dx, dy in pts:
        if dx * dx + dy * dy <= 1e-6:
            continue
        e = np.exp(2 * PI * dx)
        c = np.cos(PI * 2 * dy)
        h = hyp(e)
        t1 = xy_terms(dx, c, h)
        t2 = xy_diff_x_terms(dx, c, h)
        exact1 = restated.L.d4o_xy4(dx, dy, e, c)
        exact2 = restated.L.d4o_xy_diff_x4(dx, dy, e, c)
        worst_xy = max(worst_xy, abs(sum(t1) - exact1) / max(abs(t) for t in t1))
        scale2 = max(dx_scale(dx, c, h), max(abs(t) for t in t2))
        worst_dx = max(worst_dx, abs(sum(t2) - exact2) / scale2)
        checked += 1
    assert checked > 4500
    eps = np.finfo(np.float64).eps
    # a few ulps of the terms' magnitudes (the exact-order form rounds
    # differently); measured: 3.3 and 2.2 ulps
    assert worst_xy < 16 * eps, worst_xy
    assert worst_dx < 16 * eps, worst_dx
