"""Failure detection without a GPU fault (marked gpu).

The reference stops on input errors with exit(-1) and, in its DEBUG_VERSION
build, dumps state on non-finite values (src/simulation.cpp:754-948); without
those checks a NaN error ratio fails every attempt while getNewStepSize
doubles h forever.  Here:
  - d4_set_positions rejects non-finite and out-of-cell positions (D4_ERR_ARG);
  - a step whose error ratio is not finite (an infinite step size, so that the
    Jacobian overflows) ends d4_advance with D4_ERR_STATE instead of looping;
  - every bounded device wait gives up after its limit and reports
    D4_ERR_STATE through the host (d4_wait_selftest runs the cooperative LU's
    grid barrier with a CTA that never arrives and the block LU's tile-flag
    wait on a flag nothing sets); the context stays usable afterwards, checked
    by an attempt against the oracle.
Nothing here faults, traps or hangs the GPU: the non-finite values are
ordinary IEEE arithmetic, and the waits end by their own limits.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def make_engine(pkg, n, seed, mode=None):
    x, y, _ = pkg.dconf.generate_internal(n, seed)
    sd = pkg.SimulationData()
    sd.set_positions(x, y)
    sd.precision = 1e-8
    if mode is not None:
        sd.precision_mode = mode
    return pkg.Engine(sd), x, y


def attempt_matches_oracle(pkg, e, x, y):
    import pyoracle
    r, xb, xh, x2 = e.attempt(0.0, 1e-5)
    ora = pyoracle.Restated()
    p = ora.params(position_precision=1e-8)
    mps, _, _, _ = ora.derived(p, len(x))
    xb_o, xh_o, x2_o, _, ratio_o, id_o = ora.attempt(x, y, 0.0, 1e-5, p, np.full(len(x), mps))
    return max(np.abs(xb - xb_o).max(), np.abs(x2 - x2_o).max()) < 1e-14 and r.max_id == id_o


def test_set_positions_rejects_bad_values(pkg):
    e, x, y = make_engine(pkg, 64, 1000)
    lib = e.lib
    for bad in (np.nan, np.inf, 0.5, -0.75):
        xx = x.copy()
        xx[7] = bad
        st = lib.d4_set_positions(e.ctx, pkg._lib.ptr(xx), pkg._lib.ptr(y))
        assert st == pkg._lib.D4_ERR_ARG
        assert b"dislocation 7" in lib.d4_last_error(e.ctx)
    # the context still holds the last valid positions
    assert np.array_equal(e.positions()[0], x)
    e.close()


@pytest.mark.parametrize("mixed", [False, True])
def test_nonfinite_ratio_stops_the_loop(pkg, mixed):
    mode = pkg._lib.D4_PREC_MIXED if mixed else pkg._lib.D4_PREC_FP64
    e, x, y = make_engine(pkg, 256 if mixed else 64, 1000, mode)
    # an infinite step size: the Jacobian and residuals overflow, the positions
    # and the error ratio become NaN (a large finite h is no test: the implicit
    # step's displacement stays finite)
    e._call("d4_set_time", C.c_double(0.0), C.c_double(float("inf")))
    r = pkg._lib.RunResult()
    st = e.lib.d4_advance(e.ctx, C.c_longlong(1), C.byref(r))
    assert st == pkg._lib.D4_ERR_STATE
    assert b"non-finite error ratio" in e.lib.d4_last_error(e.ctx)
    e.close()


def test_bounded_waits_give_up_and_context_survives(pkg):
    e, x, y = make_engine(pkg, 64, 1000)
    for which in (0, 1):
        st = e.lib.d4_wait_selftest(e.ctx, which)
        assert st == pkg._lib.D4_ERR_STATE, which
        assert b"gave up" in e.lib.d4_last_error(e.ctx)
    assert attempt_matches_oracle(pkg, e, x, y)
    e.close()
