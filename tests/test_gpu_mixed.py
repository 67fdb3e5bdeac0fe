"""GPU checks of the mixed-precision form (marked gpu).

The mixed form keeps FP64 sweeps, matrix, residuals, updates and step
control, and runs the factorisations and triangular solves in FP32 (the
block LU on the tensor cores) inside FP64 iterative refinement against the
FP64 matrix.  Below N=2048 its sweeps are the FP64 form's exact-order ones;
from N=2048 its pair tiles form each image's quotients from one reciprocal
with product-adds contracted.  Tolerances: the speeds and the matrix to
1e-12 relative of the oracle's; one attempt's positions to 1e-10; each of
1000 accepted steps at N=4096, taken from the FP64 form's state, to 1e-10 of
the FP64 form's step; 50 free-running steps to 1e-8.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def engine(pkg, x, y, **kw):
    sd = pkg.SimulationData()
    sd.set_positions(x, y)
    sd.precision_mode = pkg._lib.D4_PREC_MIXED
    for k, v in kw.items():
        setattr(sd, k, v)
    return pkg.Engine(sd)


@pytest.mark.parametrize("n,seed", [(64, 1000), (256, 7), (1024, 1001)])
def test_mixed_speeds(pkg, restated, n, seed):
    x, y, _ = pkg.dconf.generate_internal(n, seed)
    e = engine(pkg, x, y)
    v, tol = e.speeds(x, y, 0.0)
    p = restated.params()
    mps, _, _, _ = restated.derived(p, n)
    tol_o = np.full(n, mps)
    vo = restated.speeds(x, y, 0.0, tol_o, mps)
    assert np.abs(v - vo).max() / np.abs(vo).max() < 1e-12
    assert np.array_equal(tol, tol_o)  # distances stay FP64


def test_mixed_close_pairs(pkg, golden):
    """Near-field pairs (r^2 <= 1e-6 uses the reference's Taylor branch)."""
    x = np.array([0.1, 0.1 + 3e-4, -0.2, 0.3])
    y = np.array([0.05, 0.05 - 2e-4, 0.2, -0.1])
    import pyoracle
    ro = pyoracle.Restated()
    vo = ro.speeds(x, y, 0.0)
    e = engine(pkg, x, y)
    v, _ = e.speeds(x, y, 0.0)
    assert np.abs(v - vo).max() / np.abs(vo).max() < 1e-12


def test_mixed_jacobian(pkg, restated):
    n = 256
    x, y, _ = pkg.dconf.generate_internal(n, 7)
    e = engine(pkg, x, y)
    va, vb, a, d, _ = e.jacobian(x, y, 1e-4, 0.0, 1e-4)
    p = restated.params()
    mps, _, cut, cs = restated.derived(p, n)
    vao, vbo, ao, do = restated.jacobian(x, y, 1e-4, 0.0, 0.0, cs, cut)
    assert np.abs(a - ao).max() / np.abs(ao).max() < 1e-12
    assert np.abs(d - do).max() < 1e-12


def test_mixed_fast_sweeps(pkg, restated):
    """From N=2048 the mixed form's pair tiles drop the reference's operation
    order (one reciprocal per image, contracted product-adds).  Close pairs
    give single forces of 1e5-1e6 whose row sums cancel to about 1e2, so a few
    ulps per term show as a few 1e-12 of max|v|: speeds, the matrix and d are
    held to 1e-10 relative of the oracle's (the exact-order sweeps of the plain
    form meet 1e-12), and one attempt from them to 1e-10 in positions
    (test_mixed_attempt)."""
    n = 2048
    x, y, _ = pkg.dconf.generate_internal(n, 1002)
    e = engine(pkg, x, y)
    p = restated.params()
    mps, _, cut, cs = restated.derived(p, n)

    def rel(u, w):
        return np.abs(u - w).max() / np.abs(w).max()

    v, tol = e.speeds(x, y, 0.0)
    vo = restated.speeds(x, y, 0.0, np.full(n, mps), mps)
    assert rel(v, vo) < 1e-10
    va, vb, a, d, _ = e.jacobian(x, y, 1e-6, 0.0, 1e-6)
    vao, vbo, ao, do = restated.jacobian(x, y, 1e-6, 0.0, 0.0, cs, cut)
    assert rel(a, ao) < 1e-10
    assert rel(d, do) < 1e-10
    assert rel(va, vao) < 1e-10


@pytest.mark.parametrize("n,h", [(2048, 1e-7)])
def test_mixed_attempt(pkg, restated, n, h):
    """One attempt on the FP32 path (N >= 2048) against the oracle's FP64 attempt."""
    x, y, _ = pkg.dconf.generate_internal(n, 1002)
    e = engine(pkg, x, y, external_stress=pkg.FixedRateProtocol(0.1, 0.0))
    r, xb, xh, x2 = e.attempt(0.0, h)
    p = restated.params(protocol=dict(kind=1, tau0=0.1, rate=0.0))
    mps, _, _, _ = restated.derived(p, n)
    xbo, xho, x2o, _, ro, io = restated.attempt(x, y, 0.0, h, p, np.full(n, mps))
    assert np.abs(x2 - x2o).max() < 1e-10
    assert np.abs(xb - xbo).max() < 1e-10
    assert r.refine_residual < 1e-10
    assert ro < 1  # a step size the error control accepts
    assert abs(r.ratio - ro) <= 1e-3 * ro + 1e-12
    assert e.mixed_stats()["block_factorizations"] == 3


def test_mixed_fixed_steps_vs_fp64(pkg):
    """100 accepted steps at N=2048 with the step size capped at h (P large, so
    the dipole criterion decides the few rejections): mixed vs the plain FP64
    form along the same step sequence."""
    n, h, steps = 2048, 2e-7, 100
    x, y, _ = pkg.dconf.generate_internal(n, 1002)
    out = []
    for mode in (pkg._lib.D4_PREC_FP64, pkg._lib.D4_PREC_MIXED):
        sd = pkg.SimulationData()
        sd.set_positions(x, y)
        sd.precision_mode = mode
        sd.precision = 1.0  # step size capped at h; the dipole criterion still rejects
        sd.max_step_size_limited, sd.max_stepsize_limit, sd.step_size = True, h, h
        sd.external_stress = pkg.FixedRateProtocol(0.1, 0.0)
        e = pkg.Engine(sd)
        r = e.advance(steps)
        out.append((e.positions()[0], r))
        e.close()
    # the same sequence of attempted and accepted steps in both forms
    assert out[0][1].attempts == out[1][1].attempts
    assert out[0][1].failed_steps == out[1][1].failed_steps
    d, _, _, _ = pkg.dconf.conf_compare(out[1][0], y, out[0][0], y)
    assert d < 1e-9


def pair_engines(pkg, x, y, tau):
    engs = []
    for mode in (pkg._lib.D4_PREC_FP64, pkg._lib.D4_PREC_MIXED):
        sd = pkg.SimulationData()
        sd.set_positions(x, y)
        sd.precision_mode = mode
        sd.external_stress = pkg.FixedRateProtocol(tau, 0.0)
        engs.append(pkg.Engine(sd))
    return engs


def test_mixed_1000_steps_shadowing_fp64(pkg):
    """N=4096 dense (seed 1002, constant stress 0.1): 1000 accepted steps of
    the FP64 form; before each one the mixed form restarts from the FP64 form's
    state (positions, time, step size, tolerances) and takes the same step.
    Every step: the same attempts and rejections, and positions within 1e-10 of
    the FP64 form's.  The run passes through stretches of stiff Jacobians (close
    pairs) where the block LU falls back to the pivoted FP32 LU.

    A free-running comparison over 1000 steps would measure the dynamics' own
    sensitivity instead: a 1e-15 perturbation of the initial positions, run by
    the FP64 form itself, grows to 1.2e-9 by step 50 and 1e-4 by step 100."""
    x, y, _ = pkg.dconf.generate_internal(4096, 1002)
    f64, mix = pair_engines(pkg, x, y, 0.1)
    mix.advance(0)
    worst = 0.0
    for s in range(1000):
        x0, _ = f64.positions()
        tol = f64.tolerance()
        t0 = f64.advance(0)
        mix.restore(x0, y, t0.sim_time, t0.step_size, tol)
        r64 = f64.advance(1)
        rmx = mix.advance(1)
        assert (r64.attempts, r64.failed_steps) == (rmx.attempts, rmx.failed_steps), s
        d = pkg.dconf.conf_compare(mix.positions()[0], y, f64.positions()[0], y)[0]
        worst = max(worst, d)
    assert worst <= 1e-10, worst
    st = mix.mixed_stats()
    assert st["block_factorizations"] > 0 and st["worst_refined_residual"] <= 1e-9
    f64.close()
    mix.close()


def test_mixed_free_run_50_steps(pkg):
    """The same workload, both forms free-running in lockstep for 50 accepted
    steps (inside the horizon where the FP64 form's own sensitivity to a
    1e-15 perturbation stays near 1e-9): the same attempts, positions within
    1e-8 after every step."""
    x, y, _ = pkg.dconf.generate_internal(4096, 1002)
    engs = pair_engines(pkg, x, y, 0.1)
    worst = 0.0
    for s in range(50):
        r64 = engs[0].advance(1)
        rmx = engs[1].advance(1)
        assert (r64.attempts, r64.failed_steps) == (rmx.attempts, rmx.failed_steps), s
        d = pkg.dconf.conf_compare(engs[1].positions()[0], y, engs[0].positions()[0], y)[0]
        worst = max(worst, d)
    assert worst <= 1e-8, worst
    for e in engs:
        e.close()


def test_mixed_small_systems_run_fp64(pkg):
    """Below N=2048 the mixed form's attempts run on the FP64 path (the exact
    LU is latency-bound there, FP32 factors gain nothing): the headline
    workload's steps are the FP64 form's, bit for bit."""
    import os
    z = np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden",
                             "c2_relaxed_1024.npz"))
    x, y = z["x"], z["y"]
    f64, mix = pair_engines(pkg, x, y, 0.05)
    r64 = f64.advance(20)
    rmx = mix.advance(20)
    assert (r64.attempts, r64.failed_steps) == (rmx.attempts, rmx.failed_steps)
    assert np.array_equal(f64.positions()[0], mix.positions()[0])
    st = mix.mixed_stats()
    assert st["block_factorizations"] == 0 and st["fp64_attempts"] == rmx.attempts
    f64.close()
    mix.close()
