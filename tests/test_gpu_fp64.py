"""GPU parity of the plain FP64 form against the oracle (marked gpu).

The oracle is the C restatement (oracle/d4_oracle.c), itself pinned bit for bit
to the reference's outputs (test_oracle_pin.py), and the golden reference
outputs directly.  Tolerances: the FP64 kernels keep the reference's operation
order with no FMA contraction, so they differ from the oracle only where CUDA's
exp2/cos/pow round differently from glibc (about 0.1% of calls, by one ulp);
the cancellation in cosh - cos of close pairs amplifies that to ~1e-11
relative in the field.  Whole runs must match the reference's positions within
1e-10 (conf_compare metric, cell units) after the same accepted-step count.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

FIELD_RTOL = 1e-9


def engine(pkg, x, y, **kw):
    sd = pkg.SimulationData()
    sd.set_positions(x, y)
    for k, v in kw.items():
        setattr(sd, k, v)
    return pkg.Engine(sd)


def rel_err(a, b):
    scale = max(np.abs(b).max(), 1e-300)
    return np.abs(a - b).max() / scale


def test_field_known_answers(pkg, golden):
    f = pkg.Field()
    dx, dy = golden["field_dx"], golden["field_dy"]
    xy, xyd = f.eval(dx, dy)
    for got, ref in ((xy, golden["field_xy"]), (xyd, golden["field_xyd"])):
        rel = np.abs(got - ref) / np.maximum(np.abs(ref), 1e-12)
        assert rel.max() < FIELD_RTOL, rel.max()
        assert np.median(rel) < 1e-15
        assert np.mean(got == ref) > 0.5


@pytest.mark.parametrize("case", ["fix64", "seed64", "seed256"])
def test_speeds_vs_reference(pkg, golden, case):
    x, y = golden[case + "_x"], golden[case + "_y"]
    e = engine(pkg, x, y, precision=1e-8)
    v, tol = e.speeds(x, y, 0.0)
    assert rel_err(v, golden[case + "_v"]) < 1e-11
    assert np.array_equal(tol, golden[case + "_tol"])  # distances are exact


@pytest.mark.parametrize("n,seed", [(1024, 1001), (2048, 1003)])
def test_speeds_large_vs_oracle(pkg, restated, n, seed):
    x, y, _ = pkg.dconf.generate_internal(n, seed)
    e = engine(pkg, x, y, precision=1e-5)
    v, tol = e.speeds(x, y, 0.0)
    p = restated.params()
    mps, _, _, _ = restated.derived(p, n)
    tol_o = np.full(n, mps)
    v_o = restated.speeds(x, y, 0.0, tol_o, mps)
    assert rel_err(v, v_o) < 1e-11
    assert np.array_equal(tol, tol_o)


@pytest.mark.parametrize("case", ["fix64", "seed64"])
def test_jacobian_vs_reference(pkg, golden, case):
    x, y = golden[case + "_x"], golden[case + "_y"]
    e = engine(pkg, x, y, precision=1e-8)
    va, vb, a, d, tol = e.jacobian(x, y, 1e-3, 0.0, 1e-3)
    assert rel_err(va, golden[case + "_jac_va"]) < 1e-11
    assert rel_err(vb, golden[case + "_jac_vb"]) < 1e-11
    assert rel_err(a, golden[case + "_jac_a"]) < 1e-10
    assert np.abs(d - golden[case + "_jac_d"]).max() < 1e-10
    assert np.array_equal(tol, golden[case + "_jac_tol"])


@pytest.mark.parametrize("case", ["fix64", "seed64"])
@pytest.mark.parametrize("tag,kw", [("cutg", dict(cutoff_multiplier=0.5)),
                                    ("cuth", dict(cutoff_multiplier=1.0, heaviside_cutoff=True)),
                                    ("wp", dict(weight_function="p")),
                                    ("wm", dict(weight_function="m"))])
def test_jacobian_variants_vs_reference(pkg, golden, case, tag, kw):
    x, y = golden[case + "_x"], golden[case + "_y"]
    e = engine(pkg, x, y, precision=1e-8, **kw)
    va, vb, a, d, tol = e.jacobian(x, y, 2e-3, 0.0, 2e-3)
    ref = golden["%s_%s_a" % (case, tag)]
    assert rel_err(a, ref) < 1e-10
    # the sparsity pattern (entries outside the cutoff range) is exact
    assert np.array_equal(a == 0, ref == 0)
    assert np.abs(d - golden["%s_%s_d" % (case, tag)]).max() < 1e-10


def test_jacobian_from_prev_exact(pkg, restated):
    x, y, _ = pkg.dconf.generate_internal(128, 11)
    e = engine(pkg, x, y)
    va, vb, a, d, _ = e.jacobian(x, y, 5e-3, 0.0, 5e-3)
    t0, h = 0.37, 5e-3
    factor = ((t0 + h / 2) - t0) / ((t0 + h) - t0)
    a2, d2 = e.jacobian_from_prev(factor)
    a_o, d_o = restated.jacobian_from_prev(np.ascontiguousarray(a), d, factor)
    assert np.array_equal(a2, a_o) and np.array_equal(d2, d_o)


@pytest.mark.parametrize("n,h", [(64, 1e-6), (256, 1e-6), (1024, 1e-8), (1024, 1e-6)])
def test_factor_solve_jacobian_exact(pkg, restated, n, h):
    """Jacobians, with or without row swaps under partial pivoting (the fast
    path or its pivoted fallback): solutions bit-identical to the oracle."""
    x, y, _ = pkg.dconf.generate_internal(n, 5 + n)
    e = engine(pkg, x, y)
    _, _, a, _, _ = e.jacobian(x, y, h, 0.0, h)
    assert e.factor() == 0
    g = np.random.default_rng(1).normal(size=n)
    dx, st = e.solve(g)
    dx_o, sing, piv = restated.lu_solve(np.ascontiguousarray(a), g)
    assert np.array_equal(dx, dx_o)


@pytest.mark.parametrize("n", [64, 100, 257])
def test_factor_solve_pivoted_exact(pkg, restated, n):
    """Random dense matrices need row swaps: the pivoted path, bit-identical."""
    x, y, _ = pkg.dconf.generate_internal(n + n % 2, 1)
    rng = np.random.default_rng(n)
    a = rng.normal(size=(n, n))
    if n % 2:
        a = np.pad(a, ((0, 1), (0, 1)))
        a[n, n] = 1.0
    m = a.shape[0]
    e = engine(pkg, x[:m], y[:m])
    e.set_matrix(a)
    assert e.factor() == 0
    g = rng.normal(size=m)
    dx, st = e.solve(g)
    dx_o, sing, piv = restated.lu_solve(a, g)
    assert (piv != np.arange(m)).any()
    assert np.array_equal(dx, dx_o)
    assert np.abs(a @ dx - g).max() < 1e-9
    # counters: every swap is the oracle's, and costs one extra pass over its block
    st = e.lu_stats()
    swaps = int((piv != np.arange(m)).sum())
    assert st["factorizations"] == 1 and st["swaps"] == swaps
    assert st["passes"] == -(-m // 32) + swaps


def test_factor_singular(pkg, restated):
    n = 64
    x, y, _ = pkg.dconf.generate_internal(n, 2)
    a = np.random.default_rng(0).normal(size=(n, n))
    a[:, 5] = 0.0
    e = engine(pkg, x, y)
    e.set_matrix(a)
    assert e.factor() == 1  # D4_WARN_SINGULAR, like UMFPACK
    g = np.ones(n)
    dx, st = e.solve(g)
    assert st == 1
    dx_o, sing, _ = restated.lu_solve(a, g)
    assert sing == 1
    same = (dx == dx_o) | (np.isnan(dx) & np.isnan(dx_o))
    assert same.all()


@pytest.mark.parametrize("case,h", [("fix64", 1e-5), ("seed64", 3e-4)])
def test_attempt_vs_oracle(pkg, golden, restated, case, h):
    x, y = golden[case + "_x"], golden[case + "_y"]
    e = engine(pkg, x, y, precision=1e-8)
    r, xb, xh, x2 = e.attempt(0.0, h)
    p = restated.params(position_precision=1e-8)
    mps, _, _, _ = restated.derived(p, len(x))
    xb_o, xh_o, x2_o, tol_o, ratio_o, id_o = restated.attempt(x, y, 0.0, h, p, np.full(len(x), mps))
    for a, b in ((xb, xb_o), (xh, xh_o), (x2, x2_o)):
        assert np.abs(a - b).max() < 1e-14
    assert abs(r.ratio - ratio_o) <= 1e-6 * ratio_o
    assert r.max_id == id_o and r.accepted == (ratio_o < 1)


def run_engine(pkg, x, y, **kw):
    e = engine(pkg, x, y, **kw)
    r = e.run()
    xr, _ = e.positions()
    return xr, r


@pytest.mark.parametrize("case", ["fix64", "seed64"])
def test_run_c1_vs_reference(pkg, golden, case):
    """N=64, zero stress, P = 1e-8, 1000 accepted steps (-C 999): the plain
    configuration.  Positions within 1e-10 of the reference's (conf_compare)."""
    x, y = golden[case + "_x"], golden[case + "_y"]
    xr, r = run_engine(pkg, x, y, precision=1e-8, step_count_limited=True, step_count_limit=999)
    ref = golden[case + "_run_res"]
    assert r.successful_steps == int(ref[2])
    assert r.failed_steps == int(ref[3])
    d, i, avg, _ = pkg.dconf.conf_compare(xr, y, golden[case + "_run_x"], y)
    assert d < 1e-10, (d, i)
    assert abs(r.sim_time - ref[0]) < 1e-9 * ref[0]


@pytest.mark.parametrize("case", ["fix64", "seed64"])
def test_run_constant_stress_vs_reference(pkg, golden, case):
    x, y = golden[case + "_x"], golden[case + "_y"]
    xr, r = run_engine(pkg, x, y, precision=1e-6, step_count_limited=True, step_count_limit=199,
                       calculate_strain_during_simulation=True,
                       external_stress=pkg.FixedRateProtocol(0.1, 0.0))
    ref = golden[case + "_tau_res"]
    assert (r.successful_steps, r.failed_steps) == (int(ref[2]), int(ref[3]))
    d, _, _, _ = pkg.dconf.conf_compare(xr, y, golden[case + "_tau_x"], y)
    assert d < 1e-10
    assert abs(r.strain - ref[4]) < 1e-10 * max(1.0, abs(ref[4]))


@pytest.mark.parametrize("case", ["fix64", "seed64"])
def test_run_cyclic_no_dipole_vs_reference(pkg, golden, case):
    x, y = golden[case + "_x"], golden[case + "_y"]
    xr, r = run_engine(pkg, x, y, precision=1e-6, dipole_precision=0.0, step_count_limited=True,
                       step_count_limit=149,
                       external_stress=pkg.CyclicLoadProtocol(0.0, 5.0, 0.01))
    ref = golden[case + "_cyc_res"]
    assert (r.successful_steps, r.failed_steps) == (int(ref[2]), int(ref[3]))
    d, _, _, _ = pkg.dconf.conf_compare(xr, y, golden[case + "_cyc_x"], y)
    assert d < 1e-10


def test_run_n1024_few_steps_vs_oracle(pkg, restated):
    n = 1024
    x, y, _ = pkg.dconf.generate_internal(n, 1001)
    xr, r = run_engine(pkg, x, y, step_count_limited=True, step_count_limit=2)
    p = restated.params(step_count_limit=2)
    xo, res, na, _ = restated.run(x, y, p)
    assert (r.successful_steps, r.failed_steps) == (res.successful_steps, res.failed_steps)
    d, _, _, _ = pkg.dconf.conf_compare(xr, y, xo, y)
    assert d < 1e-12


def test_field_vs_ieee_lattice_sum(pkg, golden):
    """The device field against the exact truncated image sum, the reference's
    IEEE variant (src/Fields/Field.cpp:26-168, values from its own evaluator:
    golden_runs.npz ieee_*): on the field grid the device stress and gradient
    are off the exact sum by the reference's own default formula's error
    (sandbox/ieee_hyperbolic/README.md:40-43 reports it: up to ~1e-10 relative
    in the stress, ~3e-4 in the gradient) and by no more than 1e-12 of the
    field's scale besides."""
    import os
    gr = np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden",
                              "golden_runs.npz"))
    f = pkg.Field()
    xy, xyd = f.eval(golden["field_dx"], golden["field_dy"])
    for dev, ref, exact in ((xy, golden["field_xy"], gr["ieee_xy"]),
                            (xyd, golden["field_xyd"], gr["ieee_xyd"])):
        m = np.abs(exact) > 1e-3
        scale = np.abs(exact[m])
        assert np.all(np.abs(dev[m] - exact[m]) <= np.abs(ref[m] - exact[m]) + 1e-12 * scale)
