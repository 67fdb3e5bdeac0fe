"""Pins the C restatement (oracle/d4_oracle.c) to the reference's own outputs.

golden.npz holds outputs of the reference core built from its sources
(tests/golden/make_golden.py).  The restatement must reproduce them bit for
bit; only then is it trusted as the oracle of the GPU tests.
"""
import numpy as np
import pytest

CASES = ["fix64", "seed64"]


def test_field_known_answers(golden, restated):
    L = restated.L
    xy = np.array([L.d4o_xy(a, b) for a, b in zip(golden["field_dx"], golden["field_dy"])])
    xyd = np.array([L.d4o_xy_diff_x(a, b) for a, b in zip(golden["field_dx"], golden["field_dy"])])
    assert np.array_equal(xy, golden["field_xy"])
    assert np.array_equal(xyd, golden["field_xyd"])


@pytest.mark.parametrize("case", CASES + ["seed256"])
def test_speeds(golden, restated, case):
    x, y = golden[case + "_x"], golden[case + "_y"]
    p = restated.params(position_precision=1e-8)
    mps, use, _, _ = restated.derived(p, len(x))
    tol = np.full(len(x), mps)
    v = restated.speeds(x, y, 0.0, tol, mps)
    assert np.array_equal(v, golden[case + "_v"])
    assert np.array_equal(tol, golden[case + "_tol"])


@pytest.mark.parametrize("case", CASES)
def test_jacobian(golden, restated, case):
    x, y = golden[case + "_x"], golden[case + "_y"]
    p = restated.params(position_precision=1e-8)
    mps, use, cut, cut_sq = restated.derived(p, len(x))
    tol = np.full(len(x), mps)
    va, vb, a, d = restated.jacobian(x, y, 1e-3, 0.0, 0.0, cut_sq, cut, tol=tol, min_prec_sq=mps)
    assert np.array_equal(va, golden[case + "_jac_va"])
    assert np.array_equal(vb, golden[case + "_jac_vb"])
    assert np.array_equal(a, golden[case + "_jac_a"])
    assert np.array_equal(d, golden[case + "_jac_d"])
    assert np.array_equal(tol, golden[case + "_jac_tol"])


@pytest.mark.parametrize("case", CASES)
@pytest.mark.parametrize("tag,kw", [("cutg", dict(cutoff_multiplier=0.5)),
                                    ("cuth", dict(cutoff_multiplier=1.0, heaviside_cutoff=1)),
                                    ("wp", dict(weight_function="p")),
                                    ("wm", dict(weight_function="m"))])
def test_jacobian_variants(golden, restated, case, tag, kw):
    x, y = golden[case + "_x"], golden[case + "_y"]
    p = restated.params(position_precision=1e-8, **kw)
    mps, use, cut, cut_sq = restated.derived(p, len(x))
    va, vb, a, d = restated.jacobian(x, y, 2e-3, 0.0, 0.0, cut_sq, cut,
                                     heaviside=kw.get("heaviside_cutoff", 0),
                                     wfn=kw.get("weight_function", "c"))
    assert np.array_equal(a, golden["%s_%s_a" % (case, tag)])
    assert np.array_equal(d, golden["%s_%s_d" % (case, tag)])
    if tag.startswith("cut"):
        # the dense expansion has exactly the CSC pattern's nonzeros
        assert int(golden["%s_%s_nnz" % (case, tag)]) < len(x) * len(x)


@pytest.mark.parametrize("case", CASES)
def test_run_c1(golden, restated, case):
    """1000 accepted steps at P = 1e-8, tau = 0 (the N=64 plain configuration)."""
    x, y = golden[case + "_x"], golden[case + "_y"]
    p = restated.params(position_precision=1e-8, step_count_limit=999)
    xr, res, na, recs = restated.run(x, y, p, record=5000)
    ref = golden[case + "_run_res"]
    assert np.array_equal(xr, golden[case + "_run_x"])
    assert (res.sim_time, res.step_size) == (ref[0], ref[1])
    assert (res.successful_steps, res.failed_steps) == (int(ref[2]), int(ref[3]))
    # the accepted steps' log rows: time, counts, ratio, id and step size
    log = golden[case + "_run_log"]
    acc = [r for r in recs if r[4]]
    assert len(acc) == len(log)
    assert np.array_equal(np.array([r[2] for r in acc]), log[:, 3])
    assert np.array_equal(np.array([r[3] for r in acc]), log[:, 4])
    assert np.array_equal(np.array([r[1] for r in acc]), log[:, 5])


@pytest.mark.parametrize("case", CASES)
def test_run_constant_stress(golden, restated, case):
    x, y = golden[case + "_x"], golden[case + "_y"]
    p = restated.params(position_precision=1e-6, step_count_limit=199, calculate_strain=1,
                        protocol=dict(kind=1, tau0=0.1, rate=0.0))
    xr, res, na, _ = restated.run(x, y, p)
    ref = golden[case + "_tau_res"]
    assert np.array_equal(xr, golden[case + "_tau_x"])
    assert (res.sim_time, res.step_size, res.strain) == (ref[0], ref[1], ref[4])
    assert (res.successful_steps, res.failed_steps) == (int(ref[2]), int(ref[3]))


@pytest.mark.parametrize("case", CASES)
def test_run_cyclic_no_dipole(golden, restated, case):
    x, y = golden[case + "_x"], golden[case + "_y"]
    p = restated.params(position_precision=1e-6, dipole_precision=0.0, step_count_limit=149,
                        protocol=dict(kind=2, tau0=0.0, rate=5.0, period=0.01))
    xr, res, na, _ = restated.run(x, y, p)
    ref = golden[case + "_cyc_res"]
    assert np.array_equal(xr, golden[case + "_cyc_x"])
    assert (res.successful_steps, res.failed_steps) == (int(ref[2]), int(ref[3]))


def test_ieee_field_restatement_pinned(restated):
    """The restatement of the IEEE variant of the field (src/Fields/Field.cpp:
    26-168) against the reference's own IEEE evaluator (sandbox/ieee_hyperbolic,
    built unmodified; golden_runs.npz ieee_*), bit for bit on the field grid
    (lattice of the reference's precision study, near-field and random
    points)."""
    import os
    g = np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden",
                             "golden_runs.npz"))
    gd = np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden",
                              "golden.npz"))
    fx, fy = gd["field_dx"], gd["field_dy"]
    xy = np.array([restated.L.d4o_ieee_xy(a, b) for a, b in zip(fx, fy)])
    xyd = np.array([restated.L.d4o_ieee_xy_diff_x(a, b) for a, b in zip(fx, fy)])
    assert np.array_equal(xy, g["ieee_xy"])
    assert np.array_equal(xyd, g["ieee_xyd"])
    # the non-IEEE (default) field against it: the reference's own precision
    # study reports stress errors to ~1e-10 and gradient errors to ~3e-4
    # relative (sandbox/ieee_hyperbolic/README.md:40-43)
    m = np.abs(g["ieee_xyd"]) > 1e-3
    rel_s = np.abs(gd["field_xy"] - g["ieee_xy"]) / np.maximum(np.abs(g["ieee_xy"]), 1e-300)
    rel_g = np.abs(gd["field_xyd"][m] - g["ieee_xyd"][m]) / np.abs(g["ieee_xyd"][m])
    assert np.median(rel_s) < 1e-12 and np.median(rel_g) < 1e-6
