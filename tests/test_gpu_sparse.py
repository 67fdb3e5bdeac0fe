"""GPU checks of the cutoff sparse solver (CSR + Jacobi-preconditioned GMRES).

The reference factorises the cutoff-sparse Jacobian with UMFPACK
(src/simulation.cpp:635-659); no reference test pins results at that boundary,
and the oracle solves the same matrix with a dense partial-pivot LU.  GMRES
stops at a relative residual of 1e-13, so one attempt's positions match the
oracle's to 1e-12 (the displacements are below 1e-2 and the scaled Jacobians
here are well conditioned), and whole runs take the same accept/reject
sequence with positions within 1e-9 (conf_compare metric).  The matrix pattern
is exact (entries outside the cutoff range are exact zeros of the dense
assembly), so the CSR entry count is bounded by the cutoff disc.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

CUTS = [("cutg", dict(cutoff_multiplier=0.5)),
        ("cuth", dict(cutoff_multiplier=1.0, heaviside_cutoff=True))]


def engine(pkg, x, y, **kw):
    sd = pkg.SimulationData()
    sd.set_positions(x, y)
    sd.solver = pkg._lib.D4_SOLVER_GMRES
    for k, v in kw.items():
        setattr(sd, k, v)
    return pkg.Engine(sd)


def oracle_kw(kw):
    return {k: int(v) if isinstance(v, bool) else v for k, v in kw.items()}


@pytest.mark.parametrize("case,h", [("fix64", 1e-5), ("seed64", 3e-4)])
@pytest.mark.parametrize("tag,kw", CUTS)
def test_gmres_attempt_vs_oracle(pkg, golden, restated, case, h, tag, kw):
    x, y = golden[case + "_x"], golden[case + "_y"]
    e = engine(pkg, x, y, precision=1e-8, **kw)
    r, xb, xh, x2 = e.attempt(0.0, h)
    p = restated.params(position_precision=1e-8, **oracle_kw(kw))
    mps, _, _, _ = restated.derived(p, len(x))
    xb_o, xh_o, x2_o, _, ratio_o, id_o = restated.attempt(x, y, 0.0, h, p, np.full(len(x), mps))
    for a, b in ((xb, xb_o), (xh, xh_o), (x2, x2_o)):
        assert np.abs(a - b).max() < 1e-12
    assert abs(r.ratio - ratio_o) <= 1e-6 * ratio_o
    assert r.max_id == id_o
    st = e.solver_stats()
    assert st["solves"] == 6 and st["fallbacks"] == 0
    assert len(x) <= st["nnz"] < len(x) ** 2


@pytest.mark.parametrize("case", ["fix64", "seed64"])
def test_gmres_run_vs_oracle(pkg, golden, restated, case):
    """N=64, Heaviside cutoff, P = 1e-8, 200 accepted steps."""
    x, y = golden[case + "_x"], golden[case + "_y"]
    kw = dict(cutoff_multiplier=1.0, heaviside_cutoff=True)
    e = engine(pkg, x, y, precision=1e-8, step_count_limited=True, step_count_limit=199, **kw)
    r = e.run()
    xr, _ = e.positions()
    p = restated.params(position_precision=1e-8, step_count_limit=199, **oracle_kw(kw))
    xo, res, _, _ = restated.run(x, y, p)
    assert (r.successful_steps, r.failed_steps) == (res.successful_steps, res.failed_steps)
    d, _, _, _ = pkg.dconf.conf_compare(xr, y, xo, y)
    assert d < 1e-9
    assert e.solver_stats()["fallbacks"] == 0


def test_gmres_n1024_vs_oracle(pkg, restated):
    """N=1024 with the Heaviside cutoff at c = 0.1 (u = 3.2): three accepted
    steps against the oracle's dense solves."""
    n = 1024
    x, y, _ = pkg.dconf.generate_internal(n, 1001)
    kw = dict(cutoff_multiplier=3.2, heaviside_cutoff=True)
    e = engine(pkg, x, y, step_count_limited=True, step_count_limit=2, **kw)
    r = e.run()
    xr, _ = e.positions()
    p = restated.params(step_count_limit=2, **oracle_kw(kw))
    xo, res, _, _ = restated.run(x, y, p)
    assert (r.successful_steps, r.failed_steps) == (res.successful_steps, res.failed_steps)
    d, _, _, _ = pkg.dconf.conf_compare(xr, y, xo, y)
    assert d < 1e-11
    st = e.solver_stats()
    assert st["fallbacks"] == 0
    # pi c^2 n ~ 32 neighbours per row (+ the diagonal)
    assert st["nnz"] < 64 * n


def test_gmres_mixed_attempt(pkg, restated):
    """Mixed form with the sparse solver: GMRES solves the FP32-stored matrix
    in FP64.  Positions within the mixed form's 1e-8 of the FP64 oracle, and
    within 1e-11 of the mixed form's dense refined solves of the same matrix."""
    n = 256
    x, y, _ = pkg.dconf.generate_internal(n, 1002)
    kw = dict(cutoff_multiplier=0.1 * np.sqrt(n), heaviside_cutoff=True,
              external_stress=pkg.FixedRateProtocol(0.1, 0.0))
    h = 5e-7
    e = engine(pkg, x, y, precision_mode=pkg._lib.D4_PREC_MIXED, **kw)
    r, xb, xh, x2 = e.attempt(0.0, h)
    assert e.solver_stats()["fallbacks"] == 0
    d = engine(pkg, x, y, precision_mode=pkg._lib.D4_PREC_MIXED,
               solver=pkg._lib.D4_SOLVER_DENSE, **kw)
    _, xb_d, xh_d, x2_d = d.attempt(0.0, h)
    kw.pop("external_stress")
    p = restated.params(protocol=dict(kind=1, tau0=0.1, rate=0.0), **oracle_kw(kw))
    mps, _, _, _ = restated.derived(p, n)
    xb_o, xh_o, x2_o, _, ratio_o, _ = restated.attempt(x, y, 0.0, h, p, np.full(n, mps))
    for a, b, c in ((xb, xb_o, xb_d), (xh, xh_o, xh_d), (x2, x2_o, x2_d)):
        assert np.abs(a - b).max() < 1e-8
        assert np.abs(a - c).max() < 1e-11


def test_solver_auto(pkg, golden):
    x, y = golden["seed64_x"], golden["seed64_y"]
    auto = pkg._lib.D4_SOLVER_AUTO
    e = engine(pkg, x, y, solver=auto, cutoff_multiplier=1.0, heaviside_cutoff=True)
    e.attempt(0.0, 1e-5)
    assert e.solver_stats()["solves"] == 6  # c^2 = 1/64 < 0.1: sparse
    e = engine(pkg, x, y, solver=auto)
    e.attempt(0.0, 1e-5)
    assert e.solver_stats()["solves"] == 0  # no cutoff: dense LU
