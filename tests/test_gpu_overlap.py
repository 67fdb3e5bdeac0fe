"""The two schedules of an attempt give identical runs (marked gpu).

By default stage I (the big step) runs on a second stream, concurrently with
stages II and III, with its own factorisation, solve scratch and copies of
the weights and end speeds; d4_set_overlap(ctx, 0) runs the stages in the
reference's order on one stream (src/simulation.cpp:88-164).  Both schedules
perform the same operations on the same values, so a run must come out bit
for bit the same: positions, step counts, time, strain, and (mixed form) the
worst refined residual of each attempt.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def run(pkg, mode, overlap, n, seed, steps):
    x, y, _ = pkg.dconf.generate_internal(n, seed)
    sd = pkg.SimulationData()
    sd.set_positions(x, y)
    sd.precision_mode = mode
    sd.precision = 1e-6
    sd.calculate_strain_during_simulation = True
    sd.external_stress = pkg.FixedRateProtocol(0.08, 0.0)
    e = pkg.Engine(sd)
    e.set_overlap(overlap)
    r = e.advance(steps)
    xe, _ = e.positions()
    st = e.lu_stats()
    e.close()
    return r, xe, st


@pytest.mark.parametrize("form,n,seed", [("fp64", 256, 11), ("fp64", 600, 12),
                                         ("mixed", 2048, 12)])
def test_overlap_matches_sequential(pkg, form, n, seed):
    """(The mixed form's FP32 factorisations run from N = 2048 on.)"""
    mode = pkg._lib.D4_PREC_MIXED if form == "mixed" else pkg._lib.D4_PREC_FP64
    ra, xa, sa = run(pkg, mode, True, n, seed, 12)
    rb, xb, sb = run(pkg, mode, False, n, seed, 12)
    assert (ra.successful_steps, ra.failed_steps) == (rb.successful_steps, rb.failed_steps)
    assert ra.sim_time == rb.sim_time and ra.step_size == rb.step_size
    assert ra.strain == rb.strain
    assert np.array_equal(xa, xb)
    assert sa == sb
    if form == "fp64":
        assert sa["factorizations"] == 3 * ra.attempts


@pytest.mark.parametrize("form", ["fp64", "mixed"])
def test_overlap_single_attempt(pkg, form):
    """One attempt from the same state: every stage's positions, the error
    ratio and the refined residual agree bit for bit."""
    mode = pkg._lib.D4_PREC_MIXED if form == "mixed" else pkg._lib.D4_PREC_FP64
    x, y, _ = pkg.dconf.generate_internal(2048 if form == "mixed" else 512, 1002)
    out = []
    for overlap in (True, False):
        sd = pkg.SimulationData()
        sd.set_positions(x, y)
        sd.precision_mode = mode
        sd.external_stress = pkg.FixedRateProtocol(0.1, 0.0)
        e = pkg.Engine(sd)
        e.set_overlap(overlap)
        out.append(e.attempt(0.0, 1e-7))
        e.close()
    (ra, *xa), (rb, *xb) = out
    for a, b in zip(xa, xb):
        assert np.array_equal(a, b)
    assert ra.ratio == rb.ratio and ra.max_id == rb.max_id
    assert ra.refine_residual == rb.refine_residual
    if form == "mixed":
        assert 0 < ra.refine_residual < 1e-10
