"""GPU checks of the batched ensemble (d4_ensemble_*, marked gpu).

Every instance of an ensemble runs the single-system engine's arithmetic: the
same pair tiles and ordered row sums, and a one-CTA LU and substitutions that
give every entry its updates in the oracle's order.  So each instance must
reproduce the single-system engine's run bit for bit (same accept/reject
sequence, same positions), uneven sizes mixed in one ensemble, and the
reference's own N=64 runs within 1e-10 (the engine's bound against the
reference).  Interrupting by time limit and continuing in several calls must
not change anything.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def make_sd(pkg, **kw):
    sd = pkg.SimulationData()
    for k, v in kw.items():
        setattr(sd, k, v)
    return sd


def single(pkg, x, y, **kw):
    sd = make_sd(pkg, **kw)
    sd.set_positions(x, y)
    e = pkg.Engine(sd)
    r = e.run()
    xr, _ = e.positions()
    e.close()
    return xr, r


def configs(pkg, golden):
    out = [(golden["fix64_x"], golden["fix64_y"]), (golden["seed64_x"], golden["seed64_y"])]
    for n, seed in ((96, 5), (250, 6), (128, 7), (40, 8)):
        x, y, _ = pkg.dconf.generate_internal(n, seed)
        out.append((x, y))
    return out


def test_ensemble_matches_single_engine(pkg, golden):
    kw = dict(precision=1e-6, step_count_limited=True, step_count_limit=29,
              calculate_strain_during_simulation=True,
              external_stress=pkg.FixedRateProtocol(0.05, 0.0))
    cfg = configs(pkg, golden)
    ens = pkg.Ensemble(make_sd(pkg, **kw), cfg)
    res = ens.run()
    for k, (x, y) in enumerate(cfg):
        xs, rs = single(pkg, x, y, **kw)
        r = res[k]
        assert (r.successful_steps, r.failed_steps) == (rs.successful_steps, rs.failed_steps), k
        assert r.sim_time == rs.sim_time and r.step_size == rs.step_size, k
        assert r.strain == rs.strain, k
        xe, ye = ens.positions(k)
        assert np.array_equal(xe, xs), k
        assert np.array_equal(ye, y)
    ens.close()


def test_ensemble_c1_vs_reference(pkg, golden):
    """The N=64 configuration (P = 1e-8, 1000 accepted steps) for both golden
    systems in one ensemble, against the reference's runs."""
    kw = dict(precision=1e-8, step_count_limited=True, step_count_limit=999)
    cases = ["fix64", "seed64"]
    ens = pkg.Ensemble(make_sd(pkg, **kw), [(golden[c + "_x"], golden[c + "_y"]) for c in cases])
    res = ens.run()
    for k, c in enumerate(cases):
        ref = golden[c + "_run_res"]
        assert (res[k].successful_steps, res[k].failed_steps) == (int(ref[2]), int(ref[3]))
        xe, _ = ens.positions(k)
        d, _, _, _ = pkg.dconf.conf_compare(xe, golden[c + "_y"], golden[c + "_run_x"],
                                            golden[c + "_y"])
        assert d < 1e-10
    ens.close()


def test_ensemble_time_limit_and_continuation(pkg, golden):
    """Stress ramp tau = 1e-3 t with a time limit (the ensemble workload's
    protocol); one call, or three rounds then the rest, give the same result,
    equal to single-system runs."""
    kw = dict(precision=1e-6, time_limited=True, time_limit=2e-3,
              external_stress=pkg.FixedRateProtocol(0.0, 1e-3))
    cfg = configs(pkg, golden)[:4]
    a = pkg.Ensemble(make_sd(pkg, **kw), cfg)
    ra = a.run()
    b = pkg.Ensemble(make_sd(pkg, **kw), cfg)
    rb3 = b.run(3)
    assert all(r.attempts == 3 for r in rb3)
    rb = b.run()
    for k, (x, y) in enumerate(cfg):
        assert ra[k].sim_time > 2e-3
        assert (ra[k].successful_steps, ra[k].failed_steps, ra[k].sim_time) == (
            rb[k].successful_steps, rb[k].failed_steps, rb[k].sim_time)
        assert np.array_equal(a.positions(k)[0], b.positions(k)[0])
        xs, rs = single(pkg, x, y, **kw)
        assert (ra[k].successful_steps, ra[k].failed_steps) == (rs.successful_steps,
                                                                 rs.failed_steps)
        assert np.array_equal(a.positions(k)[0], xs)
    a.close()
    b.close()


def test_ensemble_avalanche_limit(pkg, golden):
    """--avalanche-detection-limit 0: each instance stops when its first
    avalanche (mean |v| above the threshold, then below it) ends, at the same
    step as a single-system run with the same limit.  The threshold is twice
    the mean |v| reached after 150 steps, so the relaxation's initial
    avalanche ends within the step budget."""
    cfg = configs(pkg, golden)[2:5]
    base = dict(precision=1e-6, step_count_limited=True, step_count_limit=150)
    means = []
    for x, y in cfg:
        sd = make_sd(pkg, **base)
        sd.set_positions(x, y)
        e = pkg.Engine(sd)
        e.run()
        xe, ye = e.positions()
        v, _ = e.speeds(xe, ye, 0.0)
        means.append(np.abs(v).mean())
        e.close()
    kw = dict(precision=1e-6, step_count_limited=True, step_count_limit=400,
              count_avalanches=True, trigger_limit_for_avalanche_count=0,
              avalanche_speed_threshold=2 * max(means))
    ens = pkg.Ensemble(make_sd(pkg, **kw), cfg)
    res = ens.run()
    stopped_early = 0
    for k, (x, y) in enumerate(cfg):
        xs, rs = single(pkg, x, y, **kw)
        assert (res[k].successful_steps, res[k].failed_steps) == (rs.successful_steps,
                                                                  rs.failed_steps), k
        assert np.array_equal(ens.positions(k)[0], xs), k
        stopped_early += rs.successful_steps <= 400
    assert stopped_early > 0
    ens.close()
