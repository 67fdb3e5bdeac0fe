"""The plain FP64 form against runs of the reference itself (marked gpu).

Fixtures: tests/golden/golden_runs.npz, written by
tests/golden/make_golden_runs.py from the reference core built from its own
sources.  Parity bar: identical accepted and failed step counts and positions
within 1e-10 (conf_compare's periodic max |dx|), the bar of the plain form.

The dynamics are chaotic: the FP64 form started from positions moved by 1e-15
departs from its own unperturbed run by 2.4e-11 after 100 steps of the headline
workload and by 2e-6 after 150, and the engine differs from the reference's
glibc build in the last bit of some exp/cos results.  So each run is compared
over a horizon inside which that sensitivity stays below the bar, and the
quantities that are small differences of two solutions (the error ratio, hence
the step size and the simulation time) get a relative bar of 1e-7.
  - the headline workload's own step sequence: 100 accepted steps at constant
    stress 0.05 from the relaxed N=1024 state (src/simulation.cpp:30-281);
  - N=4096, dense, tau = 0.1, 20 accepted steps;
  - the 15-column log of a 100-step run with strain and order parameter on,
    column by column (10 and 14 are wall times and are only checked for
    sanity), and its sub-configuration dumps by name and content
    (src/simulation.cpp:52-83,184-247, src/simulation_data.cpp:231-246);
  - a run stopped by the avalanche detection limit (src/simulation.cpp:215-230,
    722-750).
"""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))


@pytest.fixture(scope="module")
def gr():
    return np.load(os.path.join(HERE, "golden", "golden_runs.npz"))


def sim_data(pkg, x, y, **kw):
    sd = pkg.SimulationData()
    sd.set_positions(x, y)
    for k, v in kw.items():
        setattr(sd, k, v)
    return sd


def test_c2_headline_trajectory(pkg, gr):
    z = np.load(os.path.join(HERE, "golden", "c2_relaxed_1024.npz"))
    x, y = z["x"], z["y"]
    e = pkg.Engine(sim_data(pkg, x, y, external_stress=pkg.FixedRateProtocol(0.05, 0.0)))
    r = e.advance(100)
    ref = gr["c2_res"]
    assert (r.successful_steps, r.failed_steps) == (int(ref[2]), int(ref[3]))
    assert abs(r.sim_time - ref[0]) <= 1e-7 * ref[0]
    d, i, _, _ = pkg.dconf.conf_compare(e.positions()[0], y, gr["c2_x"], y)
    assert d < 1e-10, (d, i)
    e.close()


def test_n4096_fp64_trajectory(pkg, gr):
    x, y, _ = pkg.dconf.generate_internal(4096, 1002)
    e = pkg.Engine(sim_data(pkg, x, y, external_stress=pkg.FixedRateProtocol(0.1, 0.0)))
    r = e.advance(20)
    ref = gr["c3_res"]
    assert (r.successful_steps, r.failed_steps) == (int(ref[2]), int(ref[3]))
    d, i, _, _ = pkg.dconf.conf_compare(e.positions()[0], y, gr["c3_x"], y)
    assert d < 1e-10, (d, i)
    e.close()


def parse_log(path):
    rows = []
    with open(path) as f:
        for line in f:
            if line.startswith("#"):
                continue
            t = line.rstrip("\n").split("\t")
            rows.append([np.nan if v.strip() == "-" else float(v) for v in t[:15]])
    return np.array(rows)


def test_log_and_sub_configurations(pkg, golden, gr, tmp_path):
    sd = sim_data(pkg, golden["fix64_x"], golden["fix64_y"], precision=1e-6,
                  step_count_limited=True, step_count_limit=99,
                  external_stress=pkg.FixedRateProtocol(0.1, 0.0),
                  calculate_strain_during_simulation=True, calculate_order_parameter=True,
                  save_sub_configs=True, sub_config_path=str(tmp_path / "sub_"),
                  sub_config_delay=5, sub_config_times=2e-4, sub_config_times_type="a",
                  logfile_path=str(tmp_path / "run.log"))
    sd.order = golden["fix64_order"]
    sim = pkg.Simulation(sd)
    r = sim.run()
    ref = gr["log_res"]
    assert (r.successful_steps, r.failed_steps) == (int(ref[2]), int(ref[3]))
    rows, want = parse_log(str(tmp_path / "run.log")), gr["log_rows"]
    assert rows.shape == want.shape
    exact = [1, 2, 4]  # successfulSteps, failedSteps, maxErrorRatioID
    # simTime, maxErrorRatioSqr and stepSize follow the error ratio
    close = {0: 1e-7, 3: 1e-7, 14: 1e-7, 5: 1e-9, 6: 1e-9, 7: 1e-9, 8: 1e-9, 10: 1e-9, 11: 1e-9,
             12: 1e-9}
    assert np.array_equal(rows[:, exact], want[:, exact])
    for col, bar in close.items():
        a, b = rows[:, col], want[:, col]
        assert np.array_equal(np.isnan(a), np.isnan(b)), col
        m = ~np.isnan(b)
        assert np.all(np.abs(a[m] - b[m]) <= bar * np.maximum(np.abs(b[m]), 1e-6)), col
    # wall-time columns: '-' in the first row, then non-negative seconds, the
    # elapsed time non-decreasing
    assert np.isnan(rows[0, 9]) and np.all(rows[1:, 9] >= 0)
    assert rows[0, 13] == 0 and np.all(np.diff(rows[:, 13]) >= 0)
    names = sorted(f[len("sub_"):] for f in os.listdir(tmp_path) if f.startswith("sub_"))
    assert names == list(gr["log_sub_names"])
    for k, nm in enumerate(names):
        got = np.loadtxt(str(tmp_path / ("sub_" + nm)), ndmin=2)
        want_k = gr["log_sub_%d" % k]
        assert np.array_equal(got[:, 2], want_k[:, 2])
        d = np.abs(got[:, :2] - want_k[:, :2])
        assert np.minimum(d, 1 - d).max() < 1e-10, nm


def test_avalanche_limit_run(pkg, golden, gr):
    sd = sim_data(pkg, golden["fix64_x"], golden["fix64_y"], precision=1e-8,
                  count_avalanches=True, trigger_limit_for_avalanche_count=0,
                  avalanche_speed_threshold=0.05)
    e = pkg.Engine(sd)
    r = e.run()
    ref = gr["aval_res"]
    assert (r.successful_steps, r.failed_steps) == (int(ref[2]), int(ref[3]))
    assert abs(r.sim_time - ref[0]) <= 1e-7 * ref[0]
    # 6502 accepted steps of relaxation at P = 1e-8: the same step counts and
    # final positions within 1e-9, a tenth of the run's own position precision
    d, _, _, _ = pkg.dconf.conf_compare(e.positions()[0], golden["fix64_y"], gr["aval_x"],
                                        golden["fix64_y"])
    assert d < 1e-9
    e.close()
