"""The command line (``python -m 2d4_b200``) against the reference program's
option handling (src/project_parser.cpp:28-333): defaults, the mapping of
every flag onto SimulationData, the checks with their messages and exit
statuses, and the stress-protocol selection.  The parse tests need no GPU; the
last test runs the N=64 golden case through the command line on the GPU and
holds the written configuration to the reference's run (1e-10, as the run
tests do)."""
import importlib
import io
import os

import numpy as np
import pytest

cli = importlib.import_module("2d4_b200.cli")


@pytest.fixture
def conf(tmp_path, pkg):
    x, y, _ = pkg.dconf.generate_internal(16, 5)
    path = str(tmp_path / "in.dconf")
    pkg.dconf.write_internal(path, x, y, np.arange(16, dtype=np.uint32))
    return path, str(tmp_path / "out.dconf"), tmp_path


def parse(argv):
    return cli.parse(["-c"] + argv, io.StringIO())


def stop(argv):
    with pytest.raises(cli.CliExit) as e:
        parse(argv)
    return e.value


def test_defaults(conf, pkg):
    i, o, _ = conf
    args, sd = parse(["-I", i, "-O", o])
    assert (sd.precision, sd.dipole_precision, sd.cutoff_multiplier) == (1e-5, 0.05, 1e20)
    assert sd.step_size == sd.initial_step_size == 1e-6
    assert sd.weight_function == "c" and not sd.heaviside_cutoff
    assert not (sd.time_limited or sd.step_count_limited or sd.strain_increase_limted
                or sd.max_step_size_limited or sd.count_avalanches or sd.save_sub_configs)
    assert type(sd.external_stress) is pkg.StressProtocol
    assert sd.final_dislocation_configuration_path == o and os.path.exists(o)
    assert sd.dislocation_count == 16
    assert sd.precision_mode == pkg._lib.D4_PREC_FP64


def test_flags_map_onto_simulation_data(conf, pkg):
    i, o, tmp = conf
    log = str(tmp / "run.log")
    args, sd = parse(["-I", i, "-O", o, "-P1e-8", "-p", "0", "-u", "6.4", "-h", "-w", "m",
                      "--initial-stepsize", "1e-7", "-M", "0.5", "-t", "200", "-C", "999",
                      "--strain-increase-limit", "0.3", "--avalanche-detection-limit", "4",
                      "--avalanche-speed-threshold", "2e-3", "-S", "-l", "-L", log,
                      "-o", str(tmp / "sub"), "-N", "7", "-T", "2.5", "-b", "b", "-n", "3",
                      "--precision-mode", "mixed", "--solver", "auto", "--field", "tabulated",
                      "--table-size", "512"])
    assert sd.precision == 1e-8 and sd.dipole_precision == 0.0
    assert sd.cutoff_multiplier == 6.4 and sd.heaviside_cutoff and sd.weight_function == "m"
    assert sd.step_size == sd.initial_step_size == 1e-7
    assert sd.max_step_size_limited and sd.max_stepsize_limit == 0.5
    assert sd.time_limited and sd.time_limit == 200
    assert sd.step_count_limited and sd.step_count_limit == 999
    assert sd.strain_increase_limted and sd.total_accumulated_strain_increase_limit == 0.3
    assert sd.count_avalanches and sd.trigger_limit_for_avalanche_count == 4
    assert sd.avalanche_speed_threshold == 2e-3
    assert sd.calculate_strain_during_simulation and sd.calculate_order_parameter
    assert sd.logfile_path == log and os.path.exists(log)
    assert sd.save_sub_configs and sd.sub_config_path == str(tmp / "sub")
    assert (sd.sub_config_delay, sd.sub_config_times, sd.sub_config_times_type) == (7, 2.5, "b")
    assert sd.sub_config_delay_during_avalanche == 3
    assert sd.precision_mode == pkg._lib.D4_PREC_MIXED
    assert sd.solver == pkg._lib.D4_SOLVER_AUTO and sd.field == pkg._lib.D4_FIELD_TABULATED
    assert sd.table_size == 512


def test_long_name_prefixes(conf):
    i, o, _ = conf
    _, sd = parse(["--dislocation-conf", i, "--result-dis", o, "--position-prec", "3e-6"])
    assert sd.precision == 3e-6


@pytest.mark.parametrize("argv,kind", [
    ([], "none"),
    (["-s", "0.1"], "none"),  # -s alone: the base protocol, zero stress at all times
    (["-s", "0.1", "-r", "0"], "fixed"),
    (["-s", "0.1", "-r", "1e-3", "-i", "2"], "cyclic"),
    (["-s", "0.1", "-r", "1e-3", "-i", "2", "-A", "0.5"], "increasing"),
])
def test_protocol_selection(conf, pkg, argv, kind):
    i, o, _ = conf
    _, sd = parse(["-I", i, "-O", o] + argv)
    cls = {"none": pkg.StressProtocol, "fixed": pkg.FixedRateProtocol,
           "cyclic": pkg.CyclicLoadProtocol, "increasing": pkg.IncreasingCyclicLoadProtocol}
    assert type(sd.external_stress) is cls[kind]
    if kind == "none":
        assert sd.external_stress.ext_stress(10.0) == 0.0
    else:
        assert sd.external_stress.init_ext_stress == 0.1


@pytest.mark.parametrize("argv,status,text", [
    (["-A", "1"], 255, "apmlitude-rate is set then cyclic-external-stress"),
    (["-A", "1", "-i", "2"], 255, "fixed-rate-external-stress must be also set"),
    (["-i", "2"], 255, "fixed-rate-external-stress must be also set"),
    (["-w", "x"], 255, "Unsupported weight-function x"),
    (["-o", "sub", "-T", "0"], 254, "T<=0"),
    (["-o", "sub", "-T", "0.5", "-b", "b"], 254, "T<1"),
    (["--point-defect-configuration", "pd"], 255, "point defects"),
    (["--no-such-option", "1"], 255, "unrecognized"),
    (["-C", "-3"], 255, ""),
])
def test_checks(conf, argv, status, text):
    i, o, _ = conf
    e = stop(["-I", i, "-O", o] + argv)
    assert e.status == status and text in e.message


def test_required_and_files(conf):
    i, o, tmp = conf
    assert stop(["-O", o]).message == "dislocation-configuration is missing!"
    assert stop(["-I", i]).message == "result-dislocation-configuration is missing!"
    log = tmp / "exists.log"
    log.write_text("old")
    e = stop(["-I", i, "-O", o, "-L", str(log)])
    assert e.status == 255 and e.message == "Error: %s exists. Program terminates." % log
    _, sd = parse(["-I", i, "-O", o, "-L", str(log), "-W"])  # -W: overwritten
    assert sd.logfile_path == str(log) and log.read_text() == ""
    e = stop(["-I", i, "-O", str(tmp / "no" / "such" / "dir" / "out.dconf")])
    assert e.status == 255 and e.message.startswith("Cannot create result dislocation")


def test_help_and_banner():
    out = io.StringIO()
    assert cli.main(["--help"], out, io.StringIO()) == 0
    text = out.getvalue()
    assert "2d4_b200:" in text.splitlines()[0] and "--position-precision" in text
    out = io.StringIO()
    assert cli.main(["-c", "--help"], out, io.StringIO()) == 0
    assert not out.getvalue().startswith("2d4_b200:")


@pytest.mark.gpu
def test_cli_run_c1_vs_reference(pkg, golden, tmp_path):
    """-P 1e-8 -C 999 on the N=64 fixture through the command line: 1000
    accepted steps (the reference's -C rule), the limit message, and the
    written configuration within 1e-10 of the reference's run."""
    x, y = golden["fix64_x"], golden["fix64_y"]
    inp, outp = str(tmp_path / "in.dconf"), str(tmp_path / "out.dconf")
    pkg.dconf.write_internal(inp, x, y, np.arange(len(x), dtype=np.uint32))
    out, err = io.StringIO(), io.StringIO()
    assert cli.main(["-c", "-I", inp, "-O", outp, "-P", "1e-8", "-C", "999"], out, err) == 0
    text = out.getvalue()
    ref = golden["fix64_run_res"]
    assert "step-count-limit (999) has been reached, succesfulSteps = 1000" in text
    assert "Simulation is done (" in text and " and %d steps)." % (int(ref[2]) + int(ref[3])) in text
    xo, yo, _ = pkg.dconf.load(outp)
    d, _, _, _ = pkg.dconf.conf_compare(xo, yo, golden["fix64_run_x"], y)
    assert d < 1e-10
