"""Command line of the engine, flag for flag the reference program's.

``python -m 2d4_b200 -I in.dconf -O out.dconf -P 1e-8 -C 999 ...`` takes the
options of the reference's 2D4_sim (option table src/project_parser.cpp:28-77,
processing src/project_parser.cpp:155-333, driver src/main.cpp:6-18), so run
scripts written for it drive the GPU engine unchanged:

- the same long and short names, defaults, unambiguous long-name prefixes and
  sticky short values (``-P1e-8``), as Boost.program_options accepts them;
- the same checks in the same order, with the reference's messages and exit
  statuses (``exit(-1)`` is 255, ``exit(-2)`` is 254): missing -I/-O, an
  unknown weight function, an existing log file without -W, sub-configuration
  times that cannot be reached, and the stress-protocol combinations;
- the same protocol selection, including that ``-s`` without ``-r`` gives the
  base protocol, whose stress is 0 at all times (stress_protocol.cpp:13-16);
- ``-C n`` stops after n + 1 accepted steps (simulation.cpp:736), as the
  reference's loop does; the engine's run loop keeps that rule;
- the start and end lines and the limit messages of Simulation::run and
  Simulation::interrupt (simulation.cpp:34-37,280,722-750).

Options with no counterpart in the reference select the engine's forms:
``--precision-mode fp64|mixed``, ``--solver dense|gmres|auto``,
``--field analytic|tabulated``, ``--table-size``, ``--device``.
``--point-defect-configuration`` is rejected: the reference's point-defect
code does not compile.  ``--spring-constant`` is accepted and has no effect,
as in the reference (declared, never read).  The licence text the reference
prints is replaced by a one-line banner, hidden by -c as there.
"""
import argparse
import os
import sys
import time

from . import _lib
from .simulation import (CyclicLoadProtocol, FixedRateProtocol, IncreasingCyclicLoadProtocol,
                         SimulationData, StressProtocol)

EXIT_ERR = 255    # exit(-1)
EXIT_ERR2 = 254   # exit(-2)


class CliExit(Exception):
    """A stop of the command line before any simulation: message and status."""

    def __init__(self, message, status=EXIT_ERR, stream="err"):
        super().__init__(message)
        self.message, self.status, self.stream = message, status, stream


def _char(v):
    if len(v) != 1:
        raise argparse.ArgumentTypeError("'%s' is not a single character" % v)
    return v


def _unsigned(v):
    n = int(v)
    if n < 0:
        raise argparse.ArgumentTypeError("'%s' is not an unsigned integer" % v)
    return n


class _Parser(argparse.ArgumentParser):
    def error(self, message):
        raise CliExit(message)


def build_parser():
    """The option table of src/project_parser.cpp:28-77 (defaults included),
    plus the engine's own selectors."""
    p = _Parser(prog="2d4_b200", add_help=False, allow_abbrev=True)
    a = p.add_argument
    # required (checked by name after parsing, as the reference does)
    a("-I", "--dislocation-configuration", metavar="PATH")
    a("-O", "--result-dislocation-configuration", metavar="PATH")
    # input / output
    a("-L", "--logfile-path", metavar="PATH")
    a("-W", "--logfile-overwrite", action="store_true")
    a("-o", "--save-sub-configurations", metavar="PREFIX")
    a("-N", "--sub-configuration-delay", type=_unsigned, default=5)
    a("-T", "--sub-config-times", type=float)
    a("-b", "--sub-config-times-type", type=_char, default="a")
    a("-n", "--sub-configuration-delay-during-avalanche", type=_unsigned, default=1)
    a("--point-defect-configuration", metavar="PATH")
    # precision
    a("-P", "--position-precision", type=float, default=1e-5)
    a("-u", "--cutoff-multiplier", type=float, default=1e20)
    a("-h", "--heaviside-cutoff", action="store_true")
    a("--initial-stepsize", type=float, default=1e-6)
    a("-M", "--max-stepsize", type=float)
    a("-w", "--weight-function", type=_char, default="c")
    a("-p", "--dipole-precision", type=float, default=0.05)
    # limits
    a("-t", "--time-limit", type=float)
    a("-C", "--step-count-limit", type=_unsigned)
    a("--strain-increase-limit", type=float)
    a("--avalanche-detection-limit", type=_unsigned)
    # in-run analysis
    a("-S", "--calculate-strain", action="store_true")
    a("--avalanche-speed-threshold", type=float, default=1e-3)
    a("-l", "--calculate-order-parameter", action="store_true")
    # external stress
    a("-s", "--const-external-stress", type=float, default=0.0)
    a("-r", "--fixed-rate-external-stress", type=float)
    a("-i", "--cyclic-external-stress", type=float)
    a("-A", "--amplitude-rate", type=float)
    a("--spring-constant", type=float)
    # general
    a("--help", action="store_true")
    a("-c", "--hide-copyright", action="store_true")
    # the engine's forms (no counterpart in the reference)
    a("--precision-mode", choices=("fp64", "mixed"), default="fp64")
    a("--solver", choices=("dense", "gmres", "auto"), default="dense")
    a("--field", choices=("analytic", "tabulated"), default="analytic")
    a("--table-size", type=int, default=1024)
    a("--device", type=int, default=0)
    return p


def _protocol(args):
    """Protocol selection of src/project_parser.cpp:286-326."""
    s = args.const_external_stress
    if args.amplitude_rate is not None:
        if args.cyclic_external_stress is None:
            raise CliExit("Error: if apmlitude-rate is set then cyclic-external-stress must be "
                          "also set. Program terminates.")
        if args.fixed_rate_external_stress is None:
            raise CliExit("Error: if cyclic-external-stress is set then "
                          "fixed-rate-external-stress must be also set. Program terminates.")
        return IncreasingCyclicLoadProtocol(s, args.fixed_rate_external_stress,
                                            args.cyclic_external_stress, args.amplitude_rate)
    if args.cyclic_external_stress is not None:
        if args.fixed_rate_external_stress is None:
            raise CliExit("Error: if cyclic-external-stress is set then "
                          "fixed-rate-external-stress must be also set. Program terminates.")
        return CyclicLoadProtocol(s, args.fixed_rate_external_stress, args.cyclic_external_stress)
    if args.fixed_rate_external_stress is not None:
        return FixedRateProtocol(s, args.fixed_rate_external_stress)
    return StressProtocol(s)  # zero at all times, whatever -s says


def parse(argv, out=None):
    """Options -> (args, SimulationData), with the reference's checks in its
    order (src/project_parser.cpp:105-333).  Creates the result file and the
    log file as the reference does at this point (so a bad path stops before
    the run).  Raises CliExit for every stop (--help included: status 0)."""
    out = out or sys.stdout
    p = build_parser()
    args = p.parse_args(argv)
    if not args.hide_copyright:
        print("2d4_b200: B200 engine for the 2D4_sim implicit step (the reference's "
              "command line; -c hides this line)", file=out)
    if args.help:
        raise CliExit(p.format_help(), 0, "out")
    if not args.dislocation_configuration:
        raise CliExit("dislocation-configuration is missing!")
    if not args.result_dislocation_configuration:
        raise CliExit("result-dislocation-configuration is missing!")
    if args.point_defect_configuration:
        raise CliExit("Error: point defects are not supported (the reference's point-defect "
                      "code does not compile). Program terminates.")
    try:
        sd = SimulationData(args.dislocation_configuration)
    except (OSError, ValueError) as e:
        raise CliExit(str(e))
    if args.time_limit is not None:
        sd.time_limited, sd.time_limit = True, args.time_limit
    sd.step_size = sd.initial_step_size = args.initial_stepsize
    sd.precision = args.position_precision
    sd.dipole_precision = args.dipole_precision
    sd.weight_function = args.weight_function
    if sd.weight_function not in ("c", "p", "m"):
        raise CliExit("Unsupported weight-function %s, supported values are c, p and m. "
                      "Program terminates." % sd.weight_function)
    sd.cutoff_multiplier = args.cutoff_multiplier
    sd.heaviside_cutoff = args.heaviside_cutoff
    if args.strain_increase_limit is not None:
        sd.strain_increase_limted = True
        sd.total_accumulated_strain_increase_limit = args.strain_increase_limit
    if args.max_stepsize is not None:
        sd.max_step_size_limited, sd.max_stepsize_limit = True, args.max_stepsize
    sd.calculate_strain_during_simulation = args.calculate_strain
    sd.calculate_order_parameter = args.calculate_order_parameter
    if args.logfile_path:
        f = args.logfile_path
        if not args.logfile_overwrite and os.path.exists(f):
            raise CliExit("Error: %s exists. Program terminates." % f)
        try:
            open(f, "w").close()
        except OSError:
            raise CliExit("Error: cannot create logfile for writing with name %s. "
                          "Program terminates." % f)
        sd.logfile_path = f
    if args.step_count_limit is not None:
        sd.step_count_limited, sd.step_count_limit = True, args.step_count_limit
    if args.avalanche_detection_limit is not None:
        sd.count_avalanches = True
        sd.trigger_limit_for_avalanche_count = args.avalanche_detection_limit
        sd.avalanche_speed_threshold = args.avalanche_speed_threshold
    if args.save_sub_configurations:
        sd.save_sub_configs = True
        sd.sub_config_path = args.save_sub_configurations
        sd.sub_config_delay = args.sub_configuration_delay
        sd.sub_config_times_type = args.sub_config_times_type
        if args.sub_config_times is not None:
            sd.sub_config_times = args.sub_config_times
            if sd.sub_config_times_type == "a" and sd.sub_config_times <= 0:
                raise CliExit("Error: T<=0 but subconfigs are asked to be printed out at T*n. "
                              "Please use T>0 or `sub-config-times-type -b` with T>1 to print "
                              "out subconfigs at initial-stepsize * T^n.\nProgram terminates.",
                              EXIT_ERR2)
            if sd.sub_config_times_type == "b" and sd.sub_config_times < 1:
                raise CliExit("Error: T<1 but subconfigs are asked to be printed out at "
                              "initial-stepsize * T^n. Please use T>1 or `sub-config-times-type "
                              "-a` with T>0 to print out subconfigs at T*n.\nProgram terminates.",
                              EXIT_ERR2)
        else:
            sd.sub_config_times = 0.0
        sd.sub_config_delay_during_avalanche = args.sub_configuration_delay_during_avalanche
    sd.final_dislocation_configuration_path = args.result_dislocation_configuration
    try:
        open(sd.final_dislocation_configuration_path, "w").close()
    except OSError:
        raise CliExit("Cannot create result dislocation configuration file at %s. Program "
                      "terminates." % sd.final_dislocation_configuration_path)
    sd.external_stress = _protocol(args)
    sd.precision_mode = {"fp64": _lib.D4_PREC_FP64, "mixed": _lib.D4_PREC_MIXED}[args.precision_mode]
    sd.solver = {"dense": _lib.D4_SOLVER_DENSE, "gmres": _lib.D4_SOLVER_GMRES,
                 "auto": _lib.D4_SOLVER_AUTO}[args.solver]
    sd.field = {"analytic": _lib.D4_FIELD_ANALYTIC,
                "tabulated": _lib.D4_FIELD_TABULATED}[args.field]
    sd.table_size = args.table_size
    return args, sd


def _stop_message(sd, r):
    """The line Simulation::interrupt prints for the limit that ended the run
    (src/simulation.cpp:722-750), from the run's totals; None if no limit did."""
    if sd.time_limited and r.sim_time > sd.time_limit:
        return "time-limit (%g) has been reached, simTime = %g" % (sd.time_limit, r.sim_time)
    if sd.strain_increase_limted and (sd.total_accumulated_strain_increase >
                                      sd.total_accumulated_strain_increase_limit):
        return "strain-increase-limit (%g) has been reached, strain = %g" % (
            sd.total_accumulated_strain_increase_limit, sd.total_accumulated_strain_increase)
    if sd.step_count_limited and r.successful_steps > sd.step_count_limit:
        return "step-count-limit (%d) has been reached, succesfulSteps = %d" % (
            sd.step_count_limit, r.successful_steps)
    if sd.count_avalanches:
        return "avalanche-detection-limit (%d) has been reached" % sd.trigger_limit_for_avalanche_count
    return None


def main(argv=None, out=None, err=None):
    """Runs the program; returns the exit status (src/main.cpp:6-18)."""
    from .simulation import Simulation

    out, err = out or sys.stdout, err or sys.stderr
    try:
        args, sd = parse(sys.argv[1:] if argv is None else argv, out)
    except CliExit as e:
        print(e.message, file=out if e.stream == "out" else err)
        return e.status
    print("Simulation started on %s\n" % time.ctime(), file=out)
    wall0 = time.time()
    sim = Simulation(sd, device=args.device)
    try:
        r = sim.run()
    finally:
        sim.engine.close()
    msg = _stop_message(sd, r)
    if msg:
        print(msg, file=out)
    print("Simulation is done (%g s and %d steps)." % (time.time() - wall0,
                                                       r.successful_steps + r.failed_steps),
          file=out)
    return 0
