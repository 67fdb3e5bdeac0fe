/*
 * d4ref: command-line front end of the reference-core oracle.  TEST AND
 * BASELINE INFRASTRUCTURE ONLY.
 *
 * Accepts the subset of the reference's flags (src/project_parser.cpp:28-68)
 * that the stepping loop reads, resolves them the way processInput does
 * (src/project_parser.cpp:176-326; note that -s alone selects the base
 * StressProtocol, which returns 0, and that -C n stops after n+1 accepted
 * steps, src/simulation.cpp:736), runs Simulation::run and prints one JSON line
 * with the counts and the wall time of the stepping loop (file I/O excluded).
 */
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>

#include "ref_driver.h"

static void usage() {
    std::fprintf(stderr,
                 "usage: d4ref -I in.dconf -O out.dconf [-L log] [-P prec] [-p dipole_prec]\n"
                 "             [-u cutoff_mult] [-h] [--initial-stepsize h0] [-M max_h]\n"
                 "             [-w c|p|m] [-t time_limit] [-C step_count_limit]\n"
                 "             [--strain-increase-limit s] [-S] [-l] [-s tau0] [-r rate]\n"
                 "             [-i period] [-A amplitude_rate] [-c]\n");
}

int main(int argc, char **argv) {
    d4ref_params p;
    d4ref_default_params(&p);
    std::string in, out, log;
    for (int k = 1; k < argc; ++k) {
        std::string a = argv[k];
        auto val = [&](void) -> const char * {
            if (k + 1 >= argc) {
                usage();
                std::exit(-1);
            }
            return argv[++k];
        };
        if (a == "-I" || a == "--dislocation-configuration") in = val();
        else if (a == "-O" || a == "--result-dislocation-configuration") out = val();
        else if (a == "-L" || a == "--logfile-path") log = val();
        else if (a == "-P" || a == "--position-precision") p.position_precision = std::atof(val());
        else if (a == "-p" || a == "--dipole-precision") p.dipole_precision = std::atof(val());
        else if (a == "-u" || a == "--cutoff-multiplier") p.cutoff_multiplier = std::atof(val());
        else if (a == "-h" || a == "--heaviside-cutoff") p.heaviside_cutoff = 1;
        else if (a == "--initial-stepsize") p.initial_stepsize = std::atof(val());
        else if (a == "-M" || a == "--max-stepsize") p.max_stepsize = std::atof(val());
        else if (a == "-w" || a == "--weight-function") p.weight_function = val()[0];
        else if (a == "-t" || a == "--time-limit") p.time_limit = std::atof(val());
        else if (a == "-C" || a == "--step-count-limit") p.step_count_limit = std::atoll(val());
        else if (a == "--strain-increase-limit") p.strain_increase_limit = std::atof(val());
        else if (a == "-S" || a == "--calculate-strain") p.calculate_strain = 1;
        else if (a == "-l" || a == "--calculate-order-parameter") p.calculate_order_parameter = 1;
        else if (a == "-s" || a == "--const-external-stress") p.const_external_stress = std::atof(val());
        else if (a == "-r" || a == "--fixed-rate-external-stress") {
            p.has_rate = 1;
            p.rate = std::atof(val());
        } else if (a == "-i" || a == "--cyclic-external-stress") {
            p.has_cyclic = 1;
            p.cyclic_period = std::atof(val());
        } else if (a == "-A" || a == "--amplitude-rate") {
            p.has_amplitude_rate = 1;
            p.amplitude_rate = std::atof(val());
        } else if (a == "-c" || a == "--hide-copyright" || a == "-W" || a == "--logfile-overwrite") {
        } else {
            usage();
            return -1;
        }
    }
    if (in.empty() || out.empty()) {
        usage();
        return -1;
    }
    if (p.weight_function != 'c' && p.weight_function != 'p' && p.weight_function != 'm') {
        std::fprintf(stderr, "Unsupported weight-function %c\n", p.weight_function);
        return -1;
    }
    d4ref_result r;
    double wall = 0;
    d4ref_run(in.c_str(), out.c_str(), log.empty() ? nullptr : log.c_str(), &p, &r, nullptr,
              nullptr, &wall);
    std::printf(
        "{\"n\": %d, \"successful_steps\": %lld, \"failed_steps\": %lld, \"sim_time\": %.17g, "
        "\"step_size\": %.17g, \"strain\": %.17g, \"wall_s\": %.6f}\n",
        r.n, r.successful_steps, r.failed_steps, r.sim_time, r.step_size, r.strain, wall);
    return 0;
}
