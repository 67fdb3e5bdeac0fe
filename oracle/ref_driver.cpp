/*
 * Driver for the reference-core oracle.  TEST INFRASTRUCTURE ONLY.
 *
 * Compiled together with the reference's own core sources (unmodified, read in
 * place by oracle/Makefile) and the project-written UMFPACK shim.  It stands in
 * for the Boost-based ProjectParser (src/project_parser.cpp:155-333) and opens
 * Simulation's private sweeps to the tests: access specifiers are widened for
 * this translation unit only, which changes no layout and no code of the
 * reference.
 */
// Standard headers first, so that only the reference's own classes are widened.
#include <algorithm>
#include <cassert>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <iomanip>
#include <iostream>
#include <map>
#include <memory>
#include <numeric>
#include <sstream>
#include <string>
#include <vector>

#define private public
#define protected public
#include "simulation.h"
#undef private
#undef protected

#include <suitesparse/umfpack.h>

#include "ref_driver.h"

using namespace sdddstCore;

extern "C" void d4ref_default_params(d4ref_params *p) {
    std::memset(p, 0, sizeof(*p));
    p->position_precision = 1e-5;
    p->dipole_precision = 0.05;
    p->cutoff_multiplier = 1e20;
    p->heaviside_cutoff = 0;
    p->initial_stepsize = 1e-6;
    p->max_stepsize = -1;
    p->weight_function = 'c';
    p->time_limit = -1;
    p->step_count_limit = -1;
    p->strain_increase_limit = -1;
    p->const_external_stress = 0;
    p->sub_config_path = nullptr;
    p->sub_config_delay = 5;
    p->sub_config_delay_during_avalanche = 1;
    p->sub_config_times = 0;
    p->sub_config_times_type = 'a';
    p->avalanche_limit = -1;
    p->avalanche_speed_threshold = 1e-3;
}

namespace {

// Mirrors ProjectParser::processInput (src/project_parser.cpp:176-326) for the
// flags in d4ref_params.
std::shared_ptr<SimulationData> make_data(const char *in_path, const d4ref_params *p,
                                          const char *log_path) {
    std::shared_ptr<SimulationData> sD(new SimulationData(in_path, ""));
    if (p->time_limit >= 0) {
        sD->isTimeLimit = true;
        sD->timeLimit = p->time_limit;
    }
    sD->stepSize = p->initial_stepsize;
    sD->initStepSize = p->initial_stepsize;
    sD->prec = p->position_precision;
    sD->dipole_prec = p->dipole_precision;
    sD->weightFunc = p->weight_function;
    sD->cutOffMultiplier = p->cutoff_multiplier;
    sD->heavisideCutoff = p->heaviside_cutoff != 0;
    sD->updateCutOff();
    if (p->strain_increase_limit >= 0) {
        sD->isStrainIncreaseLimit = true;
        sD->totalAccumulatedStrainIncreaseLimit = p->strain_increase_limit;
    }
    if (p->max_stepsize > 0) {
        sD->maxStepSizeLimit = p->max_stepsize;
        sD->isMaxStepSizeLimit = true;
    }
    sD->calculateStrainDuringSimulation = p->calculate_strain != 0;
    sD->orderParameterCalculationIsOn = p->calculate_order_parameter != 0;
    if (log_path && *log_path) sD->standardOutputLog.open(log_path);
    if (p->step_count_limit >= 0) {
        sD->isStepCountLimit = true;
        sD->stepCountLimit = (unsigned int)p->step_count_limit;
    }
    if (p->avalanche_limit >= 0) {  // src/project_parser.cpp:244-249
        sD->countAvalanches = true;
        sD->avalancheTriggerLimit = (unsigned int)p->avalanche_limit;
        sD->avalancheSpeedThreshold = p->avalanche_speed_threshold;
    }
    if (p->sub_config_path) {  // src/project_parser.cpp:251-276
        sD->isSaveSubConfigs = true;
        sD->subConfigPath = p->sub_config_path;
        sD->subConfigDelay = p->sub_config_delay;
        sD->subConfigTimesType = p->sub_config_times_type;
        sD->subConfigTimes = p->sub_config_times > 0 ? p->sub_config_times : 0;
        sD->subConfigDelayDuringAvalanche = p->sub_config_delay_during_avalanche;
        sD->nextWriteOutTime = sD->getNextWriteOutTime();
    }
    const double s = p->const_external_stress;
    if (p->has_amplitude_rate && p->has_cyclic && p->has_rate)
        sD->externalStressProtocol.reset(
            new IncreasingCyclicLoadProtocol(s, p->rate, p->cyclic_period, p->amplitude_rate));
    else if (p->has_cyclic && p->has_rate)
        sD->externalStressProtocol.reset(new CyclicLoadProtocol(s, p->rate, p->cyclic_period));
    else if (p->has_rate)
        sD->externalStressProtocol.reset(new FixedRateProtocol(s, p->rate));
    else
        sD->externalStressProtocol.reset(new StressProtocol(s));
    return sD;
}

void set_positions(SimulationData &sD, const double *x, const double *y) {
    for (unsigned i = 0; i < sD.dc; ++i) {
        sD.disl_sorted[i].x = x[i];
        sD.disl_sorted[i].y = y[i];
    }
}

}  // namespace

extern "C" int d4ref_run(const char *in_path, const char *out_path, const char *log_path,
                         const d4ref_params *p, d4ref_result *res, double *x_sorted,
                         double *y_sorted, double *wall_seconds) {
    std::shared_ptr<SimulationData> sD = make_data(in_path, p, log_path);
    sD->endDislocationConfigurationPath = out_path ? out_path : "/dev/null";
    Simulation sim(sD);
    auto t0 = std::chrono::steady_clock::now();
    sim.run();
    auto t1 = std::chrono::steady_clock::now();
    if (wall_seconds) *wall_seconds = std::chrono::duration<double>(t1 - t0).count();
    if (res) {
        res->sim_time = sD->simTime;
        res->step_size = sD->stepSize;
        res->strain = sD->totalAccumulatedStrainIncrease;
        res->successful_steps = (long long)sD->succesfulSteps;
        res->failed_steps = (long long)sD->failedSteps;
        res->n = (int)sD->dc;
    }
    for (unsigned i = 0; i < sD->dc; ++i) {
        if (x_sorted) x_sorted[i] = sD->disl_sorted[i].x;
        if (y_sorted) y_sorted[i] = sD->disl_sorted[i].y;
    }
    return 0;
}

extern "C" int d4ref_load(const char *in_path, int *n, double *x, double *y, unsigned *order,
                          int cap) {
    SimulationData sD(in_path, "");
    *n = (int)sD.dc;
    if ((int)sD.dc > cap) return -1;
    for (unsigned i = 0; i < sD.dc; ++i) {
        x[i] = sD.disl_sorted[i].x;
        y[i] = sD.disl_sorted[i].y;
        order[i] = sD.disl_order[i];
    }
    return 0;
}

extern "C" int d4ref_speeds(const char *in_path, const d4ref_params *p, const double *x,
                            const double *y, double sim_time, double *v, double *tol) {
    std::shared_ptr<SimulationData> sD = make_data(in_path, p, nullptr);
    set_positions(*sD, x, y);
    Simulation sim(sD);
    std::vector<double> forces(sD->dc);
    sim.calculateSpeedsAtTime(sD->disl_sorted, forces, sim_time);
    for (unsigned i = 0; i < sD->dc; ++i) {
        v[i] = forces[i];
        if (tol) tol[i] = sim.pH->use_dipoleCrit ? sim.pH->tolerance[i] : sim.pH->minPrecisitySq;
    }
    return 0;
}

extern "C" int d4ref_jacobian(const char *in_path, const d4ref_params *p, const double *x,
                              const double *y, double stepsize, double t_a, double t_b,
                              double *v_a, double *v_b, double *a_dense, double *dvec,
                              double *tol, int *nnz) {
    std::shared_ptr<SimulationData> sD = make_data(in_path, p, nullptr);
    set_positions(*sD, x, y);
    Simulation sim(sD);
    const unsigned n = sD->dc;
    std::vector<double> fa(n), fb(n);
    int cnt = sim.calcJacobianAndSpeedsAtTimes(stepsize, sD->disl_sorted, fa, fb, t_a, t_b);
    if (nnz) *nnz = cnt;
    std::memset(a_dense, 0, sizeof(double) * (size_t)n * n);
    for (unsigned j = 0; j < n; ++j)
        for (int q = sD->Ap[j]; q < sD->Ap[j + 1]; ++q)
            a_dense[(size_t)sD->Ai[q] * n + j] = sD->Ax[q];
    for (unsigned i = 0; i < n; ++i) {
        v_a[i] = fa[i];
        v_b[i] = fb[i];
        dvec[i] = sD->dVec[i];
        if (tol) tol[i] = sim.pH->use_dipoleCrit ? sim.pH->tolerance[i] : sim.pH->minPrecisitySq;
    }
    umfpack_di_free_numeric(&sD->Numeric);
    return 0;
}

extern "C" double d4ref_xy(double dx, double dy) { return Field().xy(dx, dy); }
extern "C" double d4ref_xy_diff_x(double dx, double dy) { return Field().xy_diff_x(dx, dy); }
extern "C" double d4ref_xy4(double dx, double dy, double e, double c) {
    return Field().xy(dx, dy, e, c);
}
extern "C" double d4ref_xy_diff_x4(double dx, double dy, double e, double c) {
    return Field().xy_diff_x(dx, dy, e, c);
}
