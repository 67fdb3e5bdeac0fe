/*
 * C interface of the reference-core oracle (oracle/_ref/libd4ref*.so).
 *
 * TEST INFRASTRUCTURE ONLY.  The library is the reference's own core
 * (src/simulation.cpp, src/Fields/Field.cpp, src/precision_handler.cpp,
 * src/sim_utils.cpp, src/simulation_data.cpp, src/stress_protocol.cpp,
 * src/dislocation.cpp) compiled unmodified from its source tree, linked with the
 * project-written UMFPACK shim and this driver.  The driver replaces the
 * Boost-based ProjectParser (src/project_parser.cpp:155-333): it fills a
 * SimulationData the way processInput does and calls Simulation::run or the
 * individual private sweeps of Simulation.
 */
#ifndef D4_REF_DRIVER_H
#define D4_REF_DRIVER_H

#ifdef __cplusplus
extern "C" {
#endif

/* Flag set of src/project_parser.cpp:28-68, resolved the way processInput
 * (:176-326) resolves it.  A value < 0 in an "optional" slot means "flag not
 * given". */
typedef struct d4ref_params {
    double position_precision;  /* -P, default 1e-5 */
    double dipole_precision;    /* -p, default 0.05; 0 disables */
    double cutoff_multiplier;   /* -u, default 1e20 */
    int heaviside_cutoff;       /* -h */
    double initial_stepsize;    /* --initial-stepsize, default 1e-6 */
    double max_stepsize;        /* -M, < 0: not given */
    char weight_function;       /* -w: 'c', 'p' or 'm' */
    double time_limit;          /* -t, < 0: not given */
    long long step_count_limit; /* -C, < 0: not given */
    double strain_increase_limit; /* < 0: not given */
    int calculate_strain;       /* -S */
    int calculate_order_parameter; /* -l */
    double const_external_stress; /* -s, default 0 */
    int has_rate;               /* -r given */
    double rate;                /* -r */
    int has_cyclic;             /* -i given */
    double cyclic_period;       /* -i */
    int has_amplitude_rate;     /* -A given */
    double amplitude_rate;      /* -A */
    const char *sub_config_path; /* -o (null: not given) */
    unsigned sub_config_delay;  /* -N, default 5 */
    unsigned sub_config_delay_during_avalanche; /* -n, default 1 */
    double sub_config_times;    /* -T, <= 0: not given */
    char sub_config_times_type; /* -b, default 'a' */
    long long avalanche_limit;  /* --avalanche-detection-limit, < 0: not given */
    double avalanche_speed_threshold; /* default 1e-3 */
} d4ref_params;

typedef struct d4ref_result {
    double sim_time;
    double step_size;
    double strain;
    long long successful_steps;
    long long failed_steps;
    int n;
} d4ref_result;

void d4ref_default_params(d4ref_params *p);

/* Whole run (Simulation::run, src/simulation.cpp:30-281).  Writes the final
 * configuration to out_path in the reference's .dconf format (14 digits) and,
 * when x_sorted/y_sorted are non-null, the final state in the reference's
 * internal (sorted) order at full precision.  log_path may be null. */
int d4ref_run(const char *in_path, const char *out_path, const char *log_path,
              const d4ref_params *p, d4ref_result *res, double *x_sorted, double *y_sorted,
              double *wall_seconds);

/* Sorted load (src/simulation_data.cpp:76-154): positions in internal order and
 * disl_order (original index -> sorted index). */
int d4ref_load(const char *in_path, int *n, double *x, double *y, unsigned *order, int cap);

/* One stress sweep, Simulation::calculateSpeedsAtTime (src/simulation.cpp:287-333),
 * on positions given in internal order.  tol receives PrecisionHandler's
 * per-dislocation tolerance after the sweep. */
int d4ref_speeds(const char *in_path, const d4ref_params *p, const double *x, const double *y,
                 double sim_time, double *v, double *tol);

/* One fused sweep, Simulation::calcJacobianAndSpeedsAtTimes
 * (src/simulation.cpp:345-527), expanded to a dense row-major N x N matrix. */
int d4ref_jacobian(const char *in_path, const d4ref_params *p, const double *x, const double *y,
                   double stepsize, double t_a, double t_b, double *v_a, double *v_b,
                   double *a_dense, double *dvec, double *tol, int *nnz);

/* Field::xy and Field::xy_diff_x (src/Fields/Field.cpp:295-346). */
double d4ref_xy(double dx, double dy);
double d4ref_xy_diff_x(double dx, double dy);
double d4ref_xy4(double dx, double dy, double exp2pix, double cos2piy);
double d4ref_xy_diff_x4(double dx, double dy, double exp2pix, double cos2piy);

#ifdef __cplusplus
}
#endif

#endif
