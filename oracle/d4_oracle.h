/*
 * d4_oracle: plain-C restatement of the 2D4_sim implicit-step hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  Only tests/, __graft_entry__.smoke() and the
 * cpu_baseline leg of bench.py may load this library, and only as the checker.
 * The product (2d4_b200/) never links or calls it.
 *
 * Every function restates the reference's algorithm in the same floating-point
 * operation order (file:line of danieltuzes/2D4 cited at each definition), so
 * that, built with the flags of oracle/Makefile (-O2 -ffp-contract=off), it
 * agrees bit for bit with the reference core built the same way
 * (oracle/_ref/libd4ref_exact.so).  tests/test_oracle_pin.py pins that.
 *
 * Layout: positions are given in the reference's internal order (sorted by
 * y+b descending, src/simulation_data.cpp:116), so b_i = +1 for i < n/2 and -1
 * otherwise (src/simulation_data.cpp:265-270).
 */
#ifndef D4_ORACLE_H
#define D4_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct d4o_protocol {
    int kind;          /* 0 StressProtocol (always 0), 1 FixedRate, 2 Cyclic, 3 IncreasingCyclic */
    double tau0;       /* initExtStress */
    double rate;       /* m_rate */
    double period;     /* m_timePeriod */
    double amp_rate;   /* m_amplitudeRate */
} d4o_protocol;

typedef struct d4o_params {
    double position_precision;
    double dipole_precision;
    double cutoff_multiplier;
    int heaviside_cutoff;
    double initial_stepsize;
    double max_stepsize;          /* <= 0: no limit */
    char weight_function;         /* 'c', 'p', 'm' */
    double time_limit;            /* < 0: none */
    long long step_count_limit;   /* < 0: none */
    double strain_increase_limit; /* < 0: none */
    int calculate_strain;
    long long avalanche_limit;    /* < 0: none */
    double avalanche_speed_threshold;
    int save_sub_configs;
    unsigned sub_config_delay;
    unsigned sub_config_delay_during_avalanche;
    double sub_config_times;      /* 0: none */
    char sub_config_times_type;   /* 'a' or 'b' */
    d4o_protocol protocol;
} d4o_params;

typedef struct d4o_result {
    double sim_time;
    double step_size;
    double strain;
    long long successful_steps;
    long long failed_steps;
    double energy;
} d4o_result;

/* One record per attempted step. */
typedef struct d4o_attempt {
    double sim_time;    /* at the start of the attempt */
    double step_size;   /* h tried */
    double ratio;       /* getMaxErrorRatioSqr() */
    int max_id;         /* maxErrorRatioID() */
    int accepted;
} d4o_attempt;

void d4o_default_params(d4o_params *p);

/* Field (src/Fields/Field.cpp:172-346, include/constants.h:40-80). */
double d4o_xy(double dx, double dy);
double d4o_xy_diff_x(double dx, double dy);
double d4o_xy4(double dx, double dy, double exp2pix, double cos2piy);
double d4o_xy_diff_x4(double dx, double dy, double exp2pix, double cos2piy);
/* The IEEE variant (USE_IEEE_HYPERBOLIC 1), src/Fields/Field.cpp:26-168. */
double d4o_ieee_xy(double dx, double dy);
double d4o_ieee_xy_diff_x(double dx, double dy);

double d4o_normalize(double v);
double d4o_weight(double s, char t);
double d4o_weight_inv(double w, char t);
double d4o_ext_stress(const d4o_protocol *p, double t);

/* Internal order of a configuration (src/simulation_data.cpp:86-123).
 * order[original] = sorted index; returns 0, or -1 if sum(b) != 0 or b is not
 * an integer. */
int d4o_sort(int n, const double *x, const double *y, const double *b, double *xs, double *ys,
             int *order);

/* Stress sweep (src/simulation.cpp:287-333).  tol (length n) is updated in
 * place like PrecisionHandler::updateTolerance; pass min_prec_sq <= 0 to skip. */
void d4o_speeds(int n, const double *x, const double *y, double ext_stress, double *v,
                double *tol, double min_prec_sq);

/* Fused sweep (src/simulation.cpp:345-527), dense row-major a[n*n]. */
void d4o_jacobian(int n, const double *x, const double *y, double stepsize, double ext_a,
                  double ext_b, double cutoff_sq, double cutoff, int heaviside, char weight_fn,
                  double *v_a, double *v_b, double *a, double *dvec, double *tol,
                  double min_prec_sq);

/* Half-step rescale (src/simulation.cpp:546-608), dense row-major. */
void d4o_jacobian_from_prev(int n, double *a, double *dvec, double factor, char weight_fn);

/* Dense LU with partial pivoting on a column-major copy, and the solve
 * (the UMFPACK stand-in of oracle/shim/umfpack_shim.cpp).  Returns 1 on an
 * exact zero pivot (UMFPACK_WARNING_singular_matrix), else 0. */
int d4o_lu(int n, double *a_colmajor, int *piv);
void d4o_lu_solve(int n, const double *lu_colmajor, const int *piv, double *x);

/* Whole run (Simulation::run, src/simulation.cpp:30-281) on positions in
 * internal order; x, y are updated in place.  rec (may be null) receives up to
 * rec_cap attempt records; the number of attempts is returned. */
long long d4o_run(int n, double *x, double *y, const d4o_params *p, d4o_result *res,
                  d4o_attempt *rec, long long rec_cap);

/* One attempted step (stages I-IV without the acceptance bookkeeping):
 * from x0 (internal order) and h, produce the big-step and two half-step
 * positions, the error ratio and its argmax, starting from tolerances tol
 * (length n, updated in place). */
void d4o_attempt_step(int n, const double *x0, const double *y, double t0, double h,
                      const d4o_params *p, double *x_big, double *x_half, double *x_two,
                      double *tol, double *ratio, int *max_id);

#ifdef __cplusplus
}
#endif

#endif
