/*
 * d4core.h: C ABI of the B200 engine for the 2D4_sim implicit-step hot path.
 *
 * Library: 2d4_b200/lib/libd4core.so (CUDA, sm_100a).  Plain C types only; every
 * function returns an int status: D4_OK (0), D4_WARN_SINGULAR (1, mirrors
 * UMFPACK_WARNING_singular_matrix) or a negative error.  Nothing crosses this
 * boundary as an exception or an exit().  d4_last_error() gives the message of
 * the last failure on a context.
 *
 * Positions are passed in the reference's internal order (sorted by y+b
 * descending, src/simulation_data.cpp:116), so the Burgers vector of
 * dislocation i is +1 for i < n/2 and -1 otherwise
 * (src/simulation_data.cpp:265-270).  Host pointers are copied in and out;
 * results are complete when a call returns.  A context is not thread-safe;
 * separate contexts may be used from separate threads.
 *
 * What each entry point replaces in the reference (danieltuzes/2D4):
 *   d4_speeds            Simulation::calculateSpeedsAtTime   src/simulation.cpp:287-333
 *   d4_jacobian          Simulation::calcJacobianAndSpeedsAtTimes src/simulation.cpp:345-527
 *   d4_jacobian_from_prev Simulation::calcJacobianAndSpeedsFromPrev src/simulation.cpp:546-608
 *   d4_set_matrix        the CSC arrays Ap/Ai/Ax handed to UMFPACK  src/simulation.cpp:637-638
 *   d4_factor            calculateSparseFormForJacobian ->
 *                        umfpack_di_symbolic/numeric     src/simulation.cpp:635-640
 *   d4_solve             Simulation::solveEQSys -> umfpack_di_solve src/simulation.cpp:643-659
 *   d4_attempt           stages I-III + calculateXError   src/simulation.cpp:90-161,692-700
 *   d4_run               Simulation::run                  src/simulation.cpp:30-281
 *   d4_advance           the body of Simulation::run's loop  src/simulation.cpp:88-277
 *   d4_field_eval        Field::xy / Field::xy_diff_x    src/Fields/Field.cpp:333-346
 */
#ifndef D4CORE_H
#define D4CORE_H

#ifdef __cplusplus
extern "C" {
#endif

enum {
    D4_OK = 0,
    D4_WARN_SINGULAR = 1,
    D4_ERR_ARG = -1,
    D4_ERR_CUDA = -2,
    D4_ERR_NOMEM = -3,
    D4_ERR_STATE = -4,
    D4_ERR_IO = -5
};

/* Arithmetic of the hot path. */
enum {
    D4_PREC_FP64 = 0,  /* plain form: FP64 throughout, reference operation order */
    D4_PREC_MIXED = 1  /* FP64 sweeps and matrix; FP32 tensor-core LU and solves inside
                          FP64 iterative refinement */
};

/* Linear solver of the implicit step.  The reference factorises the (cutoff-
   sparse) Jacobian with UMFPACK, src/simulation.cpp:635-659. */
enum {
    D4_SOLVER_DENSE = 0, /* dense LU (exact reference order in the FP64 form) */
    D4_SOLVER_GMRES = 1, /* CSR of the cutoff Jacobian + Jacobi-preconditioned GMRES(40),
                            relative residual 1e-13; dense LU when it does not converge */
    D4_SOLVER_AUTO = 2   /* GMRES when the Jacobian's support radius^2 < 0.1, else dense */
};

/* Field of a pair.  The reference's core uses the analytic image sum
   (src/Fields/Field.cpp:172-346); its Python binding also names a tabulated
   field (PeriodicShearStressELTE, python/src/periodic_shear_stress_ELTE_wrapper.cpp:43-44)
   whose tables are not part of the reference. */
enum {
    D4_FIELD_ANALYTIC = 0,  /* Field::xy / Field::xy_diff_x */
    D4_FIELD_TABULATED = 1  /* table of the smooth remainder after the free-space
                               core on a table_size^2 grid, bicubic (four-point
                               Lagrange) interpolation + the analytic core;
                               FP64 form only */
};

/* External stress protocol (src/stress_protocol.cpp:13-73). */
enum {
    D4_STRESS_NONE = 0,        /* StressProtocol: always 0 (even with tau0, as -s alone) */
    D4_STRESS_FIXED_RATE = 1,  /* FixedRateProtocol: tau0 + rate*t */
    D4_STRESS_CYCLIC = 2,      /* CyclicLoadProtocol */
    D4_STRESS_INC_CYCLIC = 3   /* IncreasingCyclicLoadProtocol */
};

typedef struct d4_protocol {
    int kind;
    double tau0;           /* initExtStress (-s) */
    double rate;           /* m_rate (-r) */
    double period;         /* m_timePeriod (-i) */
    double amplitude_rate; /* m_amplitudeRate (-A) */
} d4_protocol;

/* The flags of src/project_parser.cpp:28-68 that the stepping loop reads. */
typedef struct d4_params {
    double position_precision;    /* -P, default 1e-5 */
    double dipole_precision;      /* -p, default 0.05; 0 disables */
    double cutoff_multiplier;     /* -u, default 1e20 (no cutoff) */
    int heaviside_cutoff;         /* -h */
    double initial_stepsize;      /* --initial-stepsize, default 1e-6 */
    double max_stepsize;          /* -M; <= 0: none */
    char weight_function;         /* -w: 'c' (default), 'p' or 'm' */
    double time_limit;            /* -t; < 0: none */
    long long step_count_limit;   /* -C; < 0: none (n stops after n+1 accepted steps) */
    double strain_increase_limit; /* < 0: none */
    int calculate_strain;         /* -S */
    int calculate_order_parameter;/* -l */
    long long avalanche_limit;    /* --avalanche-detection-limit; < 0: none */
    double avalanche_speed_threshold; /* default 1e-3 */
    int save_sub_configs;         /* -o given */
    unsigned sub_config_delay;    /* -N, default 5 */
    unsigned sub_config_delay_during_avalanche; /* -n, default 1 */
    double sub_config_times;      /* -T; 0: none */
    char sub_config_times_type;   /* -b: 'a' (default) or 'b' */
    d4_protocol protocol;
    int precision;                /* D4_PREC_FP64 or D4_PREC_MIXED (d4_set_matrix,
                                     d4_factor, d4_solve: FP64 form only) */
    int device;                   /* CUDA device ordinal */
    int solver;                   /* D4_SOLVER_*: linear solver of the step (replaces the
                                     UMFPACK calls of src/simulation.cpp:635-659) */
    int field;                    /* D4_FIELD_*, default analytic */
    int table_size;               /* intervals per axis of the tabulated field, default
                                     1024 (loadStress(..., 1024)); 16..4096 */
} d4_params;

/* Result of one attempted step (stages I-IV before acceptance). */
typedef struct d4_attempt_result {
    double ratio;       /* PrecisionHandler::getMaxErrorRatioSqr() */
    int max_id;         /* PrecisionHandler::maxErrorRatioID() */
    int accepted;       /* ratio < 1 */
    int singular;       /* a factorisation met an exact zero pivot */
    int pivoted;        /* number of factorisations that needed row swaps */
    double refine_residual; /* mixed form: worst max|g - A dx| / max|g| of the
                               attempt's refined solves (0 for the FP64 form) */
} d4_attempt_result;

typedef struct d4_run_result {
    double sim_time;
    double step_size;
    double strain;
    double energy;
    long long successful_steps;
    long long failed_steps;
    long long attempts;
    long long pivoted_factorizations;
    long long singular_factorizations;
    double device_seconds; /* CUDA-event time of the stepping loop */
} d4_run_result;

/* Optional outputs of d4_run (all may be null). */
typedef struct d4_run_io {
    const char *log_path;          /* 15-column log, src/simulation.cpp:52-83,184-209 */
    const char *sub_config_prefix; /* sub-configuration files prefix (-o) */
    const char *end_config_path;   /* final configuration (-O) */
    const unsigned *order;         /* original index -> internal index, for output */
    long long max_attempts;        /* > 0: stop after this many attempts */
} d4_run_io;

void d4_default_params(d4_params *p);

int d4_create(void **ctx, int n, const d4_params *p);
int d4_destroy(void *ctx);
const char *d4_last_error(void *ctx);

/* Positions must be finite and inside the cell [-0.5, 0.5)^2 (where the
 * reference's normalize keeps them, src/sim_utils.cpp:6-13); d4_set_positions
 * and d4_ensemble_set_positions reject others with D4_ERR_ARG.  d4_run,
 * d4_advance and d4_ensemble_run return D4_ERR_STATE when an attempt's error
 * ratio is not finite, where the reference (without its DEBUG_VERSION checks,
 * src/simulation.cpp:754-948) would fail every attempt while doubling h. */
int d4_set_positions(void *ctx, const double *x, const double *y);
/* The check itself: the index of the first offending dislocation, -1 when all
 * n are valid (-2 for bad arguments).  No device work. */
int d4_check_positions(int n, const double *x, const double *y);
int d4_get_positions(void *ctx, double *x, double *y);
int d4_set_time(void *ctx, double sim_time, double step_size);

/* Stress sweep on positions x, y (host, length n) at sim_time.  v receives the
 * speeds; tol (may be null) receives the per-dislocation tolerance after the
 * sweep, starting from the context's current tolerances. */
int d4_speeds(void *ctx, const double *x, const double *y, double sim_time, double *v,
              double *tol);

/* Fused sweep: speeds at t_a and t_b, the scaled Jacobian A = I + D J kept on
 * the device (and copied to a_colmajor when non-null), and dvec. */
int d4_jacobian(void *ctx, const double *x, const double *y, double stepsize, double t_a,
                double t_b, double *v_a, double *v_b, double *a_colmajor, double *dvec,
                double *tol);

/* Half-step rescale of the device Jacobian and dvec with
 * factor = (t_new - t_base) / (t_old - t_base); a_colmajor/dvec may be null. */
int d4_jacobian_from_prev(void *ctx, double factor, double *a_colmajor, double *dvec);

/* Replace the device matrix by a dense column-major n x n matrix (the
 * umfpack_di_numeric input of src/simulation.cpp:638, expanded from CSC). */
int d4_set_matrix(void *ctx, const double *a_colmajor);

/* Factorise the device Jacobian.  Returns D4_WARN_SINGULAR on an exact zero
 * pivot, like umfpack_di_numeric.  Mixed form: its FP32 rounding, by the block
 * LU (rows in the order of the last pivoted factorisation), or by the pivoted
 * FP32 LU when a diagonal tile met a zero or non-finite pivot. */
int d4_factor(void *ctx);

/* Solve A dx = g with the last factorisation (UMFPACK_A).  Returns
 * D4_WARN_SINGULAR like umfpack_di_solve and, like it, leaves the result as
 * computed; d4_attempt/d4_run apply solveEQSys's zeroing of entries outside
 * (-1, 1) (src/simulation.cpp:646-658) themselves.  Mixed form: the FP32
 * factors' solves refined in FP64 against the FP64 matrix (at most 6 sweeps,
 * stopping at max|g - A dx| <= 1e-12 max|g|). */
int d4_solve(void *ctx, const double *g, double *dx);

/* Reset the per-dislocation tolerances (PrecisionHandler::reset). */
int d4_reset_tolerance(void *ctx);
/* The per-dislocation tolerances (length n).  With d4_get_positions and the
 * run result's sim_time and step_size they are the whole state the stepping
 * loop carries from one accepted step to the next, so d4_set_positions,
 * d4_set_time and d4_set_tolerance restart a context exactly where another
 * (or a saved copy) stood.  The tolerances are squared distances;
 * d4_set_tolerance rejects negative or non-finite values with D4_ERR_ARG. */
int d4_get_tolerance(void *ctx, double *tol);
int d4_set_tolerance(void *ctx, const double *tol);

/* One attempted step from the context's positions at t0 with step h. The
 * big-step and two half-step positions stay on the device (d4_get_attempt). */
int d4_attempt(void *ctx, double t0, double h, d4_attempt_result *res);
int d4_get_attempt(void *ctx, double *x_big, double *x_half, double *x_two);

/* Simulation::run on the context's positions; positions are updated. */
int d4_run(void *ctx, const d4_run_io *io, d4_run_result *res);

/* Continue the stepping loop of d4_run for exactly `accepted_steps` accepted
 * steps (failed attempts in between included), keeping the loop state (time,
 * step size, write-out suggestion, counters) in the context between calls.  No
 * initial sweep and no log.  res (may be null) gets the totals of this call,
 * device_seconds the CUDA-event span of the call on the context's stream. */
int d4_advance(void *ctx, long long accepted_steps, d4_run_result *res);

/* Per-category device timing of the hot kernels (CUDA events on the context's
 * stream).  Categories: 0 stress sweep, 1 fused Jacobian sweep, 2 factorisation,
 * 3 solve, 4 half-step rescale.  d4_profile(ctx, 1) clears and starts; the
 * totals (milliseconds) and call counts accumulate until read. */
enum { D4_CAT_SPEEDS = 0, D4_CAT_JACOBIAN = 1, D4_CAT_FACTOR = 2, D4_CAT_SOLVE = 3,
       D4_CAT_RESCALE = 4, D4_CAT_COUNT = 5 };
int d4_profile(void *ctx, int enable);
int d4_profile_read(void *ctx, double *ms, long long *calls);

/* Counters of the cutoff sparse solver (D4_SOLVER_GMRES): GMRES solves run,
 * Krylov iterations summed over them, solves that did not converge and were
 * redone by the dense LU, and the entry count of the last CSR matrix.  No
 * counterpart in the reference (UMFPACK's Info array is not read,
 * src/simulation.cpp:637-645). */
int d4_solver_stats(void *ctx, long long *solves, long long *iterations, long long *fallbacks,
                    long long *nnz);

/* Counters of the dense cooperative LU (plain and mixed forms): factorisations
 * run, passes over their 32-column blocks summed over them (one per block,
 * plus one per row swap found after a block's optimistic pass), and row swaps
 * (pivots off the diagonal).  No counterpart in the reference. */
int d4_lu_stats(void *ctx, long long *factorizations, long long *passes, long long *swaps);

/* Mixed form's factorisations (no counterpart in the reference): block LU
 * factorisations run (128 x 128 tiles on the tensor cores, no row interchanges
 * between tiles, rows in the order of the last pivoted factorisation);
 * fallbacks: block-LU attempts in which a diagonal tile met a zero or
 * non-finite pivot or the refinement left max|g - A dx| above 1e-9 max|g|;
 * attempts run with the pivoted FP32 LU (each fallback redone, and the
 * attempts after the b-th fallback in a row, 2^(b-1) - 1 of them, at most
 * 63; the next block LUs use its row order); attempts that ran on the FP64
 * form's path (an attempt that the pivoted FP32 LU could not refine either,
 * and the attempts after the f-th such in a row, 2^(f-1) of them, at most
 * 64); and the worst refined residual of the FP32 attempts that stood. */
int d4_mixed_stats(void *ctx, long long *block_factorizations, long long *fallbacks,
                   long long *pivoted_attempts, long long *fp64_attempts, double *worst_refined);

/* Mixed form: enable = 1 (the default) runs attempts on the block LU with the
 * fallback that d4_mixed_stats describes; 0 runs every attempt on the FP64
 * form's factorisations and solves.  No counterpart in the reference. */
int d4_set_block_lu(void *ctx, int enable);

/* Pair-tile autotuner (no counterpart in the reference): the FP64 form's pair
 * kernels evaluate each 32 x 32 tile of pairs with 32 x threads_y threads;
 * the first d4_run or d4_advance on a context picks threads_y from {2, 4, 8}
 * by timing each on the context's positions (once per device, n and field in
 * the process; the results do not depend on the choice).  threads_y = 0 until
 * then. */
int d4_pair_tile_threads(void *ctx, int *threads_y);

/* Batched ensemble of independent systems: the many-realisation statistics
 * workload, where the reference runs one system per process
 * (src/simulation.cpp:30-281).  FP64 form, analytic field, dense LU; every
 * instance shares the parameters p (protocol, precisions, limits, cutoff
 * multiplier) and instance k has n[k] dislocations (even, 2..8192, internal
 * order).  Each attempt round runs stages I-IV for every active instance with
 * one launch per phase (all instances' pair tiles and row blocks in one grid;
 * one CTA per instance for an exact-order LU and the substitutions, so each
 * instance reproduces d4_run's arithmetic), then applies each instance's step
 * control as d4_run does (src/simulation.cpp:88-277; no log, sub-configuration
 * or write-out clipping).  An instance stays active until interrupt() holds
 * (time, strain, step-count or avalanche limit, src/simulation.cpp:722-750;
 * avalanches are counted as d4_run counts them). */
int d4_ensemble_create(void **ens, int count, const int *n, const d4_params *p);
int d4_ensemble_destroy(void *ens);
const char *d4_ensemble_last_error(void *ens);
int d4_ensemble_set_positions(void *ens, int k, const double *x, const double *y);
/* The ensemble's pair-tile autotuner (as d4_pair_tile_threads, over all the
 * active instances at the first d4_ensemble_run; 0 until then). */
int d4_ensemble_pair_tile_threads(void *ens, int *threads_y);
int d4_ensemble_get_positions(void *ens, int k, double *x, double *y);
/* Runs attempt rounds until no instance is active or max_rounds rounds
 * (<= 0: no cap) have run in this call; may be called again to continue.
 * res[count] receives each instance's totals (sim_time, step_size, strain,
 * successful and failed steps, attempts, singular factorisations) and, in
 * every entry, device_seconds = the CUDA-event span of this call. */
int d4_ensemble_run(void *ens, long long max_rounds, d4_run_result *res);

/* Direct-Fourier pattern analysis of one configuration (the reference's
 * xpattern tool, method df, xpattern/xpattern.cpp:393-423).  With K = res/2+1
 * and F_m(kx, ky) = sum_i w_m(b_i) exp(-2 pi i (kx x_i + ky y_i)) for the four
 * densities m = rho_t (w = 1), kappa (w = b), rho_p (b = +1) and rho_n
 * (b = -1), adds sum_ky |F_m(kx, ky)|^2 (ky ascending) to acc[m*K + kx],
 * kx = 0..K-1, so that repeated calls sum over configurations as the tool
 * does over its input files.  x, y, b: host arrays of n entries; acc: host,
 * 4*K entries, read and updated.  FP64 throughout; 2 <= res <= 65536.  Uses
 * the current device and allocates its scratch (two n x K tables and 4 K^2
 * doubles) for the call. */
int d4_xpattern_df(int n, const double *x, const double *y, const int *b, int res, double *acc);

/* Schedule of an attempt (dense plain and mixed forms): enable = 1 (the
 * default) runs stage I, the big step, on a second stream concurrently with
 * stages II and III; 0 runs the stages one after the other on the context's
 * stream (for a caller sharing the GPU with other work).  Both give identical
 * results.  Ignored by the cutoff GMRES path, which is always sequential.  No
 * counterpart in the reference (src/simulation.cpp:88-164 runs the stages in
 * sequence). */
int d4_set_overlap(void *ctx, int enable);

/* Recording of accepted steps: while enabled, d4_run and d4_advance append
 * each accepted step's start time and size (the t and h of
 * src/simulation.cpp:88-164) to the context's list.  enable = 1 clears the
 * list and starts, 0 stops.  d4_recorded_steps copies up to `count` entries. */
int d4_record_steps(void *ctx, int enable);
long long d4_recorded_count(void *ctx);
int d4_recorded_steps(void *ctx, long long count, double *t0s, double *hs);

/* Differentiation of a fixed sequence of accepted steps (no counterpart in the
 * reference).  The forward map replays steps (t0s[k], hs[k]) from positions
 * x0 (internal order, the context's y): the stages II and III of
 * Simulation::run's attempt (src/simulation.cpp:115-150) with the engine's
 * FP64 kernels, then normalize; the loss is the accumulated strain
 * sum_k sum_i b_i (x2_i - x0_i) (src/simulation.cpp:713-720).  Step sizes are
 * constants.  proto may be null (the context's protocol); tau0 is its tau0.
 * FP64 form, analytic field, dense solver, no cutoff; the context's positions
 * and tolerances are left as they were.
 *   d4_replay   strain and final positions (x_end may be null)
 *   d4_tangent  strain and its directional derivative along (dx0, dtau0)
 *   d4_adjoint  strain, d strain / d x0 and d strain / d tau0, with positions
 *               checkpointed every checkpoint_every steps, each segment
 *               recomputed in the backward sweep and the step's LU factors
 *               reused for the transposed solves (device memory: about
 *               2 checkpoint_every n^2 doubles for the segment's factors). */
int d4_replay(void *ctx, long long steps, const double *t0s, const double *hs,
              const d4_protocol *proto, const double *x0, double *x_end, double *strain);
int d4_tangent(void *ctx, long long steps, const double *t0s, const double *hs,
               const d4_protocol *proto, const double *x0, const double *dx0, double dtau0,
               double *strain, double *dstrain);
int d4_adjoint(void *ctx, long long steps, const double *t0s, const double *hs,
               const d4_protocol *proto, int checkpoint_every, const double *x0, double *strain,
               double *grad_x0, double *grad_tau0);

/* Number of kernels this library has launched in the process so far. */
long long d4_kernel_launches(void);

/* Self-test of the kernels' bounded waits (no counterpart in the reference):
 * which = 0 runs the cooperative LU's grid barrier with one CTA that never
 * arrives, which = 1 the block LU's tile-flag wait on a flag that nothing
 * sets.  The wait gives up after its normal limit (about a second), the
 * kernel records the timeout and returns, and the call returns D4_ERR_STATE
 * (D4_OK would mean the wait did not give up); the context stays usable. */
int d4_wait_selftest(void *ctx, int which);

/* Number of device allocations (cudaMalloc) this library has made in the
 * process so far.  No counterpart in the reference. */
long long d4_device_allocations(void);

/* Allocation-free FP64 stress sweep (no counterpart in the reference: an
 * addition of this library).  For callers that cannot allocate device memory,
 * such as code running under CUDA-graph stream capture, real-time loops that
 * must not wait on an allocator, or hosts whose device memory belongs to
 * another framework's allocator.  Same result as d4_speeds of a context with
 * the analytic field (no table; every form runs the plain form's exact-order
 * sweeps at these sizes): speeds v[n] and the tolerance update of tol[n] (may
 * be null; starts from the caller's values,
 * clamped below min_prec_sq as PrecisionHandler::updateTolerance does) for
 * positions x[n], y[n] in internal order at external stress ext_stress.  All
 * pointers are DEVICE pointers owned by the caller; the work is queued on
 * `stream` (a cudaStream_t, null for the default stream) and the call returns
 * without waiting.  The n x n scratch is a file-scope device array of
 * D4_NOALLOC_MAX_N^2 doubles (8 MiB) that every GPU loading the library holds
 * until exit: n > D4_NOALLOC_MAX_N is rejected with D4_ERR_ARG, as are odd n.
 * The first call on a device looks the array up (cudaGetSymbolAddress) and
 * must come before any stream capture; so must the first call after a device
 * reset, which looks it up again (the address is cached per device and CUDA
 * context).  Calls share the array, so calls that overlap on the GPU race and
 * must be serialised by the caller. */
#define D4_NOALLOC_MAX_N 1024
int d4_speeds_noalloc(int n, const double *x, const double *y, double ext_stress, double *v,
                      double *tol, double min_prec_sq, void *stream);

/* Single field evaluations on the device, for checks: the context's field
 * (analytic FP64 Field::xy / Field::xy_diff_x, or the tabulated field). */
int d4_field_eval(void *ctx, int count, const double *dx, const double *dy, double *xy,
                  double *xy_diff_x);

#ifdef __cplusplus
}
#endif

#endif
