// d4_internal.h: device state and kernel entry points shared by the
// translation units of libd4core.so.
#pragma once

#include <cuda_runtime.h>

#include <atomic>
#include <string>
#include <vector>

#include "d4core.h"

namespace d4 {

constexpr int kTile = 32;          // pair tile edge
constexpr int kLuNb = 32;          // LU block width (FP64 path)
// Cooperative LU buffers: per launch one mask word per possible pass, then
// the FP64 form's schedule words (tickets, strip counters, look-ahead epoch);
// after the two Q halves (2 x n x 32) the published diagonal block and its
// reciprocals.
constexpr int lu_pass_words(int nblk) { return nblk * 33 + 8; }
constexpr int lu_mask_words_for(int nblk) { return lu_pass_words(nblk) + nblk + 64; }
constexpr int kLuDiagWords = kLuNb * (kLuNb + 1) + kLuNb + kLuNb * kLuNb;
constexpr int kSolveThreads = 1024;
constexpr int kMaxSolveN = 8192;   // x and g of the one-CTA solve live in shared memory

// Device flag words (ints in one small buffer).
enum FlagSlot {
    kFlagNeedPivot = 0,  // fast LU met |a_ik| > |a_kk| or a_kk == 0: partial pivoting would swap
    kFlagSingular = 1,   // pivoted LU met an exact zero pivot
    kFlagBarrierTimeout = 2,  // a bounded grid-barrier wait gave up
    kFlagPasses = 3,     // cooperative LU: passes over the column blocks
    kFlagSwaps = 4,      // cooperative LU: row swaps (pivots off the diagonal)
    kFlagCount = 8
};

// wave_err words: [0..4] triangular-solve wait diagnostics, [5] a row-sum pipeline
// wait gave up.
constexpr int kWaveErrRows = 5;

// Buffers of one LU factorisation (factors, pivot bookkeeping, flags).
struct LuBufs {
    double *LU = nullptr, *P0 = nullptr, *Q = nullptr;
    unsigned *mask = nullptr, *bar = nullptr;
    int *flags = nullptr, *perm = nullptr, *piv = nullptr;
};

// Launch counters of one block-LU buffer set (host side): epochs of its tile
// and solve flags.
struct BluState {
    int lu_epoch = 0, solve_epoch = 0;
};

// Buffers of the mixed form's block LU and block solves (d4_blu32.cu): the
// packed tensor-core operands of every tile (TF32 hi and lo parts), the
// schedule, ticket counters ([0] factorisation, [1] the solves), the tile
// flags, the solves' tagged block values and the solution.
struct BluBufs {
    unsigned char *op = nullptr;
    const int *tasks = nullptr;
    int *ticket = nullptr;
    int *ready = nullptr;
    unsigned long long *yt = nullptr, *xt = nullptr;  // tagged block values of the solves
    float *xs = nullptr;
    BluState *state = nullptr;
};

// Buffers of one FP32 factorisation and its refined solves (mixed form): the
// matrix the refinement's residual multiplies, the factors and the pivot
// bookkeeping, the refinement vectors and the ring of residual maxima.
struct Mix32Bufs {
    double *A64 = nullptr;  // the FP64 matrix the refinement's residual multiplies
    float *A32 = nullptr, *LU32 = nullptr, *P0 = nullptr, *Q = nullptr;
    unsigned *mask = nullptr, *bar = nullptr;
    int *flags = nullptr, *perm = nullptr, *piv = nullptr;
    double *g = nullptr, *r = nullptr, *dx = nullptr, *dx2 = nullptr;
    double *part = nullptr;  // ceil(n / 256) x n: the residual product's column-chunk sums
    unsigned *cnt = nullptr; // ceil(n / 256): chunk blocks finished per row block (k_resid_fused)
    unsigned long long *conv = nullptr;  // kIrMax + 1: max|g|, then max|r| after each sweep
    float *c32 = nullptr, *w1 = nullptr;
    unsigned long long *resid = nullptr;  // 8 pairs (max |r|, max |g|)
    int *resid_count = nullptr;           // host: next slot of resid
    BluBufs blu;                          // block LU path (Ctx::m_fast)
    int *blk = nullptr;                   // host: LU32 holds block-LU factors (else pivoted)
};

// Buffers of the solves of one stage chain: the weights read by the
// residual, the forward-solve scratch and the correction.
struct SolveBufs {
    const double *dvec = nullptr;
    double *xw1 = nullptr, *xw2 = nullptr, *dx = nullptr;
};

// State of Simulation::run's loop kept between d4_advance calls.
struct RunState {
    bool started = false;
    double strain = 0, energy = 0, h_before_writeout = 0, next_wo = 0;
    long long ok = 0, failed = 0, attempts = 0, pivoted = 0, singular = 0;
    long long aval_count = 0;
    bool in_aval = false;
    unsigned sub_counter = 0;
    double wall_start = 0, wall_last = 0;  // log columns 14 and 10 (seconds)
};

struct Prof {
    bool on = false;
    std::vector<cudaEvent_t> pool;      // pairs (start, stop)
    std::vector<int> cat;               // category per pair in use
    size_t used = 0;
    double ms[D4_CAT_COUNT] = {};
    long long calls[D4_CAT_COUNT] = {};
};

struct Ctx {
    int n = 0;
    d4_params p{};
    cudaStream_t stream = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    std::string err, err_detail;

    // derived scalars (host, reference rounding)
    double min_prec_sq = 0, dipole_prec_sq = 1;
    int use_dipole = 0;
    double cutoff = 0, cutoff_sq = 0, range_sq = 49;

    // host-side state of the stepping loop
    double sim_time = 0, step_size = 0;
    int selected_id = 0;
    int factor_singular = 0;
    int factor_pivoted = 0;
    int lu_pivoted_path = 0;  // current factorisation came from the pivoted kernels

    // device buffers (FP64)
    double *x0 = nullptr, *y = nullptr, *xb = nullptr, *xh = nullptr, *x2 = nullptr;
    double *xs_tmp = nullptr, *ys_tmp = nullptr;  // staging for d4_speeds / d4_jacobian
    double *v_init = nullptr, *v_init2 = nullptr, *speed = nullptr, *speed2 = nullptr;
    double *dvec = nullptr, *dvec_new = nullptr, *fac = nullptr, *dx = nullptr, *tol = nullptr;
    double *A = nullptr;   // scaled Jacobian, column-major n x n
    double *LU = nullptr;  // factorisation of A, column-major
    double *F = nullptr;   // signed pair-force matrix (column-major) of one sweep
    int *piv = nullptr, *perm = nullptr;
    int *flags = nullptr;
    double *red = nullptr;  // reduction results
    // pinned host mirror of the small results
    double *h_red = nullptr;
    int *h_flags = nullptr;

    // triangular solves: intermediate vectors and the error words of bounded
    // waits (wave_err, see kWaveErrRows)
    int *wave_err = nullptr;
    double *xw1 = nullptr, *xw2 = nullptr;
    // row sums of the FP64 fused sweep: subSum_i and the row scale (1 + d_i)/2
    double *rowsub = nullptr, *rowsc = nullptr;
    // cooperative LU: saved block columns, pre-division values, per-pass masks,
    // grid barrier words
    double *lu_p0 = nullptr, *lu_q = nullptr;
    unsigned *lu_mask = nullptr, *lu_bar = nullptr;
    int lu_mask_words = 0, lu_grid = 0;

    // mixed form: FP32 matrix and factors, FP64 accumulators and refinement
    float *A32 = nullptr, *LU32 = nullptr, *lu32_p0 = nullptr, *lu32_q = nullptr;
    int lu32_grid = 0;
    double *m_g = nullptr, *m_r = nullptr, *m_dx = nullptr, *m_dx2 = nullptr;
    unsigned *m_cnt = nullptr;
    unsigned long long *m_conv = nullptr;
    int *spiv = nullptr;  // static pivots of the block LU: row of A at each position of P A
    float *m_c32 = nullptr, *m_w1 = nullptr;
    double *m_part = nullptr;  // residual product's column-chunk sums (Mix32Bufs::part)
    unsigned long long *m_resid = nullptr;  // 8 pairs (max |r|, max |g|) of recent solves
    int m_resid_count = 0;
    int ir_iters = 2;
    // block LU path of the mixed form (d4_blu32.cu): on by default; an attempt
    // whose block factorisation met a bad pivot, or whose refined residual
    // stayed above kRefineLimit, is redone on the FP64 form's path
    int m_fast = 1;
    int *blu_tasks = nullptr;
    BluBufs blu;  // the primary buffer set's block-LU buffers
    BluState blu_state, blu_state_b;
    int m_blk = 0, m_blk_b = 0;  // Mix32Bufs::blk of the primary and stage-I buffer sets
    long long m_blocklu = 0, m_fallbacks = 0, m_fp64_attempts = 0;
    int m_skip = 0;          // attempts left on the FP64 path (backoff)
    int m_fallback_run = 0;  // attempts in a row that no FP32 factorisation refined
    int m_piv_skip = 0;      // attempts left on the pivoted FP32 LU (backoff)
    int m_block_run = 0;     // block-LU failures in a row
    long long m_pivoted32 = 0;  // attempts run with the pivoted FP32 LU
    double m_worst_refine = 0;

    // cutoff sparse path: CSR of the matrix and the GMRES work space
    int use_gmres = 0;
    int sp_grid = 0, sp_nch = 0, sp_cap = 0, sp_nnz = 0, sp_dense_ready = 0;
    int *sp_cnt = nullptr, *sp_off = nullptr, *sp_rp = nullptr, *sp_ci = nullptr;
    int *sp_flags = nullptr;
    unsigned *sp_bar = nullptr;
    double *sp_val = nullptr, *sp_dinv = nullptr, *sp_V = nullptr, *sp_z = nullptr,
           *sp_w = nullptr, *sp_g = nullptr, *sp_x = nullptr, *sp_part = nullptr;
    long long sp_solves = 0, sp_iters = 0, sp_fallbacks = 0;
    // cooperative LU counters (d4_lu_stats)
    long long lu_count = 0, lu_passes = 0, lu_swaps = 0;

    // tabulated field (null: analytic field)
    double2 *tab = nullptr;
    int tab_T = 0;

    // accepted steps (t0, h) recorded by the run loop (d4_record_steps)
    bool recording = false;
    std::vector<double> rec_t0, rec_h;

    // stage I (the big step) on a second stream, concurrent with stages II
    // and III (FP64 dense form): its own factorisation, force scratch,
    // weights and speed copies, solve scratch, and the three factorisations'
    // flags of an attempt
    int overlap = 0;
    cudaStream_t stream_b = nullptr;
    cudaEvent_t ev_fork = nullptr, ev_copy = nullptr, ev_join = nullptr;
    LuBufs lub;
    double *F_b = nullptr, *dvec_b = nullptr, *speed_b = nullptr, *speed2_b = nullptr,
           *xw1_b = nullptr, *xw2_b = nullptr, *dx_b = nullptr;
    int *flags3 = nullptr;  // 3 x kFlagCount
    // mixed form: stage I's FP64 matrix copy and FP32 buffers
    Mix32Bufs m32b;
    int m_resid_count_b = 0;

    // pair-tile autotuner (FP64 pair kernels): threads per 32x32 tile along j
    int pair_ty = 8;
    // the mixed form's sweeps (N >= kMixedMinN, analytic field) use the pair
    // tiles and row sums of d4_fp64_fast.cu, with chunk partials and counters
    // per stream ([1]: stage I's sweeps on stream_b)
    int fast_pairs = 0;
    double *fr_part[2] = {nullptr, nullptr};
    unsigned *fr_cnt[2] = {nullptr, nullptr};
    bool pair_tuned = false;

    RunState rs;
    Prof prof;
};

// Category timing: returns the index of an event pair (or -1 when off).
int prof_begin(Ctx &c, int cat, cudaStream_t st = nullptr);  // null: the context's stream
void prof_end(Ctx &c, int idx, cudaStream_t st = nullptr);
void prof_collect(Ctx &c);  // after a stream sync: folds finished pairs into totals

struct ProfScope {
    Ctx &c;
    int idx;
    cudaStream_t st;
    ProfScope(Ctx &cc, int cat, cudaStream_t s = nullptr)
        : c(cc), idx(prof_begin(cc, cat, s)), st(s) {}
    ~ProfScope() { prof_end(c, idx, st); }
};

extern std::atomic<long long> g_launches;
extern std::atomic<long long> g_allocs;

// Every device allocation of the library goes through this wrapper, which
// counts it (d4_device_allocations).
template <typename T>
inline cudaError_t dmalloc(T **p, size_t bytes) {
    g_allocs.fetch_add(1, std::memory_order_relaxed);
    return cudaMalloc((void **)p, bytes);
}

// ---- FP64 pair sweeps (d4_fp64.cu) ----
// Stress sweep: F (signed pair forces) and tolerance update, then ordered row sums.
void speeds64(Ctx &c, const double *x, const double *y, double ext, double *v);
// Fused sweep: F and raw J, row sums, dvec, scaling to A = I + D J.
void jacobian64(Ctx &c, const double *x, const double *y, double h, double ext_a, double ext_b,
                double *v_a, double *v_b);
void jacobian_from_prev64(Ctx &c, double factor);
void half_weights64(Ctx &c, double factor);  // dvec_new and fac of the half step
void shift_speed64(Ctx &c, double *v, double dif);
void reset_tol64(Ctx &c);
void error_ratio64(Ctx &c, const double *xb, const double *x2);  // -> red[0], red[1]
void normalize64(Ctx &c, double *x_dst, const double *x_src);
void strain_increment64(Ctx &c, const double *x_old, const double *x_new, double *out);
void field_eval64(Ctx &c, int count, const double *dx, const double *dy, double *xy,
                  double *xyd);

// Pair-tile autotuner (d4_fp64.cu): picks the threads per pair tile of the FP64
// pair kernels by timing the candidates on the context's positions, once per
// (device, n, field) in the process; results do not depend on the choice.
void autotune_pairs(Ctx &c);
// The candidates and the timing shared with the ensemble's tuner.
constexpr int kPairTyCandidates[3] = {2, 4, 8};

// ---- FP64 factorisation and solves (d4_lu64.cu) ----
// Factorises A into LU; returns via flags whether the pivoted path ran and
// whether the matrix is singular.  Host-synchronising.
int factor64(Ctx &c);                 // d4_lu_coop64.cu
void factor64_async(Ctx &c, const LuBufs &L, const double *A, int grid, cudaStream_t st,
                    cudaEvent_t after_copy);
LuBufs primary_lu(Ctx &c);
// Adds one factorisation's pass and swap counts (its flag words) to the
// context's counters.
inline void count_lu(Ctx &c, const int *fl) {
    ++c.lu_count;
    c.lu_passes += fl[kFlagPasses];
    c.lu_swaps += fl[kFlagSwaps];
}
int coop_grid_size(int n);            // CTAs of the cooperative LU (-1: n too large)
enum GMode { kGBig = 0, kGHalf = 1, kGNewton = 2 };
// g built from (gmode, hval, dvec, s_end, s_init, x_new, x_old); solve; out = base - dx.
void solve_update64(Ctx &c, int gmode, double hval, const double *s_end, const double *s_init,
                    const double *x_new, const double *x_old, const double *base, double *out);
void solve_update64_with(Ctx &c, const LuBufs &L, const SolveBufs &S, cudaStream_t st, int gmode,
                         double hval, const double *s_end, const double *s_init,
                         const double *x_new, const double *x_old, const double *base,
                         double *out);
// The mixed form's pair tiles (d4_fp64_fast.cu): forces into F and, for jac,
// the raw Jacobian entries into c.A, as the plain pair tiles write them.
void pairs64_fast(Ctx &c, bool jac, const double *x, const double *y, double *F, double h,
                  cudaStream_t st);
// ... and their row sums: speeds v_a (and v_b), for jac d, rowsub, rowsc.
void rows64_fast(Ctx &c, bool jac, const double *F, double ext_a, double ext_b, double *v_a,
                 double *v_b, cudaStream_t st);
void speeds64_with(Ctx &c, double *F, cudaStream_t st, const double *x, const double *y,
                   double ext, double *v);
// Plain solve of A dx = g (g on device, dx written to c.dx).
void solve_plain64(Ctx &c, const double *g);
// Mixed form: refined solve of A32 dx = g with the last factorisation (g on
// device, dx written to c.dx); the block LU's factorisation falls back to the
// pivoted one by itself when a diagonal tile met a bad pivot (factor32).
void solve_plain32(Ctx &c, const double *g);

// ---- mixed form (d4_mixed.cu) ----
// Refinement sweeps: at most kIrMax, stopping once max|r| <= kIrStop max|g|.
constexpr int kIrMax = 6;
constexpr double kIrStop = 1e-12;
// The context's own buffers (stages II and III, and the sequential attempt).
Mix32Bufs primary_mix32(Ctx &c);
// FP32 factorisation of the FP64 matrix A into B on `st` with up to `grid`
// CTAs, without waiting; with copy_matrix, A is first copied into B.A64 (the
// matrix stage I's refinement multiplies) and `after_copy` (may be null) is
// recorded once it is taken.
void factor32_async(Ctx &c, const Mix32Bufs &B, const double *A, bool copy_matrix, int grid,
                    cudaStream_t st, cudaEvent_t after_copy);
// The primary buffers' last pivoted factorisation gives the block LU's pivots.
void adopt_pivots(Ctx &c);
// solve_update32 with explicit buffers, weights, correction output and stream.
void solve_update32_with(Ctx &c, const Mix32Bufs &B, const double *dvec, double *dx_out,
                         cudaStream_t st, int gmode, double hval, const double *s_end,
                         const double *s_init, const double *x_new, const double *x_old,
                         const double *base, double *out);
int factor32(Ctx &c);
int coop_grid_size32(int n);

// ---- mixed form's block LU (d4_blu32.cu) ----
constexpr double kRefineLimit = 1e-9;  // refined max|r| / max|g| above this: exact path
int blu_tiles(int n);
size_t blu_op_bytes(int n);
std::vector<int> blu_schedule(int n);
void blu_alloc(BluBufs &B, int n, const int *tasks, BluState *state);
void blu_free(BluBufs &B);
// Factorises A (FP32, column-major n x n) into LU (block factors, plain) and the
// packed operands of B, on `st` with up to `grid` CTAs; flags receives
// kFlagSingular (a diagonal tile's Gauss-Jordan met a bad pivot) and
// kFlagBarrierTimeout (a bounded wait gave up).
void blu_factor_async(const BluBufs &B, int n, const float *A, float *LU, int *flags, int grid,
                      cudaStream_t st);
// Runs a bounded wait on a barrier or flag that nothing completes (d4_wait_selftest).
int wait_selftest(int which);
// x = (block LU of P A)^-1 P b in FP32 (b FP64; perm: the rows of P, null for
// the identity); the result is B.xs (padded to 128-row blocks).  Refinement
// sweep `it`: returns at once when conv says sweep it - 1 converged.
void blu_solve_async(const BluBufs &B, int n, const float *LU, const double *b, const int *perm,
                     const unsigned long long *conv, int it, int *flags, cudaStream_t st);
void solve_update32(Ctx &c, int gmode, double hval, const double *s_end, const double *s_init,
                    const double *x_new, const double *x_old, const double *base, double *out);

// tau_ext(t) of the stress protocol (d4_api.cu).
double ext_stress_host(const d4_protocol &p, double t);

// ---- tabulated field (d4_table.cu) ----
void table_build(Ctx &c);  // allocates c.tab (T = c.tab_T) and fills it on c.stream

// ---- cutoff sparse path (d4_sparse.cu) ----
bool gmres_selected(const Ctx &c);
void sparse_alloc(Ctx &c);
void sparse_free(Ctx &c);
void sparse_prepare(Ctx &c);  // CSR of A (or A32); host-synchronising
// GMRES solve of the stage; false when it did not converge (dense LU then).
bool sparse_solve_update(Ctx &c, int gmode, double hval, const double *s_end,
                         const double *s_init, const double *x_new, const double *x_old,
                         const double *base, double *out);

}  // namespace d4

#define D4_CUDA_OK(expr)                                                       \
    do {                                                                       \
        cudaError_t e_ = (expr);                                               \
        if (e_ != cudaSuccess) throw d4::CudaError(e_, #expr, __FILE__, __LINE__); \
    } while (0)

namespace d4 {
struct CudaError {
    cudaError_t code;
    std::string what;
    CudaError(cudaError_t c, const char *expr, const char *file, int line)
        : code(c),
          what(std::string(cudaGetErrorString(c)) + " at " + file + ":" + std::to_string(line) +
               " (" + expr + ")") {}
};
struct StateError {
    std::string what;
    explicit StateError(const char *w) : what(w) {}
};
inline void check_launch(const char *name) {
    g_launches.fetch_add(1, std::memory_order_relaxed);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) throw CudaError(e, name, __FILE__, __LINE__);
}
}  // namespace d4
