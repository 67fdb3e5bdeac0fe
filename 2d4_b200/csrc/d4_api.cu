// d4_api.cu: C ABI of libd4core.so and the host side of the stepping loop.
//
// The loop mirrors Simulation::run (src/simulation.cpp:30-281): the hot path
// (pair sweeps, Jacobian, factorisations, solves, error reduction) runs on the
// device; the scalar control (accept/reject, PrecisionHandler::getNewStepSize,
// write-out clipping, stop conditions, log lines) runs here on the host in the
// reference's own double arithmetic, with one 16-byte read-back per attempt.
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <iomanip>
#include <algorithm>
#include <chrono>
#include <new>
#include <sstream>
#include <string>
#include <vector>

#include "d4_internal.h"

using d4::Ctx;
using d4::CudaError;

namespace d4 {
std::atomic<long long> g_launches{0};
std::atomic<long long> g_allocs{0};

int prof_begin(Ctx &c, int cat, cudaStream_t st) {
    if (!c.prof.on) return -1;
    if (c.prof.used * 2 + 2 > c.prof.pool.size()) {
        for (int k = 0; k < 64; ++k) {
            cudaEvent_t e;
            D4_CUDA_OK(cudaEventCreate(&e));
            c.prof.pool.push_back(e);
        }
    }
    const int idx = (int)c.prof.used++;
    if ((size_t)idx >= c.prof.cat.size()) c.prof.cat.resize(idx + 1);
    c.prof.cat[idx] = cat;
    D4_CUDA_OK(cudaEventRecord(c.prof.pool[2 * idx], st ? st : c.stream));
    return idx;
}

void prof_end(Ctx &c, int idx, cudaStream_t st) {
    if (idx < 0) return;
    cudaEventRecord(c.prof.pool[2 * idx + 1], st ? st : c.stream);
}

void prof_collect(Ctx &c) {
    for (size_t k = 0; k < c.prof.used; ++k) {
        float ms = 0;
        if (cudaEventElapsedTime(&ms, c.prof.pool[2 * k], c.prof.pool[2 * k + 1]) == cudaSuccess) {
            c.prof.ms[c.prof.cat[k]] += ms;
            c.prof.calls[c.prof.cat[k]] += 1;
        }
    }
    c.prof.used = 0;
}

// StressProtocol family, src/stress_protocol.cpp:13-73.
double ext_stress_host(const d4_protocol &p, double t) {
    switch (p.kind) {
    case D4_STRESS_FIXED_RATE:
        return t * p.rate + p.tau0;
    case D4_STRESS_CYCLIC:
    case D4_STRESS_INC_CYCLIC: {
        double periodic = t - std::floor((t / p.period + 1. / 4)) * p.period;
        double stress = p.rate * periodic + p.tau0;
        if (periodic > p.period / 4) stress = p.rate * p.period / 2 - stress + p.tau0;
        if (p.kind == D4_STRESS_INC_CYCLIC) return stress * p.amplitude_rate * t;
        return stress;
    }
    default:
        return 0;
    }
}
}  // namespace d4

namespace {

inline double ext_stress(const d4_protocol &p, double t) { return d4::ext_stress_host(p, t); }

// get_wall_time, src/sim_utils.cpp:22-33: seconds of the wall clock, at the
// reference's millisecond resolution.
double wall_time() {
    const auto ms = std::chrono::time_point_cast<std::chrono::milliseconds>(
        std::chrono::high_resolution_clock::now());
    return static_cast<double>(ms.time_since_epoch().count()) / 1000.;
}

// SimulationData::getNextWriteOutTime, src/simulation_data.cpp:231-246.
double next_write_out(const d4_params &p, double sim_time) {
    if (p.sub_config_times == 0) return INFINITY;
    if (p.sub_config_times_type == 'a')
        return (double)((size_t)(sim_time / p.sub_config_times) + 1) * p.sub_config_times;
    if (p.sub_config_times_type == 'b') {
        double exponent =
            std::nextafter(std::log(sim_time / p.initial_stepsize) / std::log(p.sub_config_times),
                           INFINITY);
        int next_exp = std::max((int)exponent + 1, 1);
        return p.initial_stepsize * std::pow(p.sub_config_times, next_exp);
    }
    return INFINITY;
}

template <typename T>
void dalloc(T **p, size_t count) {
    D4_CUDA_OK(d4::dmalloc((void **)p, sizeof(T) * (count > 0 ? count : 1)));
}

void free_all(Ctx *c) {
    void *bufs[] = {c->x0, c->y, c->xb, c->xh, c->x2, c->xs_tmp, c->ys_tmp, c->v_init,
                    c->v_init2, c->speed, c->speed2, c->dvec, c->dvec_new, c->fac, c->dx,
                    c->tol, c->A, c->LU, c->F, c->piv, c->perm, c->flags, c->red,
                    c->wave_err, c->xw1, c->xw2,
                    c->rowsub, c->rowsc,
                    c->lu_p0, c->lu_q, c->lu_mask, c->lu_bar, c->A32, c->LU32, c->lu32_p0,
                    c->lu32_q, c->m_g, c->m_r, c->m_dx, c->m_c32, c->m_w1, c->m_resid,
                    c->m_part, c->m_dx2, c->m_cnt, c->m_conv, c->spiv};
    for (void *b : bufs)
        if (b) cudaFree(b);
    d4::sparse_free(*c);
    d4::blu_free(c->blu);
    d4::blu_free(c->m32b.blu);
    if (c->blu_tasks) cudaFree(c->blu_tasks);
    const d4::Mix32Bufs &B = c->m32b;
    void *ob[] = {c->lub.LU, c->lub.P0, c->lub.Q, c->lub.mask, c->lub.bar, c->lub.perm,
                  c->lub.piv, c->flags3, c->F_b, c->dvec_b, c->speed_b, c->speed2_b, c->xw1_b,
                  c->xw2_b, c->dx_b, B.A32, B.LU32, B.P0, B.Q, B.mask, B.bar, B.perm, B.piv,
                  B.g, B.r, B.dx, B.part, B.c32, B.w1, B.resid, B.dx2, B.cnt, B.conv, B.A64,
                  c->fr_part[0], c->fr_part[1], c->fr_cnt[0], c->fr_cnt[1]};
    for (void *b : ob)
        if (b) cudaFree(b);
    if (c->ev_fork) cudaEventDestroy(c->ev_fork);
    if (c->ev_copy) cudaEventDestroy(c->ev_copy);
    if (c->ev_join) cudaEventDestroy(c->ev_join);
    if (c->stream_b) cudaStreamDestroy(c->stream_b);
    if (c->tab) cudaFree(c->tab);
    if (c->h_red) cudaFreeHost(c->h_red);
    if (c->h_flags) cudaFreeHost(c->h_flags);
    for (cudaEvent_t e : c->prof.pool) cudaEventDestroy(e);
    if (c->ev0) cudaEventDestroy(c->ev0);
    if (c->ev1) cudaEventDestroy(c->ev1);
    if (c->stream) cudaStreamDestroy(c->stream);
}

int fail(Ctx *c, int code, const std::string &msg) {
    if (c) c->err = msg;
    return code;
}

#define D4_GUARD_BEGIN try {
#define D4_GUARD_END(c)                                         \
    }                                                           \
    catch (const CudaError &e) {                                \
        return fail((c), D4_ERR_CUDA, e.what);                  \
    }                                                           \
    catch (const d4::StateError &e) {                           \
        return fail((c), D4_ERR_STATE, e.what);                 \
    }                                                           \
    catch (const std::bad_alloc &) {                            \
        return fail((c), D4_ERR_NOMEM, "host allocation failed"); \
    }

void upload(Ctx &c, double *dst, const double *src) {
    D4_CUDA_OK(cudaMemcpyAsync(dst, src, sizeof(double) * c.n, cudaMemcpyHostToDevice, c.stream));
}

void download(Ctx &c, double *dst, const double *src) {
    D4_CUDA_OK(cudaMemcpyAsync(dst, src, sizeof(double) * c.n, cudaMemcpyDeviceToHost, c.stream));
}

void sync(Ctx &c) { D4_CUDA_OK(cudaStreamSynchronize(c.stream)); }

// Errors that kernels record instead of hanging (bounded waits), read back
// into h_flags[0..5] from wave_err after a stream sync.
void check_async_errors(Ctx &c) {
    const int *werr = c.h_flags;
    if (werr[0]) {
        c.err_detail = "triangular solve wait timed out: block " + std::to_string(werr[1]) +
                       " waiting for block " + std::to_string(werr[2]);
        throw d4::StateError(c.err_detail.c_str());
    }
    if (werr[d4::kWaveErrRows]) throw d4::StateError("row-sum pipeline wait timed out");
}

void read_async_errors(Ctx &c) {
    D4_CUDA_OK(cudaMemcpyAsync(c.h_flags, c.wave_err, sizeof(int) * 6, cudaMemcpyDeviceToHost,
                               c.stream));
    sync(c);
    check_async_errors(c);
}

// Mixed form backoff: after the f-th attempt in a row that neither the block
// LU nor the pivoted FP32 LU could refine, the next 2^(f-1) attempts (at most
// kMaxSkip) run on the FP64 path; after the b-th block-LU failure in a row the
// next 2^(b-1) - 1 attempts use the pivoted FP32 LU directly.  A successful
// block-LU attempt resets b, an attempt that FP32 factors refine resets f, so
// a stretch of states that defeats a path wastes at most one try of it in
// kMaxSkip attempts.
constexpr int kMaxSkip = 64;

// Below this order the mixed form's attempts run on the FP64 path: there the
// exact LU is bound by its per-block latency, not by its arithmetic, so FP32
// factors save little, while their refinement (and, for the stiff Jacobians of
// close pairs, the fallbacks) costs more than the FP64 solves (measured at
// N = 1024 over 300 steps of the relaxed state: 0.6x the FP64 form).
constexpr int kMixedMinN = 2048;

// Grid split of an attempt's two concurrent cooperative factorisations:
// stage I's chain (one LU, two solves, one sweep) is the shorter one, so it
// gets 40% of the co-resident CTAs and stage II's factorisation the rest.
// Neither gets fewer than one thread per row (n / 256 CTAs), as the full
// grid's size check requires.
static void stage_split(int grid, int n, int &g1, int &g2) {
    const int need = (n + 255) / 256;
    g1 = std::max(need, grid * 2 / 5);
    g2 = grid - g1;
    if (g2 < need) g1 = g2 = std::max(1, grid / 2);
}

// Stages I-IV with stage I on a second stream (FP64 dense form).  Stage I
// (the big step: LU of A1, two solves, one stress sweep) feeds only the error
// ratio, and stage II starts from the unfactored A1, so once A1 is copied into
// stage I's factor buffer the two chains are independent: stage I runs on
// stream_b with its own factors, force scratch and copies of d and the end
// speed, while stages II and III run on the context's stream.  The two
// concurrent cooperative factorisations take half the CTAs each, so both are
// co-resident; stage III's runs on the full grid.  Every operation is the
// sequential attempt's, so the results are identical; the factorisations'
// flags go to separate slots and are read once at the end.
static void attempt_overlap(Ctx &c, double t0, double h, int *singular_out) {
    using d4::ProfScope;
    const d4_protocol &pr = c.p.protocol;
    const double t1 = t0 + h, th = t0 + h / 2;
    const int n = c.n;
    d4::LuBufs L1 = c.lub, L2 = d4::primary_lu(c), L3 = d4::primary_lu(c);
    L1.flags = c.flags3;
    L2.flags = c.flags3 + d4::kFlagCount;
    L3.flags = c.flags3 + 2 * d4::kFlagCount;
    d4::SolveBufs Sa, Sb;
    Sa.dvec = c.dvec;
    Sa.xw1 = c.xw1;
    Sa.xw2 = c.xw2;
    Sa.dx = c.dx;
    Sb.dvec = c.dvec_b;
    Sb.xw1 = c.xw1_b;
    Sb.xw2 = c.xw2_b;
    Sb.dx = c.dx_b;
    int g1, g2;
    stage_split(c.lu_grid, n, g1, g2);
    cudaStream_t sa = c.stream, sb = c.stream_b;
    {
        ProfScope ps(c, D4_CAT_JACOBIAN);
        d4::jacobian64(c, c.x0, c.y, h, ext_stress(pr, t0), ext_stress(pr, t1), c.v_init, c.speed);
    }
    D4_CUDA_OK(cudaMemcpyAsync(c.dvec_b, c.dvec, sizeof(double) * n, cudaMemcpyDeviceToDevice, sa));
    D4_CUDA_OK(cudaMemcpyAsync(c.speed_b, c.speed, sizeof(double) * n, cudaMemcpyDeviceToDevice, sa));
    D4_CUDA_OK(cudaEventRecord(c.ev_fork, sa));
    D4_CUDA_OK(cudaStreamWaitEvent(sb, c.ev_fork, 0));
    // stage I on stream_b
    {
        ProfScope ps(c, D4_CAT_FACTOR, sb);
        d4::factor64_async(c, L1, c.A, g1, sb, c.ev_copy);
    }
    {
        ProfScope ps(c, D4_CAT_SOLVE, sb);
        d4::solve_update64_with(c, L1, Sb, sb, d4::kGBig, h, c.speed_b, c.v_init, nullptr, nullptr,
                                c.x0, c.xb);
    }
    {
        ProfScope ps(c, D4_CAT_SPEEDS, sb);
        d4::speeds64_with(c, c.F_b, sb, c.xb, c.y, ext_stress(pr, t1), c.speed2_b);
    }
    {
        ProfScope ps(c, D4_CAT_SOLVE, sb);
        d4::solve_update64_with(c, L1, Sb, sb, d4::kGNewton, h, c.speed2_b, c.v_init, c.xb, c.x0,
                                c.xb, c.xb);
    }
    D4_CUDA_OK(cudaEventRecord(c.ev_join, sb));
    // stage II on the context's stream, once A1 is copied
    D4_CUDA_OK(cudaStreamWaitEvent(sa, c.ev_copy, 0));
    {
        ProfScope ps(c, D4_CAT_RESCALE);
        d4::jacobian_from_prev64(c, (th - t0) / (t1 - t0));
    }
    {
        ProfScope ps(c, D4_CAT_FACTOR);
        d4::factor64_async(c, L2, c.A, g2, sa, nullptr);
    }
    d4::shift_speed64(c, c.speed, ext_stress(pr, th) - ext_stress(pr, t1));
    {
        ProfScope ps(c, D4_CAT_SOLVE);
        d4::solve_update64_with(c, L2, Sa, sa, d4::kGHalf, h, c.speed, c.v_init, nullptr, nullptr,
                                c.x0, c.xh);
    }
    {
        ProfScope ps(c, D4_CAT_SPEEDS);
        d4::speeds64(c, c.xh, c.y, ext_stress(pr, th), c.speed2);
    }
    {
        ProfScope ps(c, D4_CAT_SOLVE);
        d4::solve_update64_with(c, L2, Sa, sa, d4::kGNewton, h / 2, c.speed2, c.v_init, c.xh, c.x0,
                                c.xh, c.xh);
    }
    // stage III
    {
        ProfScope ps(c, D4_CAT_JACOBIAN);
        d4::jacobian64(c, c.xh, c.y, h / 2, ext_stress(pr, th), ext_stress(pr, t1), c.v_init2,
                       c.speed2);
    }
    {
        ProfScope ps(c, D4_CAT_FACTOR);
        d4::factor64_async(c, L3, c.A, c.lu_grid, sa, nullptr);
    }
    {
        ProfScope ps(c, D4_CAT_SOLVE);
        d4::solve_update64_with(c, L3, Sa, sa, d4::kGHalf, h, c.speed2, c.v_init2, nullptr, nullptr,
                                c.xh, c.x2);
    }
    {
        ProfScope ps(c, D4_CAT_SPEEDS);
        d4::speeds64(c, c.x2, c.y, ext_stress(pr, t1), c.speed2);
    }
    {
        ProfScope ps(c, D4_CAT_SOLVE);
        d4::solve_update64_with(c, L3, Sa, sa, d4::kGNewton, h / 2, c.speed2, c.v_init2, c.x2,
                                c.xh, c.x2, c.x2);
    }
    D4_CUDA_OK(cudaStreamWaitEvent(sa, c.ev_join, 0));
    d4::error_ratio64(c, c.xb, c.x2);
    D4_CUDA_OK(cudaMemcpyAsync(c.h_red, c.red, sizeof(double) * 2, cudaMemcpyDeviceToHost, sa));
    D4_CUDA_OK(cudaMemcpyAsync(c.h_flags, c.wave_err, sizeof(int) * 6, cudaMemcpyDeviceToHost, sa));
    int fl[3 * d4::kFlagCount];
    D4_CUDA_OK(cudaMemcpyAsync(fl, c.flags3, sizeof(fl), cudaMemcpyDeviceToHost, sa));
    sync(c);
    if (c.prof.on) d4::prof_collect(c);
    check_async_errors(c);
    int singular = 0;
    for (int k = 0; k < 3; ++k) {
        if (fl[k * d4::kFlagCount + d4::kFlagBarrierTimeout])
            throw d4::StateError("LU grid barrier timed out");
        singular |= fl[k * d4::kFlagCount + d4::kFlagSingular] != 0;
        d4::count_lu(c, fl + k * d4::kFlagCount);
    }
    // the last factorisation's flags stand for the context's (d4_solve etc.)
    D4_CUDA_OK(cudaMemcpyAsync(c.flags, L3.flags, sizeof(int) * d4::kFlagCount,
                               cudaMemcpyDeviceToDevice, sa));
    c.factor_singular = fl[2 * d4::kFlagCount + d4::kFlagSingular] != 0;
    c.factor_pivoted = 0;
    *singular_out = singular;
}

// Worst refined residual max|r| / max|g| over a ring of 8 (max |r|, max |g|)
// pairs (as ordered bits of non-negatives), 0 where nothing was recorded.
static double worst_refined(const unsigned long long *rb) {
    double worst = 0;
    for (int k = 0; k < 8; ++k) {
        double r, g;
        std::memcpy(&r, &rb[2 * k], 8);
        std::memcpy(&g, &rb[2 * k + 1], 8);
        if (std::isnan(r) || std::isnan(g)) return NAN;  // a NaN must fail the checks
        if (g > 0) {
            const double q = r / g;
            if (!std::isfinite(q)) return NAN;  // inf / inf as well
            worst = std::max(worst, q);
        }
    }
    return worst;
}

// The mixed form's stages I-IV with stage I on a second stream, as
// attempt_overlap: the FP64 form's sweeps and rescale, the factorisations and
// refined solves of d4_mixed.cu.  Stage I copies A1 into its own FP64 matrix
// (the one its refinement multiplies) before factorising it, and runs its two
// solves and its stress sweep on stream_b with its own buffers; stages II and
// III run on the context's stream.  Every operation is the sequential
// attempt's, so the results are identical.  *refine_out: the worst refined
// residual of the attempt's six solves.
static void attempt_overlap_mixed(Ctx &c, double t0, double h, int *singular_out,
                                  double *refine_out) {
    using d4::ProfScope;
    const d4_protocol &pr = c.p.protocol;
    const double t1 = t0 + h, th = t0 + h / 2;
    const int n = c.n;
    d4::Mix32Bufs B1 = c.m32b, B2 = d4::primary_mix32(c), B3 = d4::primary_mix32(c);
    B1.flags = c.flags3;
    B2.flags = c.flags3 + d4::kFlagCount;
    B3.flags = c.flags3 + 2 * d4::kFlagCount;
    int g1, g2;
    stage_split(c.lu32_grid, n, g1, g2);
    cudaStream_t sa = c.stream, sb = c.stream_b;
    {
        ProfScope ps(c, D4_CAT_JACOBIAN);
        d4::jacobian64(c, c.x0, c.y, h, ext_stress(pr, t0), ext_stress(pr, t1), c.v_init, c.speed);
    }
    D4_CUDA_OK(cudaMemcpyAsync(c.dvec_b, c.dvec, sizeof(double) * n, cudaMemcpyDeviceToDevice, sa));
    D4_CUDA_OK(cudaMemcpyAsync(c.speed_b, c.speed, sizeof(double) * n, cudaMemcpyDeviceToDevice, sa));
    D4_CUDA_OK(cudaEventRecord(c.ev_fork, sa));
    D4_CUDA_OK(cudaStreamWaitEvent(sb, c.ev_fork, 0));
    // stage I on stream_b
    {
        ProfScope ps(c, D4_CAT_FACTOR, sb);
        d4::factor32_async(c, B1, c.A, true, g1, sb, c.ev_copy);
    }
    {
        ProfScope ps(c, D4_CAT_SOLVE, sb);
        d4::solve_update32_with(c, B1, c.dvec_b, c.dx_b, sb, d4::kGBig, h, c.speed_b, c.v_init,
                                nullptr, nullptr, c.x0, c.xb);
    }
    {
        ProfScope ps(c, D4_CAT_SPEEDS, sb);
        d4::speeds64_with(c, c.F_b, sb, c.xb, c.y, ext_stress(pr, t1), c.speed2_b);
    }
    {
        ProfScope ps(c, D4_CAT_SOLVE, sb);
        d4::solve_update32_with(c, B1, c.dvec_b, c.dx_b, sb, d4::kGNewton, h, c.speed2_b,
                                c.v_init, c.xb, c.x0, c.xb, c.xb);
    }
    D4_CUDA_OK(cudaEventRecord(c.ev_join, sb));
    // stage II on the context's stream, once A1 is copied
    D4_CUDA_OK(cudaStreamWaitEvent(sa, c.ev_copy, 0));
    {
        ProfScope ps(c, D4_CAT_RESCALE);
        d4::jacobian_from_prev64(c, (th - t0) / (t1 - t0));
    }
    {
        ProfScope ps(c, D4_CAT_FACTOR);
        d4::factor32_async(c, B2, c.A, false, g2, sa, nullptr);
    }
    d4::shift_speed64(c, c.speed, ext_stress(pr, th) - ext_stress(pr, t1));
    {
        ProfScope ps(c, D4_CAT_SOLVE);
        d4::solve_update32_with(c, B2, c.dvec, c.dx, sa, d4::kGHalf, h, c.speed, c.v_init, nullptr,
                                nullptr, c.x0, c.xh);
    }
    {
        ProfScope ps(c, D4_CAT_SPEEDS);
        d4::speeds64(c, c.xh, c.y, ext_stress(pr, th), c.speed2);
    }
    {
        ProfScope ps(c, D4_CAT_SOLVE);
        d4::solve_update32_with(c, B2, c.dvec, c.dx, sa, d4::kGNewton, h / 2, c.speed2, c.v_init,
                                c.xh, c.x0, c.xh, c.xh);
    }
    // stage III
    {
        ProfScope ps(c, D4_CAT_JACOBIAN);
        d4::jacobian64(c, c.xh, c.y, h / 2, ext_stress(pr, th), ext_stress(pr, t1), c.v_init2,
                       c.speed2);
    }
    {
        ProfScope ps(c, D4_CAT_FACTOR);
        d4::factor32_async(c, B3, c.A, false, c.lu32_grid, sa, nullptr);
    }
    {
        ProfScope ps(c, D4_CAT_SOLVE);
        d4::solve_update32_with(c, B3, c.dvec, c.dx, sa, d4::kGHalf, h, c.speed2, c.v_init2,
                                nullptr, nullptr, c.xh, c.x2);
    }
    {
        ProfScope ps(c, D4_CAT_SPEEDS);
        d4::speeds64(c, c.x2, c.y, ext_stress(pr, t1), c.speed2);
    }
    {
        ProfScope ps(c, D4_CAT_SOLVE);
        d4::solve_update32_with(c, B3, c.dvec, c.dx, sa, d4::kGNewton, h / 2, c.speed2,
                                c.v_init2, c.x2, c.xh, c.x2, c.x2);
    }
    D4_CUDA_OK(cudaStreamWaitEvent(sa, c.ev_join, 0));
    d4::error_ratio64(c, c.xb, c.x2);
    D4_CUDA_OK(cudaMemcpyAsync(c.h_red, c.red, sizeof(double) * 2, cudaMemcpyDeviceToHost, sa));
    D4_CUDA_OK(cudaMemcpyAsync(c.h_flags, c.wave_err, sizeof(int) * 6, cudaMemcpyDeviceToHost, sa));
    int fl[3 * d4::kFlagCount];
    D4_CUDA_OK(cudaMemcpyAsync(fl, c.flags3, sizeof(fl), cudaMemcpyDeviceToHost, sa));
    unsigned long long rb[2][16];
    D4_CUDA_OK(cudaMemcpyAsync(rb[0], c.m_resid, sizeof(rb[0]), cudaMemcpyDeviceToHost, sa));
    D4_CUDA_OK(cudaMemcpyAsync(rb[1], c.m32b.resid, sizeof(rb[1]), cudaMemcpyDeviceToHost, sa));
    sync(c);
    if (c.prof.on) d4::prof_collect(c);
    check_async_errors(c);
    int singular = 0;
    for (int k = 0; k < 3; ++k) {
        if (fl[k * d4::kFlagCount + d4::kFlagBarrierTimeout])
            throw d4::StateError("LU grid barrier timed out");
        singular |= fl[k * d4::kFlagCount + d4::kFlagSingular] != 0;
        d4::count_lu(c, fl + k * d4::kFlagCount);
    }
    // the last factorisation's flags stand for the context's (d4_solve etc.)
    D4_CUDA_OK(cudaMemcpyAsync(c.flags, B3.flags, sizeof(int) * d4::kFlagCount,
                               cudaMemcpyDeviceToDevice, sa));
    D4_CUDA_OK(cudaMemsetAsync(c.m_resid, 0, sizeof(rb[0]), sa));
    D4_CUDA_OK(cudaMemsetAsync(c.m32b.resid, 0, sizeof(rb[1]), sa));
    c.factor_singular = fl[2 * d4::kFlagCount + d4::kFlagSingular] != 0;
    c.factor_pivoted = 0;
    *singular_out = singular;
    *refine_out = std::max(worst_refined(rb[0]), worst_refined(rb[1]));
}

// Stages I-IV of src/simulation.cpp:90-161 on the device.
// fp64: in the mixed form, run this attempt on the FP64 form's factorisations
// and solves (with stage I overlapped when the context holds the FP64 form's
// stage-I buffers, as below kMixedMinN; else in sequence).
static int attempt_once(Ctx &c, double t0, double h, d4_attempt_result *res, bool fp64 = false) {
    const bool mixed_path = c.p.precision == D4_PREC_MIXED && !fp64;
    if (c.overlap && (mixed_path || c.lub.LU)) {
        int singular = 0;
        double refine = 0;
        if (mixed_path)
            attempt_overlap_mixed(c, t0, h, &singular, &refine);
        else
            attempt_overlap(c, t0, h, &singular);
        const int idx = (int)c.h_red[1];
        if (idx >= 0) c.selected_id = idx;
        res->ratio = c.h_red[0] / c.dipole_prec_sq;
        res->max_id = c.selected_id;
        res->accepted = res->ratio < 1;
        res->singular = singular;
        res->pivoted = 0;
        res->refine_residual = refine;
        return D4_OK;
    }
    using d4::ProfScope;
    const d4_protocol &pr = c.p.protocol;
    const double t_1__ = t0 + h;
    const double t_1p2 = t0 + h / 2;
    int singular = 0, pivoted = 0;
    const bool mixed = c.p.precision == D4_PREC_MIXED && !fp64;
    auto jac = [&](const double *x, double hh, double ta, double tb, double *va, double *vb) {
        ProfScope ps(c, D4_CAT_JACOBIAN);
        d4::jacobian64(c, x, c.y, hh, ext_stress(pr, ta), ext_stress(pr, tb), va, vb);
    };
    const bool gmres = c.use_gmres != 0;
    auto dense_fac = [&]() {
        const int st = mixed ? d4::factor32(c) : d4::factor64(c);
        singular |= st == D4_WARN_SINGULAR;
        pivoted += c.factor_pivoted;
    };
    auto fac = [&]() {
        ProfScope ps(c, D4_CAT_FACTOR);
        if (gmres)
            d4::sparse_prepare(c);
        else
            dense_fac();
    };
    auto spd = [&](const double *x, double t, double *v) {
        ProfScope ps(c, D4_CAT_SPEEDS);
        d4::speeds64(c, x, c.y, ext_stress(pr, t), v);
    };
    auto slv = [&](int gmode, double hv, const double *se, const double *si, const double *xn,
                   const double *xo, const double *base, double *out) {
        ProfScope ps(c, D4_CAT_SOLVE);
        if (gmres) {
            if (d4::sparse_solve_update(c, gmode, hv, se, si, xn, xo, base, out)) return;
            if (!c.sp_dense_ready) {  // GMRES did not converge: dense LU of the same matrix
                dense_fac();
                c.sp_dense_ready = 1;
            }
        }
        if (mixed)
            d4::solve_update32(c, gmode, hv, se, si, xn, xo, base, out);
        else
            d4::solve_update64(c, gmode, hv, se, si, xn, xo, base, out);
    };
    // stage I: one large step
    jac(c.x0, h, t0, t_1__, c.v_init, c.speed);
    fac();
    slv(d4::kGBig, h, c.speed, c.v_init, nullptr, nullptr, c.x0, c.xb);
    spd(c.xb, t_1__, c.speed2);
    slv(d4::kGNewton, h, c.speed2, c.v_init, c.xb, c.x0, c.xb, c.xb);
    // stage II: first small step, Jacobian from the previous one
    {
        const double factor = (t_1p2 - t0) / (t_1__ - t0);
        {
            ProfScope ps(c, D4_CAT_RESCALE);
            d4::jacobian_from_prev64(c, factor);
        }
        fac();
        const double dif = ext_stress(pr, t_1p2) - ext_stress(pr, t_1__);
        d4::shift_speed64(c, c.speed, dif);
    }
    slv(d4::kGHalf, h, c.speed, c.v_init, nullptr, nullptr, c.x0, c.xh);
    spd(c.xh, t_1p2, c.speed2);
    slv(d4::kGNewton, h / 2, c.speed2, c.v_init, c.xh, c.x0, c.xh, c.xh);
    // stage III: second small step
    jac(c.xh, h / 2, t_1p2, t_1__, c.v_init2, c.speed2);
    fac();
    slv(d4::kGHalf, h, c.speed2, c.v_init2, nullptr, nullptr, c.xh, c.x2);
    spd(c.x2, t_1__, c.speed2);
    slv(d4::kGNewton, h / 2, c.speed2, c.v_init2, c.x2, c.xh, c.x2, c.x2);
    // stage IV: error ratio
    d4::error_ratio64(c, c.xb, c.x2);
    D4_CUDA_OK(cudaMemcpyAsync(c.h_red, c.red, sizeof(double) * 2, cudaMemcpyDeviceToHost,
                               c.stream));
    D4_CUDA_OK(cudaMemcpyAsync(c.h_flags, c.wave_err, sizeof(int) * 6, cudaMemcpyDeviceToHost,
                               c.stream));
    sync(c);
    if (c.prof.on) d4::prof_collect(c);
    check_async_errors(c);
    const int idx = (int)c.h_red[1];
    if (idx >= 0) c.selected_id = idx;
    res->ratio = c.h_red[0] / c.dipole_prec_sq;
    res->max_id = c.selected_id;
    res->accepted = res->ratio < 1;
    res->singular = singular;
    res->pivoted = pivoted;
    res->refine_residual = 0;
    if (mixed) {
        unsigned long long rb[16];
        D4_CUDA_OK(cudaMemcpy(rb, c.m_resid, sizeof(rb), cudaMemcpyDeviceToHost));
        res->refine_residual = worst_refined(rb);
        D4_CUDA_OK(cudaMemset(c.m_resid, 0, sizeof(rb)));
    }
    return D4_OK;
}

// One attempted step.  In the mixed form the factorisations are block LUs
// without row interchanges between tiles (d4_blu32.cu); when one of them met
// a zero or non-finite pivot in a diagonal tile, or a refined solve kept a
// residual above kRefineLimit, the attempt is redone with the pivoted FP32 LU
// and, if its refinement fails too, with the FP64 form's attempt, so an
// accepted result always carries a refined residual within kRefineLimit or
// the FP64 form's solves.
int attempt(Ctx &c, double t0, double h, d4_attempt_result *res) {
    if (c.p.precision != D4_PREC_MIXED) return attempt_once(c, t0, h, res);
    auto fp32_ok = [&]() {
        return !res->singular && res->refine_residual <= d4::kRefineLimit &&
               std::isfinite(res->ratio);
    };
    auto fp64_attempt = [&]() {
        ++c.m_fp64_attempts;
        attempt_once(c, t0, h, res, true);
        d4::adopt_pivots(c);  // the next block LUs factorise P A with this attempt's P
    };
    auto pivoted_attempt = [&]() {
        ++c.m_pivoted32;
        c.m_fast = 0;
        try {
            attempt_once(c, t0, h, res);
        } catch (...) {
            c.m_fast = 1;
            throw;
        }
        c.m_fast = 1;
        d4::adopt_pivots(c);
    };
    if (!c.m_fast || c.m_skip > 0 || c.n < kMixedMinN) {
        // the FP64 form's attempt: block LU switched off, a recent attempt
        // that FP32 factors could not refine, or a system too small to gain
        if (c.m_skip > 0) --c.m_skip;
        fp64_attempt();
        return D4_OK;
    }
    if (c.m_piv_skip > 0) {
        // a recent block-LU failure: the pivoted FP32 LU directly
        --c.m_piv_skip;
        pivoted_attempt();
        if (fp32_ok()) {
            if (res->refine_residual > c.m_worst_refine) c.m_worst_refine = res->refine_residual;
            return D4_OK;
        }
    } else {
        const long long before = c.m_blocklu;
        attempt_once(c, t0, h, res);
        if (c.m_blocklu == before) return D4_OK;  // no dense factorisation ran (GMRES)
        if (fp32_ok()) {
            if (res->refine_residual > c.m_worst_refine) c.m_worst_refine = res->refine_residual;
            c.m_block_run = 0;
            c.m_fallback_run = 0;
            return D4_OK;
        }
        // a diagonal tile met a bad pivot or the refinement did not converge:
        // the explicit inverses of the diagonal tiles lose accuracy when a tile
        // is ill-conditioned (close pairs), which the backward-stable pivoted
        // FP32 LU does not; it redoes the attempt, and the next block LUs wait
        // 2^(b-1) attempts after the b-th failure in a row (at most kMaxSkip)
        ++c.m_fallbacks;
        c.m_piv_skip = std::min(kMaxSkip, 1 << std::min(c.m_block_run, 6)) - 1;
        ++c.m_block_run;
        pivoted_attempt();
        if (fp32_ok()) {
            if (res->refine_residual > c.m_worst_refine) c.m_worst_refine = res->refine_residual;
            c.m_fallback_run = 0;
            return D4_OK;
        }
    }
    // the Jacobian is too ill-conditioned for FP32 factors: the FP64 form's
    // attempt, and the next attempts go there directly (backing off, kMaxSkip)
    c.m_skip = std::min(kMaxSkip, 1 << std::min(c.m_fallback_run, 6));
    ++c.m_fallback_run;
    fp64_attempt();
    return D4_OK;
}

// Stress sweep (both forms use the FP64 sweeps).
void sweep_speeds(Ctx &c, const double *x, const double *y, double ext, double *v) {
    d4::speeds64(c, x, y, ext, v);
}

// Device matrix (FP64 in both forms) to a host buffer.
void copy_matrix_out(Ctx &c, double *dst) {
    if (!dst) return;
    const size_t nn = (size_t)c.n * c.n;
    D4_CUDA_OK(cudaMemcpyAsync(dst, c.A, sizeof(double) * nn, cudaMemcpyDeviceToHost, c.stream));
}

double host_abs_sum(const std::vector<double> &v) {
    double s = 0;
    for (double x : v) s = s + std::fabs(x);
    return s;
}

double host_sq_sum(const std::vector<double> &v) {
    double s = 0;
    for (double x : v) s = s + x * x;
    return s;
}

void write_config(Ctx &c, const std::string &path, const unsigned *order) {
    std::vector<double> x(c.n), y(c.n);
    download(c, x.data(), c.x0);
    download(c, y.data(), c.y);
    sync(c);
    std::ofstream of(path);
    if (!of) return;
    // src/simulation_data.cpp:177-191: original order, 14 significant digits
    of << std::setprecision(14);
    for (int k = 0; k < c.n; ++k) {
        const unsigned id = order ? order[k] : (unsigned)k;
        of << x[id] << "\t" << y[id] << "\t" << (id < (unsigned)c.n / 2 ? 1 : -1) << "\n";
    }
}

}  // namespace

extern "C" {

int d4_check_positions(int n, const double *x, const double *y) {
    if (n < 0 || (n > 0 && (!x || !y))) return -2;
    for (int i = 0; i < n; ++i) {
        // finite and inside the periodic cell, where normalize
        // (src/sim_utils.cpp:6-13) keeps every position
        if (!(x[i] >= -0.5 && x[i] < 0.5 && y[i] >= -0.5 && y[i] < 0.5)) return i;
    }
    return -1;
}

void d4_default_params(d4_params *p) {
    std::memset(p, 0, sizeof(*p));
    p->position_precision = 1e-5;
    p->dipole_precision = 0.05;
    p->cutoff_multiplier = 1e20;
    p->initial_stepsize = 1e-6;
    p->max_stepsize = -1;
    p->weight_function = 'c';
    p->time_limit = -1;
    p->step_count_limit = -1;
    p->strain_increase_limit = -1;
    p->avalanche_limit = -1;
    p->avalanche_speed_threshold = 1e-3;
    p->sub_config_delay = 5;
    p->sub_config_delay_during_avalanche = 1;
    p->sub_config_times_type = 'a';
    p->precision = D4_PREC_FP64;
    p->device = 0;
    p->solver = D4_SOLVER_DENSE;
    p->field = D4_FIELD_ANALYTIC;
    p->table_size = 1024;
}

int d4_create(void **out, int n, const d4_params *p) {
    if (!out || !p) return D4_ERR_ARG;
    *out = nullptr;
    if (n < 2 || n % 2 != 0 || n > d4::kMaxSolveN) return D4_ERR_ARG;
    if (p->weight_function != 'c' && p->weight_function != 'p' && p->weight_function != 'm')
        return D4_ERR_ARG;
    if (p->precision != D4_PREC_FP64 && p->precision != D4_PREC_MIXED) return D4_ERR_ARG;
    if (p->solver < D4_SOLVER_DENSE || p->solver > D4_SOLVER_AUTO) return D4_ERR_ARG;
    if (p->field != D4_FIELD_ANALYTIC && p->field != D4_FIELD_TABULATED) return D4_ERR_ARG;
    if (p->field == D4_FIELD_TABULATED &&
        (p->precision != D4_PREC_FP64 || p->table_size < 16 || p->table_size > 4096))
        return D4_ERR_ARG;
    Ctx *c = new (std::nothrow) Ctx();
    if (!c) return D4_ERR_NOMEM;
    try {
        c->n = n;
        c->p = *p;
        D4_CUDA_OK(cudaSetDevice(p->device));
        D4_CUDA_OK(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking));
        D4_CUDA_OK(cudaEventCreate(&c->ev0));
        D4_CUDA_OK(cudaEventCreate(&c->ev1));
        // PrecisionHandler::setMinPrecisity + setDipolePrecisity
        // (src/precision_handler.cpp:65-89, src/simulation.cpp:24-26)
        c->min_prec_sq = p->position_precision * p->position_precision;
        if (p->dipole_precision == 0) {
            c->use_dipole = 0;
            c->dipole_prec_sq = 1;
        } else {
            c->use_dipole = 1;
            c->dipole_prec_sq = p->dipole_precision * p->dipole_precision;
            c->min_prec_sq /= p->dipole_precision * p->dipole_precision;
        }
        // SimulationData::updateCutOff, src/simulation_data.cpp:253-262
        double mult = p->cutoff_multiplier;
        if (!p->heaviside_cutoff && p->cutoff_multiplier >= std::sqrt(2 * (double)n) / 12)
            mult = 1e20;
        c->cutoff = mult / std::sqrt((double)n);
        c->cutoff_sq = c->cutoff * c->cutoff;
        c->range_sq = p->heaviside_cutoff ? 1 : 49;
        c->step_size = p->initial_stepsize;
        const size_t nn = (size_t)n * n;
        double **vecs[] = {&c->x0, &c->y, &c->xb, &c->xh, &c->x2, &c->xs_tmp, &c->ys_tmp,
                           &c->v_init, &c->v_init2, &c->speed, &c->speed2, &c->dvec,
                           &c->dvec_new, &c->fac, &c->dx, &c->tol};
        for (double **v : vecs) dalloc(v, (size_t)n);
        const bool mixed = p->precision == D4_PREC_MIXED;
        // both forms: the FP64 matrix and pair-force scratch of the FP64 sweeps;
        // the FP64 factors only in the FP64 form
        dalloc(&c->A, nn);
        dalloc(&c->LU, nn);  // the mixed form's FP64 attempts factorise here too
        dalloc(&c->F, nn);
        if (mixed) {
            dalloc(&c->A32, nn);
            dalloc(&c->LU32, nn);
            dalloc(&c->lu32_p0, (size_t)n * 32);
            dalloc(&c->lu32_q, (size_t)n * 64);
            double **mv[] = {&c->m_g, &c->m_r, &c->m_dx, &c->m_dx2};
            for (double **v : mv) dalloc(v, (size_t)n);
            dalloc(&c->m_cnt, (size_t)(n + 255) / 256);
            D4_CUDA_OK(cudaMemset(c->m_cnt, 0, sizeof(unsigned) * ((n + 255) / 256)));
            dalloc(&c->m_conv, (size_t)d4::kIrMax + 1);
            dalloc(&c->m_c32, (size_t)n);
            dalloc(&c->m_w1, (size_t)n);
            dalloc(&c->m_part, (size_t)((n + 255) / 256) * n);
            dalloc(&c->m_resid, 16);
            D4_CUDA_OK(cudaMemset(c->m_resid, 0, sizeof(unsigned long long) * 16));
            std::vector<int> ident(n);
            for (int i = 0; i < n; ++i) ident[i] = i;
            dalloc(&c->spiv, (size_t)n);
            D4_CUDA_OK(cudaMemcpy(c->spiv, ident.data(), sizeof(int) * n, cudaMemcpyHostToDevice));
            c->lu32_grid = d4::coop_grid_size32(n);
            if (c->lu32_grid < 0) throw d4::StateError("n too large for the cooperative LU");
            const std::vector<int> sched = d4::blu_schedule(n);
            dalloc(&c->blu_tasks, sched.size());
            D4_CUDA_OK(cudaMemcpy(c->blu_tasks, sched.data(), sizeof(int) * sched.size(),
                                  cudaMemcpyHostToDevice));
            d4::blu_alloc(c->blu, n, c->blu_tasks, &c->blu_state);
        }
        dalloc(&c->piv, (size_t)n);
        dalloc(&c->perm, (size_t)n);
        dalloc(&c->flags, (size_t)d4::kFlagCount);
        dalloc(&c->red, 8);
        const int nblk = (n + 31) / 32;
        dalloc(&c->wave_err, 8);
        dalloc(&c->xw1, (size_t)n);
        dalloc(&c->xw2, (size_t)n);
        dalloc(&c->rowsub, (size_t)n);
        dalloc(&c->rowsc, (size_t)n);
        D4_CUDA_OK(cudaMemset(c->wave_err, 0, sizeof(int) * 8));
        D4_CUDA_OK(cudaMallocHost((void **)&c->h_red, sizeof(double) * 8));
        D4_CUDA_OK(cudaMallocHost((void **)&c->h_flags, sizeof(int) * d4::kFlagCount));
        D4_CUDA_OK(cudaMemset(c->A, 0, sizeof(double) * nn));
        D4_CUDA_OK(cudaMemset(c->F, 0, sizeof(double) * nn));
        D4_CUDA_OK(cudaMemset(c->dvec, 0, sizeof(double) * n));
        D4_CUDA_OK(cudaMemset(c->flags, 0, sizeof(int) * d4::kFlagCount));
        c->lu_grid = d4::coop_grid_size(n);
        if (c->lu_grid < 0) throw d4::StateError("n too large for the cooperative LU");
        dalloc(&c->lu_p0, (size_t)n * 32);
        dalloc(&c->lu_q, (size_t)n * 64 + d4::kLuDiagWords);
        c->lu_mask_words = d4::lu_mask_words_for(nblk);
        dalloc(&c->lu_mask, (size_t)c->lu_mask_words);
        dalloc(&c->lu_bar, 64);
        if (p->field == D4_FIELD_TABULATED) {
            c->tab_T = p->table_size;
            d4::table_build(*c);
        }
        c->use_gmres = d4::gmres_selected(*c) ? 1 : 0;
        if (c->use_gmres) d4::sparse_alloc(*c);
        // the mixed form's dense attempts from kMixedMinN on: pair tiles
        // without the reference's operation order (d4_fp64_fast.cu)
        c->fast_pairs = (mixed && n >= kMixedMinN && !c->tab && !c->use_gmres) ? 1 : 0;
        if (c->fast_pairs)
            for (int s = 0; s < 2; ++s) {
                const int rb = (n + 255) / 256, nch = (n + 255) / 256;
                dalloc(&c->fr_part[s], (size_t)2 * nch * n);
                dalloc(&c->fr_cnt[s], (size_t)rb);
                D4_CUDA_OK(cudaMemset(c->fr_cnt[s], 0, sizeof(unsigned) * rb));
            }
        if (!c->use_gmres) {
            // stage I's own stream and buffers (attempt_overlap, attempt_overlap_mixed)
            c->overlap = 1;
            D4_CUDA_OK(cudaStreamCreateWithFlags(&c->stream_b, cudaStreamNonBlocking));
            D4_CUDA_OK(cudaEventCreateWithFlags(&c->ev_fork, cudaEventDisableTiming));
            D4_CUDA_OK(cudaEventCreateWithFlags(&c->ev_copy, cudaEventDisableTiming));
            D4_CUDA_OK(cudaEventCreateWithFlags(&c->ev_join, cudaEventDisableTiming));
            dalloc(&c->flags3, (size_t)3 * d4::kFlagCount);
            double **bv[] = {&c->dvec_b, &c->speed_b, &c->speed2_b, &c->xw1_b, &c->xw2_b,
                             &c->dx_b};
            for (double **v : bv) dalloc(v, (size_t)n);
            dalloc(&c->F_b, nn);
            if (!mixed || n < kMixedMinN) {
                // the FP64 form's stage I (also the mixed form's attempts below
                // kMixedMinN, which run on the FP64 path)
                dalloc(&c->lub.LU, nn);
                dalloc(&c->lub.P0, (size_t)n * 32);
                dalloc(&c->lub.Q, (size_t)n * 64 + d4::kLuDiagWords);
                dalloc(&c->lub.mask, (size_t)c->lu_mask_words);
                dalloc(&c->lub.bar, 64);
                dalloc(&c->lub.perm, (size_t)n);
                dalloc(&c->lub.piv, (size_t)n);
            }
            if (mixed) {
                d4::Mix32Bufs &B = c->m32b;
                dalloc(&B.A64, nn);
                dalloc(&B.conv, (size_t)d4::kIrMax + 1);
                dalloc(&B.A32, nn);
                dalloc(&B.LU32, nn);
                dalloc(&B.P0, (size_t)n * 32);
                dalloc(&B.Q, (size_t)n * 64);
                dalloc(&B.mask, (size_t)c->lu_mask_words);
                dalloc(&B.bar, 64);
                dalloc(&B.perm, (size_t)n);
                dalloc(&B.piv, (size_t)n);
                dalloc(&B.g, (size_t)n);
                dalloc(&B.r, (size_t)n);
                dalloc(&B.dx, (size_t)n);
                dalloc(&B.dx2, (size_t)n);
                dalloc(&B.cnt, (size_t)(n + 255) / 256);
                D4_CUDA_OK(cudaMemset(B.cnt, 0, sizeof(unsigned) * ((n + 255) / 256)));
                dalloc(&B.part, (size_t)((n + 255) / 256) * n);
                dalloc(&B.c32, (size_t)n);
                dalloc(&B.w1, (size_t)n);
                dalloc(&B.resid, 16);
                D4_CUDA_OK(cudaMemset(B.resid, 0, sizeof(unsigned long long) * 16));
                B.resid_count = &c->m_resid_count_b;
                B.blk = &c->m_blk_b;
                d4::blu_alloc(B.blu, n, c->blu_tasks, &c->blu_state_b);
            }
        }
        d4::reset_tol64(*c);
        sync(*c);
    } catch (const CudaError &e) {
        free_all(c);
        delete c;
        return D4_ERR_CUDA;
    } catch (const d4::StateError &e) {
        free_all(c);
        delete c;
        return D4_ERR_STATE;
    }
    *out = c;
    return D4_OK;
}

int d4_destroy(void *ctx) {
    Ctx *c = (Ctx *)ctx;
    if (!c) return D4_ERR_ARG;
    if (c->stream) cudaStreamSynchronize(c->stream);
    free_all(c);
    delete c;
    return D4_OK;
}

const char *d4_last_error(void *ctx) {
    Ctx *c = (Ctx *)ctx;
    return c ? c->err.c_str() : "null context";
}

int d4_set_positions(void *ctx, const double *x, const double *y) {
    Ctx *c = (Ctx *)ctx;
    if (!c || !x || !y) return D4_ERR_ARG;
    const int bad = d4_check_positions(c->n, x, y);
    if (bad >= 0)
        return fail(c, D4_ERR_ARG,
                    "d4_set_positions: dislocation " + std::to_string(bad) +
                        " is not finite or outside the cell [-0.5, 0.5)^2");
    D4_GUARD_BEGIN
    upload(*c, c->x0, x);
    upload(*c, c->y, y);
    sync(*c);
    return D4_OK;
    D4_GUARD_END(c)
}

int d4_get_positions(void *ctx, double *x, double *y) {
    Ctx *c = (Ctx *)ctx;
    if (!c || !x) return D4_ERR_ARG;
    D4_GUARD_BEGIN
    download(*c, x, c->x0);
    if (y) download(*c, y, c->y);
    sync(*c);
    return D4_OK;
    D4_GUARD_END(c)
}

int d4_set_time(void *ctx, double sim_time, double step_size) {
    Ctx *c = (Ctx *)ctx;
    if (!c) return D4_ERR_ARG;
    c->sim_time = sim_time;
    c->step_size = step_size;
    return D4_OK;
}

int d4_reset_tolerance(void *ctx) {
    Ctx *c = (Ctx *)ctx;
    if (!c) return D4_ERR_ARG;
    D4_GUARD_BEGIN
    d4::reset_tol64(*c);
    sync(*c);
    return D4_OK;
    D4_GUARD_END(c)
}

int d4_get_tolerance(void *ctx, double *tol) {
    Ctx *c = (Ctx *)ctx;
    if (!c || !tol) return D4_ERR_ARG;
    D4_GUARD_BEGIN
    download(*c, tol, c->tol);
    sync(*c);
    return D4_OK;
    D4_GUARD_END(c)
}

int d4_set_tolerance(void *ctx, const double *tol) {
    Ctx *c = (Ctx *)ctx;
    if (!c || !tol) return D4_ERR_ARG;
    for (int i = 0; i < c->n; ++i)
        if (!(std::isfinite(tol[i]) && tol[i] >= 0))
            return fail(c, D4_ERR_ARG,
                        "d4_set_tolerance: entry " + std::to_string(i) +
                            " is not a finite non-negative number");
    D4_GUARD_BEGIN
    upload(*c, c->tol, tol);
    sync(*c);
    return D4_OK;
    D4_GUARD_END(c)
}

int d4_speeds(void *ctx, const double *x, const double *y, double sim_time, double *v,
              double *tol) {
    Ctx *c = (Ctx *)ctx;
    if (!c || !x || !y || !v) return D4_ERR_ARG;
    D4_GUARD_BEGIN
    upload(*c, c->xs_tmp, x);
    upload(*c, c->ys_tmp, y);
    d4::speeds64(*c, c->xs_tmp, c->ys_tmp, ext_stress(c->p.protocol, sim_time), c->speed2);
    download(*c, v, c->speed2);
    if (tol) download(*c, tol, c->tol);
    read_async_errors(*c);
    return D4_OK;
    D4_GUARD_END(c)
}

int d4_jacobian(void *ctx, const double *x, const double *y, double stepsize, double t_a,
                double t_b, double *v_a, double *v_b, double *a_colmajor, double *dvec,
                double *tol) {
    Ctx *c = (Ctx *)ctx;
    if (!c || !x || !y || !v_a || !v_b) return D4_ERR_ARG;
    D4_GUARD_BEGIN
    upload(*c, c->xs_tmp, x);
    upload(*c, c->ys_tmp, y);
    d4::jacobian64(*c, c->xs_tmp, c->ys_tmp, stepsize, ext_stress(c->p.protocol, t_a),
                   ext_stress(c->p.protocol, t_b), c->v_init, c->speed);
    download(*c, v_a, c->v_init);
    download(*c, v_b, c->speed);
    if (dvec) download(*c, dvec, c->dvec);
    if (tol) download(*c, tol, c->tol);
    copy_matrix_out(*c, a_colmajor);
    read_async_errors(*c);
    return D4_OK;
    D4_GUARD_END(c)
}

int d4_jacobian_from_prev(void *ctx, double factor, double *a_colmajor, double *dvec) {
    Ctx *c = (Ctx *)ctx;
    if (!c) return D4_ERR_ARG;
    D4_GUARD_BEGIN
    d4::jacobian_from_prev64(*c, factor);
    if (dvec) download(*c, dvec, c->dvec);
    copy_matrix_out(*c, a_colmajor);
    sync(*c);
    return D4_OK;
    D4_GUARD_END(c)
}

int d4_set_matrix(void *ctx, const double *a_colmajor) {
    Ctx *c = (Ctx *)ctx;
    if (!c || !a_colmajor) return D4_ERR_ARG;
    D4_GUARD_BEGIN
    const size_t nn = (size_t)c->n * c->n;
    D4_CUDA_OK(cudaMemcpyAsync(c->A, a_colmajor, sizeof(double) * nn, cudaMemcpyHostToDevice,
                               c->stream));
    sync(*c);
    return D4_OK;
    D4_GUARD_END(c)
}

int d4_factor(void *ctx) {
    Ctx *c = (Ctx *)ctx;
    if (!c) return D4_ERR_ARG;
    D4_GUARD_BEGIN
    if (c->p.precision == D4_PREC_MIXED) return d4::factor32(*c);
    return d4::factor64(*c);
    D4_GUARD_END(c)
}

int d4_solve(void *ctx, const double *g, double *dx) {
    Ctx *c = (Ctx *)ctx;
    if (!c || !g || !dx) return D4_ERR_ARG;
    D4_GUARD_BEGIN
    upload(*c, c->xs_tmp, g);
    if (c->p.precision == D4_PREC_MIXED) {
        d4::solve_plain32(*c, c->xs_tmp);
        download(*c, dx, c->dx);
        read_async_errors(*c);
        int fl[d4::kFlagCount];
        D4_CUDA_OK(cudaMemcpy(fl, c->flags, sizeof(fl), cudaMemcpyDeviceToHost));
        if (fl[d4::kFlagBarrierTimeout]) throw d4::StateError("block solve wait timed out");
        return c->factor_singular ? D4_WARN_SINGULAR : D4_OK;
    }
    d4::solve_plain64(*c, c->xs_tmp);
    download(*c, dx, c->dx);
    sync(*c);
    return c->factor_singular ? D4_WARN_SINGULAR : D4_OK;
    D4_GUARD_END(c)
}

int d4_attempt(void *ctx, double t0, double h, d4_attempt_result *res) {
    Ctx *c = (Ctx *)ctx;
    if (!c || !res) return D4_ERR_ARG;
    D4_GUARD_BEGIN
    return attempt(*c, t0, h, res);
    D4_GUARD_END(c)
}

int d4_get_attempt(void *ctx, double *x_big, double *x_half, double *x_two) {
    Ctx *c = (Ctx *)ctx;
    if (!c) return D4_ERR_ARG;
    D4_GUARD_BEGIN
    if (x_big) download(*c, x_big, c->xb);
    if (x_half) download(*c, x_half, c->xh);
    if (x_two) download(*c, x_two, c->x2);
    sync(*c);
    return D4_OK;
    D4_GUARD_END(c)
}

int d4_field_eval(void *ctx, int count, const double *dx, const double *dy, double *xy,
                  double *xyd) {
    Ctx *c = (Ctx *)ctx;
    if (!c || count < 0 || !dx || !dy || !xy || !xyd) return D4_ERR_ARG;
    D4_GUARD_BEGIN
    double *d = nullptr;
    D4_CUDA_OK(d4::dmalloc((void **)&d, sizeof(double) * 4 * (size_t)(count > 0 ? count : 1)));
    const size_t b = sizeof(double) * (size_t)count;
    cudaMemcpyAsync(d, dx, b, cudaMemcpyHostToDevice, c->stream);
    cudaMemcpyAsync(d + count, dy, b, cudaMemcpyHostToDevice, c->stream);
    d4::field_eval64(*c, count, d, d + count, d + 2 * count, d + 3 * count);
    cudaMemcpyAsync(xy, d + 2 * count, b, cudaMemcpyDeviceToHost, c->stream);
    cudaMemcpyAsync(xyd, d + 3 * count, b, cudaMemcpyDeviceToHost, c->stream);
    cudaError_t e = cudaStreamSynchronize(c->stream);
    cudaFree(d);
    D4_CUDA_OK(e);
    return D4_OK;
    D4_GUARD_END(c)
}

// One pass of Simulation::run's loop body per attempt (src/simulation.cpp:88-277),
// until `target` accepted steps (target < 0: until interrupt()).
static int run_loop(Ctx *c, const d4_run_io *io, std::ofstream *log, long long target) {
    const d4_params &p = c->p;
    const int n = c->n;
    d4::RunState &rs = c->rs;
    const bool want_log = log && log->is_open();
    std::vector<double> hv(n), hv2(n), hv3(n);
    double *d_strain = c->red + 4;
    const long long ok_start = rs.ok;
    for (;;) {
        if (target >= 0) {
            if (rs.ok - ok_start >= target) break;
        } else {
            // interrupt(), src/simulation.cpp:722-750
            if (p.time_limit >= 0 && c->sim_time > p.time_limit) break;
            if (p.strain_increase_limit >= 0 && rs.strain > p.strain_increase_limit) break;
            if (p.step_count_limit >= 0 && rs.ok > p.step_count_limit) break;
            if (p.avalanche_limit >= 0 && rs.aval_count > p.avalanche_limit) break;
        }
        if (io && io->max_attempts > 0 && rs.attempts >= io->max_attempts) break;

        const double h = c->step_size;
        d4_attempt_result ar;
        attempt(*c, c->sim_time, h, &ar);
        if (!std::isfinite(ar.ratio)) {
            // a NaN ratio fails every attempt while getNewStepSize keeps
            // doubling h (min(2, NaN^(-1/6)) is 2): stop with an error instead,
            // as the reference's DEBUG_VERSION checks stop on non-finite state
            // (src/simulation.cpp:754-948)
            c->err_detail = "non-finite error ratio at t = " + std::to_string(c->sim_time) +
                            ", h = " + std::to_string(h) + ": positions or speeds are not finite";
            throw d4::StateError(c->err_detail.c_str());
        }
        ++rs.attempts;
        rs.pivoted += ar.pivoted;
        rs.singular += ar.singular;
        if (ar.ratio < 1) {
            if (c->recording) {
                c->rec_t0.push_back(c->sim_time);
                c->rec_h.push_back(h);
            }
            c->sim_time += h;
            ++rs.ok;
            if (p.calculate_strain) {
                d4::strain_increment64(*c, c->x0, c->xh, d_strain);
                d4::strain_increment64(*c, c->xh, c->x2, d_strain + 1);
                D4_CUDA_OK(cudaMemcpyAsync(c->h_red + 4, d_strain, sizeof(double) * 2,
                                           cudaMemcpyDeviceToHost, c->stream));
                sync(*c);
                rs.strain += c->h_red[4];
                rs.strain += c->h_red[5];
            }
            d4::normalize64(*c, c->x0, c->x2);
            const bool need_speed = want_log || p.avalanche_limit >= 0;
            double sum_avg = 0;
            if (need_speed) {
                download(*c, hv2.data(), c->v_init2);
                sync(*c);
                sum_avg = host_abs_sum(hv2) / n;
            }
            if (want_log) {
                download(*c, hv.data(), c->v_init);
                download(*c, hv3.data(), c->speed2);
                sync(*c);
                const double vsq_end = host_sq_sum(hv3);
                rs.energy += (host_sq_sum(hv) + 2 * host_sq_sum(hv2) + vsq_end) * h / 4;
                *log << c->sim_time << "\t" << rs.ok << "\t" << rs.failed << "\t" << ar.ratio
                     << "\t" << ar.max_id << "\t" << sum_avg << "\t" << c->cutoff << "\t";
                if (p.calculate_order_parameter) {
                    download(*c, hv3.data(), c->speed);
                    sync(*c);
                    double op = 0;
                    for (int i = 0; i < n; ++i) op += (i < n / 2 ? 1 : -1) * hv3[i];
                    *log << op << "\t";
                } else
                    *log << "-\t";
                // columns 10 and 14: wall time since the previous log line and
                // since the start of the run (src/simulation.cpp:197,206)
                *log << ext_stress(p.protocol, c->sim_time) << "\t" << wall_time() - rs.wall_last
                     << "\t";
                if (p.calculate_strain)
                    *log << rs.strain << "\t";
                else
                    *log << "-\t";
                *log << vsq_end << "\t" << rs.energy << "\t" << wall_time() - rs.wall_start
                     << "\t" << h << "\n";
                rs.wall_last = wall_time();
            }
            if (p.avalanche_limit >= 0) {
                if (rs.in_aval && sum_avg < p.avalanche_speed_threshold) {
                    ++rs.aval_count;
                    rs.in_aval = false;
                } else if (sum_avg > p.avalanche_speed_threshold)
                    rs.in_aval = true;
            }
            if (p.save_sub_configs) {
                if ((!rs.in_aval && p.sub_config_delay <= rs.sub_counter) ||
                    (rs.in_aval && p.sub_config_delay_during_avalanche <= rs.sub_counter) ||
                    rs.next_wo <= c->sim_time) {
                    rs.sub_counter = 0;
                    rs.next_wo = next_write_out(p, c->sim_time);
                    if (io && io->sub_config_prefix) {
                        std::stringstream ss;
                        ss << std::setprecision(9) << c->sim_time;
                        write_config(*c, std::string(io->sub_config_prefix) + ss.str() + ".dconf",
                                     io->order);
                    }
                } else
                    ++rs.sub_counter;
            }
        } else
            ++rs.failed;
        // PrecisionHandler::getNewStepSize (src/precision_handler.cpp:57-62) and
        // the write-out clipping of src/simulation.cpp:253-274
        double hn = 0.9 * h * std::min(2., std::pow(ar.ratio, -1. / 6));
        if (rs.h_before_writeout != 0) {
            if (ar.ratio < 1) hn = std::max(hn, rs.h_before_writeout);
            rs.h_before_writeout = 0;
        }
        const double rem = std::nextafter(rs.next_wo, INFINITY) - c->sim_time;
        if (rem < hn) {
            rs.h_before_writeout = hn;
            hn = rem;
        }
        if (c->use_dipole) d4::reset_tol64(*c);
        if (p.max_stepsize > 0 && p.max_stepsize < hn) hn = p.max_stepsize;
        c->step_size = hn;
    }
    return D4_OK;
}

static void fill_result(Ctx *c, const d4::RunState &before, float ms, d4_run_result *res) {
    if (!res) return;
    const d4::RunState &rs = c->rs;
    res->sim_time = c->sim_time;
    res->step_size = c->step_size;
    res->strain = rs.strain - before.strain;
    res->energy = rs.energy - before.energy;
    res->successful_steps = rs.ok - before.ok;
    res->failed_steps = rs.failed - before.failed;
    res->attempts = rs.attempts - before.attempts;
    res->pivoted_factorizations = rs.pivoted - before.pivoted;
    res->singular_factorizations = rs.singular - before.singular;
    res->device_seconds = ms / 1000.0;
}

static void start_state(Ctx *c) {
    c->rs = d4::RunState();
    c->rs.started = true;
    c->rs.next_wo = c->p.save_sub_configs ? next_write_out(c->p, c->sim_time) : INFINITY;
}

// Simulation::run, src/simulation.cpp:30-281.
int d4_run(void *ctx, const d4_run_io *io, d4_run_result *res) {
    Ctx *c = (Ctx *)ctx;
    if (!c) return D4_ERR_ARG;
    D4_GUARD_BEGIN
    const d4_params &p = c->p;
    const int n = c->n;
    std::ofstream log;
    if (io && io->log_path && *io->log_path) {
        log.open(io->log_path);
        if (!log) return fail(c, D4_ERR_IO, std::string("cannot open log ") + io->log_path);
        log << std::scientific << std::setprecision(16);
    }
    d4::autotune_pairs(*c);  // both forms run the FP64 pair kernels
    start_state(c);
    c->rs.wall_start = c->rs.wall_last = wall_time();
    const d4::RunState before = c->rs;
    D4_CUDA_OK(cudaEventRecord(c->ev0, c->stream));
    // src/simulation.cpp:46: initial speeds (also seeds the tolerances)
    sweep_speeds(*c, c->x0, c->y, ext_stress(p.protocol, c->sim_time), c->v_init);
    if (log.is_open()) {
        std::vector<double> hv(n);
        download(*c, hv.data(), c->v_init);
        sync(*c);
        log << "# simTime(1)\tsuccessfullSteps(2)\tfailedSteps(3)\tmaxErrorRatioSqr(4)\t"
               "maxErrorRatioID(5)\tsumAvgSp(6)\tcutOff(7)\torderParameter(8)\t"
               "externalStress(9)\ttimeStageI - III(10)\tstrain(11)\tvSquare(12)\t"
               "energy(13)\twallTimeElapsed(14)\tstepSize(15)\t\n";
        log << c->sim_time << "\t" << 0 << "\t" << 0 << "\t" << 0 << "\t" << 0 << "\t"
            << host_abs_sum(hv) / n << "\t" << c->cutoff << "\t-\t"
            << ext_stress(p.protocol, c->sim_time) << "\t-\t" << 0.0 << "\t" << host_sq_sum(hv)
            << "\t" << 0.0 << "\t" << 0 << "\t" << c->step_size << "\n";
    }
    run_loop(c, io, &log, -1);
    D4_CUDA_OK(cudaEventRecord(c->ev1, c->stream));
    sync(*c);
    float ms = 0;
    D4_CUDA_OK(cudaEventElapsedTime(&ms, c->ev0, c->ev1));
    if (io && io->end_config_path) write_config(*c, io->end_config_path, io->order);
    fill_result(c, before, ms, res);
    return D4_OK;
    D4_GUARD_END(c)
}

int d4_advance(void *ctx, long long accepted_steps, d4_run_result *res) {
    Ctx *c = (Ctx *)ctx;
    if (!c || accepted_steps < 0) return D4_ERR_ARG;
    D4_GUARD_BEGIN
    d4::autotune_pairs(*c);  // both forms run the FP64 pair kernels
    if (!c->rs.started) {
        start_state(c);
        // the first attempt's tolerances include the initial sweep of run()
        sweep_speeds(*c, c->x0, c->y, ext_stress(c->p.protocol, c->sim_time), c->v_init);
    }
    const d4::RunState before = c->rs;
    D4_CUDA_OK(cudaEventRecord(c->ev0, c->stream));
    run_loop(c, nullptr, nullptr, accepted_steps);
    D4_CUDA_OK(cudaEventRecord(c->ev1, c->stream));
    sync(*c);
    float ms = 0;
    D4_CUDA_OK(cudaEventElapsedTime(&ms, c->ev0, c->ev1));
    fill_result(c, before, ms, res);
    return D4_OK;
    D4_GUARD_END(c)
}

int d4_profile(void *ctx, int enable) {
    Ctx *c = (Ctx *)ctx;
    if (!c) return D4_ERR_ARG;
    c->prof.on = enable != 0;
    c->prof.used = 0;
    for (int k = 0; k < D4_CAT_COUNT; ++k) {
        c->prof.ms[k] = 0;
        c->prof.calls[k] = 0;
    }
    return D4_OK;
}

int d4_profile_read(void *ctx, double *ms, long long *calls) {
    Ctx *c = (Ctx *)ctx;
    if (!c || !ms || !calls) return D4_ERR_ARG;
    D4_GUARD_BEGIN
    sync(*c);
    d4::prof_collect(*c);
    for (int k = 0; k < D4_CAT_COUNT; ++k) {
        ms[k] = c->prof.ms[k];
        calls[k] = c->prof.calls[k];
    }
    return D4_OK;
    D4_GUARD_END(c)
}

int d4_solver_stats(void *ctx, long long *solves, long long *iterations, long long *fallbacks,
                    long long *nnz) {
    Ctx *c = (Ctx *)ctx;
    if (!c || !solves || !iterations || !fallbacks || !nnz) return D4_ERR_ARG;
    *solves = c->sp_solves;
    *iterations = c->sp_iters;
    *fallbacks = c->sp_fallbacks;
    *nnz = c->sp_nnz;
    return D4_OK;
}

int d4_set_overlap(void *ctx, int enable) {
    Ctx *c = (Ctx *)ctx;
    if (!c) return D4_ERR_ARG;
    c->overlap = (enable && c->stream_b) ? 1 : 0;  // the second stream exists unless GMRES
    return D4_OK;
}

int d4_lu_stats(void *ctx, long long *factorizations, long long *passes, long long *swaps) {
    Ctx *c = (Ctx *)ctx;
    if (!c || !factorizations || !passes || !swaps) return D4_ERR_ARG;
    *factorizations = c->lu_count;
    *passes = c->lu_passes;
    *swaps = c->lu_swaps;
    return D4_OK;
}

int d4_mixed_stats(void *ctx, long long *block_factorizations, long long *fallbacks,
                   long long *pivoted_attempts, long long *fp64_attempts, double *worst_refined) {
    Ctx *c = (Ctx *)ctx;
    if (!c || !block_factorizations || !fallbacks || !pivoted_attempts || !fp64_attempts ||
        !worst_refined)
        return D4_ERR_ARG;
    *block_factorizations = c->m_blocklu;
    *fallbacks = c->m_fallbacks;
    *pivoted_attempts = c->m_pivoted32;
    *fp64_attempts = c->m_fp64_attempts;
    *worst_refined = c->m_worst_refine;
    return D4_OK;
}

int d4_pair_tile_threads(void *ctx, int *threads_y) {
    Ctx *c = (Ctx *)ctx;
    if (!c || !threads_y) return D4_ERR_ARG;
    *threads_y = c->pair_tuned ? c->pair_ty : 0;
    return D4_OK;
}

int d4_set_block_lu(void *ctx, int enable) {
    Ctx *c = (Ctx *)ctx;
    if (!c) return D4_ERR_ARG;
    if (c->p.precision != D4_PREC_MIXED) return fail(c, D4_ERR_ARG, "d4_set_block_lu: mixed form only");
    c->m_fast = enable ? 1 : 0;
    return D4_OK;
}

int d4_record_steps(void *ctx, int enable) {
    Ctx *c = (Ctx *)ctx;
    if (!c) return D4_ERR_ARG;
    if (enable) {
        c->rec_t0.clear();
        c->rec_h.clear();
    }
    c->recording = enable != 0;
    return D4_OK;
}

long long d4_recorded_count(void *ctx) {
    Ctx *c = (Ctx *)ctx;
    return c ? (long long)c->rec_t0.size() : -1;
}

int d4_recorded_steps(void *ctx, long long count, double *t0s, double *hs) {
    Ctx *c = (Ctx *)ctx;
    if (!c || count < 0 || (count > 0 && (!t0s || !hs))) return D4_ERR_ARG;
    const long long m = std::min<long long>(count, (long long)c->rec_t0.size());
    for (long long k = 0; k < m; ++k) {
        t0s[k] = c->rec_t0[k];
        hs[k] = c->rec_h[k];
    }
    return D4_OK;
}

long long d4_kernel_launches(void) { return d4::g_launches.load(); }

long long d4_device_allocations(void) { return d4::g_allocs.load(); }

int d4_wait_selftest(void *ctx, int which) {
    Ctx *c = (Ctx *)ctx;
    if (!c || which < 0 || which > 1) return D4_ERR_ARG;
    D4_GUARD_BEGIN
    D4_CUDA_OK(cudaSetDevice(c->p.device));
    const int st = d4::wait_selftest(which);
    if (st == D4_ERR_STATE)
        return fail(c, st, which == 0 ? "grid barrier wait gave up (self-test)"
                                      : "tile flag wait gave up (self-test)");
    return st;
    D4_GUARD_END(c)
}

}  // extern "C"
