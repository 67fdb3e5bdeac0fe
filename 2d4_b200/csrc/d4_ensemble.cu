// d4_ensemble.cu: batched ensemble of independent systems (FP64 form,
// compiled with --fmad=false).
//
// The reference runs one system per process (src/simulation.cpp:30-281);
// statistics over many realisations mean many such runs.  Here all systems of
// an ensemble advance together: each attempt round runs stages I-IV
// (src/simulation.cpp:90-161) for every active instance with ONE launch per
// phase:
//   pair tiles     all instances' upper-triangle tiles in one grid (block ->
//                  instance by a prefix table), the same tile body as the
//                  single-system engine (d4_sweep64.cuh);
//   row sums       all instances' 32-row blocks in one grid (same pipeline);
//   LU, solves     one CTA per instance: an exact-order blocked LU (panel of
//                  32 columns, U12 by column, trailing update in 64x64 tiles
//                  from shared memory) and column-oriented substitutions,
//                  each entry receiving its updates in the oracle's order, so
//                  every instance reproduces the single-system result bit
//                  for bit;
//   elementwise    one CTA per instance, or a prefix table for n^2 work.
// Instances are ordered by decreasing n, so the largest (whose one-CTA LU is
// the longest) start first.  After each round the host applies each
// instance's step control exactly as d4_run does (acceptance, new step size,
// limits), and the next round's per-instance scalars are uploaded in one copy.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <numeric>
#include <string>
#include <vector>

#include "d4_sweep64.cuh"

namespace d4 {
namespace ens {

enum Vec {
    kX0, kY, kXB, kXH, kX2, kVI, kVI2, kSP, kSP2, kDV, kDVN, kFAC, kTOL, kRSUB, kRSC,
    kNumVec
};

struct Inst {
    int n;
    int pad;
    long long voff;  // offset of the instance's vectors in every vector pool
    long long moff;  // offset of its n x n matrices in every matrix pool
    double cutoff, cut_sq, one_per_cut_sq;
};

// Per-instance scalars of one attempt round.
struct Sc {
    double h;
    double ext[3];  // tau_ext at t0, t0 + h, t0 + h/2
    double factor;  // (t_half - t0) / (t1 - t0) of calcJacobianAndSpeedsFromPrev
    double dif;     // tau_ext(t_half) - tau_ext(t1)
};

struct Pools {
    double *v[kNumVec];
    double *F, *A, *LU;
    int *piv;
    int *sing;        // per instance: the current factorisation met a zero pivot
    int *sing_any;    // per instance: some factorisation of the round did
    double *ratio;    // per instance: {max err^2/tol, index}
    double *strain;   // per instance: accumulated strain
    int *acc;         // per instance: accepted this round
    int *err;         // row-pipeline wait failure
};

struct Common {
    double min_prec_sq;
    int use_dipole;
    double range_sq;
    int heaviside;
    char wfn;
    int calc_strain;
};

// Slot of block b in a prefix table pre[0..na] (pre[s] <= b < pre[s + 1]).
__device__ __forceinline__ int find_slot(const int *pre, int na, int b) {
    int lo = 0, hi = na - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (pre[mid] <= b)
            lo = mid;
        else
            hi = mid - 1;
    }
    return lo;
}

template <bool kJac>
__global__ void __launch_bounds__(256) k_ens_pairs(Pools P, const Inst *ins, const Sc *sc,
                                                   const int *act, const int *pre, int na,
                                                   Common cm, int xsel, double hmul) {
    const int s = find_slot(pre, na, blockIdx.x);
    const int k = act[s];
    const Inst in = ins[k];
    PairArgs a;
    a.n = in.n;
    a.x = P.v[xsel] + in.voff;
    a.y = P.v[kY] + in.voff;
    a.F = P.F + in.moff;
    a.A = P.A + in.moff;
    a.tol = cm.use_dipole ? P.v[kTOL] + in.voff : nullptr;
    a.min_prec_sq = cm.min_prec_sq;
    a.h = kJac ? sc[k].h * hmul : 0;
    a.cut_sq = in.cut_sq;
    a.cutoff = in.cutoff;
    a.range_sq = cm.range_sq;
    a.one_per_cut_sq = in.one_per_cut_sq;
    a.heaviside = cm.heaviside;
    a.tb.t = nullptr;
    a.tb.T = a.tb.W = 0;
    pair_tile<kJac, false>(a, blockIdx.x - pre[s]);
}

template <bool kJac>
__global__ void __launch_bounds__(64) k_ens_rows(Pools P, const Inst *ins, const Sc *sc,
                                                 const int *act, const int *pre, int na,
                                                 Common cm, int ea, int eb, int va, int vb) {
    const int s = find_slot(pre, na, blockIdx.x);
    const int k = act[s];
    const Inst in = ins[k];
    RowArgs r;
    r.n = in.n;
    r.F = P.F + in.moff;
    r.A = P.A + in.moff;
    r.ext_a = sc[k].ext[ea];
    r.ext_b = kJac ? sc[k].ext[eb] : 0;
    r.v_a = P.v[va] + in.voff;
    r.v_b = kJac ? P.v[vb] + in.voff : nullptr;
    r.dvec = P.v[kDV] + in.voff;
    r.rowsub = P.v[kRSUB] + in.voff;
    r.rowsc = P.v[kRSC] + in.voff;
    r.wfn = cm.wfn;
    r.err = P.err;
    row_block<kJac>(r, blockIdx.x - pre[s]);
}

constexpr int kElemChunk = 2048;  // n^2 elements per block of the matrix kernels

// Row scaling (src/simulation.cpp:516-522) or the half-step rescale
// (src/simulation.cpp:584-594) of all instances' matrices.
template <bool kHalf>
__global__ void __launch_bounds__(256) k_ens_matrix(Pools P, const Inst *ins, const int *act,
                                                    const int *pre, int na) {
    const int s = find_slot(pre, na, blockIdx.x);
    const Inst in = ins[act[s]];
    const int n = in.n;
    double *A = P.A + in.moff;
    const double *rsub = P.v[kRSUB] + in.voff, *rsc = P.v[kRSC] + in.voff;
    const double *fac = P.v[kFAC] + in.voff;
    const size_t base = (size_t)(blockIdx.x - pre[s]) * kElemChunk;
    const size_t total = (size_t)n * n;
    for (size_t idx = base + threadIdx.x; idx < min(total, base + kElemChunk); idx += 256) {
        const int r = (int)(idx % n), c = (int)(idx / n);
        if (kHalf) {
            const double f = fac[r];
            const double e = A[idx];
            A[idx] = (r == c) ? 1 + (e - 1) / 2 * f : e / 2 * f;
        } else {
            const double scv = rsc[r];
            A[idx] = (r == c) ? rsub[r] * scv + 1 : A[idx] * scv;
        }
    }
}

__device__ __forceinline__ double bs(int i, int n) { return i < n / 2 ? 1.0 : -1.0; }

// calcJacobianAndSpeedsFromPrev weights and speed shift (src/simulation.cpp:552-608).
__global__ void k_ens_half_weights(Pools P, const Inst *ins, const Sc *sc, const int *act,
                                   Common cm) {
    const int k = act[blockIdx.x];
    const Inst in = ins[k];
    double *dv = P.v[kDV] + in.voff, *fac = P.v[kFAC] + in.voff;
    for (int i = threadIdx.x; i < in.n; i += blockDim.x) {
        const double old = dv[i];
        double w = 0.;
        if (old != 0) w = f64::weight(f64::weight_inv(old, cm.wfn) * sc[k].factor, cm.wfn);
        P.v[kDVN][in.voff + i] = w;
        fac[i] = (1 + w) / (1 + old);
    }
}

__global__ void k_ens_half_finish(Pools P, const Inst *ins, const Sc *sc, const int *act) {
    const int k = act[blockIdx.x];
    const Inst in = ins[k];
    for (int i = threadIdx.x; i < in.n; i += blockDim.x) {
        P.v[kDV][in.voff + i] = P.v[kDVN][in.voff + i];
        P.v[kSP][in.voff + i] += sc[k].dif * bs(i, in.n);
    }
}

// ---- one-CTA exact-order LU -------------------------------------------------
constexpr int kLuT = 256;
constexpr int kPan = 32;
constexpr int kTt = 64;  // trailing tile edge

__device__ __forceinline__ void argmax_combine(double &v, int &i, double ov, int oi) {
    if (oi >= 0 && (ov > v || (ov == v && (i < 0 || oi < i)))) {
        v = ov;
        i = oi;
    }
}

// Factorises the instance's A into LU with the operation sequence of the
// oracle's partial-pivot LU (first maximum wins, whole-row swaps, column
// divided by the pivot, each entry updated k ascending with the product and
// the difference rounded separately, and updates with u_kj == 0 skipped).
__global__ void __launch_bounds__(kLuT) k_ens_lu(Pools P, const Inst *ins, const int *act) {
    __shared__ double sL[kTt][kPan + 1];
    __shared__ double sU[kPan][kTt + 1];
    __shared__ double rv[kLuT / 32];
    __shared__ int ri[kLuT / 32];
    __shared__ int s_piv;
    __shared__ double prow[kPan];
    const int k = act[blockIdx.x];
    const Inst in = ins[k];
    const int n = in.n, tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
    double *a = P.LU + in.moff;
    const double *a0 = P.A + in.moff;
    int *piv = P.piv + in.voff;
    const size_t nn = (size_t)n * n;
    for (size_t idx = tid; idx < nn; idx += kLuT) a[idx] = a0[idx];
    __syncthreads();
    int singular = 0;
    for (int k0 = 0; k0 < n; k0 += kPan) {
        const int kw = min(kPan, n - k0);
        // panel: columns k0 .. k0 + kw - 1, unblocked
        for (int kk = k0; kk < k0 + kw; ++kk) {
            const double akk = fabs(a[kk + (size_t)kk * n]);
            double bv = -1;
            int bi = -1;
#pragma unroll 4
            for (int i = kk + 1 + tid; i < n; i += kLuT) {
                const double v = fabs(a[i + (size_t)kk * n]);
                if (v > bv) {
                    bv = v;
                    bi = i;
                }
            }
            for (int o = 16; o > 0; o >>= 1) {
                const double ov = __shfl_down_sync(0xffffffffu, bv, o);
                const int oi = __shfl_down_sync(0xffffffffu, bi, o);
                argmax_combine(bv, bi, ov, oi);
            }
            if (lane == 0) {
                rv[wid] = bv;
                ri[wid] = bi;
            }
            __syncthreads();
            if (tid == 0) {
                double v = rv[0];
                int i = ri[0];
                for (int w = 1; w < kLuT / 32; ++w) argmax_combine(v, i, rv[w], ri[w]);
                // the sequential scan starts from |a_kk| and replaces only on a
                // strictly greater value (a NaN |a_kk| is never replaced)
                s_piv = (i >= 0 && v > akk) ? i : kk;
                piv[kk] = s_piv;
            }
            __syncthreads();
            const int p = s_piv;
            if (a[p + (size_t)kk * n] == 0.0) {
                singular = 1;
                __syncthreads();
                continue;
            }
            if (p != kk)
                for (int j = tid; j < n; j += kLuT) {
                    const double t = a[kk + (size_t)j * n];
                    a[kk + (size_t)j * n] = a[p + (size_t)j * n];
                    a[p + (size_t)j * n] = t;
                }
            __syncthreads();
            const double d = a[kk + (size_t)kk * n];
#pragma unroll 4
            for (int i = kk + 1 + tid; i < n; i += kLuT) a[i + (size_t)kk * n] /= d;
            __syncthreads();
            // rank-1 update of the panel's remaining columns: a thread per row,
            // the row's loads issued together (one memory round trip per row)
            const int ncol = k0 + kw - kk - 1;
            if (tid < kPan) prow[tid] = tid < ncol ? a[kk + (size_t)(kk + 1 + tid) * n] : 0.0;
            __syncthreads();
            for (int i = kk + 1 + tid; i < n; i += kLuT) {
                const double l = a[i + (size_t)kk * n];
                double v[kPan - 1];
#pragma unroll
                for (int q = 0; q < kPan - 1; ++q)
                    v[q] = q < ncol ? a[i + (size_t)(kk + 1 + q) * n] : 0.0;
#pragma unroll
                for (int q = 0; q < kPan - 1; ++q) {
                    const double t = prow[q];
                    if (q < ncol && t != 0.0) a[i + (size_t)(kk + 1 + q) * n] = v[q] - l * t;
                }
            }
            __syncthreads();
        }
        const int j1 = k0 + kw;
        if (j1 >= n) break;
        // U12: rows k0 .. k0 + kw - 1 of columns j >= j1 (unit lower L11 from sL)
        for (int t = tid; t < kPan * kPan; t += kLuT) {
            const int r = t % kPan, c = t / kPan;
            sL[r][c] = (r < kw && c < kw) ? a[(k0 + r) + (size_t)(k0 + c) * n] : 0.0;
        }
        __syncthreads();
        for (int j = j1 + tid; j < n; j += kLuT) {
            double u[kPan];
            double *col = a + k0 + (size_t)j * n;
#pragma unroll
            for (int r = 0; r < kPan; ++r) u[r] = r < kw ? col[r] : 0.0;
#pragma unroll
            for (int c = 0; c < kPan; ++c) {
                const double t = u[c];
                if (c < kw && t != 0.0) {
#pragma unroll
                    for (int r = c + 1; r < kPan; ++r)
                        if (r < kw) u[r] -= sL[r][c] * t;
                }
            }
#pragma unroll
            for (int r = 0; r < kPan; ++r)
                if (r < kw) col[r] = u[r];
        }
        __syncthreads();
        // trailing update in kTt x kTt tiles: thread (tr, tc) owns rows
        // i0 + tr + 16 q and columns j0 + tc + 16 w (q, w = 0..3)
        const int tr = tid & 15, tc = tid >> 4;
        for (int i0 = j1; i0 < n; i0 += kTt) {
            for (int jt = j1; jt < n; jt += kTt) {
                for (int t = tid; t < kTt * kPan; t += kLuT) {
                    const int r = t % kTt, c = t / kTt;
                    sL[r][c] = (i0 + r < n && c < kw) ? a[(i0 + r) + (size_t)(k0 + c) * n] : 0.0;
                }
                for (int t = tid; t < kTt * kPan; t += kLuT) {
                    const int r = t % kPan, c = t / kPan;
                    sU[r][c] = (jt + c < n && r < kw) ? a[(k0 + r) + (size_t)(jt + c) * n] : 0.0;
                }
                __syncthreads();
                double acc[4][4];
#pragma unroll
                for (int q = 0; q < 4; ++q)
#pragma unroll
                    for (int w = 0; w < 4; ++w) {
                        const int i = i0 + tr + 16 * q, j = jt + tc + 16 * w;
                        acc[q][w] = (i < n && j < n) ? a[i + (size_t)j * n] : 0.0;
                    }
                for (int c = 0; c < kw; ++c) {
                    double lv[4], uv[4];
#pragma unroll
                    for (int q = 0; q < 4; ++q) lv[q] = sL[tr + 16 * q][c];
#pragma unroll
                    for (int w = 0; w < 4; ++w) uv[w] = sU[c][tc + 16 * w];
                    // the oracle skips an update whose u_kj is 0; when no u of
                    // this warp's columns is 0 (the dense case) the plain
                    // product-difference is the same and needs no select
                    const bool nz = uv[0] != 0.0 && uv[1] != 0.0 && uv[2] != 0.0 && uv[3] != 0.0;
                    if (__all_sync(0xffffffffu, nz)) {
#pragma unroll
                        for (int q = 0; q < 4; ++q)
#pragma unroll
                            for (int w = 0; w < 4; ++w) acc[q][w] = acc[q][w] - lv[q] * uv[w];
                    } else {
#pragma unroll
                        for (int q = 0; q < 4; ++q)
#pragma unroll
                            for (int w = 0; w < 4; ++w) {
                                const double nv = acc[q][w] - lv[q] * uv[w];
                                acc[q][w] = uv[w] != 0.0 ? nv : acc[q][w];
                            }
                    }
                }
#pragma unroll
                for (int q = 0; q < 4; ++q)
#pragma unroll
                    for (int w = 0; w < 4; ++w) {
                        const int i = i0 + tr + 16 * q, j = jt + tc + 16 * w;
                        if (i < n && j < n) a[i + (size_t)j * n] = acc[q][w];
                    }
                __syncthreads();
            }
        }
    }
    if (tid == 0) {
        P.sing[k] = singular;
        P.sing_any[k] |= singular;
    }
}

// ---- one-CTA solve with the LU factors (the oracle's substitution order) ----
constexpr int kSolT = 512;

__global__ void __launch_bounds__(kSolT) k_ens_solve(Pools P, const Inst *ins, const Sc *sc,
                                                     const int *act, int gmode, double hmul,
                                                     int se, int si, int xn, int xo, int base,
                                                     int out) {
    extern __shared__ double xs[];
    const int k = act[blockIdx.x];
    const Inst in = ins[k];
    const int n = in.n, tid = threadIdx.x;
    const double *a = P.LU + in.moff;
    const int *piv = P.piv + in.voff;
    const double hv = sc[k].h * hmul;
    const double *dv = P.v[kDV] + in.voff;
    const double *s_end = P.v[se] + in.voff, *s_init = P.v[si] + in.voff;
    for (int r = tid; r < n; r += kSolT) {
        // residual of the stage, src/simulation.cpp:101,123,142,621
        const double d = dv[r];
        const double X = (1 + d) * s_end[r] + (1 - d) * s_init[r];
        double g;
        if (gmode == kGBig)
            g = -hv * X / 2;
        else if (gmode == kGHalf)
            g = -hv / 2 * X / 2;
        else
            g = P.v[xn][in.voff + r] - P.v[xo][in.voff + r] - hv * X / 2;
        xs[r] = g;
    }
    __syncthreads();
    if (tid == 0)
        for (int q = 0; q < n; ++q) {
            const int p = piv[q];
            if (p != q) {
                const double t = xs[q];
                xs[q] = xs[p];
                xs[p] = t;
            }
        }
    __syncthreads();
    for (int q = 0; q < n; ++q) {
        const double t = xs[q];
        if (t != 0.0) {
            const double *cq = a + (size_t)q * n;
            for (int i = q + 1 + tid; i < n; i += kSolT) xs[i] -= cq[i] * t;
        }
        __syncthreads();
    }
    for (int q = n - 1; q >= 0; --q) {
        if (tid == 0) xs[q] /= a[q + (size_t)q * n];
        __syncthreads();
        const double t = xs[q];
        if (t != 0.0) {
            const double *cq = a + (size_t)q * n;
            for (int i = tid; i < q; i += kSolT) xs[i] -= cq[i] * t;
        }
        __syncthreads();
    }
    const int singular = P.sing[k];
    for (int r = tid; r < n; r += kSolT) {
        double d = xs[r];
        if (singular && !((-1 < d) && (d < 1))) d = 0;  // src/simulation.cpp:652-657
        P.v[out][in.voff + r] = P.v[base][in.voff + r] - d;
    }
}

__global__ void __launch_bounds__(1024) k_ens_error(Pools P, const Inst *ins, const int *act,
                                                    Common cm) {
    const int k = act[blockIdx.x];
    const Inst in = ins[k];
    error_ratio_block(in.n, P.v[kXB] + in.voff, P.v[kX2] + in.voff, P.v[kTOL] + in.voff,
                      cm.min_prec_sq, cm.use_dipole, P.ratio + 2 * k);
}

// After the round: strain increments and normalisation of accepted instances,
// tolerance reset of all (src/simulation.cpp:164-252).
__global__ void k_ens_accept(Pools P, const Inst *ins, const int *act, Common cm) {
    const int k = act[blockIdx.x];
    const Inst in = ins[k];
    const int n = in.n;
    if (P.acc[k]) {
        if (cm.calc_strain && threadIdx.x == 0) {
            const double *x0 = P.v[kX0] + in.voff, *xh = P.v[kXH] + in.voff,
                         *x2 = P.v[kX2] + in.voff;
            double r1 = 0, r2 = 0;
            for (int i = 0; i < n; ++i) r1 += bs(i, n) * (xh[i] - x0[i]);
            for (int i = 0; i < n; ++i) r2 += bs(i, n) * (x2[i] - xh[i]);
            P.strain[k] += r1;
            P.strain[k] += r2;
        }
        __syncthreads();
        for (int i = threadIdx.x; i < n; i += blockDim.x)
            P.v[kX0][in.voff + i] = f64::normalize(P.v[kX2][in.voff + i]);
    }
    if (cm.use_dipole)
        for (int i = threadIdx.x; i < n; i += blockDim.x) P.v[kTOL][in.voff + i] = cm.min_prec_sq;
}

__global__ void k_ens_fill_tol(Pools P, const Inst *ins, const int *act, double v) {
    const Inst in = ins[act[blockIdx.x]];
    for (int i = threadIdx.x; i < in.n; i += blockDim.x) P.v[kTOL][in.voff + i] = v;
}

inline int cdiv(long long a, long long b) { return (int)((a + b - 1) / b); }

struct HostInst {
    int n;
    double sim_time, step_size;
    long long ok = 0, failed = 0, attempts = 0, singular = 0;
    double strain = 0;
    int selected_id = 0;
    bool started = false;
    long long aval_count = 0;  // avalanche detection (src/simulation.cpp:184-199)
    bool in_aval = false;
};

struct Ensemble {
    int count = 0;
    d4_params p{};
    Common cm{};
    double dipole_prec_sq = 1;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    std::string err;
    std::vector<HostInst> hi;
    std::vector<Inst> hins;
    Pools P{};
    Inst *d_ins = nullptr;
    Sc *d_sc = nullptr;
    int *d_act = nullptr, *d_pre_pair = nullptr, *d_pre_row = nullptr, *d_pre_mat = nullptr;
    std::vector<Sc> hsc;
    std::vector<int> act, pre_pair, pre_row, pre_mat;
    int solve_smem = 0;
    long long launches = 0;
    long long vtot = 0;  // entries of each per-dislocation vector pool
    int pair_ty = 8;     // threads per pair tile along j (autotuned, first run)
    bool tuned = false;
};

void check(const char *name) {
    g_launches.fetch_add(1, std::memory_order_relaxed);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) throw CudaError(e, name, __FILE__, __LINE__);
}

// Upload the active list (sorted by n descending) and its prefix tables.
void set_active(Ensemble &E, const std::vector<int> &active) {
    E.act = active;
    std::stable_sort(E.act.begin(), E.act.end(),
                     [&](int a, int b) { return E.hi[a].n > E.hi[b].n; });
    const int na = (int)E.act.size();
    E.pre_pair.assign(na + 1, 0);
    E.pre_row.assign(na + 1, 0);
    E.pre_mat.assign(na + 1, 0);
    for (int s = 0; s < na; ++s) {
        const int n = E.hi[E.act[s]].n;
        const int T = (n + kTile - 1) / kTile;
        E.pre_pair[s + 1] = E.pre_pair[s] + T * (T + 1) / 2;
        E.pre_row[s + 1] = E.pre_row[s] + cdiv(n, kRowRows);
        E.pre_mat[s + 1] = E.pre_mat[s] + cdiv((long long)n * n, kElemChunk);
    }
    if (na == 0) return;
    D4_CUDA_OK(cudaMemcpyAsync(E.d_act, E.act.data(), sizeof(int) * na, cudaMemcpyHostToDevice,
                               E.stream));
    D4_CUDA_OK(cudaMemcpyAsync(E.d_pre_pair, E.pre_pair.data(), sizeof(int) * (na + 1),
                               cudaMemcpyHostToDevice, E.stream));
    D4_CUDA_OK(cudaMemcpyAsync(E.d_pre_row, E.pre_row.data(), sizeof(int) * (na + 1),
                               cudaMemcpyHostToDevice, E.stream));
    D4_CUDA_OK(cudaMemcpyAsync(E.d_pre_mat, E.pre_mat.data(), sizeof(int) * (na + 1),
                               cudaMemcpyHostToDevice, E.stream));
    D4_CUDA_OK(cudaStreamSynchronize(E.stream));  // host vectors may change next round
}

template <bool kJac>
void sweep(Ensemble &E, int xsel, double hmul, int ea, int eb, int va, int vb) {
    const int na = (int)E.act.size();
    k_ens_pairs<kJac><<<E.pre_pair[na], dim3(kTile, E.pair_ty), 0, E.stream>>>(
        E.P, E.d_ins, E.d_sc, E.d_act, E.d_pre_pair, na, E.cm, xsel, hmul);
    check("k_ens_pairs");
    constexpr int bytes = row_smem_bytes<kJac>();
    k_ens_rows<kJac><<<E.pre_row[na], 64, bytes, E.stream>>>(
        E.P, E.d_ins, E.d_sc, E.d_act, E.d_pre_row, na, E.cm, ea, eb, va, vb);
    check("k_ens_rows");
    if (kJac) {
        k_ens_matrix<false><<<E.pre_mat[na], 256, 0, E.stream>>>(E.P, E.d_ins, E.d_act,
                                                                 E.d_pre_mat, na);
        check("k_ens_matrix<scale>");
    }
}

// Pair-tile autotuner of the ensemble: threads per tile from the candidates,
// by timing the stress and fused pair kernels of every active instance
// (tolerances off; F and A are scratch that every attempt rewrites), one
// untimed and three timed runs each; the fastest total wins.  Each pair is
// evaluated by one thread whatever the choice, so results do not depend on it.
void autotune(Ensemble &E) {
    if (E.tuned || E.act.empty()) return;
    Common cm = E.cm;
    cm.use_dipole = 0;
    const int na = (int)E.act.size();
    float best = 1e30f;
    int best_ty = 8;
    cudaEvent_t e0, e1;  // own events: E.ev0 times the whole d4_ensemble_run call
    D4_CUDA_OK(cudaEventCreate(&e0));
    D4_CUDA_OK(cudaEventCreate(&e1));
    for (int ty : kPairTyCandidates) {
        float total = 0;
        for (int rep = 0; rep < 4; ++rep) {
            D4_CUDA_OK(cudaEventRecord(e0, E.stream));
            k_ens_pairs<false><<<E.pre_pair[na], dim3(kTile, ty), 0, E.stream>>>(
                E.P, E.d_ins, E.d_sc, E.d_act, E.d_pre_pair, na, cm, kX0, 1.0);
            k_ens_pairs<true><<<E.pre_pair[na], dim3(kTile, ty), 0, E.stream>>>(
                E.P, E.d_ins, E.d_sc, E.d_act, E.d_pre_pair, na, cm, kX0, 1.0);
            check("k_ens_pairs<tune>");
            D4_CUDA_OK(cudaEventRecord(e1, E.stream));
            D4_CUDA_OK(cudaEventSynchronize(e1));
            float ms = 0;
            D4_CUDA_OK(cudaEventElapsedTime(&ms, e0, e1));
            if (rep > 0) total += ms;
        }
        if (total < best) {
            best = total;
            best_ty = ty;
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    E.pair_ty = best_ty;
    E.tuned = true;
}

void lu(Ensemble &E) {
    k_ens_lu<<<(int)E.act.size(), kLuT, 0, E.stream>>>(E.P, E.d_ins, E.d_act);
    check("k_ens_lu");
}

void solve(Ensemble &E, int gmode, double hmul, int se, int si, int xn, int xo, int base,
           int out) {
    k_ens_solve<<<(int)E.act.size(), kSolT, E.solve_smem, E.stream>>>(
        E.P, E.d_ins, E.d_sc, E.d_act, gmode, hmul, se, si, xn < 0 ? 0 : xn, xo < 0 ? 0 : xo,
        base, out);
    check("k_ens_solve");
}

// Stages I-IV for every active instance (the sequence of attempt() in d4_api.cu).
void attempt_round(Ensemble &E) {
    const int na = (int)E.act.size();
    D4_CUDA_OK(cudaMemsetAsync(E.P.sing_any, 0, sizeof(int) * E.count, E.stream));
    sweep<true>(E, kX0, 1.0, 0, 1, kVI, kSP);
    lu(E);
    solve(E, kGBig, 1.0, kSP, kVI, -1, -1, kX0, kXB);
    sweep<false>(E, kXB, 0, 1, 0, kSP2, 0);
    solve(E, kGNewton, 1.0, kSP2, kVI, kXB, kX0, kXB, kXB);
    k_ens_half_weights<<<na, 256, 0, E.stream>>>(E.P, E.d_ins, E.d_sc, E.d_act, E.cm);
    check("k_ens_half_weights");
    k_ens_matrix<true><<<E.pre_mat[na], 256, 0, E.stream>>>(E.P, E.d_ins, E.d_act, E.d_pre_mat,
                                                            na);
    check("k_ens_matrix<half>");
    k_ens_half_finish<<<na, 256, 0, E.stream>>>(E.P, E.d_ins, E.d_sc, E.d_act);
    check("k_ens_half_finish");
    lu(E);
    solve(E, kGHalf, 1.0, kSP, kVI, -1, -1, kX0, kXH);
    sweep<false>(E, kXH, 0, 2, 0, kSP2, 0);
    solve(E, kGNewton, 0.5, kSP2, kVI, kXH, kX0, kXH, kXH);
    sweep<true>(E, kXH, 0.5, 2, 1, kVI2, kSP2);
    lu(E);
    solve(E, kGHalf, 1.0, kSP2, kVI2, -1, -1, kXH, kX2);
    sweep<false>(E, kX2, 0, 1, 0, kSP2, 0);
    solve(E, kGNewton, 0.5, kSP2, kVI2, kX2, kXH, kX2, kX2);
    k_ens_error<<<na, 1024, 0, E.stream>>>(E.P, E.d_ins, E.d_act, E.cm);
    check("k_ens_error");
}

bool interrupted(const Ensemble &E, const HostInst &h) {
    const d4_params &p = E.p;
    if (p.time_limit >= 0 && h.sim_time > p.time_limit) return true;
    if (p.strain_increase_limit >= 0 && h.strain > p.strain_increase_limit) return true;
    if (p.step_count_limit >= 0 && h.ok > p.step_count_limit) return true;
    if (p.avalanche_limit >= 0 && h.aval_count > p.avalanche_limit) return true;
    return false;
}

}  // namespace ens
}  // namespace d4

using d4::ens::Ensemble;

extern "C" {

int d4_ensemble_create(void **out, int count, const int *n, const d4_params *p) {
    using namespace d4::ens;
    if (!out || !n || !p || count <= 0) return D4_ERR_ARG;
    if (p->precision != D4_PREC_FP64 || p->field != D4_FIELD_ANALYTIC ||
        p->solver == D4_SOLVER_GMRES)
        return D4_ERR_ARG;
    if (p->weight_function != 'c' && p->weight_function != 'p' && p->weight_function != 'm')
        return D4_ERR_ARG;
    for (int k = 0; k < count; ++k)
        if (n[k] < 2 || n[k] % 2 != 0 || n[k] > d4::kMaxSolveN) return D4_ERR_ARG;
    Ensemble *E = new (std::nothrow) Ensemble();
    if (!E) return D4_ERR_NOMEM;
    try {
        E->count = count;
        E->p = *p;
        D4_CUDA_OK(cudaSetDevice(p->device));
        D4_CUDA_OK(cudaStreamCreateWithFlags(&E->stream, cudaStreamNonBlocking));
        D4_CUDA_OK(cudaEventCreate(&E->ev0));
        D4_CUDA_OK(cudaEventCreate(&E->ev1));
        // as d4_create: PrecisionHandler and SimulationData::updateCutOff
        double mps = p->position_precision * p->position_precision;
        if (p->dipole_precision == 0) {
            E->cm.use_dipole = 0;
        } else {
            E->cm.use_dipole = 1;
            E->dipole_prec_sq = p->dipole_precision * p->dipole_precision;
            mps /= p->dipole_precision * p->dipole_precision;
        }
        E->cm.min_prec_sq = mps;
        E->cm.range_sq = p->heaviside_cutoff ? 1 : 49;
        E->cm.heaviside = p->heaviside_cutoff;
        E->cm.wfn = p->weight_function;
        E->cm.calc_strain = p->calculate_strain;
        long long voff = 0, moff = 0, smax = 0;
        E->hi.resize(count);
        E->hins.resize(count);
        for (int k = 0; k < count; ++k) {
            HostInst &h = E->hi[k];
            h.n = n[k];
            h.sim_time = 0;
            h.step_size = p->initial_stepsize;
            Inst &in = E->hins[k];
            in.n = n[k];
            in.pad = 0;
            in.voff = voff;
            in.moff = moff;
            double mult = p->cutoff_multiplier;
            if (!p->heaviside_cutoff && p->cutoff_multiplier >= std::sqrt(2 * (double)n[k]) / 12)
                mult = 1e20;
            in.cutoff = mult / std::sqrt((double)n[k]);
            in.cut_sq = in.cutoff * in.cutoff;
            in.one_per_cut_sq = 1 / in.cut_sq;
            voff += n[k] + (n[k] & 1) + 2;  // keep every vector 16-byte aligned
            voff += voff & 1;
            moff += (long long)n[k] * n[k];
            smax = std::max<long long>(smax, n[k]);
        }
        E->vtot = voff;
        for (int v = 0; v < kNumVec; ++v) {
            D4_CUDA_OK(d4::dmalloc((void **)&E->P.v[v], sizeof(double) * voff));
            D4_CUDA_OK(cudaMemsetAsync(E->P.v[v], 0, sizeof(double) * voff, E->stream));
        }
        D4_CUDA_OK(d4::dmalloc((void **)&E->P.F, sizeof(double) * moff));
        D4_CUDA_OK(d4::dmalloc((void **)&E->P.A, sizeof(double) * moff));
        D4_CUDA_OK(d4::dmalloc((void **)&E->P.LU, sizeof(double) * moff));
        D4_CUDA_OK(cudaMemsetAsync(E->P.A, 0, sizeof(double) * moff, E->stream));
        D4_CUDA_OK(d4::dmalloc((void **)&E->P.piv, sizeof(int) * voff));
        D4_CUDA_OK(d4::dmalloc((void **)&E->P.sing, sizeof(int) * count));
        D4_CUDA_OK(d4::dmalloc((void **)&E->P.sing_any, sizeof(int) * count));
        D4_CUDA_OK(d4::dmalloc((void **)&E->P.ratio, sizeof(double) * 2 * count));
        D4_CUDA_OK(d4::dmalloc((void **)&E->P.strain, sizeof(double) * count));
        D4_CUDA_OK(cudaMemsetAsync(E->P.strain, 0, sizeof(double) * count, E->stream));
        D4_CUDA_OK(d4::dmalloc((void **)&E->P.acc, sizeof(int) * count));
        D4_CUDA_OK(d4::dmalloc((void **)&E->P.err, sizeof(int) * 4));
        D4_CUDA_OK(cudaMemsetAsync(E->P.err, 0, sizeof(int) * 4, E->stream));
        D4_CUDA_OK(d4::dmalloc((void **)&E->d_ins, sizeof(Inst) * count));
        D4_CUDA_OK(cudaMemcpyAsync(E->d_ins, E->hins.data(), sizeof(Inst) * count,
                                   cudaMemcpyHostToDevice, E->stream));
        D4_CUDA_OK(d4::dmalloc((void **)&E->d_sc, sizeof(Sc) * count));
        D4_CUDA_OK(d4::dmalloc((void **)&E->d_act, sizeof(int) * count));
        D4_CUDA_OK(d4::dmalloc((void **)&E->d_pre_pair, sizeof(int) * (count + 1)));
        D4_CUDA_OK(d4::dmalloc((void **)&E->d_pre_row, sizeof(int) * (count + 1)));
        D4_CUDA_OK(d4::dmalloc((void **)&E->d_pre_mat, sizeof(int) * (count + 1)));
        E->hsc.resize(count);
        E->solve_smem = (int)(sizeof(double) * smax);
        D4_CUDA_OK(cudaFuncSetAttribute(k_ens_solve, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        E->solve_smem));
        D4_CUDA_OK(cudaFuncSetAttribute(k_ens_rows<true>,
                                        cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        d4::row_smem_bytes<true>()));
        D4_CUDA_OK(cudaFuncSetAttribute(k_ens_rows<false>,
                                        cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        d4::row_smem_bytes<false>()));
        D4_CUDA_OK(cudaStreamSynchronize(E->stream));
    } catch (const d4::CudaError &e) {
        d4_ensemble_destroy(E);
        return D4_ERR_CUDA;
    }
    *out = E;
    return D4_OK;
}

int d4_ensemble_destroy(void *ens) {
    Ensemble *E = (Ensemble *)ens;
    if (!E) return D4_ERR_ARG;
    if (E->stream) cudaStreamSynchronize(E->stream);
    for (int v = 0; v < d4::ens::kNumVec; ++v)
        if (E->P.v[v]) cudaFree(E->P.v[v]);
    void *bufs[] = {E->P.F, E->P.A, E->P.LU, E->P.piv, E->P.sing, E->P.sing_any, E->P.ratio,
                    E->P.strain,
                    E->P.acc, E->P.err, E->d_ins, E->d_sc, E->d_act, E->d_pre_pair,
                    E->d_pre_row, E->d_pre_mat};
    for (void *b : bufs)
        if (b) cudaFree(b);
    if (E->ev0) cudaEventDestroy(E->ev0);
    if (E->ev1) cudaEventDestroy(E->ev1);
    if (E->stream) cudaStreamDestroy(E->stream);
    delete E;
    return D4_OK;
}

const char *d4_ensemble_last_error(void *ens) {
    Ensemble *E = (Ensemble *)ens;
    return E ? E->err.c_str() : "null ensemble";
}

int d4_ensemble_pair_tile_threads(void *ens, int *threads_y) {
    Ensemble *E = (Ensemble *)ens;
    if (!E || !threads_y) return D4_ERR_ARG;
    *threads_y = E->tuned ? E->pair_ty : 0;
    return D4_OK;
}

int d4_ensemble_set_positions(void *ens, int k, const double *x, const double *y) {
    Ensemble *E = (Ensemble *)ens;
    if (!E || k < 0 || k >= E->count || !x || !y) return D4_ERR_ARG;
    const d4::ens::Inst &in = E->hins[k];
    const int bad = d4_check_positions(in.n, x, y);
    if (bad >= 0) {
        E->err = "d4_ensemble_set_positions: instance " + std::to_string(k) + ", dislocation " +
                 std::to_string(bad) + " is not finite or outside the cell [-0.5, 0.5)^2";
        return D4_ERR_ARG;
    }
    const size_t b = sizeof(double) * in.n;
    if (cudaMemcpy(E->P.v[d4::ens::kX0] + in.voff, x, b, cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(E->P.v[d4::ens::kY] + in.voff, y, b, cudaMemcpyHostToDevice) != cudaSuccess)
        return D4_ERR_CUDA;
    return D4_OK;
}

int d4_ensemble_get_positions(void *ens, int k, double *x, double *y) {
    Ensemble *E = (Ensemble *)ens;
    if (!E || k < 0 || k >= E->count || !x || !y) return D4_ERR_ARG;
    const d4::ens::Inst &in = E->hins[k];
    const size_t b = sizeof(double) * in.n;
    if (cudaStreamSynchronize(E->stream) != cudaSuccess ||
        cudaMemcpy(x, E->P.v[d4::ens::kX0] + in.voff, b, cudaMemcpyDeviceToHost) != cudaSuccess ||
        cudaMemcpy(y, E->P.v[d4::ens::kY] + in.voff, b, cudaMemcpyDeviceToHost) != cudaSuccess)
        return D4_ERR_CUDA;
    return D4_OK;
}

int d4_ensemble_run(void *ens, long long max_rounds, d4_run_result *res) {
    using namespace d4::ens;
    Ensemble *E = (Ensemble *)ens;
    if (!E) return D4_ERR_ARG;
    try {
        const d4_params &p = E->p;
        std::vector<int> active;
        for (int k = 0; k < E->count; ++k)
            if (!interrupted(*E, E->hi[k])) active.push_back(k);
        D4_CUDA_OK(cudaEventRecord(E->ev0, E->stream));
        // start of run(): tolerances reset and the initial stress sweep
        // (src/simulation.cpp:46), for instances that have not started
        {
            std::vector<int> fresh;
            for (int k : active)
                if (!E->hi[k].started) fresh.push_back(k);
            if (!fresh.empty()) {
                set_active(*E, fresh);
                for (int k : fresh) {
                    E->hsc[k].ext[0] = d4::ext_stress_host(p.protocol, E->hi[k].sim_time);
                    E->hi[k].started = true;
                }
                D4_CUDA_OK(cudaMemcpyAsync(E->d_sc, E->hsc.data(), sizeof(Sc) * E->count,
                                           cudaMemcpyHostToDevice, E->stream));
                k_ens_fill_tol<<<(int)fresh.size(), 256, 0, E->stream>>>(E->P, E->d_ins, E->d_act,
                                                                         E->cm.min_prec_sq);
                check("k_ens_fill_tol");
                sweep<false>(*E, kX0, 0, 0, 0, kVI, 0);
            }
        }
        if (!E->tuned) {
            if (E->act.empty()) set_active(*E, active);
            autotune(*E);
        }
        std::vector<double> ratio(2 * E->count);
        std::vector<int> acc(E->count);
        long long rounds = 0;
        for (;;) {
            std::vector<int> next;
            for (int k : active)
                if (!interrupted(*E, E->hi[k])) next.push_back(k);
            active.swap(next);
            if (active.empty() || (max_rounds > 0 && rounds >= max_rounds)) break;
            if (active.size() != E->act.size() ||
                !std::equal(active.begin(), active.end(), E->act.begin()) || rounds == 0)
                set_active(*E, active);
            for (int k : active) {
                HostInst &h = E->hi[k];
                Sc &s = E->hsc[k];
                const double t0 = h.sim_time, hh = h.step_size;
                const double t1 = t0 + hh, th = t0 + hh / 2;
                s.h = hh;
                s.ext[0] = d4::ext_stress_host(p.protocol, t0);
                s.ext[1] = d4::ext_stress_host(p.protocol, t1);
                s.ext[2] = d4::ext_stress_host(p.protocol, th);
                s.factor = (th - t0) / (t1 - t0);
                s.dif = s.ext[2] - s.ext[1];
            }
            D4_CUDA_OK(cudaMemcpyAsync(E->d_sc, E->hsc.data(), sizeof(Sc) * E->count,
                                       cudaMemcpyHostToDevice, E->stream));
            attempt_round(*E);
            D4_CUDA_OK(cudaMemcpyAsync(ratio.data(), E->P.ratio, sizeof(double) * 2 * E->count,
                                       cudaMemcpyDeviceToHost, E->stream));
            std::vector<int> sing(E->count);
            D4_CUDA_OK(cudaMemcpyAsync(sing.data(), E->P.sing_any, sizeof(int) * E->count,
                                       cudaMemcpyDeviceToHost, E->stream));
            int perr = 0;
            D4_CUDA_OK(cudaMemcpyAsync(&perr, E->P.err, sizeof(int), cudaMemcpyDeviceToHost,
                                       E->stream));
            D4_CUDA_OK(cudaStreamSynchronize(E->stream));
            if (perr) throw d4::StateError("row-sum pipeline wait timed out");
            for (int k : active) {
                HostInst &h = E->hi[k];
                const double hh = h.step_size;
                const int idx = (int)ratio[2 * k + 1];
                if (idx >= 0) h.selected_id = idx;
                const double r = ratio[2 * k] / E->dipole_prec_sq;
                if (!std::isfinite(r))  // as d4_run: stop instead of doubling h forever
                    throw d4::StateError("non-finite error ratio: an instance's positions or "
                                         "speeds are not finite");
                ++h.attempts;
                h.singular += sing[k] != 0;
                acc[k] = r < 1;
                if (acc[k]) {
                    h.sim_time += hh;
                    ++h.ok;
                } else {
                    ++h.failed;
                }
                // PrecisionHandler::getNewStepSize (src/precision_handler.cpp:57-62)
                double hn = 0.9 * hh * std::min(2., std::pow(r, -1. / 6));
                if (p.max_stepsize > 0 && p.max_stepsize < hn) hn = p.max_stepsize;
                h.step_size = hn;
            }
            if (p.avalanche_limit >= 0) {
                // the accepted instances' mean |v| at the half-step position
                // (v_init2), summed on the host in index order as d4_run does,
                // drives the same two-state avalanche counter
                std::vector<double> v2(E->vtot);
                D4_CUDA_OK(cudaMemcpyAsync(v2.data(), E->P.v[kVI2], sizeof(double) * E->vtot,
                                           cudaMemcpyDeviceToHost, E->stream));
                D4_CUDA_OK(cudaStreamSynchronize(E->stream));
                for (int k : active) {
                    if (!acc[k]) continue;
                    HostInst &h = E->hi[k];
                    const Inst &in = E->hins[k];
                    double sum = 0;
                    for (int i = 0; i < in.n; ++i) sum = sum + std::fabs(v2[in.voff + i]);
                    const double sum_avg = sum / in.n;
                    if (h.in_aval && sum_avg < p.avalanche_speed_threshold) {
                        ++h.aval_count;
                        h.in_aval = false;
                    } else if (sum_avg > p.avalanche_speed_threshold)
                        h.in_aval = true;
                }
            }
            D4_CUDA_OK(cudaMemcpyAsync(E->P.acc, acc.data(), sizeof(int) * E->count,
                                       cudaMemcpyHostToDevice, E->stream));
            k_ens_accept<<<(int)active.size(), 256, 0, E->stream>>>(E->P, E->d_ins, E->d_act,
                                                                    E->cm);
            check("k_ens_accept");
            if (p.calculate_strain) {
                std::vector<double> st(E->count);
                D4_CUDA_OK(cudaMemcpyAsync(st.data(), E->P.strain, sizeof(double) * E->count,
                                           cudaMemcpyDeviceToHost, E->stream));
                D4_CUDA_OK(cudaStreamSynchronize(E->stream));
                for (int k : active) E->hi[k].strain = st[k];
            }
            ++rounds;
        }
        D4_CUDA_OK(cudaEventRecord(E->ev1, E->stream));
        D4_CUDA_OK(cudaStreamSynchronize(E->stream));
        float ms = 0;
        D4_CUDA_OK(cudaEventElapsedTime(&ms, E->ev0, E->ev1));
        if (res)
            for (int k = 0; k < E->count; ++k) {
                const HostInst &h = E->hi[k];
                d4_run_result &r = res[k];
                std::memset(&r, 0, sizeof(r));
                r.sim_time = h.sim_time;
                r.step_size = h.step_size;
                r.strain = h.strain;
                r.successful_steps = h.ok;
                r.failed_steps = h.failed;
                r.attempts = h.attempts;
                r.singular_factorizations = h.singular;
                r.device_seconds = ms / 1000.0;
            }
        return D4_OK;
    } catch (const d4::CudaError &e) {
        E->err = e.what;
        return D4_ERR_CUDA;
    } catch (const d4::StateError &e) {
        E->err = e.what;
        return D4_ERR_STATE;
    } catch (const std::bad_alloc &) {
        E->err = "host allocation failed";
        return D4_ERR_NOMEM;
    }
}

}  // extern "C"
