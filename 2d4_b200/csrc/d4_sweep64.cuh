// d4_sweep64.cuh: the FP64 pair-sweep building blocks (pair tiles, pipelined
// ordered row sums, row scaling), shared by the single-system engine
// (d4_fp64.cu) and the batched ensemble (d4_ensemble.cu), which are compiled
// with --fmad=false; d4_fp64_fast.cu builds the mixed form's pair tiles from it
// with another field.
//
// Design.  The reference visits each unordered pair (i, j), i < j, once and
// scatters its force antisymmetrically (src/simulation.cpp:292-311,444-483), so
// speed i is the sum, in the order j = 0..n-1 (j != i), of -f(j,i) for j < i and
// +f(i,j) for j > i, plus tau_ext*b_i.  A 2-D grid of 32x32 pair tiles (upper
// triangle only, so each pair is evaluated once, like the reference) evaluates
// the field and writes the signed pair force into an n x n matrix F
// (column-major, transposed half via shared memory so both halves store
// coalesced), and, in the fused sweep, the raw Jacobian entry into A.  The row
// pipeline then sums row i of F and of A in ascending j, which reproduces the
// reference's summation order exactly, computes d_i and the row scale of
// A = I + D J.  The per-dislocation nearest distance
// (PrecisionHandler::updateTolerance) is a min, reduced with 64-bit atomicMin on
// the bit pattern of the non-negative distance.
#pragma once
#include <cstdint>

#include "d4_bulk.cuh"
#include "d4_field64.cuh"
#include "d4_internal.h"
#include "d4_table.cuh"

// The field of the pair tiles: d4::f64 (the reference's operation order) unless
// the including file names another with the same interface (d4_fp64_fast.cu:
// d4::f64fast for the mixed form).
#ifndef D4_PAIR_FIELD
#define D4_PAIR_FIELD f64
#endif

namespace d4 {
namespace {

__device__ __forceinline__ double bsign(int i, int n) { return i < n / 2 ? 1.0 : -1.0; }

__device__ __forceinline__ void tol_min(double *tol, int idx, double d) {
    // d >= 0 here, so the IEEE bit patterns order like the values.
    atomicMin(reinterpret_cast<unsigned long long *>(tol + idx),
              static_cast<unsigned long long>(__double_as_longlong(d)));
}

// Enumerates upper-triangular tiles (ti <= tj) from a linear block index.
__device__ __forceinline__ void tile_of(int t, int T, int &ti, int &tj) {
    // row ti holds T - ti tiles; walk rows (T is small: <= 256 for n <= 8192)
    int r = 0;
    int rem = t;
    while (rem >= T - r) {
        rem -= T - r;
        ++r;
    }
    ti = r;
    tj = r + rem;
}

struct PairArgs {
    int n;
    const double *x, *y;
    double *F;      // signed pair forces, column-major
    double *A;      // raw Jacobian entries (fused sweep only)
    double *tol;    // tolerance (may be null)
    double min_prec_sq;
    double h;       // step size of the Jacobian
    double cut_sq, cutoff, range_sq, one_per_cut_sq;
    int heaviside;
    tab::Table tb;  // tabulated field (kTab kernels only)
};

// The pair sweep's arguments for a context: positions x, y, the context's
// force matrix, Jacobian, tolerances, cutoff and table.
inline PairArgs pair_args(const Ctx &c, const double *x, const double *y) {
    PairArgs a;
    a.n = c.n;
    a.x = x;
    a.y = y;
    a.F = c.F;
    a.A = c.A;
    a.tol = c.use_dipole ? c.tol : nullptr;
    a.min_prec_sq = c.min_prec_sq;
    a.h = 0;
    a.cut_sq = c.cutoff_sq;
    a.cutoff = c.cutoff;
    a.range_sq = c.range_sq;
    a.one_per_cut_sq = 1 / c.cutoff_sq;
    a.heaviside = c.p.heaviside_cutoff;
    a.tb.t = c.tab;
    a.tb.T = c.tab_T;
    a.tb.W = c.tab_T + 1 + 2 * tab::kGuard;
    return a;
}

inline int pair_blocks(int n) {
    const int T = (n + kTile - 1) / kTile;
    return T * (T + 1) / 2;
}

// One 32x32 tile of pairs per block; threadIdx.x = local i (coalesced column
// stores), threadIdx.y steps local j.  kTab: the field and its x-derivative come
// from the table (d4_table.cuh) instead of the analytic image sums.
template <bool kJac, bool kTab>
__device__ __forceinline__ void pair_tile(const PairArgs &a, int tile) {
    const int T = (a.n + kTile - 1) / kTile;
    int ti, tj;
    tile_of(tile, T, ti, tj);
    __shared__ double sxi[kTile], syi[kTile], sxj[kTile], syj[kTile];
    __shared__ double sf[kTile][kTile + 1];
    __shared__ double sv[kJac ? kTile : 1][kJac ? kTile + 1 : 1];
    const int tx = threadIdx.x, ty = threadIdx.y;
    const int i0 = ti * kTile, j0 = tj * kTile;
    if (ty == 0) {
        int i = i0 + tx, j = j0 + tx;
        sxi[tx] = i < a.n ? a.x[i] : 0;
        syi[tx] = i < a.n ? a.y[i] : 0;
        sxj[tx] = j < a.n ? a.x[j] : 0;
        syj[tx] = j < a.n ? a.y[j] : 0;
    }
    __syncthreads();
    const int i = i0 + tx;
    const double bi = bsign(i, a.n);
    double row_min = 1e300;
    for (int lj = ty; lj < kTile; lj += blockDim.y) {
        const int j = j0 + lj;
        double f = 0, v = 0;
        if (i < a.n && j < a.n && i < j) {
            double dx = D4_PAIR_FIELD::normalize(sxi[tx] - sxj[lj]);
            double dy = D4_PAIR_FIELD::normalize(syi[tx] - syj[lj]);
            double dist_sq = dx * dx + dy * dy;
            if (a.tol && dist_sq < a.min_prec_sq) {
                row_min = fmin(row_min, dist_sq);
                tol_min(a.tol, j, dist_sq);
            }
            const double bj = bsign(j, a.n);
            double fxy, fdx = 0;
            if (kTab) {
                const double2 t = tab::eval<kJac>(a.tb, dx, dy);
                fxy = t.x;
                fdx = t.y;
            } else {
                D4_PAIR_FIELD::Hyp hp(D4_PAIR_FIELD::exp2pix(dx));
                double c = D4_PAIR_FIELD::cos2piy(dy);
                fxy = D4_PAIR_FIELD::xy(dx, dy, hp, c);
                if (kJac && dist_sq < a.range_sq * a.cut_sq)
                    fdx = D4_PAIR_FIELD::xy_diff_x(dx, dy, hp, c);
            }
            f = fxy * bi * bj;
            if (kJac) {
                if (dist_sq < a.range_sq * a.cut_sq) {
                    v = a.h * bj * bi * fdx;
                    if (!a.heaviside && dist_sq > a.cut_sq) {
                        double t = sqrt(dist_sq) - a.cutoff;
                        v *= exp(-(t * t) * a.one_per_cut_sq);
                    }
                }
            }
            a.F[(size_t)i + (size_t)j * a.n] = f;
            if (kJac) a.A[(size_t)i + (size_t)j * a.n] = v;
        }
        sf[tx][lj] = f;
        if (kJac) sv[tx][lj] = v;
    }
    if (a.tol && i < a.n && row_min < a.min_prec_sq) tol_min(a.tol, i, row_min);
    __syncthreads();
    // transposed half: row j gets -f(i, j) at column i; lanes now walk j
    const int j = j0 + tx;
    for (int li = ty; li < kTile; li += blockDim.y) {
        const int ii = i0 + li;
        if (ii < a.n && j < a.n && ii < j) {
            a.F[(size_t)j + (size_t)ii * a.n] = -sf[li][tx];
            if (kJac) a.A[(size_t)j + (size_t)ii * a.n] = sv[li][tx];
        }
    }
}

template <bool kJac, bool kTab = false>
__global__ void __launch_bounds__(256) k_pairs64(PairArgs a) {
    pair_tile<kJac, kTab>(a, blockIdx.x);
}

// Ordered row sums, pipelined.  Block b owns rows i0 = 32 b .. i0 + 31; F (and,
// in the fused sweep, the raw Jacobian A) are column-major, so the 32 rows of
// one column are 256 contiguous bytes.  Warp 1 streams them column chunk by
// column chunk into shared memory with bulk copies (kRowStages chunks of
// kRowCols columns in flight, each completing on its stage's mbarrier); warp 0
// has one lane per row and adds the entries in ascending j, exactly the
// reference's summation order (src/simulation.cpp:292-311,444-503).  The fused
// sweep then writes subSum, d_i = weight(subSum) and the row scale (1 + d_i)/2
// for k_scale_rows64.  A wait that gives up records err[0] = 1 and the block
// drains its copies in flight before it returns.
constexpr int kRowRows = 32, kRowCols = 64, kRowStages = 4;

struct RowArgs {
    int n;
    const double *F, *A;
    double ext_a, ext_b;
    double *v_a, *v_b;  // stress sweep: v_a only
    double *dvec, *rowsub, *rowsc;
    char wfn;
    int *err;
};

template <bool kJac>
constexpr int row_smem_bytes() {
    return (kJac ? 2 : 1) * kRowStages * kRowCols * kRowRows * (int)sizeof(double);
}

template <bool kJac>
__device__ __forceinline__ void row_block(const RowArgs &a, int rb) {
    extern __shared__ __align__(128) unsigned char row_smem[];
    double *bf = reinterpret_cast<double *>(row_smem);  // [stage][col][row]
    double *ba = bf + kRowStages * kRowCols * kRowRows;
    __shared__ __align__(8) uint64_t full[kRowStages], empty[kRowStages];
    __shared__ int issued_s, consumed_s;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int n = a.n;
    const int i0 = rb * kRowRows;
    const int rows = min(kRowRows, n - i0);
    const int nst = (n + kRowCols - 1) / kRowCols;
    if (threadIdx.x == 0) {
        for (int s = 0; s < kRowStages; ++s) {
            bulk::init(&full[s], 1);
            bulk::init(&empty[s], 1);
        }
        bulk::fence_init();
        issued_s = 0;
        consumed_s = 0;
    }
    __syncthreads();
    if (warp == 1) {
        // producer
        const uint32_t col_bytes = rows * (uint32_t)sizeof(double);
        int st = 0;
        for (; st < nst; ++st) {
            const int s = st % kRowStages;
            const uint32_t use = st / kRowStages;
            if (use > 0 && !__all_sync(0xffffffffu, bulk::wait(&empty[s], (use - 1) & 1))) {
                if (lane == 0) atomicOr(a.err, 1);
                break;
            }
            const int j0 = st * kRowCols, nc = min(kRowCols, n - j0);
            if (lane == 0) bulk::arrive_expect_tx(&full[s], nc * col_bytes * (kJac ? 2 : 1));
            __syncwarp();
            for (int k = lane; k < nc; k += 32) {
                const size_t off = (size_t)i0 + (size_t)(j0 + k) * n;
                const int slot = (s * kRowCols + k) * kRowRows;
                bulk::g2s(bf + slot, a.F + off, col_bytes, &full[s]);
                if (kJac) bulk::g2s(ba + slot, a.A + off, col_bytes, &full[s]);
            }
        }
        if (lane == 0) issued_s = st;
    } else {
        // consumer: lane = row
        const int i = i0 + lane;
        double sum = 0, sub = 0;
        int st = 0;
        for (; st < nst; ++st) {
            const int s = st % kRowStages;
            if (!__all_sync(0xffffffffu, bulk::wait(&full[s], (st / kRowStages) & 1))) {
                if (lane == 0) atomicOr(a.err, 1);
                break;
            }
            const int j0 = st * kRowCols, nc = min(kRowCols, n - j0);
            const double *cf = bf + s * kRowCols * kRowRows + lane;
            const double *ca = ba + s * kRowCols * kRowRows + lane;
            for (int k = 0; k < nc; ++k) {
                if (j0 + k == i) continue;
                sum += cf[k * kRowRows];
                if (kJac) sub -= ca[k * kRowRows];
            }
            __syncwarp();
            if (lane == 0) bulk::arrive(&empty[s]);
        }
        if (lane == 0) consumed_s = st;
        if (st == nst && lane < rows) {
            const double b = bsign(i, n);
            if (kJac) {
                a.v_b[i] = sum + a.ext_b * b;
                a.v_a[i] = sum + a.ext_a * b;
                const double d = f64::weight(sub, a.wfn);
                a.dvec[i] = d;
                a.rowsub[i] = sub;
                a.rowsc[i] = (1 + d) / 2;
            } else {
                a.v_a[i] = sum + a.ext_a * b;
            }
        }
    }
    __syncthreads();
    // after a failed wait: let the copies in flight land before the block exits
    if (threadIdx.x == 32)
        for (int st = consumed_s; st < issued_s; ++st)
            bulk::wait(&full[st % kRowStages], (st / kRowStages) & 1);
}

template <bool kJac>
__global__ void __launch_bounds__(64) k_rows64(RowArgs a) {
    row_block<kJac>(a, blockIdx.x);
}

// Row scaling of the fused sweep (src/simulation.cpp:516-522): A[i,i] =
// subSum_i * sc_i + 1, A[i,j] *= sc_i otherwise (coalesced, column-major).
__global__ void k_scale_rows64(int n, double *A, const double *rowsub, const double *rowsc) {
    const size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= (size_t)n * n) return;
    const int r = (int)(idx % n), c = (int)(idx / n);
    const double sc = rowsc[r];
    A[idx] = (r == c) ? rowsub[r] * sc + 1 : A[idx] * sc;
}

// calculateXError + updateMaxErrorToleranceRatioSq (src/simulation.cpp:692-700,
// src/precision_handler.cpp:41-54): max of err^2/tol with the first index
// winning ties; out[0] = max, out[1] = index (or -1 when no value beats 0).
__device__ __forceinline__ void error_ratio_block(int n, const double *xb, const double *x2,
                                                  const double *tol, double min_prec_sq,
                                                  int use_dipole, double *out) {
    __shared__ double sv[32];
    __shared__ int si[32];
    double best = 0;
    int bi = -1;
    int bad = 0;
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        double e = fabs(xb[i] - x2[i]);
        double t = use_dipole ? e * e / tol[i] : e * e / min_prec_sq;
        bad |= !isfinite(e);
        if (t > best) {
            best = t;
            bi = i;
        }
    }
    // the reference's maximum skips a NaN (src/simulation.cpp:692-700); a
    // position that is not finite makes the ratio NaN here, which the host
    // turns into an error instead of a step
    bad = __syncthreads_or(bad);
    for (int o = 16; o > 0; o >>= 1) {
        double ov = __shfl_down_sync(0xffffffffu, best, o);
        int oi = __shfl_down_sync(0xffffffffu, bi, o);
        if (oi >= 0 && (ov > best || (ov == best && (bi < 0 || oi < bi)))) {
            best = ov;
            bi = oi;
        }
    }
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    if (l == 0) {
        sv[w] = best;
        si[w] = bi;
    }
    __syncthreads();
    if (w == 0) {
        const int nw = blockDim.x >> 5;
        best = l < nw ? sv[l] : 0;
        bi = l < nw ? si[l] : -1;
        for (int o = 16; o > 0; o >>= 1) {
            double ov = __shfl_down_sync(0xffffffffu, best, o);
            int oi = __shfl_down_sync(0xffffffffu, bi, o);
            if (oi >= 0 && (ov > best || (ov == best && (bi < 0 || oi < bi)))) {
                best = ov;
                bi = oi;
            }
        }
        if (l == 0) {
            out[0] = bad ? __longlong_as_double(0x7ff8000000000000ll) : best;
            out[1] = bi;
        }
    }
}

}  // namespace
}  // namespace d4
