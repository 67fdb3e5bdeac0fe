// d4_fp64.cu: FP64 pair sweeps of the plain form (compiled with --fmad=false).
//
// Design.  The reference visits each unordered pair (i, j), i < j, once and
// scatters its force antisymmetrically (src/simulation.cpp:292-311,444-483), so
// speed i is the sum, in the order j = 0..n-1 (j != i), of -f(j,i) for j < i and
// +f(i,j) for j > i, plus tau_ext*b_i.  Here a 2-D grid of 32x32 pair tiles
// (upper triangle only, so each pair is evaluated once, like the reference)
// evaluates the field and writes the signed pair force into an n x n matrix F
// (column-major, transposed half via shared memory so both halves store
// coalesced), and, in the fused sweep, the raw Jacobian entry into A.  A second
// kernel with one thread per row then sums row i of F and of A in ascending j,
// which reproduces the reference's summation order exactly, computes d_i and
// applies the row scaling A = I + D J.  The per-dislocation nearest distance
// (PrecisionHandler::updateTolerance) is a min, reduced with 64-bit atomicMin on
// the bit pattern of the non-negative distance.
#include <cstdint>
#include <mutex>

#include "d4_bulk.cuh"
#include "d4_field64.cuh"
#include "d4_internal.h"
#include "d4_table.cuh"

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

// One 32x32 tile of pairs per block; threadIdx.x = local i (coalesced column
// stores), threadIdx.y steps local j.  kTab: the field and its x-derivative come
// from the table (d4_table.cuh) instead of the analytic image sums.
template <bool kJac, bool kTab = false>
__global__ void __launch_bounds__(256) k_pairs64(PairArgs a) {
    const int T = (a.n + kTile - 1) / kTile;
    int ti, tj;
    tile_of(blockIdx.x, T, ti, tj);
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
            double dx = f64::normalize(sxi[tx] - sxj[lj]);
            double dy = f64::normalize(syi[tx] - syj[lj]);
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
                f64::Hyp hp(f64::exp2pix(dx));
                double c = f64::cos2piy(dy);
                fxy = f64::xy(dx, dy, hp, c);
                if (kJac && dist_sq < a.range_sq * a.cut_sq) fdx = f64::xy_diff_x(dx, dy, hp, c);
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

// Ordered row sums of the stress sweep: v_i = sum_j F[i, j] + ext * b_i.
// Loads are issued 8 at a time ahead of the (sequential, ordered) additions.
__global__ void k_rows_speed64(int n, const double *__restrict__ F, double ext, double *v) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double s = 0;
    const double *col = F + i;
    int j = 0;
    for (; j + 8 <= n; j += 8) {
        double t[8];
#pragma unroll
        for (int u = 0; u < 8; ++u) t[u] = __ldg(col + (size_t)(j + u) * n);
#pragma unroll
        for (int u = 0; u < 8; ++u)
            if (j + u != i) s += t[u];
    }
    for (; j < n; ++j)
        if (j != i) s += col[(size_t)j * n];
    v[i] = s + ext * bsign(i, n);
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
__global__ void __launch_bounds__(64) k_rows64(RowArgs a) {
    extern __shared__ __align__(128) unsigned char row_smem[];
    double *bf = reinterpret_cast<double *>(row_smem);  // [stage][col][row]
    double *ba = bf + kRowStages * kRowCols * kRowRows;
    __shared__ __align__(8) uint64_t full[kRowStages], empty[kRowStages];
    __shared__ int issued_s, consumed_s;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int n = a.n;
    const int i0 = blockIdx.x * kRowRows;
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

// Row scaling of the fused sweep (src/simulation.cpp:516-522): A[i,i] =
// subSum_i * sc_i + 1, A[i,j] *= sc_i otherwise (coalesced, column-major).
__global__ void k_scale_rows64(int n, double *A, const double *rowsub, const double *rowsc) {
    const size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= (size_t)n * n) return;
    const int r = (int)(idx % n), c = (int)(idx / n);
    const double sc = rowsc[r];
    A[idx] = (r == c) ? rowsub[r] * sc + 1 : A[idx] * sc;
}

// calcJacobianAndSpeedsFromPrev weights (src/simulation.cpp:552-582).
__global__ void k_half_weights64(int n, const double *dvec, double factor, char wfn,
                                 double *dnew, double *fac) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double old = dvec[i];
    double w = 0.;
    if (old != 0) w = f64::weight(f64::weight_inv(old, wfn) * factor, wfn);
    dnew[i] = w;
    fac[i] = (1 + w) / (1 + old);
}

// Elementwise rescale (src/simulation.cpp:584-594): factor of the row.
__global__ void k_half_rescale64(int n, double *A, const double *fac) {
    const size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    const size_t total = (size_t)n * n;
    if (idx >= total) return;
    const int r = (int)(idx % n), c = (int)(idx / n);
    const double f = fac[r];
    double e = A[idx];
    A[idx] = (r == c) ? 1 + (e - 1) / 2 * f : e / 2 * f;
}

__global__ void k_shift_speed64(int n, double *v, double dif) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) v[i] += dif * bsign(i, n);
}

__global__ void k_fill64(int n, double *v, double val) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) v[i] = val;
}

// calculateXError + updateMaxErrorToleranceRatioSq (src/simulation.cpp:692-700,
// src/precision_handler.cpp:41-54): max of err^2/tol with the first index
// winning ties; out[0] = max, out[1] = index (or -1 when no value beats 0).
__global__ void __launch_bounds__(1024) k_error_ratio64(int n, const double *xb, const double *x2,
                                                        const double *tol, double min_prec_sq,
                                                        int use_dipole, double *out) {
    __shared__ double sv[32];
    __shared__ int si[32];
    double best = 0;
    int bi = -1;
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        double e = fabs(xb[i] - x2[i]);
        double t = use_dipole ? e * e / tol[i] : e * e / min_prec_sq;
        if (t > best) {
            best = t;
            bi = i;
        }
    }
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
            out[0] = best;
            out[1] = bi;
        }
    }
}

__global__ void k_normalize64(int n, double *dst, const double *src) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) dst[i] = f64::normalize(src[i]);
}

// calculateStrainIncrement (src/simulation.cpp:713-720), sequential order.
__global__ void k_strain64(int n, const double *old, const double *nw, double *out) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    double r = 0;
    for (int i = 0; i < n; ++i) r += bsign(i, n) * (nw[i] - old[i]);
    *out = r;
}

// The tabulated field at given points.
__global__ void k_field_tab64(tab::Table tb, int count, const double *dx, const double *dy,
                              double *xy, double *xyd) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= count) return;
    const double2 t = tab::eval<true>(tb, dx[k], dy[k]);
    xy[k] = t.x;
    xyd[k] = t.y;
}

// Field::xy (2-arg, exp2) and Field::xy_diff_x (2-arg, exp) at given points.
__global__ void k_field64(int count, const double *dx, const double *dy, double *xy,
                          double *xyd) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= count) return;
    const double x = dx[k], y = dy[k];
    const double c = f64::cos2piy(y);
    f64::Hyp h2(f64::exp2pix(x));
    xy[k] = f64::xy(x, y, h2, c);
    f64::Hyp he(exp(f64::kPi * 2 * x));
    xyd[k] = f64::xy_diff_x(x, y, he, c);
}

inline int blocks(long long n, int t) { return (int)((n + t - 1) / t); }

}  // namespace

static PairArgs pair_args(Ctx &c, const double *x, const double *y) {
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

template <bool kJac>
static void launch_rows(Ctx &c, const RowArgs &r) {
    constexpr int bytes = row_smem_bytes<kJac>();
    D4_CUDA_OK(cudaFuncSetAttribute(k_rows64<kJac>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    bytes));
    k_rows64<kJac><<<(c.n + kRowRows - 1) / kRowRows, 64, bytes, c.stream>>>(r);
    check_launch(kJac ? "k_rows64<jacobian>" : "k_rows64<speeds>");
}

static int pair_blocks(int n) {
    const int T = (n + kTile - 1) / kTile;
    return T * (T + 1) / 2;
}

void speeds64(Ctx &c, const double *x, const double *y, double ext, double *v) {
    PairArgs a = pair_args(c, x, y);
    if (c.tab)
        k_pairs64<false, true><<<pair_blocks(c.n), dim3(kTile, 8), 0, c.stream>>>(a);
    else
        k_pairs64<false><<<pair_blocks(c.n), dim3(kTile, 8), 0, c.stream>>>(a);
    check_launch("k_pairs64<speeds>");
    RowArgs r{};
    r.n = c.n;
    r.F = c.F;
    r.ext_a = ext;
    r.v_a = v;
    r.err = c.wave_err + kWaveErrRows;
    launch_rows<false>(c, r);
}

void jacobian64(Ctx &c, const double *x, const double *y, double h, double ext_a, double ext_b,
                double *v_a, double *v_b) {
    PairArgs a = pair_args(c, x, y);
    a.h = h;
    if (c.tab)
        k_pairs64<true, true><<<pair_blocks(c.n), dim3(kTile, 8), 0, c.stream>>>(a);
    else
        k_pairs64<true><<<pair_blocks(c.n), dim3(kTile, 8), 0, c.stream>>>(a);
    check_launch("k_pairs64<jacobian>");
    RowArgs r{};
    r.n = c.n;
    r.F = c.F;
    r.A = c.A;
    r.ext_a = ext_a;
    r.ext_b = ext_b;
    r.v_a = v_a;
    r.v_b = v_b;
    r.dvec = c.dvec;
    r.rowsub = c.rowsub;
    r.rowsc = c.rowsc;
    r.wfn = c.p.weight_function;
    r.err = c.wave_err + kWaveErrRows;
    launch_rows<true>(c, r);
    k_scale_rows64<<<blocks((long long)c.n * c.n, 256), 256, 0, c.stream>>>(c.n, c.A, c.rowsub,
                                                                           c.rowsc);
    check_launch("k_scale_rows64");
}

void jacobian_from_prev64(Ctx &c, double factor) {
    k_half_weights64<<<blocks(c.n, 128), 128, 0, c.stream>>>(c.n, c.dvec, factor,
                                                             c.p.weight_function, c.dvec_new,
                                                             c.fac);
    check_launch("k_half_weights64");
    k_half_rescale64<<<blocks((long long)c.n * c.n, 256), 256, 0, c.stream>>>(c.n, c.A, c.fac);
    check_launch("k_half_rescale64");
    D4_CUDA_OK(cudaMemcpyAsync(c.dvec, c.dvec_new, sizeof(double) * c.n, cudaMemcpyDeviceToDevice,
                               c.stream));
}

void half_weights64(Ctx &c, double factor) {
    k_half_weights64<<<blocks(c.n, 128), 128, 0, c.stream>>>(c.n, c.dvec, factor,
                                                             c.p.weight_function, c.dvec_new,
                                                             c.fac);
    check_launch("k_half_weights64");
}

void shift_speed64(Ctx &c, double *v, double dif) {
    k_shift_speed64<<<blocks(c.n, 128), 128, 0, c.stream>>>(c.n, v, dif);
    check_launch("k_shift_speed64");
}

void reset_tol64(Ctx &c) {
    k_fill64<<<blocks(c.n, 128), 128, 0, c.stream>>>(c.n, c.tol, c.min_prec_sq);
    check_launch("k_fill64");
}

void error_ratio64(Ctx &c, const double *xb, const double *x2) {
    k_error_ratio64<<<1, 1024, 0, c.stream>>>(c.n, xb, x2, c.tol, c.min_prec_sq, c.use_dipole,
                                              c.red);
    check_launch("k_error_ratio64");
}

void normalize64(Ctx &c, double *dst, const double *src) {
    k_normalize64<<<blocks(c.n, 128), 128, 0, c.stream>>>(c.n, dst, src);
    check_launch("k_normalize64");
}

void strain_increment64(Ctx &c, const double *x_old, const double *x_new, double *out) {
    k_strain64<<<1, 32, 0, c.stream>>>(c.n, x_old, x_new, out);
    check_launch("k_strain64");
}

void field_eval64(Ctx &c, int count, const double *dx, const double *dy, double *xy,
                  double *xyd) {
    if (c.tab) {
        PairArgs a = pair_args(c, nullptr, nullptr);
        k_field_tab64<<<blocks(count, 128), 128, 0, c.stream>>>(a.tb, count, dx, dy, xy, xyd);
        check_launch("k_field_tab64");
        return;
    }
    k_field64<<<blocks(count, 128), 128, 0, c.stream>>>(count, dx, dy, xy, xyd);
    check_launch("k_field64");
}

}  // namespace d4

// ---------------------------------------------------------------------------
// Allocation-free stress sweep.
//
// Some callers cannot allocate device memory at all: code that runs while a
// stream is being captured into a CUDA graph (an allocation there breaks the
// capture), real-time stepping loops that must not block on the allocator,
// and hosts whose device memory is owned by another framework's allocator
// that this library must not bypass.  For them, d4_speeds_noalloc runs the
// FP64 stress sweep with its n x n pair-force scratch in the file-scope device
// array below instead of a context buffer.  The caller passes device pointers
// for the inputs and outputs; the function calls no cudaMalloc/cudaFree and no
// allocating library routine.
//
// Limit: n <= D4_NOALLOC_MAX_N (1024), i.e. 8 MiB of scratch, held on every
// GPU that loads the library until the process exits.  Every call shares the
// array and it keeps the last call's contents; every entry a call reads is
// written by the same call first, so nothing needs clearing, but calls that
// overlap on the GPU (different streams, or different host threads) race on
// it and must be serialised by the caller.  The first call on a device looks
// up the array's device address (cudaGetSymbolAddress) with that device
// current; make that first call before any stream capture begins.
static __device__ __align__(256) double g_noalloc_pair_force[D4_NOALLOC_MAX_N * D4_NOALLOC_MAX_N];

namespace {
constexpr int kMaxDevices = 64;
std::mutex g_noalloc_mu;
double *g_noalloc_addr[kMaxDevices] = {};
}  // namespace

extern "C" int d4_speeds_noalloc(int n, const double *x, const double *y, double ext_stress,
                                 double *v, double *tol, double min_prec_sq, void *stream) {
    if (n < 2 || n % 2 != 0 || !x || !y || !v) return D4_ERR_ARG;
    if (n > D4_NOALLOC_MAX_N) return D4_ERR_ARG;  // scratch holds at most 1024 x 1024 forces
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return D4_ERR_CUDA;
    double *scratch = nullptr;
    {
        std::lock_guard<std::mutex> lk(g_noalloc_mu);
        if (!g_noalloc_addr[dev]) {
            void *p = nullptr;
            if (cudaGetSymbolAddress(&p, g_noalloc_pair_force) != cudaSuccess || !p)
                return D4_ERR_CUDA;
            g_noalloc_addr[dev] = static_cast<double *>(p);
        }
        scratch = g_noalloc_addr[dev];
    }
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    using namespace d4;
    PairArgs a;
    a.n = n;
    a.x = x;
    a.y = y;
    a.F = scratch;
    a.A = nullptr;
    a.tol = tol;
    a.min_prec_sq = min_prec_sq;
    a.h = 0;
    a.cut_sq = a.cutoff = a.range_sq = a.one_per_cut_sq = 0;
    a.heaviside = 0;
    k_pairs64<false><<<pair_blocks(n), dim3(kTile, 8), 0, st>>>(a);
    g_launches.fetch_add(1, std::memory_order_relaxed);
    if (cudaGetLastError() != cudaSuccess) return D4_ERR_CUDA;
    k_rows_speed64<<<blocks(n, 128), 128, 0, st>>>(n, scratch, ext_stress, v);
    g_launches.fetch_add(1, std::memory_order_relaxed);
    if (cudaGetLastError() != cudaSuccess) return D4_ERR_CUDA;
    return D4_OK;
}
