// d4_lu64.cu: FP64 LU factorisation and solves of the plain form (--fmad=false).
//
// Replaces umfpack_di_numeric/umfpack_di_solve (src/simulation.cpp:635-659)
// for the dense Jacobian.  The CPU oracle factorises with right-looking
// Gaussian elimination with partial pivoting, where every entry a_ij receives
// its updates a_ij -= l_ik * u_kj one k at a time, in increasing k, each product
// and difference rounded separately.  Any schedule that keeps that per-entry
// sequence gives bit-identical factors, so the kernels below are blocked
// (32-wide) but keep it: no FMA contraction, k innermost in ascending order.
//
// Partial pivoting puts a reduction over the whole remaining column on the
// critical path of every column.  The Jacobian A = I + D J is usually
// diagonally dominant enough that partial pivoting never swaps, so the fast
// path factorises without pivoting and checks, for every column k, the exact
// condition under which partial pivoting would have swapped (some
// |a_ik| > |a_kk| below the diagonal, or a_kk == 0).  If it never holds, the
// result is bit-identical to the pivoted factorisation.  If it holds anywhere,
// the factorisation is redone by the pivoted kernels (panel in one CTA with
// first-max pivot search, row swaps, same TRSM and update kernels).
#include <cstdint>
#include <vector>

#include "d4_internal.h"

namespace d4 {
namespace {

constexpr int NB = kLuNb;

// Factor the kw x kw diagonal block at (k0, k0) without pivoting; flag when
// partial pivoting would swap.  blockDim = (32, 32): x = row, y = column.
__global__ void __launch_bounds__(1024) k_lu_diag64(int n, double *A, int k0, int kw, int *flags) {
    __shared__ double s[NB][NB + 1];
    const int r = threadIdx.x, col = threadIdx.y;
    if (r < kw && col < kw) s[r][col] = A[(size_t)(k0 + r) + (size_t)(k0 + col) * n];
    __syncthreads();
    for (int k = 0; k < kw; ++k) {
        if (col == k && r > k && r < kw) {
            const double d = s[k][k], a = s[r][k];
            if (fabs(a) > fabs(d) || d == 0.0) atomicOr(&flags[kFlagNeedPivot], 1);
            s[r][k] = a / d;
        }
        if (col == k && r == k && k == kw - 1 && s[k][k] == 0.0)
            atomicOr(&flags[kFlagNeedPivot], 1);
        __syncthreads();
        if (r > k && col > k && r < kw && col < kw) s[r][col] = s[r][col] - s[r][k] * s[k][col];
        __syncthreads();
    }
    if (r < kw && col < kw) A[(size_t)(k0 + r) + (size_t)(k0 + col) * n] = s[r][col];
}

// L21 = A21 U11^-1, one thread per row below the diagonal block, with the
// partial-pivoting check on each column's pre-division value.
__global__ void __launch_bounds__(128) k_lu_l21_64(int n, double *A, int k0, int kw, int *flags) {
    __shared__ double u[NB][NB + 1];
    for (int t = threadIdx.x; t < kw * kw; t += blockDim.x) {
        const int rr = t % kw, cc = t / kw;
        u[rr][cc] = A[(size_t)(k0 + rr) + (size_t)(k0 + cc) * n];
    }
    __syncthreads();
    const int i = k0 + kw + blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double r[NB];
#pragma unroll
    for (int k = 0; k < NB; ++k)
        if (k < kw) r[k] = A[(size_t)i + (size_t)(k0 + k) * n];
    int need = 0;
#pragma unroll
    for (int k = 0; k < NB; ++k) {
        if (k < kw) {
            const double d = u[k][k];
            if (fabs(r[k]) > fabs(d) || d == 0.0) need = 1;
            const double l = r[k] / d;
            r[k] = l;
#pragma unroll
            for (int kk = k + 1; kk < NB; ++kk)
                if (kk < kw) r[kk] = r[kk] - l * u[k][kk];
        }
    }
    if (need) atomicOr(&flags[kFlagNeedPivot], 1);
#pragma unroll
    for (int k = 0; k < NB; ++k)
        if (k < kw) A[(size_t)i + (size_t)(k0 + k) * n] = r[k];
}

// U12 = L11^-1 A12 (unit lower L11), one warp per column right of the block.
__global__ void __launch_bounds__(256) k_lu_u12_64(int n, double *A, int k0, int kw) {
    __shared__ double l[NB][NB + 1];
    for (int t = threadIdx.x; t < kw * kw; t += blockDim.x) {
        const int rr = t % kw, cc = t / kw;
        l[rr][cc] = A[(size_t)(k0 + rr) + (size_t)(k0 + cc) * n];
    }
    __syncthreads();
    const int lane = threadIdx.x & 31;
    const int j = k0 + kw + blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    if (j >= n) return;
    double a = lane < kw ? A[(size_t)(k0 + lane) + (size_t)j * n] : 0;
    for (int k = 0; k < kw; ++k) {
        const double t = __shfl_sync(0xffffffffu, a, k);
        if (lane > k && lane < kw && t != 0.0) a = a - l[lane][k] * t;
    }
    if (lane < kw) A[(size_t)(k0 + lane) + (size_t)j * n] = a;
}

// A22 -= L21 U12 with the updates applied one k at a time (mul, then sub).
// 64x64 tile per block, 256 threads, 4x4 entries per thread.
__global__ void __launch_bounds__(256) k_lu_gemm64(int n, double *A, int k0, int kw) {
    __shared__ double Ls[NB][64 + 1];
    __shared__ double Us[NB][64 + 1];
    const int base = k0 + kw;
    const int i0 = base + blockIdx.x * 64, j0 = base + blockIdx.y * 64;
    const int tid = threadIdx.x;
    for (int t = tid; t < 64 * NB; t += 256) {
        const int ii = t % 64, k = t / 64;  // L: contiguous in ii
        const int gi = i0 + ii;
        Ls[k][ii] = (k < kw && gi < n) ? A[(size_t)gi + (size_t)(k0 + k) * n] : 0;
        const int k2 = t % NB, jj = t / NB;  // U: contiguous in k
        const int gj = j0 + jj;
        Us[k2][jj] = (k2 < kw && gj < n) ? A[(size_t)(k0 + k2) + (size_t)gj * n] : 0;
    }
    __syncthreads();
    const int tr = tid % 16, tc = tid / 16;  // 16 x 16 threads, each 4 rows x 4 cols
    double acc[4][4];
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
        for (int b = 0; b < 4; ++b) {
            const int gi = i0 + tr + 16 * a, gj = j0 + tc + 16 * b;
            acc[a][b] = (gi < n && gj < n) ? A[(size_t)gi + (size_t)gj * n] : 0;
        }
    for (int k = 0; k < kw; ++k) {
        double lv[4], uv[4];
#pragma unroll
        for (int a = 0; a < 4; ++a) lv[a] = Ls[k][tr + 16 * a];
#pragma unroll
        for (int b = 0; b < 4; ++b) uv[b] = Us[k][tc + 16 * b];
#pragma unroll
        for (int a = 0; a < 4; ++a)
#pragma unroll
            for (int b = 0; b < 4; ++b)
                if (uv[b] != 0.0) acc[a][b] = acc[a][b] - lv[a] * uv[b];
    }
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
        for (int b = 0; b < 4; ++b) {
            const int gi = i0 + tr + 16 * a, gj = j0 + tc + 16 * b;
            if (gi < n && gj < n) A[(size_t)gi + (size_t)gj * n] = acc[a][b];
        }
}

// Pivoted panel: columns [k0, k0+kw), rows [k0, n), one CTA, entries in global
// memory.  Pivot = first index of the largest |a_ik| (the oracle's strict >
// scan); an exact zero pivot marks the matrix singular and skips the column.
__global__ void __launch_bounds__(1024) k_lu_panel_piv64(int n, double *A, int k0, int kw,
                                                         int *piv, int *flags) {
    __shared__ double sv[32];
    __shared__ int si[32];
    __shared__ int s_p;
    __shared__ double s_row[NB];
    const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
    for (int kk = 0; kk < kw; ++kk) {
        const int k = k0 + kk;
        const double *ck = A + (size_t)k * n;
        double best = -1;
        int bi = n;
        for (int i = k + tid; i < n; i += blockDim.x) {
            const double v = fabs(ck[i]);
            if (v > best) {
                best = v;
                bi = i;
            }
        }
        for (int o = 16; o > 0; o >>= 1) {
            const double ov = __shfl_down_sync(0xffffffffu, best, o);
            const int oi = __shfl_down_sync(0xffffffffu, bi, o);
            if (ov > best || (ov == best && oi < bi)) {
                best = ov;
                bi = oi;
            }
        }
        if (lane == 0) {
            sv[w] = best;
            si[w] = bi;
        }
        __syncthreads();
        if (w == 0) {
            const int nw = blockDim.x >> 5;
            best = lane < nw ? sv[lane] : -1;
            bi = lane < nw ? si[lane] : n;
            for (int o = 16; o > 0; o >>= 1) {
                const double ov = __shfl_down_sync(0xffffffffu, best, o);
                const int oi = __shfl_down_sync(0xffffffffu, bi, o);
                if (ov > best || (ov == best && oi < bi)) {
                    best = ov;
                    bi = oi;
                }
            }
            if (lane == 0) {
                // |a_kk| NaN: nothing compares greater, the oracle keeps k
                int p = isnan(fabs(ck[k])) ? k : (bi < n ? bi : k);
                // NaN entries below never win; a best of -1 means all NaN
                if (best < 0) p = k;
                // the oracle only moves off k on a strictly larger value
                if (p != k && !(fabs(ck[p]) > fabs(ck[k]))) p = k;
                s_p = p;
                piv[k] = p;
            }
        }
        __syncthreads();
        const int p = s_p;
        if (ck[p] == 0.0) {
            if (tid == 0) atomicOr(&flags[kFlagSingular], 1);
            __syncthreads();
            continue;
        }
        if (p != k && tid < kw) {
            double *cj = A + (size_t)(k0 + tid) * n;
            const double t = cj[k];
            cj[k] = cj[p];
            cj[p] = t;
        }
        __syncthreads();
        if (tid < kw) s_row[tid] = A[(size_t)k + (size_t)(k0 + tid) * n];
        __syncthreads();
        const double d = s_row[kk];
        for (int i = k + 1 + tid; i < n; i += blockDim.x) {
            const double l = ck[i] / d;
            A[(size_t)i + (size_t)k * n] = l;
            for (int j = kk + 1; j < kw; ++j) {
                const double u = s_row[j];
                if (u != 0.0) {
                    double *e = A + (size_t)i + (size_t)(k0 + j) * n;
                    *e = *e - l * u;
                }
            }
        }
        __syncthreads();
    }
}

// Applies the panel's row swaps, in order, to the columns outside the panel.
__global__ void k_lu_swap64(int n, double *A, int k0, int kw, const int *piv) {
    int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n - kw) return;
    if (j >= k0) j += kw;
    double *cj = A + (size_t)j * n;
    for (int kk = 0; kk < kw; ++kk) {
        const int k = k0 + kk, p = piv[k];
        if (p != k) {
            const double t = cj[k];
            cj[k] = cj[p];
            cj[p] = t;
        }
    }
}

// Row permutation of the right-hand side implied by the sequential swaps.
__global__ void k_perm64(int n, const int *piv, int *perm) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    for (int i = 0; i < n; ++i) perm[i] = i;
    for (int k = 0; k < n; ++k) {
        const int p = piv[k];
        if (p != k) {
            const int t = perm[k];
            perm[k] = perm[p];
            perm[p] = t;
        }
    }
}

__global__ void k_iota(int n, int *v) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) v[i] = i;
}

struct GArgs {
    int gmode;
    double hval;
    const double *dvec, *s_end, *s_init, *x_new, *x_old, *g_in;
    const double *base;
    double *out;
    double *dx_out;
    int fix_singular;  // apply the zeroing of src/simulation.cpp:652-657
};

// One-CTA solve A dx = g with the LU factors (column-major, unit lower L):
// g from the residual formula of the stage (src/simulation.cpp:101,123,142,621),
// permuted, forward and backward substitution in the oracle's per-entry order,
// the singular-matrix fix of src/simulation.cpp:646-658, and out = base - dx.
__global__ void __launch_bounds__(kSolveThreads) k_solve64(int n, const double *__restrict__ LU,
                                                           const int *__restrict__ perm,
                                                           const int *__restrict__ flags,
                                                           GArgs ga) {
    extern __shared__ double sm[];
    double *g = sm;      // n
    double *x = sm + n;  // n
    const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
    for (int i = tid; i < n; i += blockDim.x) {
        double gi;
        if (ga.gmode < 0) {
            gi = ga.g_in[i];
        } else {
            const double d = ga.dvec[i];
            const double X = (1 + d) * ga.s_end[i] + (1 - d) * ga.s_init[i];
            if (ga.gmode == kGBig)
                gi = -ga.hval * X / 2;
            else if (ga.gmode == kGHalf)
                gi = -ga.hval / 2 * X / 2;
            else
                gi = ga.x_new[i] - ga.x_old[i] - ga.hval * X / 2;
        }
        g[i] = gi;
    }
    __syncthreads();
    for (int i = tid; i < n; i += blockDim.x) x[i] = g[perm[i]];
    __syncthreads();
    const int nblk = (n + 31) / 32;
    // forward: unit lower triangular, entry order k ascending
    for (int b = 0; b < nblk; ++b) {
        const int k0 = b * 32, kw = min(32, n - k0);
        if (w == 0) {
            double xi = lane < kw ? x[k0 + lane] : 0;
            for (int k = 0; k < kw; ++k) {
                const double t = __shfl_sync(0xffffffffu, xi, k);
                if (lane > k && lane < kw && t != 0.0)
                    xi = xi - LU[(size_t)(k0 + lane) + (size_t)(k0 + k) * n] * t;
            }
            if (lane < kw) x[k0 + lane] = xi;
        }
        __syncthreads();
        for (int i = k0 + kw + tid; i < n; i += blockDim.x) {
            double xi = x[i];
            for (int k = 0; k < kw; ++k) {
                const double t = x[k0 + k];
                if (t != 0.0) xi = xi - LU[(size_t)i + (size_t)(k0 + k) * n] * t;
            }
            x[i] = xi;
        }
        __syncthreads();
    }
    // backward: upper triangular, k descending
    for (int b = nblk - 1; b >= 0; --b) {
        const int k0 = b * 32, kw = min(32, n - k0);
        if (w == 0) {
            double xi = lane < kw ? x[k0 + lane] : 0;
            for (int k = kw - 1; k >= 0; --k) {
                if (lane == k) xi = xi / LU[(size_t)(k0 + k) + (size_t)(k0 + k) * n];
                const double t = __shfl_sync(0xffffffffu, xi, k);
                if (lane < k && t != 0.0)
                    xi = xi - LU[(size_t)(k0 + lane) + (size_t)(k0 + k) * n] * t;
            }
            if (lane < kw) x[k0 + lane] = xi;
        }
        __syncthreads();
        for (int i = tid; i < k0; i += blockDim.x) {
            double xi = x[i];
            for (int k = kw - 1; k >= 0; --k) {
                const double t = x[k0 + k];
                if (t != 0.0) xi = xi - LU[(size_t)i + (size_t)(k0 + k) * n] * t;
            }
            x[i] = xi;
        }
        __syncthreads();
    }
    const int singular = flags[kFlagSingular];
    for (int i = tid; i < n; i += blockDim.x) {
        double d = x[i];
        if (ga.fix_singular && singular && !((-1 < d) && (d < 1))) d = 0;
        if (ga.dx_out) ga.dx_out[i] = d;
        if (ga.out) ga.out[i] = ga.base[i] - d;
    }
}

// Residual of the stage for row r (src/simulation.cpp:101,123,142,621).
__device__ __forceinline__ double g_of(const GArgs &ga, int r) {
    if (ga.gmode < 0) return ga.g_in[r];
    const double d = ga.dvec[r];
    const double X = (1 + d) * ga.s_end[r] + (1 - d) * ga.s_init[r];
    if (ga.gmode == kGBig) return -ga.hval * X / 2;
    if (ga.gmode == kGHalf) return -ga.hval / 2 * X / 2;
    return ga.x_new[r] - ga.x_old[r] - ga.hval * X / 2;
}

__device__ __forceinline__ unsigned ld_acquire(const unsigned *p) {
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ void st_release(unsigned *p, unsigned v) {
    asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

constexpr int kWaveThreads = 128;       // warp 0 computes, warps 1-3 prefetch tiles
constexpr int kWaveRing = 4;            // L/U tiles in flight per CTA
constexpr long long kSpinLimit = 1ll << 26;

// Triangular solve as a wavefront over 32-row blocks, one block per CTA (all
// CTAs co-resident: cooperative launch).  Each entry receives its updates in
// the oracle's order (forward: k ascending; backward: k descending, then the
// division), so the result is bit-identical to the sequential substitution.
// A CTA publishes its 32 finished values and then raises its flag to `epoch`
// (release); consumers acquire the flag before reading.  Spin-waits give up
// after kSpinLimit polls, record the failure in err and finish without
// waiting, so no launch can hang.
template <bool kFwd>
__global__ void __launch_bounds__(kWaveThreads) k_trsv_wave(int n, const double *__restrict__ LU,
                                                            const int *__restrict__ perm,
                                                            const int *__restrict__ flags, GArgs ga,
                                                            double *xg, const double *xin,
                                                            unsigned *done, unsigned epoch,
                                                            int *err) {
    __shared__ double tile[kWaveRing][32][33];
    __shared__ int abort_s;
    const int nblk = (n + 31) / 32;
    const int b = blockIdx.x;
    const int rb = kFwd ? b : nblk - 1 - b;  // row block of this CTA
    const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
    const int i = rb * 32 + lane;
    const bool row_ok = i < n;
    if (tid == 0) abort_s = 0;
    // column blocks this CTA applies, in order, then its diagonal block
    const int count = kFwd ? rb : (nblk - 1 - rb);
    auto col_block = [&](int s) { return kFwd ? s : nblk - 1 - s; };  // s-th applied block
    auto load_tile = [&](int slot, int kb) {
        // tile[slot][l][k] = M[(rb*32 + l) + (kb*32 + k) * n]
        for (int t = tid - 32; t < 32 * 32; t += kWaveThreads - 32) {
            const int k = t >> 5, l = t & 31;
            const int r = rb * 32 + l, cidx = kb * 32 + k;
            tile[slot][l][k] = (r < n && cidx < n) ? LU[(size_t)r + (size_t)cidx * n] : 0.0;
        }
    };
    double xi = 0;
    if (w == 0 && row_ok) xi = kFwd ? g_of(ga, perm[i]) : xin[i];
    // prefetch the first two tiles (the diagonal tile is step `count`)
    if (w > 0) {
        for (int s = 0; s < 2 && s <= count; ++s) load_tile(s % kWaveRing, s < count ? col_block(s) : rb);
    }
    __syncthreads();
    for (int s = 0; s < count; ++s) {
        if (w > 0 && s + 2 <= count)
            load_tile((s + 2) % kWaveRing, s + 2 < count ? col_block(s + 2) : rb);
        if (w == 0) {
            const int kb = col_block(s);
            if (!abort_s) {
                // every lane acquires the flag itself before reading the values
                long long spins = 0;
                while (!__all_sync(0xffffffffu, ld_acquire(done + kb) == epoch)) {
                    if (++spins > kSpinLimit) {
                        if (lane == 0) {
                            abort_s = 1;
                            atomicExch(err, 1);
                        }
                        break;
                    }
                }
                __syncwarp();
            }
            const int kbase = kb * 32;
            double xk = (kbase + lane < n) ? __ldcg(xg + kbase + lane) : 0.0;
            const double(*T)[33] = tile[s % kWaveRing];
            if (kFwd) {
                for (int k = 0; k < 32; ++k) {
                    const double t = __shfl_sync(0xffffffffu, xk, k);
                    if (t != 0.0) xi = xi - T[lane][k] * t;
                }
            } else {
                for (int k = 31; k >= 0; --k) {
                    const double t = __shfl_sync(0xffffffffu, xk, k);
                    if (t != 0.0) xi = xi - T[lane][k] * t;
                }
            }
        }
        __syncthreads();
    }
    if (w == 0) {
        const double(*T)[33] = tile[count % kWaveRing];
        const int kw = min(32, n - rb * 32);
        if (kFwd) {
            for (int k = 0; k < kw; ++k) {
                const double t = __shfl_sync(0xffffffffu, xi, k);
                if (lane > k && t != 0.0) xi = xi - T[lane][k] * t;
            }
        } else {
            for (int k = kw - 1; k >= 0; --k) {
                if (lane == k) xi = xi / T[k][k];
                const double t = __shfl_sync(0xffffffffu, xi, k);
                if (lane < k && t != 0.0) xi = xi - T[lane][k] * t;
            }
        }
        if (row_ok) xg[i] = xi;
        __threadfence();
        __syncwarp();
        if (lane == 0) st_release(done + rb, epoch);
        if (!kFwd && row_ok) {
            double d = xi;
            if (ga.fix_singular && flags[kFlagSingular] && !((-1 < d) && (d < 1))) d = 0;
            if (ga.dx_out) ga.dx_out[i] = d;
            if (ga.out) ga.out[i] = ga.base[i] - d;
        }
    }
}

void lu_blocked(Ctx &c, bool pivoted) {
    const int n = c.n;
    for (int k0 = 0; k0 < n; k0 += NB) {
        const int kw = min(NB, n - k0);
        const int rest = n - k0 - kw;
        if (pivoted) {
            k_lu_panel_piv64<<<1, 1024, 0, c.stream>>>(n, c.LU, k0, kw, c.piv, c.flags);
            check_launch("k_lu_panel_piv64");
            if (n - kw > 0) {
                k_lu_swap64<<<(n - kw + 127) / 128, 128, 0, c.stream>>>(n, c.LU, k0, kw, c.piv);
                check_launch("k_lu_swap64");
            }
        } else {
            k_lu_diag64<<<1, dim3(NB, NB), 0, c.stream>>>(n, c.LU, k0, kw, c.flags);
            check_launch("k_lu_diag64");
            if (rest > 0) {
                k_lu_l21_64<<<(rest + 127) / 128, 128, 0, c.stream>>>(n, c.LU, k0, kw, c.flags);
                check_launch("k_lu_l21_64");
            }
        }
        if (rest > 0) {
            k_lu_u12_64<<<(rest + 7) / 8, 256, 0, c.stream>>>(n, c.LU, k0, kw);
            check_launch("k_lu_u12_64");
            const int tb = (rest + 63) / 64;
            k_lu_gemm64<<<dim3(tb, tb), 256, 0, c.stream>>>(n, c.LU, k0, kw);
            check_launch("k_lu_gemm64");
        }
    }
}

}  // namespace

void init_lu64() {
    D4_CUDA_OK(cudaFuncSetAttribute(k_solve64, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (int)(sizeof(double) * 2 * kMaxSolveN)));
}

int factor64(Ctx &c) {
    const size_t bytes = sizeof(double) * (size_t)c.n * c.n;
    D4_CUDA_OK(cudaMemsetAsync(c.flags, 0, sizeof(int) * kFlagCount, c.stream));
    D4_CUDA_OK(cudaMemcpyAsync(c.LU, c.A, bytes, cudaMemcpyDeviceToDevice, c.stream));
    lu_blocked(c, false);
    D4_CUDA_OK(cudaMemcpyAsync(c.h_flags, c.flags, sizeof(int) * kFlagCount,
                               cudaMemcpyDeviceToHost, c.stream));
    D4_CUDA_OK(cudaStreamSynchronize(c.stream));
    c.lu_pivoted_path = 0;
    if (c.h_flags[kFlagNeedPivot]) {
        c.lu_pivoted_path = 1;
        D4_CUDA_OK(cudaMemsetAsync(c.flags, 0, sizeof(int) * kFlagCount, c.stream));
        D4_CUDA_OK(cudaMemcpyAsync(c.LU, c.A, bytes, cudaMemcpyDeviceToDevice, c.stream));
        lu_blocked(c, true);
        k_perm64<<<1, 1, 0, c.stream>>>(c.n, c.piv, c.perm);
        check_launch("k_perm64");
        D4_CUDA_OK(cudaMemcpyAsync(c.h_flags, c.flags, sizeof(int) * kFlagCount,
                                   cudaMemcpyDeviceToHost, c.stream));
        D4_CUDA_OK(cudaStreamSynchronize(c.stream));
    } else {
        k_iota<<<(c.n + 255) / 256, 256, 0, c.stream>>>(c.n, c.perm);
        check_launch("k_iota");
    }
    c.factor_singular = c.h_flags[kFlagSingular] != 0;
    c.factor_pivoted = c.lu_pivoted_path;
    return c.factor_singular ? D4_WARN_SINGULAR : D4_OK;
}

static void launch_solve(Ctx &c, const GArgs &ga) {
    const int nblk = (c.n + 31) / 32;
    unsigned e1 = ++c.wave_epoch;
    unsigned e2 = ++c.wave_epoch;
    GArgs g = ga;
    const double *xin_null = nullptr;
    void *args1[] = {(void *)&c.n, (void *)&c.LU, (void *)&c.perm, (void *)&c.flags, (void *)&g,
                     (void *)&c.xw1, (void *)&xin_null, (void *)&c.wave_done, (void *)&e1,
                     (void *)&c.wave_err};
    D4_CUDA_OK(cudaLaunchCooperativeKernel((const void *)k_trsv_wave<true>, dim3(nblk),
                                           dim3(kWaveThreads), args1, 0, c.stream));
    check_launch("k_trsv_wave<fwd>");
    void *args2[] = {(void *)&c.n, (void *)&c.LU, (void *)&c.perm, (void *)&c.flags, (void *)&g,
                     (void *)&c.xw2, (void *)&c.xw1, (void *)&c.wave_done2, (void *)&e2,
                     (void *)&c.wave_err};
    D4_CUDA_OK(cudaLaunchCooperativeKernel((const void *)k_trsv_wave<false>, dim3(nblk),
                                           dim3(kWaveThreads), args2, 0, c.stream));
    check_launch("k_trsv_wave<bwd>");
}

void solve_update64(Ctx &c, int gmode, double hval, const double *s_end, const double *s_init,
                    const double *x_new, const double *x_old, const double *base, double *out) {
    GArgs ga{};
    ga.gmode = gmode;
    ga.hval = hval;
    ga.dvec = c.dvec;
    ga.s_end = s_end;
    ga.s_init = s_init;
    ga.x_new = x_new;
    ga.x_old = x_old;
    ga.base = base;
    ga.out = out;
    ga.dx_out = c.dx;
    ga.fix_singular = 1;
    launch_solve(c, ga);
}

void solve_plain64(Ctx &c, const double *g) {
    GArgs ga{};
    ga.gmode = -1;
    ga.g_in = g;
    ga.dx_out = c.dx;
    launch_solve(c, ga);
}

}  // namespace d4
