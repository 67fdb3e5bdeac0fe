// d4_lu_coop.cuh: the cooperative LU kernel, templated on the scalar type
// (double: plain form, --fmad=false; float: mixed form).  See d4_lu_coop64.cu.
#pragma once
#include <cstdint>

#include "d4_internal.h"

namespace d4 {
namespace coop {

constexpr int NB = 32;
constexpr int kThreads = 256;
constexpr long long kSpinLimit = 1ll << 24;  // x >= 64 ns each: > 1 s
constexpr int kGenWord = 32;
template <typename T>
constexpr size_t kRowBufBytes() { return sizeof(T) * kThreads * (NB + 1); }

template <typename T>
struct CoopArgs {
    int n;
    T *A;            // column-major n x n, factorised in place
    T *P0;           // n x 32: the current block's columns before the block
    T *Q;            // 2 x n x 32: pre-division values of a pass (double-buffered)
    unsigned *mask;  // one word per pass (zeroed before the launch): flagged columns
    int *perm;       // n: original row of each position (receives the row swaps)
    int *piv;        // n pivot rows
    int *flags;      // kFlagSingular, kFlagBarrierTimeout
    unsigned *bar;   // grid barrier: [0] arrivals, [kGenWord] generation
};

__device__ __forceinline__ unsigned ld_acq(const unsigned *p) {
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

// Generation barrier over all CTAs of the grid, bounded.  After kSpinLimit
// polls, or as soon as any CTA has given up (kFlagBarrierTimeout), a CTA stops
// waiting for good (dead_s), so the launch always ends; the host then reports
// the error and discards the result.
static __device__ void grid_barrier(unsigned *bar, int *flags, unsigned &gen, int *dead_s) {
    // bar[0]: arrivals; bar[kGenWord]: generation, on its own 128-byte line so
    // the spinning loads do not contend with the arrivals' atomics
    __syncthreads();
    if (threadIdx.x == 0) {
        const unsigned target = gen + 1;
        __threadfence();
        const unsigned arrived = atomicAdd(bar, 1u) + 1;
        if (arrived == gridDim.x) {
            atomicExch(bar, 0u);
            __threadfence();
            atomicExch(bar + kGenWord, target);
        } else if (!*dead_s) {
            long long spins = 0;
            while (ld_acq(bar + kGenWord) != target) {
                __nanosleep(64);
                if ((++spins & 255) == 0 &&
                    (spins > kSpinLimit || ld_acq((const unsigned *)&flags[kFlagBarrierTimeout]))) {
                    atomicOr(&flags[kFlagBarrierTimeout], 1);
                    *dead_s = 1;
                    break;
                }
            }
        }
        gen = target;
    }
    __syncthreads();
}

// Source row in P0 of position r after the block's transpositions (applied in
// order to the arrangement): walk the list backwards.
__device__ __forceinline__ int src_row(int r, const int *sa, const int *sb, int ns) {
    for (int t = ns - 1; t >= 0; --t) {
        if (r == sa[t])
            r = sb[t];
        else if (r == sb[t])
            r = sa[t];
    }
    return r;
}

// Diagonal block of the pass, in every CTA, by all its threads on shared
// memory (two block barriers per column).  Pre-division values go to Q (CTA
// 0), flags into the returned mask (meaningful in thread 0's and the column
// owners' copies; they are OR-ed over the CTA).
template <typename T>
__device__ __noinline__ unsigned diag_block(const CoopArgs<T> &a, T *Q, T (*s)[NB + 1],
                                            int k0, int kw, const int *sa, const int *sb, int ns,
                                            unsigned skip, bool write_q) {
    const int n = a.n;
    const int tid = threadIdx.x;
    unsigned msk = 0;
    for (int t = tid; t < NB * NB; t += kThreads) {
        const int r = t % NB, k = t / NB;
        T v = 0.0;
        if (r < kw && k < kw) v = a.P0[(size_t)src_row(k0 + r, sa, sb, ns) + (size_t)k * n];
        s[r][k] = v;
    }
    __syncthreads();
    for (int k = 0; k < kw; ++k) {
        const T d = s[k][k];
        const bool sk = (skip >> k) & 1u;
        if (tid < NB) {
            const int r = tid;
            if (write_q && r >= k && r < kw) Q[(size_t)(k0 + r) + (size_t)k * n] = s[r][k];
            if (!sk) {
                if (r == 0 && d == 0.0) msk |= 1u << k;
                if (r > k && r < kw) {
                    const T v = s[r][k];
                    if (fabs(v) > fabs(d)) msk |= 1u << k;
                    s[r][k] = v / d;
                }
            }
        }
        __syncthreads();
        if (!sk) {
            for (int t = tid; t < NB * NB; t += kThreads) {
                const int r = t % NB, j = t / NB;
                if (r > k && j > k && r < kw && j < kw) {
                    const T u = s[k][j];
                    if (u != 0.0) s[r][j] = s[r][j] - s[r][k] * u;
                }
            }
        }
        __syncthreads();
    }
    return msk;
}

// Rows below the diagonal block, 8 lanes per row: lane q of a group owns the
// columns q, q+8, q+16, q+24 of its row in registers.  Column k's owner divides
// and broadcasts the multiplier by shuffle; every lane then updates its own
// columns j > k.  Each entry keeps the oracle's update order.  Pre-division
// values to Q, multipliers to A, flags into the returned mask.
template <int KW, typename T>
__device__ __forceinline__ unsigned rows_below_t(const CoopArgs<T> &a, T *Q,
                                                 const T (*s)[NB + 1], int r_pos, int sr,
                                                 int k0, unsigned skip, bool active) {
    const int n = a.n;
    const int lane = threadIdx.x & 31, q = lane & 7, gbase = lane & ~7;
    unsigned msk = 0;
    T c[4];
#pragma unroll
    for (int t = 0; t < 4; ++t) {
        const int col = q + 8 * t;
        c[t] = (active && col < KW) ? a.P0[(size_t)sr + (size_t)col * n] : T(0);
    }
#pragma unroll
    for (int k = 0; k < KW; ++k) {
        const int own = k & 7, slot = k >> 3;
        const T v = __shfl_sync(0xffffffffu, c[slot], gbase + own);
        if (active && q == own) Q[(size_t)r_pos + (size_t)k * n] = v;
        if (!((skip >> k) & 1u)) {
            const T d = s[k][k];
            T l = 0.0;
            if (q == own) {
                if (active && fabs(v) > fabs(d)) msk |= 1u << k;
                l = v / d;
                c[slot] = l;
            }
            l = __shfl_sync(0xffffffffu, l, gbase + own);
#pragma unroll
            for (int t = 0; t < 4; ++t) {
                const int col = q + 8 * t;
                if (col > k && col < KW) {
                    const T u = s[k][col];
                    if (u != 0.0) c[t] = c[t] - l * u;
                }
            }
        }
    }
#pragma unroll
    for (int t = 0; t < 4; ++t) {
        const int col = q + 8 * t;
        if (active && col < KW) a.A[(size_t)r_pos + (size_t)(k0 + col) * n] = c[t];
    }
    return msk;
}

// Narrow last block (kw < 32): one thread per row, shared-memory row.
template <typename T>
__device__ __noinline__ unsigned rows_below_var(const CoopArgs<T> &a, T *Q,
                                                const T (*s)[NB + 1], T *rowbuf,
                                                int r_pos, int sr, int k0, int kw,
                                                unsigned skip) {
    const int n = a.n;
    T *rv = rowbuf + threadIdx.x * (NB + 1);
    for (int k = 0; k < kw; ++k) rv[k] = a.P0[(size_t)sr + (size_t)k * n];
    unsigned msk = 0;
    for (int k = 0; k < kw; ++k) {
        const T v = rv[k];
        Q[(size_t)r_pos + (size_t)k * n] = v;
        if (!((skip >> k) & 1u)) {
            const T d = s[k][k];
            if (fabs(v) > fabs(d)) msk |= 1u << k;
            const T l = v / d;
            rv[k] = l;
            for (int j = k + 1; j < kw; ++j) {
                const T u = s[k][j];
                if (u != 0.0) rv[j] = rv[j] - l * u;
            }
        }
        a.A[(size_t)r_pos + (size_t)(k0 + k) * n] = rv[k];
    }
    return msk;
}

template <typename T>
__device__ __noinline__ unsigned rows_below(const CoopArgs<T> &a, T *Q,
                                            const T (*s)[NB + 1], T *rowbuf, int k0,
                                            int kw, const int *sa, const int *sb, int ns,
                                            unsigned skip) {
    const int n = a.n;
    const int rows = n - k0 - kw;
    unsigned msk = 0;
    if (kw == NB) {
        const int per_round = gridDim.x * (kThreads / 8);
        for (int base = 0; base < rows; base += per_round) {
            const int g = base + blockIdx.x * (kThreads / 8) + (threadIdx.x >> 3);
            if (base + blockIdx.x * (kThreads / 8) >= rows) break;  // warp-uniform per CTA
            const bool active = g < rows;
            const int r_pos = k0 + kw + (active ? g : 0);
            const int sr = active ? src_row(r_pos, sa, sb, ns) : 0;
            msk |= rows_below_t<NB, T>(a, Q, s, r_pos, sr, k0, skip, active);
        }
    } else {
        for (int g = blockIdx.x * kThreads + threadIdx.x; g < rows; g += gridDim.x * kThreads) {
            const int r_pos = k0 + kw + g;
            msk |= rows_below_var(a, Q, s, rowbuf, r_pos, src_row(r_pos, sa, sb, ns), k0, kw,
                                  skip);
        }
    }
    return msk;
}

template <typename T>
__global__ void __launch_bounds__(kThreads, 1) k_lu_coop(CoopArgs<T> a) {
    extern __shared__ __align__(16) unsigned char rowbuf_raw[];
    T *rowbuf = reinterpret_cast<T *>(rowbuf_raw);  // kThreads rows of NB+1 entries
    __shared__ T s[NB][NB + 1];           // diagonal block (rows = positions k0..k0+31)
    __shared__ T Ls[NB][64 + 1];          // update: L21 tile
    __shared__ T Us[NB][64 + 1];          // update: U12 tile
    __shared__ int sa[NB], sb[NB];        // swap list of the block (positions)
    __shared__ unsigned skip_mask;        // singular columns (skipped)
    __shared__ int ns_s;
    __shared__ unsigned cta_mask;
    __shared__ T red_v[kThreads / 32];
    __shared__ int red_i[kThreads / 32];
    __shared__ int dead_s;

    const int n = a.n;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int G = gridDim.x, cta = blockIdx.x;
    unsigned gen = 0;
    if (tid == 0) dead_s = 0;
    const int nblk = (n + NB - 1) / NB;
    for (int i = cta * kThreads + tid; i < n; i += G * kThreads) a.perm[i] = i;

    // prologue: P0 = first block's columns
    for (size_t t = (size_t)cta * kThreads + tid; t < (size_t)n * NB; t += (size_t)G * kThreads) {
        const int r = (int)(t % n), k = (int)(t / n);
        a.P0[t] = k < n ? a.A[(size_t)r + (size_t)k * n] : T(0);
    }
    grid_barrier(a.bar, a.flags, gen, &dead_s);

    int pass = 0;  // global pass counter: mask word, and Q buffer by parity
    for (int kb = 0; kb < nblk; ++kb) {
        const int k0 = kb * NB, kw = min(NB, n - k0);
        if (tid == 0) {
            ns_s = 0;
            skip_mask = 0;
        }
        __syncthreads();
        int scan_from = 0;
        // ------------------------------------------------------------ passes
        for (;;) {
            const int par = pass & 1;
            T *Q = a.Q + (size_t)par * n * NB;
            const int ns = ns_s;
            const unsigned skip = skip_mask;
            if (tid == 0) cta_mask = 0;
            // diagonal block, redundantly in every CTA (warp 0), then the rows below
            unsigned my_mask = diag_block(a, Q, s, k0, kw, sa, sb, ns, skip, cta == 0);
            my_mask |= rows_below(a, Q, s, rowbuf, k0, kw, sa, sb, ns, skip);
            if (my_mask) atomicOr(&cta_mask, my_mask);
            __syncthreads();
            if (tid == 0 && cta_mask) atomicOr(&a.mask[pass], cta_mask);
            grid_barrier(a.bar, a.flags, gen, &dead_s);
            // ------------------------------------------------------- decide
            const unsigned long long mw = ld_acq(&a.mask[pass]);
            const unsigned m = scan_from >= 32 ? 0u : (unsigned)((mw >> scan_from) << scan_from);
            ++pass;
            if (m == 0 || dead_s) break;  // exact: this pass's values stand
            const int ks = __ffs(m) - 1;  // first flagged column
            const int kabs = k0 + ks;
            // exact first-max pivot over positions >= kabs of column ks
            T best = -1.0;
            int bi = n;
            for (int r = kabs + tid; r < n; r += kThreads) {
                const T v = fabs(Q[(size_t)r + (size_t)ks * n]);
                if (v > best) {
                    best = v;
                    bi = r;
                }
            }
            for (int o = 16; o > 0; o >>= 1) {
                const T ov = __shfl_down_sync(0xffffffffu, best, o);
                const int oi = __shfl_down_sync(0xffffffffu, bi, o);
                if (ov > best || (ov == best && oi < bi)) {
                    best = ov;
                    bi = oi;
                }
            }
            if (lane == 0) {
                red_v[warp] = best;
                red_i[warp] = bi;
            }
            __syncthreads();
            if (tid == 0) {
                best = red_v[0];
                bi = red_i[0];
                for (int w = 1; w < kThreads / 32; ++w)
                    if (red_v[w] > best || (red_v[w] == best && red_i[w] < bi)) {
                        best = red_v[w];
                        bi = red_i[w];
                    }
                const T dkk = Q[(size_t)kabs + (size_t)ks * n];
                const int p = (best > fabs(dkk)) ? bi : kabs;
                const T ap = Q[(size_t)p + (size_t)ks * n];
                if (ap == 0.0) {
                    skip_mask |= 1u << ks;
                    if (cta == 0) atomicOr(&a.flags[kFlagSingular], 1);
                } else {
                    sa[ns_s] = kabs;
                    sb[ns_s] = p;
                    ns_s = ns_s + 1;
                }
            }
            __syncthreads();
            scan_from = ks + 1;
        }
        // ---------------------------------------------------------- finish
        const int ns = ns_s;
        if (cta == 0) {
            for (int t = tid; t < NB * NB; t += kThreads) {
                const int r = t % NB, k = t / NB;
                if (r < kw && k < kw) a.A[(size_t)(k0 + r) + (size_t)(k0 + k) * n] = s[r][k];
            }
            for (int k = tid; k < kw; k += kThreads) {
                int p = k0 + k;
                for (int t = 0; t < ns; ++t)
                    if (sa[t] == k0 + k) p = sb[t];
                a.piv[k0 + k] = p;
            }
            if (tid == 0) {
                for (int t = 0; t < ns; ++t) {
                    const int x = a.perm[sa[t]];
                    a.perm[sa[t]] = a.perm[sb[t]];
                    a.perm[sb[t]] = x;
                }
            }
        }
        // other columns: the block's swaps, then U12 = L11^-1 A12 (warp per column)
        {
            const int warps = G * (kThreads / 32);
            for (int c = cta * (kThreads / 32) + warp; c < n - kw; c += warps) {
                const int j = c < k0 ? c : c + kw;
                T *cj = a.A + (size_t)j * n;
                if (lane == 0) {
                    for (int t = 0; t < ns; ++t) {
                        const T x = cj[sa[t]];
                        cj[sa[t]] = cj[sb[t]];
                        cj[sb[t]] = x;
                    }
                }
                __syncwarp();
                if (j >= k0 + kw) {
                    T v = lane < kw ? cj[k0 + lane] : 0.0;
                    for (int k = 0; k < kw; ++k) {
                        const T t = __shfl_sync(0xffffffffu, v, k);
                        if (lane > k && lane < kw && t != 0.0) v = v - s[lane][k] * t;
                    }
                    if (lane < kw) cj[k0 + lane] = v;
                }
            }
        }
        grid_barrier(a.bar, a.flags, gen, &dead_s);
        // ---------------------------------------------------------- update
        const int base = k0 + kw;
        const int rest = n - base;
        if (rest > 0) {
            const int tb = (rest + 63) / 64;
            const int nk0 = base, nkw = min(NB, n - base);  // next block's columns
            for (int tile = cta; tile < tb * tb; tile += G) {
                const int i0 = base + (tile % tb) * 64, j0 = base + (tile / tb) * 64;
                __syncthreads();
                for (int t = tid; t < 64 * NB; t += kThreads) {
                    const int ii = t % 64, k = t / 64;
                    const int gi = i0 + ii;
                    Ls[k][ii] = (k < kw && gi < n) ? a.A[(size_t)gi + (size_t)(k0 + k) * n] : T(0);
                    const int k2 = t % NB, jj = t / NB;
                    const int gj = j0 + jj;
                    Us[k2][jj] =
                        (k2 < kw && gj < n) ? a.A[(size_t)(k0 + k2) + (size_t)gj * n] : T(0);
                }
                __syncthreads();
                const int tr = tid % 16, tc = tid / 16;
                T acc[4][4];
#pragma unroll
                for (int p = 0; p < 4; ++p)
#pragma unroll
                    for (int q = 0; q < 4; ++q) {
                        const int gi = i0 + tr + 16 * p, gj = j0 + tc + 16 * q;
                        acc[p][q] = (gi < n && gj < n) ? a.A[(size_t)gi + (size_t)gj * n] : T(0);
                    }
                for (int k = 0; k < kw; ++k) {
                    T lv[4], uv[4];
#pragma unroll
                    for (int p = 0; p < 4; ++p) lv[p] = Ls[k][tr + 16 * p];
#pragma unroll
                    for (int q = 0; q < 4; ++q) uv[q] = Us[k][tc + 16 * q];
#pragma unroll
                    for (int p = 0; p < 4; ++p)
#pragma unroll
                        for (int q = 0; q < 4; ++q) acc[p][q] = acc[p][q] - lv[p] * uv[q];
                }
#pragma unroll
                for (int p = 0; p < 4; ++p)
#pragma unroll
                    for (int q = 0; q < 4; ++q) {
                        const int gi = i0 + tr + 16 * p, gj = j0 + tc + 16 * q;
                        if (gi < n && gj < n) {
                            a.A[(size_t)gi + (size_t)gj * n] = acc[p][q];
                            if (gj >= nk0 && gj < nk0 + nkw)
                                a.P0[(size_t)gi + (size_t)(gj - nk0) * n] = acc[p][q];
                        }
                    }
            }
            // rows of the next block's columns above the trailing matrix are
            // never read from P0 (positions >= nk0 only)
        }
        grid_barrier(a.bar, a.flags, gen, &dead_s);
    }
}

}  // namespace coop
}  // namespace d4
