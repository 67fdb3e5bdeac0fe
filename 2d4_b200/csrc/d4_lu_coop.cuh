// d4_lu_coop.cuh: the cooperative LU kernel, templated on the scalar type
// (double: plain form, --fmad=false; float: mixed form).  See d4_lu_coop64.cu.
#pragma once
#include <cstdint>
#include <type_traits>

#include "d4_internal.h"
#include "d4_qdiv.cuh"

namespace d4 {
namespace coop {

constexpr int NB = 32;
constexpr int kThreads = 256;
constexpr long long kSpinLimit = 1ll << 24;  // x >= 64 ns each: > 1 s
constexpr int kGenWord = 32;
// Dynamic shared memory: the narrow last block's rows (a row of NB + 1 entries
// per thread) and the diagonal block's pre-division values (NB rows) during a
// pass, the trailing update's second piece buffer during the update; for the
// FP32 form after them the four
// tensor-core operand tiles (L21 and U12 as TF32 hi and lo parts, 16 KiB each,
// 1 KiB aligned) plus the MMA completion barrier and the TMEM address slot.
constexpr size_t kOpTileBytes = 128 * NB * 4;
template <typename T>
__host__ __device__ constexpr size_t kRowBufRaw() { return sizeof(T) * (kThreads + NB) * (NB + 1); }
template <typename T>
__host__ __device__ constexpr size_t kTcOffset() { return (kRowBufRaw<T>() + 1023) / 1024 * 1024; }
template <typename T>
__host__ __device__ constexpr size_t kRowBufBytes() {
    return std::is_same<T, float>::value ? kTcOffset<T>() + 4 * kOpTileBytes + 1024 + 64
                                         : kRowBufRaw<T>();
}

template <typename T>
struct CoopArgs {
    int n;
    T *A;            // column-major n x n, factorised in place
    T *P0;           // n x 32: the current block's columns before the block
    T *Q;            // 2 x n x 32: pre-division values of a pass (double-buffered)
    unsigned *mask;  // one word per pass (zeroed before the launch): flagged columns
    int *perm;       // n: original row of each position (receives the row swaps)
    int *piv;        // n pivot rows
    int *flags;      // kFlagSingular, kFlagBarrierTimeout, kFlagPasses, kFlagSwaps
    unsigned *bar;   // grid barrier: [0] arrivals, [kGenWord] generation
    // FP64 form only (look-ahead of the next diagonal block during the
    // trailing update), zeroed before the launch: per block kb the update's
    // finished strip-0 tiles [kb]; [nblk] the last block whose diagonal block
    // is published
    unsigned *sched;
    T *dg;           // kLuDiagWords: see kDiagWords (null in the FP32 form)
};

// dg: the published diagonal block s (NB x (NB + 1)), its reciprocals rs (NB),
// then the next diagonal block's entries before the update (NB x NB, by column)
constexpr int kDiagWords = NB * (NB + 1) + NB;
constexpr int kSnapOffset = kDiagWords;
static_assert(kDiagWords + NB * NB == kLuDiagWords && NB == kLuNb, "buffer sizes in d4_internal.h");

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

__device__ __forceinline__ void st_rel(unsigned *p, unsigned v) {
    asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// Thread 0: wait until *p >= target, bounded as the grid barrier is (a CTA
// that gives up records kFlagBarrierTimeout and stops waiting for good).
__device__ __forceinline__ void wait_ge(const unsigned *p, unsigned target, int *flags,
                                        int *dead_s) {
    if (*dead_s) return;
    long long spins = 0;
    while (ld_acq(p) < target) {
        __nanosleep(32);
        if ((++spins & 255) == 0 &&
            (spins > kSpinLimit || ld_acq((const unsigned *)&flags[kFlagBarrierTimeout]))) {
            atomicOr(&flags[kFlagBarrierTimeout], 1);
            *dead_s = 1;
            return;
        }
    }
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
// memory (two block barriers per column).  Pre-division values are kept in
// qbuf and go to Q after the loop (CTA 0), so no block barrier waits for a
// global store; flags go into the returned mask (meaningful in thread 0's and
// the column owners' copies; they are OR-ed over the CTA).  A spare thread
// stores each pivot's correctly rounded reciprocal in rs, for the rows below.
template <typename T>
__device__ __noinline__ unsigned diag_block(const CoopArgs<T> &a, T *Q, T (*s)[NB + 1],
                                            T *rs, T (*qbuf)[NB + 1], int k0, int kw,
                                            const int *sa, const int *sb, int ns, unsigned skip,
                                            bool write_q, bool preloaded = false) {
    const int n = a.n;
    const int tid = threadIdx.x;
    unsigned msk = 0;
    if (!preloaded)
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
        if (tid == NB) rs[k] = qdiv::recip(d);
        if (tid < NB) {
            const int r = tid;
            if (write_q && r >= k && r < kw) qbuf[r][k] = s[r][k];
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
    if (write_q)
        for (int t = tid; t < NB * NB; t += kThreads) {
            const int r = t % NB, k = t / NB;
            if (r >= k && r < kw && k < kw) Q[(size_t)(k0 + r) + (size_t)k * n] = qbuf[r][k];
        }
    return msk;
}

// Rows below the diagonal block, 8 lanes per row: lane q of a group owns the
// columns q, q+8, q+16, q+24 of its row in registers.  Column k's owner divides
// and broadcasts the multiplier by shuffle; every lane then updates its own
// columns j > k.  Each entry keeps the oracle's update order; the multiplier
// is the IEEE quotient, formed from the pivot's reciprocal (rs).  Pre-division
// values to Q, multipliers to A, flags into the returned mask.
template <int KW, typename T>
__device__ __forceinline__ unsigned rows_below_t(const CoopArgs<T> &a, T *Q,
                                                 const T (*s)[NB + 1], const T *rs, int r_pos,
                                                 int sr,
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
                l = qdiv::div(v, d, rs[k]);
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
                                                const T (*s)[NB + 1], const T *rs, T *rowbuf,
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
            const T l = qdiv::div(v, d, rs[k]);
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
                                            const T (*s)[NB + 1], const T *rs, T *rowbuf, int k0,
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
            msk |= rows_below_t<NB, T>(a, Q, s, rs, r_pos, sr, k0, skip, active);
        }
    } else {
        for (int g = blockIdx.x * kThreads + threadIdx.x; g < rows; g += gridDim.x * kThreads) {
            const int r_pos = k0 + kw + g;
            msk |= rows_below_var(a, Q, s, rs, rowbuf, r_pos, src_row(r_pos, sa, sb, ns), k0, kw,
                                  skip);
        }
    }
    return msk;
}


// The block's row swaps on every other column, then U12 = L11^-1 A12 on the
// columns right of the block, a warp per column: lane r holds row r, column
// k's value reaches the lanes below by shuffle (u_kj == 0 skips its updates,
// as the oracle does).  The FP64 form also keeps the next diagonal block's
// entries (after the swaps, before the update) for the look-ahead.
template <typename T>
__device__ __noinline__ void finish_cols(const CoopArgs<T> &a, const T (*s)[NB + 1], int k0,
                                         int kw, const int *sa, const int *sb, int ns) {
    const int n = a.n, G = gridDim.x, cta = blockIdx.x;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
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
            if (a.dg && j >= k0 + kw && j < k0 + kw + NB) {
                const int nk0 = k0 + kw;
                if (nk0 + lane < n) a.dg[kSnapOffset + (j - nk0) * NB + lane] = cj[nk0 + lane];
            }
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
}

__device__ __forceinline__ void cp_async8(void *smem, const void *gmem, bool valid) {
    // 8 bytes global -> shared without registers; zero-filled when !valid
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;" ::"r"(
                     (unsigned)__cvta_generic_to_shared(smem)),
                 "l"(gmem), "r"(valid ? 8 : 0)
                 : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;" ::: "memory"); }

// Trailing update A22 -= L21 U12 of the plain form, every entry in the
// oracle's order (k ascending, product and difference rounded separately);
// tiles holding the next block's columns (strip 0) also refresh P0.  64 x 64
// tiles, 4 x 4 entries per thread.  While a tile computes, the next tile's L21
// and U12 pieces stream into the other shared-memory buffer (cp.async) and its
// entries into registers.
//
// Look-ahead: the last CTA takes no tile (unless it is the only one).  It
// forms the next block's diagonal block itself from A, L21 and U12 (the same
// operations in the same order as the tile that owns it, so the same values),
// eliminates it as diag_block does for the next block's first pass (no swaps
// yet) and publishes it: s and rs to dg, pre-division values to Q, flags into
// the next pass's mask word.  The next pass starts without a grid barrier,
// once the diagonal block is published and the strip-0 tiles (P0) are done.
template <typename T>
__device__ __noinline__ void update_la(const CoopArgs<T> &a, int k0, int kw, int kb, int pass,
                                       T *buf0, T *buf1, T (*s)[NB + 1], T *rs,
                                       T (*qbuf)[NB + 1], const int *sa, const int *sb,
                                       unsigned *la_mask_s) {
    constexpr int kLd = 64 + 1;          // row stride of the L and U pieces
    constexpr int kPiece = NB * kLd;     // one piece (L or U)
    const int n = a.n, tid = threadIdx.x, cta = blockIdx.x, G = gridDim.x;
    const int nblk = (n + NB - 1) / NB;
    const int base = k0 + kw, rest = n - base;
    const int tb = (rest + 63) / 64;
    const int nk0 = base, nkw = min(NB, n - base);  // next block's columns
    const int tr = tid % 16, tc = tid / 16;
    const int ntiles = tb * tb;
    const int gt = G > 1 ? G - 1 : 1;  // CTAs that take tiles
    if (cta == G - 1) {
        // the next block's diagonal block: L and U pieces, then 4 entries per thread
        T *Lp = buf0, *Up = buf0 + NB * (NB + 1);
        for (int t = tid; t < NB * NB; t += kThreads) {
            const int r = t % NB, k = t / NB;
            Lp[k * (NB + 1) + r] = (r < nkw && k < kw) ? a.A[(size_t)(nk0 + r) + (size_t)(k0 + k) * n] : T(0);
            const int k2 = t % NB, c = t / NB;
            Up[k2 * (NB + 1) + c] = (c < nkw && k2 < kw) ? a.A[(size_t)(k0 + k2) + (size_t)(nk0 + c) * n] : T(0);
        }
        // the entries before the update come from the snapshot finish_cols
        // took: the tile that owns them may already have overwritten A
        T v[NB * NB / kThreads];
#pragma unroll
        for (int e = 0; e < NB * NB / kThreads; ++e) {
            const int t = tid + e * kThreads, r = t % NB, c = t / NB;
            v[e] = (r < nkw && c < nkw) ? __ldcg(a.dg + kSnapOffset + c * NB + r) : T(0);
        }
        __syncthreads();
        for (int k = 0; k < kw; ++k) {
#pragma unroll
            for (int e = 0; e < NB * NB / kThreads; ++e) {
                const int t = tid + e * kThreads, r = t % NB, c = t / NB;
                v[e] = v[e] - Lp[k * (NB + 1) + r] * Up[k * (NB + 1) + c];
            }
        }
#pragma unroll
        for (int e = 0; e < NB * NB / kThreads; ++e) {
            const int t = tid + e * kThreads;
            s[t % NB][t / NB] = v[e];
        }
        if (tid == 0) *la_mask_s = 0;
        T *Qn = a.Q + (size_t)(pass & 1) * n * NB;
        const unsigned m = diag_block(a, Qn, s, rs, qbuf, nk0, nkw, sa, sb, 0, 0u, true, true);
        if (m) atomicOr(la_mask_s, m);
        for (int t = tid; t < kDiagWords; t += kThreads)
            a.dg[t] = t < NB * (NB + 1) ? s[t / (NB + 1)][t % (NB + 1)] : rs[t - NB * (NB + 1)];
        __syncthreads();
        if (tid == 0) {
            if (*la_mask_s) atomicOr(&a.mask[pass], *la_mask_s);
            __threadfence();
            st_rel(a.sched + nblk, (unsigned)(kb + 1));
        }
        if (G > 1) return;
    }
    T pa[4][4];
    auto stage = [&](int tile, T *buf) {
        const int i0 = base + (tile % tb) * 64, j0 = base + (tile / tb) * 64;
        T *Ls = buf, *Us = buf + kPiece;
#pragma unroll
        for (int r = 0; r < 64 * NB / kThreads; ++r) {
            const int t = tid + r * kThreads;
            const int ii = t % 64, k = t / 64;
            const bool vl = k < kw && i0 + ii < n;
            cp_async8(Ls + k * kLd + ii, vl ? a.A + (size_t)(i0 + ii) + (size_t)(k0 + k) * n : a.A, vl);
            const int k2 = t % NB, jj = t / NB;
            const bool vu = k2 < kw && j0 + jj < n;
            cp_async8(Us + k2 * kLd + jj, vu ? a.A + (size_t)(k0 + k2) + (size_t)(j0 + jj) * n : a.A, vu);
        }
        cp_async_commit();
#pragma unroll
        for (int p = 0; p < 4; ++p)
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const int gi = i0 + tr + 16 * p, gj = j0 + tc + 16 * q;
                pa[p][q] = (gi < n && gj < n) ? a.A[(size_t)gi + (size_t)gj * n] : T(0);
            }
    };
    if (cta < ntiles) stage(cta, buf0);
    int par = 0;
    for (int tile = cta; tile < ntiles; tile += gt, par ^= 1) {
        const int i0 = base + (tile % tb) * 64, j0 = base + (tile / tb) * 64;
        const T *Ls = par ? buf1 : buf0;
        const T *Us = Ls + kPiece;
        T acc[4][4];
#pragma unroll
        for (int p = 0; p < 4; ++p)
#pragma unroll
            for (int q = 0; q < 4; ++q) acc[p][q] = pa[p][q];
        cp_async_wait_all();
        __syncthreads();  // this tile's pieces are in; the other buffer is free
        if (tile + gt < ntiles) stage(tile + gt, par ? buf0 : buf1);
#pragma unroll 2
        for (int k = 0; k < kw; ++k) {
            T lv[4], uv[4];
#pragma unroll
            for (int p = 0; p < 4; ++p) lv[p] = Ls[k * kLd + tr + 16 * p];
#pragma unroll
            for (int q = 0; q < 4; ++q) uv[q] = Us[k * kLd + tc + 16 * q];
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
        // products done with this buffer before it is refilled; a strip-0
        // tile's stores are in before it is counted
        __syncthreads();
        if (tile < tb && tid == 0) {
            __threadfence();
            atomicAdd(a.sched + kb, 1u);
        }
    }
}

// ---------------------------------------------------------------------------
// Tensor-core trailing update of the FP32 form (tcgen05, kind::tf32).
//
// Operand tiles live in shared memory in the canonical K-major layout without
// swizzle: 8-row x 16-byte core matrices, the 8-row groups of a 4-wide K chunk
// contiguous (stride 128 B), consecutive K chunks 16 groups apart (2048 B).
// One instruction covers K = 8 (two chunks).  Each FP32 operand is split into
// TF32 hi and lo parts and the product formed as hi*hi + hi*lo + lo*hi, which
// keeps it close to FP32 accuracy (the update is memory-bound, so the three
// MMAs cost nothing).  D (128 x 128 FP32) accumulates in 128 TMEM columns.
namespace tc {

constexpr uint32_t kLBO = 2048;  // K-chunk stride
constexpr uint32_t kSBO = 128;   // 8-row group stride
// kind::tf32, D F32, A and B TF32 K-major, N = 128, M = 128
constexpr uint32_t kIdesc = (1u << 4) | (2u << 7) | (2u << 10) | ((128u >> 3) << 17) |
                            ((128u >> 4) << 24);
constexpr long long kWaitLimit = 1ll << 24;

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ uint64_t desc(uint32_t saddr) {
    return (uint64_t)((saddr & 0x3FFFFu) >> 4) | ((uint64_t)(kLBO >> 4) << 16) |
           ((uint64_t)(kSBO >> 4) << 32) | (1ull << 46);
}

// byte offset of element (row, k) of a 128 x 32 operand tile
__device__ __forceinline__ uint32_t off(int row, int k) {
    return (uint32_t)((((k >> 2) * 16 + (row >> 3)) * 128) + (row & 7) * 16 + (k & 3) * 4);
}

__device__ __forceinline__ float to_tf32(float x) {
    uint32_t r;
    asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
    return __uint_as_float(r);
}

__device__ __forceinline__ void mma(uint32_t tmem_d, uint64_t ad, uint64_t bd, uint32_t acc) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(tmem_d),
        "l"(ad), "l"(bd), "r"(kIdesc), "r"(acc));
}

__device__ __forceinline__ void commit(uint32_t mbar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
                 ::"r"(mbar) : "memory");
}

// Bounded wait for the barrier's phase `parity`; false if it gave up.
__device__ __forceinline__ bool wait(uint32_t mbar, uint32_t parity) {
    for (long long i = 0; i < kWaitLimit; ++i) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred P1;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2;\n\t"
            "selp.b32 %0, 1, 0, P1;\n\t}\n"
            : "=r"(done) : "r"(mbar), "r"(parity) : "memory");
        if (done) return true;
    }
    return false;
}

__device__ __forceinline__ void ld32(uint32_t taddr, float (&v)[32]) {
    uint32_t r[32];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,"
        "%13,%14,%15,%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
          "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]),
          "=r"(r[13]), "=r"(r[14]), "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]),
          "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]),
          "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]),
          "=r"(r[31])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int t = 0; t < 32; ++t) v[t] = __uint_as_float(r[t]);
}

__device__ __forceinline__ void fence_after() {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void fence_before() {
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}

}  // namespace tc

template <typename T>
__global__ void __launch_bounds__(kThreads, 1) k_lu_coop(CoopArgs<T> a) {
    extern __shared__ __align__(16) unsigned char rowbuf_raw[];
    T *rowbuf = reinterpret_cast<T *>(rowbuf_raw);  // see kRowBufRaw
    __shared__ T s[NB][NB + 1];           // diagonal block (rows = positions k0..k0+31)
    __shared__ T rs[NB];                  // RN(1 / pivot) of the block's columns
    __shared__ __align__(16) T LUs[2 * NB * (64 + 1)];  // update: L21 and U12 pieces (buffer 0)
    __shared__ int sa[NB], sb[NB];        // swap list of the block (positions)
    __shared__ unsigned skip_mask;        // singular columns (skipped)
    __shared__ int ns_s;
    __shared__ unsigned cta_mask;
    __shared__ T red_v[kThreads / 32];
    __shared__ int red_i[kThreads / 32];
    __shared__ int dead_s;
    __shared__ unsigned la_mask_s;        // look-ahead: flags of the diagonal block

    const int n = a.n;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int G = gridDim.x, cta = blockIdx.x;
    unsigned gen = 0;
    if (tid == 0) dead_s = 0;
    const int nblk = (n + NB - 1) / NB;
    for (int i = cta * kThreads + tid; i < n; i += G * kThreads) a.perm[i] = i;
    constexpr bool kTc = std::is_same<T, float>::value;
    unsigned char *tc_base = rowbuf_raw + kTcOffset<T>();
    uint64_t *tc_mbar = reinterpret_cast<uint64_t *>(tc_base + 4 * kOpTileBytes);
    uint32_t *tc_slot = reinterpret_cast<uint32_t *>(tc_base + 4 * kOpTileBytes + 64);
    uint32_t tmem = 0, tc_phase = 0;
    if (kTc) {
        if (warp == 0) {
            asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], 128;"
                         ::"r"(tc::smem_u32(tc_slot)) : "memory");
            asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
        }
        if (tid == 0) {
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(tc::smem_u32(tc_mbar))
                         : "memory");
            asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        }
        tc::fence_before();
        __syncthreads();
        tc::fence_after();
        tmem = *tc_slot;
    }

    // prologue: P0 = first block's columns
    for (size_t t = (size_t)cta * kThreads + tid; t < (size_t)n * NB; t += (size_t)G * kThreads) {
        const int r = (int)(t % n), k = (int)(t / n);
        a.P0[t] = k < n ? a.A[(size_t)r + (size_t)k * n] : T(0);
    }
    grid_barrier(a.bar, a.flags, gen, &dead_s);

    int swaps = 0;  // thread 0: row swaps so far
    int pass = 0;   // global pass counter: mask word, and Q buffer by parity
    for (int kb = 0; kb < nblk; ++kb) {
        const int k0 = kb * NB, kw = min(NB, n - k0);
        if (tid == 0) {
            ns_s = 0;
            skip_mask = 0;
        }
        __syncthreads();
        int scan_from = 0;
        bool first = true;
        // ------------------------------------------------------------ passes
        for (;;) {
            const int par = pass & 1;
            T *Q = a.Q + (size_t)par * n * NB;
            const int ns = ns_s;
            const unsigned skip = skip_mask;
            if (tid == 0) cta_mask = 0;
            unsigned my_mask = 0;
            if (!kTc && kb > 0 && first) {
                // the diagonal block published by the previous update's
                // look-ahead, once that update's strip 0 (P0) is done too
                if (tid == 0) {
                    wait_ge(a.sched + nblk, (unsigned)kb, a.flags, &dead_s);
                    wait_ge(a.sched + (kb - 1), (unsigned)((n - k0 + 63) / 64), a.flags, &dead_s);
                }
                __syncthreads();
                for (int t = tid; t < kDiagWords; t += kThreads) {
                    const T v = __ldcg(a.dg + t);
                    if (t < NB * (NB + 1))
                        s[t / (NB + 1)][t % (NB + 1)] = v;
                    else
                        rs[t - NB * (NB + 1)] = v;
                }
                __syncthreads();
            } else {
                // diagonal block, redundantly in every CTA
                my_mask = diag_block(a, Q, s, rs,
                                     reinterpret_cast<T (*)[NB + 1]>(rowbuf + kThreads * (NB + 1)),
                                     k0, kw, sa, sb, ns, skip, cta == 0);
            }
            first = false;
            my_mask |= rows_below(a, Q, s, rs, rowbuf, k0, kw, sa, sb, ns, skip);
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
        swaps += ns;
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
        finish_cols(a, s, k0, kw, sa, sb, ns);
        grid_barrier(a.bar, a.flags, gen, &dead_s);
        // ---------------------------------------------------------- update
        const int base = k0 + kw;
        const int rest = n - base;
        if (kTc && rest > 0) {
            const int nk0 = base, nkw = min(NB, n - base);  // next block's columns
            const int tb = (rest + 127) / 128;
            float *Ahi = reinterpret_cast<float *>(tc_base);
            float *Alo = reinterpret_cast<float *>(tc_base + kOpTileBytes);
            float *Bhi = reinterpret_cast<float *>(tc_base + 2 * kOpTileBytes);
            float *Blo = reinterpret_cast<float *>(tc_base + 3 * kOpTileBytes);
            for (int tile = cta; tile < tb * tb; tile += G) {
                const int i0 = base + (tile % tb) * 128, j0 = base + (tile / tb) * 128;
                // stage L21 (rows i0.., columns k0..) and U12 (rows k0.., columns j0..):
                // all global loads first (independent), then split and store
                {
                    constexpr int kPer = 128 * NB / kThreads;  // 16 entries per thread
                    float xa[kPer], xb[kPer];
#pragma unroll
                    for (int r = 0; r < kPer; ++r) {
                        const int t = tid + r * kThreads;
                        const int m = t & 127, k = t >> 7;
                        const int gi = i0 + m;
                        xa[r] = (k < kw && gi < n) ? (float)a.A[(size_t)gi + (size_t)(k0 + k) * n]
                                                   : 0.f;
                        const int k2 = t & 31, nn = t >> 5;
                        const int gj = j0 + nn;
                        xb[r] = (k2 < kw && gj < n) ? (float)a.A[(size_t)(k0 + k2) + (size_t)gj * n]
                                                    : 0.f;
                    }
#pragma unroll
                    for (int r = 0; r < kPer; ++r) {
                        const int t = tid + r * kThreads;
                        const uint32_t o = tc::off(t & 127, t >> 7) >> 2;
                        const float hi = tc::to_tf32(xa[r]);
                        Ahi[o] = hi;
                        Alo[o] = tc::to_tf32(xa[r] - hi);
                        const uint32_t o2 = tc::off(t >> 5, t & 31) >> 2;
                        const float yh = tc::to_tf32(xb[r]);
                        Bhi[o2] = yh;
                        Blo[o2] = tc::to_tf32(xb[r] - yh);
                    }
                }
                asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
                __syncthreads();
                if (tid == 0) {
                    tc::fence_after();
                    const uint32_t ah = tc::smem_u32(Ahi), al = tc::smem_u32(Alo);
                    const uint32_t bh = tc::smem_u32(Bhi), bl = tc::smem_u32(Blo);
#pragma unroll
                    for (int q = 0; q < NB / 8; ++q) {
                        const uint32_t ko = q * 2 * tc::kLBO;
                        tc::mma(tmem, tc::desc(ah + ko), tc::desc(bh + ko), q > 0 ? 1u : 0u);
                        tc::mma(tmem, tc::desc(ah + ko), tc::desc(bl + ko), 1u);
                        tc::mma(tmem, tc::desc(al + ko), tc::desc(bh + ko), 1u);
                    }
                    tc::commit(tc::smem_u32(tc_mbar));
                }
                const bool ok = tc::wait(tc::smem_u32(tc_mbar), tc_phase);
                tc_phase ^= 1u;
                if (!ok && tid == 0) atomicOr(&a.flags[kFlagBarrierTimeout], 1);
                tc::fence_after();
                {
                    const int q4 = warp & 3, hf = warp >> 2;
                    const int gi = i0 + 32 * q4 + lane;
#pragma unroll 1
                    for (int c = 0; c < 2; ++c) {
                        const int cb = 64 * hf + 32 * c;
                        float v[32];
                        tc::ld32(tmem + ((uint32_t)(32 * q4) << 16) + (uint32_t)cb, v);
                        if (gi < n) {
                            // loads first (independent), then the stores
                            T cv[32];
#pragma unroll
                            for (int t = 0; t < 32; ++t) {
                                const int gj = j0 + cb + t;
                                cv[t] = gj < n ? a.A[(size_t)gi + (size_t)gj * n] : T(0);
                            }
#pragma unroll
                            for (int t = 0; t < 32; ++t) {
                                const int gj = j0 + cb + t;
                                if (gj < n) {
                                    const T r = cv[t] - (T)v[t];
                                    a.A[(size_t)gi + (size_t)gj * n] = r;
                                    if (gj >= nk0 && gj < nk0 + nkw)
                                        a.P0[(size_t)gi + (size_t)(gj - nk0) * n] = r;
                                }
                            }
                        }
                    }
                }
                tc::fence_before();
                __syncthreads();
            }
        } else if (rest > 0) {
            // buffer 1 reuses the panel's buffers; rows of the next block's
            // columns above the trailing matrix are never read from P0
            // (positions >= nk0 only)
            update_la(a, k0, kw, kb, pass, LUs, rowbuf, s, rs,
                      reinterpret_cast<T (*)[NB + 1]>(rowbuf + kThreads * (NB + 1)), sa, sb,
                      &la_mask_s);
        }
        // FP64 form: the next pass waits for the look-ahead and strip 0 only;
        // the pass barrier then also closes this update
        if (kTc) grid_barrier(a.bar, a.flags, gen, &dead_s);
    }
    if (cta == 0 && tid == 0) {
        a.flags[kFlagPasses] = pass;
        a.flags[kFlagSwaps] = swaps;
    }
    if (kTc) {
        tc::fence_before();
        __syncthreads();
        if (warp == 0)
            asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, 128;" ::"r"(tmem)
                         : "memory");
    }
}

}  // namespace coop
}  // namespace d4
