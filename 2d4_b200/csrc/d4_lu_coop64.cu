// d4_lu_coop64.cu: FP64 LU with partial pivoting as one persistent kernel
// (compiled with --fmad=false).
//
// Same result, bit for bit, as the oracle's right-looking Gaussian elimination
// with partial pivoting (first index of the largest |a_ik| wins; an exact zero
// pivot skips its column and marks the matrix singular), which stands in for
// umfpack_di_numeric (src/simulation.cpp:635-640).  Every entry keeps its
// update sequence: a_ij -= l_ik * u_kj for k ascending, product and difference
// rounded separately.
//
// Schedule.  The matrix is processed in 32-column blocks by all CTAs of a
// cooperative launch, separated by a grid barrier:
//   pass   every CTA eliminates the block's 32 columns for its rows below the
//          diagonal block, and all CTAs redundantly eliminate the 32x32
//          diagonal block in shared memory, WITHOUT pivoting, starting from a
//          saved copy P0 of the block's columns with the swaps found so far
//          applied.  Pre-division values go to Q; a 32-bit mask records the
//          columns where partial pivoting would have swapped (some
//          |a_ik| > |a_kk|) or met a zero pivot.
//   decide after the barrier every CTA reads the mask.  Empty: the pass is
//          exact, go on.  Otherwise the first flagged column k* gets its exact
//          pivot from Q (first max), the swap (or the singular skip) is
//          appended to the block's list and the pass repeats.  A row swap at
//          column k commutes with the updates of earlier columns, so applying
//          the list to P0 up front is exact.
//   finish CTAs write their rows' multipliers, apply the block's swaps to the
//          other columns and solve U12 = L11^-1 A12 (warp per column).
//   update trailing A22 -= L21 U12 in 64x64 tiles; tiles that hold the next
//          block's columns also refresh P0.  The oracle skips an update whose
//          u_kj is exactly 0; here it is applied (x - l*0 == x for finite l, and
//          the multipliers of an accepted pass are finite: |l| <= 1), so the
//          factors agree bit for bit for every finite matrix.
// A block without swaps costs one pass: three barriers per block in all.
// Barrier waits are bounded: after kSpinLimit polls a CTA records an error
// and stops waiting, so a launch always ends.
#include <cstdint>

#include "d4_internal.h"

namespace d4 {
namespace {

constexpr int NB = 32;
constexpr int kThreads = 256;
constexpr long long kSpinLimit = 1ll << 24;  // x >= 64 ns each: > 1 s
constexpr int kGenWord = 32;
constexpr size_t kRowBufBytes = sizeof(double) * kThreads * (NB + 1);

struct CoopArgs {
    int n;
    double *A;       // column-major n x n, factorised in place
    double *P0;      // n x 32: the current block's columns before the block
    double *Q;       // 2 x n x 32: pre-division values of a pass (double-buffered)
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
__device__ void grid_barrier(unsigned *bar, int *flags, unsigned &gen, int *dead_s) {
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
__device__ __noinline__ unsigned diag_block(const CoopArgs &a, double *Q, double (*s)[NB + 1],
                                            int k0, int kw, const int *sa, const int *sb, int ns,
                                            unsigned skip, bool write_q) {
    const int n = a.n;
    const int tid = threadIdx.x;
    unsigned msk = 0;
    for (int t = tid; t < NB * NB; t += kThreads) {
        const int r = t % NB, k = t / NB;
        double v = 0.0;
        if (r < kw && k < kw) v = a.P0[(size_t)src_row(k0 + r, sa, sb, ns) + (size_t)k * n];
        s[r][k] = v;
    }
    __syncthreads();
    for (int k = 0; k < kw; ++k) {
        const double d = s[k][k];
        const bool sk = (skip >> k) & 1u;
        if (tid < NB) {
            const int r = tid;
            if (write_q && r >= k && r < kw) Q[(size_t)(k0 + r) + (size_t)k * n] = s[r][k];
            if (!sk) {
                if (r == 0 && d == 0.0) msk |= 1u << k;
                if (r > k && r < kw) {
                    const double v = s[r][k];
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
                    const double u = s[k][j];
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
template <int KW>
__device__ __forceinline__ unsigned rows_below_t(const CoopArgs &a, double *Q,
                                                 const double (*s)[NB + 1], int r_pos, int sr,
                                                 int k0, unsigned skip, bool active) {
    const int n = a.n;
    const int lane = threadIdx.x & 31, q = lane & 7, gbase = lane & ~7;
    unsigned msk = 0;
    double c[4];
#pragma unroll
    for (int t = 0; t < 4; ++t) {
        const int col = q + 8 * t;
        c[t] = (active && col < KW) ? a.P0[(size_t)sr + (size_t)col * n] : 0.0;
    }
#pragma unroll
    for (int k = 0; k < KW; ++k) {
        const int own = k & 7, slot = k >> 3;
        const double v = __shfl_sync(0xffffffffu, c[slot], gbase + own);
        if (active && q == own) Q[(size_t)r_pos + (size_t)k * n] = v;
        if (!((skip >> k) & 1u)) {
            const double d = s[k][k];
            double l = 0.0;
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
                    const double u = s[k][col];
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
__device__ __noinline__ unsigned rows_below_var(const CoopArgs &a, double *Q,
                                                const double (*s)[NB + 1], double *rowbuf,
                                                int r_pos, int sr, int k0, int kw,
                                                unsigned skip) {
    const int n = a.n;
    double *rv = rowbuf + threadIdx.x * (NB + 1);
    for (int k = 0; k < kw; ++k) rv[k] = a.P0[(size_t)sr + (size_t)k * n];
    unsigned msk = 0;
    for (int k = 0; k < kw; ++k) {
        const double v = rv[k];
        Q[(size_t)r_pos + (size_t)k * n] = v;
        if (!((skip >> k) & 1u)) {
            const double d = s[k][k];
            if (fabs(v) > fabs(d)) msk |= 1u << k;
            const double l = v / d;
            rv[k] = l;
            for (int j = k + 1; j < kw; ++j) {
                const double u = s[k][j];
                if (u != 0.0) rv[j] = rv[j] - l * u;
            }
        }
        a.A[(size_t)r_pos + (size_t)(k0 + k) * n] = rv[k];
    }
    return msk;
}

__device__ __noinline__ unsigned rows_below(const CoopArgs &a, double *Q,
                                            const double (*s)[NB + 1], double *rowbuf, int k0,
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
            msk |= rows_below_t<NB>(a, Q, s, r_pos, sr, k0, skip, active);
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

__global__ void __launch_bounds__(kThreads, 1) k_lu_coop64(CoopArgs a) {
    extern __shared__ double rowbuf[];    // kThreads rows of NB+1 doubles
    __shared__ double s[NB][NB + 1];      // diagonal block (rows = positions k0..k0+31)
    __shared__ double Ls[NB][64 + 1];     // update: L21 tile
    __shared__ double Us[NB][64 + 1];     // update: U12 tile
    __shared__ int sa[NB], sb[NB];        // swap list of the block (positions)
    __shared__ unsigned skip_mask;        // singular columns (skipped)
    __shared__ int ns_s;
    __shared__ unsigned cta_mask;
    __shared__ double red_v[kThreads / 32];
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
        a.P0[t] = k < n ? a.A[(size_t)r + (size_t)k * n] : 0.0;
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
            double *Q = a.Q + (size_t)par * n * NB;
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
            double best = -1.0;
            int bi = n;
            for (int r = kabs + tid; r < n; r += kThreads) {
                const double v = fabs(Q[(size_t)r + (size_t)ks * n]);
                if (v > best) {
                    best = v;
                    bi = r;
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
                const double dkk = Q[(size_t)kabs + (size_t)ks * n];
                const int p = (best > fabs(dkk)) ? bi : kabs;
                const double ap = Q[(size_t)p + (size_t)ks * n];
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
                double *cj = a.A + (size_t)j * n;
                if (lane == 0) {
                    for (int t = 0; t < ns; ++t) {
                        const double x = cj[sa[t]];
                        cj[sa[t]] = cj[sb[t]];
                        cj[sb[t]] = x;
                    }
                }
                __syncwarp();
                if (j >= k0 + kw) {
                    double v = lane < kw ? cj[k0 + lane] : 0.0;
                    for (int k = 0; k < kw; ++k) {
                        const double t = __shfl_sync(0xffffffffu, v, k);
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
                    Ls[k][ii] = (k < kw && gi < n) ? a.A[(size_t)gi + (size_t)(k0 + k) * n] : 0.0;
                    const int k2 = t % NB, jj = t / NB;
                    const int gj = j0 + jj;
                    Us[k2][jj] =
                        (k2 < kw && gj < n) ? a.A[(size_t)(k0 + k2) + (size_t)gj * n] : 0.0;
                }
                __syncthreads();
                const int tr = tid % 16, tc = tid / 16;
                double acc[4][4];
#pragma unroll
                for (int p = 0; p < 4; ++p)
#pragma unroll
                    for (int q = 0; q < 4; ++q) {
                        const int gi = i0 + tr + 16 * p, gj = j0 + tc + 16 * q;
                        acc[p][q] = (gi < n && gj < n) ? a.A[(size_t)gi + (size_t)gj * n] : 0.0;
                    }
                for (int k = 0; k < kw; ++k) {
                    double lv[4], uv[4];
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

}  // namespace

int coop_grid_size(int n) {
    int dev = 0, sms = 0, per_sm = 0;
    D4_CUDA_OK(cudaGetDevice(&dev));
    D4_CUDA_OK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    D4_CUDA_OK(cudaFuncSetAttribute(k_lu_coop64, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (int)kRowBufBytes));
    D4_CUDA_OK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_lu_coop64, kThreads,
                                                             kRowBufBytes));
    int g = sms * (per_sm < 1 ? 1 : per_sm);
    // enough threads for one row below the diagonal block per thread
    const int need = (n + kThreads - 1) / kThreads;
    if (g < need) return -1;
    return g;
}

int factor64(Ctx &c) {
    const int n = c.n;
    const size_t bytes = sizeof(double) * (size_t)n * n;
    D4_CUDA_OK(cudaMemsetAsync(c.flags, 0, sizeof(int) * kFlagCount, c.stream));
    D4_CUDA_OK(cudaMemsetAsync(c.lu_bar, 0, sizeof(unsigned) * 64, c.stream));
    D4_CUDA_OK(cudaMemsetAsync(c.lu_mask, 0, sizeof(unsigned) * c.lu_mask_words, c.stream));
    D4_CUDA_OK(cudaMemcpyAsync(c.LU, c.A, bytes, cudaMemcpyDeviceToDevice, c.stream));
    CoopArgs a;
    a.n = n;
    a.A = c.LU;
    a.P0 = c.lu_p0;
    a.Q = c.lu_q;
    a.mask = c.lu_mask;
    a.piv = c.piv;
    a.flags = c.flags;
    a.bar = c.lu_bar;
    a.perm = c.perm;
    void *args[] = {(void *)&a};
    D4_CUDA_OK(cudaLaunchCooperativeKernel((const void *)k_lu_coop64, dim3(c.lu_grid),
                                           dim3(kThreads), args, kRowBufBytes, c.stream));
    check_launch("k_lu_coop64");
    D4_CUDA_OK(cudaMemcpyAsync(c.h_flags, c.flags, sizeof(int) * kFlagCount,
                               cudaMemcpyDeviceToHost, c.stream));
    D4_CUDA_OK(cudaStreamSynchronize(c.stream));
    if (c.h_flags[kFlagBarrierTimeout]) throw StateError("LU grid barrier timed out");
    c.factor_singular = c.h_flags[kFlagSingular] != 0;
    c.factor_pivoted = 0;
    return c.factor_singular ? D4_WARN_SINGULAR : D4_OK;
}

}  // namespace d4
