// d4_trsv.cuh: wavefront triangular solves with LU factors of element type T
// (double: plain form, exact order; float: mixed form inside refinement).
#pragma once
#include "d4_internal.h"

namespace d4 {
namespace trsv {

struct GArgs {
    int gmode;
    double hval;
    const double *dvec, *s_end, *s_init, *x_new, *x_old, *g_in;
    const double *base;
    double *out;
    double *dx_out;
    int fix_singular;  // apply the zeroing of src/simulation.cpp:652-657
};

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
constexpr long long kSpinLimit = 1ll << 25;  // polls of >= 32 ns: > 1 s

// Triangular solve as a wavefront over 32-row blocks, one block per CTA (all
// CTAs co-resident: cooperative launch).  Each entry receives its updates in
// the oracle's order (forward: k ascending; backward: k descending, then the
// division), so the result is bit-identical to the sequential substitution.
// A CTA publishes its 32 finished values and then raises its flag to `epoch`
// (release); consumers acquire the flag before reading.  Spin-waits give up
// after kSpinLimit polls, record the failure in err and finish without
// waiting, so no launch can hang.
template <bool kFwd, typename T>
__global__ void __launch_bounds__(kWaveThreads) k_trsv_wave(int n, const T *__restrict__ LU,
                                                            const int *__restrict__ perm,
                                                            const int *__restrict__ flags, GArgs ga,
                                                            T *xg, const T *xin,
                                                            unsigned *done, unsigned epoch,
                                                            int *err) {
    __shared__ T tile[kWaveRing][32][33];
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
            tile[slot][l][k] = (r < n && cidx < n) ? LU[(size_t)r + (size_t)cidx * n] : T(0);
        }
    };
    T xi = 0;
    if (w == 0 && row_ok) xi = kFwd ? T(g_of(ga, perm[i])) : xin[i];
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
                    __nanosleep(32);
                    if (++spins > kSpinLimit) {
                        if (lane == 0) {
                            abort_s = 1;
                            // err[0] = 1; err[1..3] = waiting block, awaited block, flag seen
                            if (atomicCAS(err, 0, 1) == 0) {
                                err[1] = rb;
                                err[2] = kb;
                                err[3] = (int)ld_acquire(done + kb);
                                err[4] = (int)epoch;
                            }
                        }
                        break;
                    }
                }
                __syncwarp();
            }
            const int kbase = kb * 32;
            T xk = (kbase + lane < n) ? __ldcg(xg + kbase + lane) : T(0);
            const T(*Tl)[33] = tile[s % kWaveRing];
            if (kFwd) {
                for (int k = 0; k < 32; ++k) {
                    const T t = __shfl_sync(0xffffffffu, xk, k);
                    if (t != T(0)) xi = xi - Tl[lane][k] * t;
                }
            } else {
                for (int k = 31; k >= 0; --k) {
                    const T t = __shfl_sync(0xffffffffu, xk, k);
                    if (t != T(0)) xi = xi - Tl[lane][k] * t;
                }
            }
        }
        __syncthreads();
    }
    if (w == 0) {
        const T(*Tl)[33] = tile[count % kWaveRing];
        const int kw = min(32, n - rb * 32);
        if (kFwd) {
            for (int k = 0; k < kw; ++k) {
                const T t = __shfl_sync(0xffffffffu, xi, k);
                if (lane > k && t != T(0)) xi = xi - Tl[lane][k] * t;
            }
        } else {
            for (int k = kw - 1; k >= 0; --k) {
                if (lane == k) xi = xi / Tl[k][k];
                const T t = __shfl_sync(0xffffffffu, xi, k);
                if (lane < k && t != T(0)) xi = xi - Tl[lane][k] * t;
            }
        }
        if (row_ok) xg[i] = xi;
        __threadfence();
        __syncwarp();
        if (lane == 0) st_release(done + rb, epoch);
        if (!kFwd && row_ok) {
            double d = (double)xi;
            if (ga.fix_singular && flags[kFlagSingular] && !((-1 < d) && (d < 1))) d = 0;
            if (ga.dx_out) ga.dx_out[i] = d;
            if (ga.out) ga.out[i] = ga.base[i] - d;
        }
    }
}

}  // namespace trsv
}  // namespace d4
