// d4_trsv.cuh: triangular solves with LU factors of element type T (double:
// plain form, exact order; float: mixed form inside refinement), by one
// thread-block cluster with distributed shared memory.
#pragma once
#include <cstdint>

#include "d4_internal.h"
#include "d4_qdiv.cuh"

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

constexpr long long kSpinLimit = 1ll << 25;  // polls: > 1 s

// ---------------------------------------------------------------------------
// Triangular solves with LU factors of element type T (double: the plain form,
// exact order; float: the mixed form, inside refinement), by one thread-block
// cluster of kClusterCtas CTAs, one warp per 32-row block: block b belongs to
// warp b / C of CTA b % C (a warp takes further blocks b + C * warps when there
// are more blocks than warps).  A warp copies its diagonal tile into its shared
// slot when it starts the block, loads each off-diagonal factor tile straight
// into registers before it waits for that tile's x values (the load overlaps
// the wait), applies the tile, then solves its diagonal block.  A finished
// block's 32 values are pushed into EVERY CTA's shared copy of x with
// asynchronous stores (st.async ... mbarrier::complete_tx) that count down the
// transaction bytes which that CTA's mbarrier for the block expects; a consumer
// waits on its own barrier (acquire) and reads the values locally.  The
// hand-off is one distributed-shared-memory store per value, with no fence and
// no flag poll.  Each entry receives its updates in the oracle's order
// (forward: k ascending; backward: k descending, then the division; updates
// with a zero value skipped), so the result is bit-identical to the sequential
// substitution.  Waits are bounded: after kSpinLimit polls a warp records
// err[0] and stops waiting (the host then discards the results); all CTAs meet
// at a final cluster barrier, so none exits while another may still write into
// its shared memory.
constexpr int kClusterCtas = 8;
constexpr int kClusterMaxWarps = 16;

__device__ __forceinline__ unsigned cluster_rank() {
    unsigned r;
    asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(r));
    return r;
}
__device__ __forceinline__ unsigned cluster_size() {
    unsigned r;
    asm volatile("mov.u32 %0, %%cluster_nctarank;" : "=r"(r));
    return r;
}
__device__ __forceinline__ void cluster_sync_all() {
    asm volatile("barrier.cluster.arrive.release.aligned;\n\tbarrier.cluster.wait.acquire.aligned;" ::
                     : "memory");
}
__device__ __forceinline__ uint32_t mapa(uint32_t addr, unsigned cta) {
    uint32_t r;
    asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(r) : "r"(addr), "r"(cta));
    return r;
}
// Asynchronous store into another CTA's shared memory that completes
// sizeof(v) bytes of the transaction count of that CTA's mbarrier `mbar`.
__device__ __forceinline__ void st_async(uint32_t addr, double v, uint32_t mbar) {
    asm volatile("st.async.shared::cluster.mbarrier::complete_tx::bytes.f64 [%0], %1, [%2];" ::"r"(
                     addr),
                 "d"(v), "r"(mbar)
                 : "memory");
}
__device__ __forceinline__ void st_async(uint32_t addr, float v, uint32_t mbar) {
    asm volatile("st.async.shared::cluster.mbarrier::complete_tx::bytes.f32 [%0], %1, [%2];" ::"r"(
                     addr),
                 "f"(v), "r"(mbar)
                 : "memory");
}
__device__ __forceinline__ void arrive_expect_tx(uint32_t mbar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(mbar), "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ bool try_wait_cluster(uint32_t mbar) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred P1;\n\t"
        "mbarrier.try_wait.parity.acquire.cluster.shared::cta.b64 P1, [%1], 0;\n\t"
        "selp.b32 %0, 1, 0, P1;\n\t}\n"
        : "=r"(done)
        : "r"(mbar)
        : "memory");
    return done != 0;
}

__host__ __device__ constexpr int cluster_warps(int n) {
    return ((n + 31) / 32 + kClusterCtas - 1) / kClusterCtas < kClusterMaxWarps
               ? ((n + 31) / 32 + kClusterCtas - 1) / kClusterCtas
               : kClusterMaxWarps;
}

// x (n values), one mbarrier per 32-row block, and a 32 x 33 diagonal-tile
// slot per warp.
template <typename T>
__host__ __device__ constexpr size_t cluster_smem_bytes(int n) {
    return ((sizeof(T) * (size_t)n + 15) / 16) * 16 +
           ((8 * (size_t)((n + 31) / 32) + 15) / 16) * 16 +
           sizeof(T) * 32 * 33 * (size_t)kClusterMaxWarps;
}

// Tile (row block b, column block kb) of the factors into registers: lane l
// gets row 32 b + l, columns 32 kb .. 32 kb + 31.
template <typename T>
__device__ __forceinline__ void tile_regs(const T *__restrict__ LU, int n, int b, int kb, int lane,
                                          T (&t)[32]) {
    const int r = b * 32 + lane;
#pragma unroll
    for (int k = 0; k < 32; ++k) {
        const int cidx = kb * 32 + k;
        t[k] = (r < n && cidx < n) ? LU[(size_t)r + (size_t)cidx * n] : T(0);
    }
}

// kTrans: the factors are given transposed (Lt = (LU)^T) and the system is
// A^T x = g (P A = L U, so A^T = U^T L^T P): the forward pass is U^T (lower,
// divided), the backward pass L^T (unit upper), g is taken unpermuted and the
// result scattered through perm at the end.
template <bool kFwd, typename T, bool kTrans = false>
__global__ void __launch_bounds__(32 * kClusterMaxWarps) k_trsv_cluster(
    int n, const T *__restrict__ LU, const int *__restrict__ perm, const int *__restrict__ flags,
    GArgs ga, T *xg, const T *xin, int *err) {
    extern __shared__ __align__(16) unsigned char craw[];
    const int nblk = (n + 31) / 32;
    T *xall = reinterpret_cast<T *>(craw);
    uint64_t *mbar = reinterpret_cast<uint64_t *>(craw + ((sizeof(T) * (size_t)n + 15) / 16) * 16);
    T(*dslot)[32][33] = reinterpret_cast<T(*)[32][33]>(reinterpret_cast<unsigned char *>(mbar) +
                                                      ((8 * (size_t)nblk + 15) / 16) * 16);
    const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5, nw = blockDim.x >> 5;
    const int C = (int)cluster_size(), c = (int)cluster_rank();
    // one barrier per block, expecting the block's values (kw x sizeof(T)
    // bytes) from its producer's asynchronous stores
    for (int b = tid; b < nblk; b += blockDim.x) {
        const uint32_t ma = static_cast<uint32_t>(__cvta_generic_to_shared(mbar + b));
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(ma) : "memory");
        arrive_expect_tx(ma, (uint32_t)(sizeof(T) * min(32, n - b * 32)));
    }
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    __syncthreads();
    cluster_sync_all();
    bool aborted = false;
    T(*dt)[33] = dslot[w];
    // this warp's blocks, in solve order
    const int first = c + C * w, stride = C * nw;
    const int nmine = first < nblk ? (nblk - 1 - first) / stride + 1 : 0;
    for (int m = 0; m < nmine; ++m) {
        const int b = kFwd ? first + m * stride : first + (nmine - 1 - m) * stride;
        const int row = b * 32 + lane;
        const bool row_ok = row < n;
        T xi = row_ok ? (kFwd ? T(kTrans ? ga.g_in[row] : g_of(ga, perm[row])) : xin[row]) : T(0);
        T tl[32];
        // the diagonal tile, early, into this warp's shared slot (row per lane)
        tile_regs(LU, n, b, b, lane, tl);
#pragma unroll
        for (int k = 0; k < 32; ++k) dt[lane][k] = tl[k];
        __syncwarp();
        // this lane's divisor and its reciprocal, formed before the chain
        // (the quotient in the chain is still the IEEE one)
        const T dmine = dt[lane][lane];
        const T rmine = qdiv::recip(dmine);
        const int napply = kFwd ? b : nblk - 1 - b;
        for (int s = 0; s < napply; ++s) {
            const int kb = kFwd ? s : nblk - 1 - s;
            const int kw = min(32, n - kb * 32);
            tile_regs(LU, n, b, kb, lane, tl);
            if (!aborted) {
                const uint32_t ma = static_cast<uint32_t>(__cvta_generic_to_shared(mbar + kb));
                long long spins = 0;
                bool ok = true;
                while (!try_wait_cluster(ma)) {
                    if (++spins > kSpinLimit) {
                        ok = false;
                        break;
                    }
                }
                if (!__all_sync(0xffffffffu, ok)) {
                    aborted = true;
                    if (lane == 0 && atomicCAS(err, 0, 1) == 0) {
                        err[1] = b;
                        err[2] = kb;
                        err[3] = -1;
                        err[4] = -1;
                    }
                }
            }
            const T *xb = xall + kb * 32;
            if (kFwd) {
#pragma unroll
                for (int k = 0; k < 32; ++k) {
                    const T t = xb[k < kw ? k : 0];
                    if (k < kw && t != T(0)) xi = xi - tl[k] * t;
                }
            } else {
#pragma unroll
                for (int k = 31; k >= 0; --k) {
                    const T t = xb[k < kw ? k : 0];
                    if (k < kw && t != T(0)) xi = xi - tl[k] * t;
                }
            }
        }
        // diagonal block
        const int kw = min(32, n - b * 32);
        if (kFwd) {
#pragma unroll
            for (int k = 0; k < 32; ++k) {
                if (kTrans && k < kw && lane == k) xi = qdiv::div(xi, dmine, rmine);
                const T t = __shfl_sync(0xffffffffu, xi, k);
                if (k < kw && lane > k && t != T(0)) xi = xi - dt[lane][k] * t;
            }
        } else {
#pragma unroll
            for (int k = 31; k >= 0; --k) {
                if (!kTrans && k < kw && lane == k) xi = qdiv::div(xi, dmine, rmine);
                const T t = __shfl_sync(0xffffffffu, xi, k);
                if (k < kw && lane < k && t != T(0)) xi = xi - dt[lane][k] * t;
            }
        }
        // push to every CTA: asynchronous stores completing that CTA's barrier
        const uint32_t xa = static_cast<uint32_t>(__cvta_generic_to_shared(xall + b * 32 + lane));
        const uint32_t mba = static_cast<uint32_t>(__cvta_generic_to_shared(mbar + b));
        if (row_ok)
            for (int q = 0; q < C; ++q) st_async(mapa(xa, (unsigned)q), xi, mapa(mba, (unsigned)q));
        if (row_ok) {
            xg[(kTrans && !kFwd) ? perm[row] : row] = xi;
            if (!kFwd && !kTrans) {
                double d = (double)xi;
                if (ga.fix_singular && flags[kFlagSingular] && !((-1 < d) && (d < 1))) d = 0;
                if (ga.dx_out) ga.dx_out[row] = d;
                if (ga.out) ga.out[row] = ga.base[row] - d;
            }
        }
    }
    __syncthreads();
    cluster_sync_all();
}

// Forward then backward cluster solve on `stream`: x1 = forward result (global
// scratch), out = backward result.
template <typename T, bool kTrans = false>
inline void launch_cluster_solve(int n, const T *LU, const int *perm, const int *flags,
                                 const GArgs &ga, T *x1, T *out, int *err, cudaStream_t stream) {
    const size_t bytes = cluster_smem_bytes<T>(n);
    const int warps = cluster_warps(n) > 0 ? cluster_warps(n) : 1;
    static bool attr_done = false;
    if (!attr_done) {
        const int maxb = (int)cluster_smem_bytes<T>(kMaxSolveN);
        D4_CUDA_OK(cudaFuncSetAttribute(k_trsv_cluster<true, T, kTrans>,
                                        cudaFuncAttributeMaxDynamicSharedMemorySize, maxb));
        D4_CUDA_OK(cudaFuncSetAttribute(k_trsv_cluster<false, T, kTrans>,
                                        cudaFuncAttributeMaxDynamicSharedMemorySize, maxb));
        attr_done = true;
    }
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(kClusterCtas);
    cfg.blockDim = dim3(32 * warps);
    cfg.dynamicSmemBytes = bytes;
    cfg.stream = stream;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = kClusterCtas;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    const T *none = nullptr;
    D4_CUDA_OK(cudaLaunchKernelEx(&cfg, k_trsv_cluster<true, T, kTrans>, n, LU, perm, flags, ga, x1,
                                  none, err));
    check_launch("k_trsv_cluster<fwd>");
    D4_CUDA_OK(cudaLaunchKernelEx(&cfg, k_trsv_cluster<false, T, kTrans>, n, LU, perm, flags, ga,
                                  out, (const T *)x1, err));
    check_launch("k_trsv_cluster<bwd>");
}

}  // namespace trsv
}  // namespace d4
