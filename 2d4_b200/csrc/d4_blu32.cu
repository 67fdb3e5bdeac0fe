// d4_blu32.cu: the mixed form's factorisation and triangular solves.
//
// Block LU of the FP32 Jacobian in 128 x 128 tiles without row interchanges
// between tiles:
//     A = L U,  L block unit-lower, U block upper with full diagonal blocks,
//     S_ij = A_ij - sum_{k < min(i,j)} L_ik U_kj
//     i == j:  D_j = S_jj^-1   (Gauss-Jordan of the tile, kept for the solves)
//     i >  j:  L_ij = S_ij D_j
//     i <  j:  U_ij = S_ij
// so the solve of A x = b is  y_i = b_i - sum_{k<i} L_ik y_k,
// x_i = D_i (y_i - sum_{j>i} U_ij x_j).  Every product runs on the tensor
// cores (tcgen05.mma kind::tf32, FP32 accumulators in TMEM) as hi*hi + hi*lo
// + lo*hi of the operands split into TF32 hi and lo parts, which keeps the
// factors close to FP32 accuracy; the FP64 refinement of each solve (against
// the FP32 matrix, d4_mixed.cu) removes the rest.  The mixed form has no
// bit-parity duty, so the exact-order partial pivoting of the FP64 form is
// replaced by this pivot-free block form; a tile whose Gauss-Jordan meets a
// zero or non-finite pivot sets kFlagSingular, and the caller redoes the
// attempt with the pivoted cooperative LU (d4_lu_coop.cuh) — as it does when
// a refined residual stays large.
//
// Scheduling.  One persistent launch; each CTA takes the next tile from a
// ticket counter in the order ring m = 0, 1, ... (ring m: the tiles with
// min(i, j) = m, diagonal first, then the pairs (m+d, m), (m, m+d) by
// increasing d).  A tile depends only on tiles earlier in that order, which
// CTAs that are already running hold, so the launch needs no co-residency.
// Finished tiles publish an epoch flag (release); a CTA waits for its
// operands' flags (acquire, bounded) before copying them.
//
// Each finished tile is stored twice: plainly into LU (column-major n x n,
// read by the solves) and as tensor-core operands into its slot of `op`: the
// TF32 hi and lo parts (64 KiB each) in the canonical K-major layout without
// swizzle (8-row x 16-byte core matrices; 32-wide K chunks of 16 KiB), L_ik
// with rows as M, U_kj and D_j with columns as N.  A CTA streams the operand
// chunks of its accumulation with untiled bulk copies (cp.async.bulk, this
// GPU's memory only, no multicast) into a three-stage shared-memory ring;
// thread 0 issues the copies and the MMAs (one elected thread per CTA) and
// tcgen05.commit frees each stage.
#include <cstdint>

#include "d4_bulk.cuh"
#include "d4_internal.h"
#include "d4_lu_coop.cuh"

namespace d4 {
namespace blu {

constexpr int kB = 128;
constexpr int kThreads = 256;
constexpr int kStages = 3;
constexpr uint32_t kStageBytes = 65536;  // A hi, A lo, B hi, B lo chunks of 16 KiB
constexpr uint32_t kChunkBytes = 16384;
constexpr size_t kPartBytes = 65536;     // one packed 128 x 128 FP32 tile
constexpr size_t kSlotBytes = 2 * kPartBytes;
constexpr int kSp = 129;                 // row stride (floats) of the plain tile in shared memory
constexpr size_t kRingBytes = (size_t)kStages * kStageBytes;
constexpr size_t kBarOff = kRingBytes;   // barriers: full[3], empty[3], acc
constexpr size_t kSmemBytes = kRingBytes + 1024;
constexpr long long kSpin = 1ll << 24;   // flag polls (each >= 64 ns): > 1 s
static_assert((size_t)kB * kSp * 4 + 8 * kB * 4 <= kRingBytes, "plain tile and GJ buffers fit the ring");

struct Args {
    int n, T;
    const float *A;         // n x n column-major
    float *LU;              // n x n column-major: L_ij (i > j), U_ij (i < j), D_j (diagonal)
    unsigned char *op;      // T*T slots of kSlotBytes
    const int *tasks;       // T*T: (i << 16) | j in schedule order
    int *ticket;            // ticket counter (zeroed before the launch)
    int *ready;             // T*T tile flags (== epoch: done)
    int epoch;
    int *flags;             // kFlagSingular, kFlagBarrierTimeout
    int refine;             // diagonal inverses: 0 as Gauss-Jordan leaves them, 1 refined,
                            // 2 refined when the tile's condition estimate exceeds kRefineKappa
};

// Infinity-norm condition estimate ||S|| ||D|| of a diagonal tile above which
// its Gauss-Jordan inverse gets a Newton-Schulz step (refine == 2): the
// inverse's error grows faster than the condition number, and the refined
// solves need a contraction well below 1e-3 per sweep.
constexpr float kRefineKappa = 30.f;

__device__ __forceinline__ uint32_t poff(int R, int K) {
    return (uint32_t)((K >> 5) * 16384 + ((K & 31) >> 2) * 2048 + (R >> 3) * 128 + (R & 7) * 16 +
                      (K & 3) * 4);
}

__device__ __forceinline__ int ld_acq(const int *p) {
    int v;
    asm volatile("ld.acquire.gpu.global.b32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ void st_rel(int *p, int v) {
    asm volatile("st.release.gpu.global.b32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

__device__ __forceinline__ void fence_async_global() {
    asm volatile("fence.proxy.async.global;" ::: "memory");
}

__device__ __forceinline__ void fence_async_shared() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// Bounded wait for flag == epoch; false (and kFlagBarrierTimeout) if it gave up
// or another CTA already gave up.
__device__ bool wait_flag(const int *f, int epoch, int *flags) {
    long long spins = 0;
    while (ld_acq(f) != epoch) {
        __nanosleep(64);
        if ((++spins & 255) == 0 &&
            (spins > kSpin || ld_acq(&flags[kFlagBarrierTimeout]))) {
            atomicOr(&flags[kFlagBarrierTimeout], 1);
            return false;
        }
    }
    return true;
}

__device__ __forceinline__ void gave_up(int *flags) { atomicOr(&flags[kFlagBarrierTimeout], 1); }

// The 12 MMAs of one 32-wide K chunk held in stage `sb` (shared address):
// A hi/lo at +0/+16K, B hi/lo at +32K/+48K; hi*hi + hi*lo + lo*hi.
__device__ __forceinline__ void mma_chunk(uint32_t tmem_d, uint32_t sb, bool first) {
    using namespace coop::tc;
#pragma unroll
    for (int u = 0; u < 4; ++u) {
        const uint32_t o = u * 4096;
        mma(tmem_d, desc(sb + o), desc(sb + 32768 + o), (first && u == 0) ? 0u : 1u);
        mma(tmem_d, desc(sb + o), desc(sb + 49152 + o), 1u);
        mma(tmem_d, desc(sb + 16384 + o), desc(sb + 32768 + o), 1u);
    }
}

__device__ __forceinline__ void ld64(uint32_t taddr, float (&v)[64]) {
    float a[32], b[32];
    coop::tc::ld32(taddr, a);
    coop::tc::ld32(taddr + 32, b);
#pragma unroll
    for (int t = 0; t < 32; ++t) {
        v[t] = a[t];
        v[32 + t] = b[t];
    }
}

// A tile F (plain, row-major, stride kSp, in shared memory) of tile position
// (ti, tj): store_tile writes its operand slot (A format, rows as M, when
// !bfmt, else B format, columns as N), store_plain its real entries to LU.
// The slot is what other tiles wait for; LU is read only by the solves, after
// the launch, so it is written after the tile's flag is published.
__device__ void store_plain(const Args &a, const float *Sp, int ti, int tj) {
    const int tid = threadIdx.x;
    const int n = a.n;
    const int r = tid & 127, h = tid >> 7;
    const int gr = ti * kB + r;
    if (gr < n) {
        for (int c = 64 * h; c < 64 * h + 64; ++c) {
            const int gc = tj * kB + c;
            if (gc < n) a.LU[(size_t)gr + (size_t)gc * n] = Sp[r * kSp + c];
        }
    }
}

__device__ void store_tile(const Args &a, const float *Sp, int ti, int tj, bool bfmt,
                           unsigned char *slot) {
    const int tid = threadIdx.x;
#pragma unroll 4
    for (int u = 0; u < 16; ++u) {
        const int p = tid + kThreads * u;
        const int chunk = p >> 10, kg = (p >> 7) & 7, R = ((p >> 3) & 15) * 8 + (p & 7);
        const int K0 = chunk * 32 + kg * 4;
        float v[4], hi[4], lo[4];
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            v[q] = bfmt ? Sp[(K0 + q) * kSp + R] : Sp[R * kSp + K0 + q];
            hi[q] = coop::tc::to_tf32(v[q]);
            lo[q] = coop::tc::to_tf32(v[q] - hi[q]);
        }
        *reinterpret_cast<float4 *>(slot + 16 * (size_t)p) = make_float4(hi[0], hi[1], hi[2], hi[3]);
        *reinterpret_cast<float4 *>(slot + kPartBytes + 16 * (size_t)p) =
            make_float4(lo[0], lo[1], lo[2], lo[3]);
    }
}

// In-place Gauss-Jordan inverse of the 128 x 128 tile in Sp (no pivoting):
// thread (tr, tc) of a 16 x 16 grid keeps rows 8tr.. and columns 8tc.. in
// registers.  The step of pivot k is the rank-1 form
//     a_rc <- [c != k] a_rc - L_r U_c  (+1 at r = c = k)
// with L_r = a_rk (a_kk - 1 at r = k) and U_c = a_kc / a_kk (1 / a_kk at
// c = k).  Pivots go in pairs (k, k+1) with one block barrier per pair: the
// owners publish columns k, k+1 and rows k, k+1 as they stand before pivot k
// (double-buffered), and every thread forms column k+1 and row k+1 after
// pivot k for its own rows and columns with the same products the owners
// would use, so the result is the one-pivot-at-a-time inverse bit for bit.
// Returns false (on thread 0) when a pivot is zero or not finite.
__device__ bool gauss_jordan(float *Sp, float *cbuf, float *rbuf) {
    const int tid = threadIdx.x;
    const int tr = tid >> 4, tc = tid & 15;
    float a[8][8];
#pragma unroll
    for (int i = 0; i < 8; ++i)
#pragma unroll
        for (int j = 0; j < 8; ++j) a[i][j] = Sp[(8 * tr + i) * kSp + 8 * tc + j];
    bool ok = true;
    // pivots in groups of 8: the group index kb is a loop variable, the pair's
    // place kl inside the group is a compile-time index into the registers
#pragma unroll 1
    for (int kb = 0; kb < kB / 8; ++kb)
#pragma unroll
    for (int kl = 0; kl < 8; kl += 2) {
        const int k = 8 * kb + kl;
        float *cb = cbuf + ((kl >> 1) & 1) * 2 * kB;  // columns k, k+1
        float *rb = rbuf + ((kl >> 1) & 1) * 2 * kB;  // rows k, k+1
        if (tc == kb) {
#pragma unroll
            for (int i = 0; i < 8; ++i) {
                cb[8 * tr + i] = a[i][kl];
                cb[kB + 8 * tr + i] = a[i][kl + 1];
            }
        }
        if (tr == kb) {
#pragma unroll
            for (int j = 0; j < 8; ++j) {
                rb[8 * tc + j] = a[kl][j];
                rb[kB + 8 * tc + j] = a[kl + 1][j];
            }
        }
        __syncthreads();
        // ---- pivot k
        const float akk = rb[k];
        const float p = 1.0f / akk;
        if (tid == 0 && !(isfinite(p) && akk != 0.f)) ok = false;
        float L[8], U[8], C1[8], R1[8];
#pragma unroll
        for (int i = 0; i < 8; ++i) L[i] = cb[8 * tr + i];
#pragma unroll
        for (int j = 0; j < 8; ++j) U[j] = rb[8 * tc + j] * p;
        if (tc == kb) U[kl] = p;
        if (tr == kb) L[kl] = akk - 1.f;
        // column k+1 (own rows) and row k+1 (own columns) after pivot k
        const float uk1 = rb[k + 1] * p;  // U at column k+1
        const float lk1 = rb[kB + k];     // L at row k+1: a_{k+1,k}
#pragma unroll
        for (int i = 0; i < 8; ++i) C1[i] = fmaf(-L[i], uk1, cb[kB + 8 * tr + i]);
#pragma unroll
        for (int j = 0; j < 8; ++j) {
            const float r0 = rb[kB + 8 * tc + j];
            R1[j] = (tc == kb && j == kl) ? -lk1 * U[j] : fmaf(-lk1, U[j], r0);
        }
        const float ak1 = fmaf(-lk1, uk1, rb[kB + k + 1]);  // a_{k+1,k+1} after pivot k
#pragma unroll
        for (int i = 0; i < 8; ++i) {
#pragma unroll
            for (int j = 0; j < 8; ++j) {
                if (j == kl)
                    a[i][j] = (tc == kb) ? -L[i] * U[j] : fmaf(-L[i], U[j], a[i][j]);
                else
                    a[i][j] = fmaf(-L[i], U[j], a[i][j]);
            }
        }
        if (tr == kb && tc == kb) a[kl][kl] += 1.f;
        // ---- pivot k+1
        const float p2 = 1.0f / ak1;
        if (tid == 0 && !(isfinite(p2) && ak1 != 0.f)) ok = false;
#pragma unroll
        for (int j = 0; j < 8; ++j) U[j] = R1[j] * p2;
        if (tc == kb) U[kl + 1] = p2;
#pragma unroll
        for (int i = 0; i < 8; ++i) L[i] = C1[i];
        if (tr == kb) L[kl + 1] = ak1 - 1.f;
#pragma unroll
        for (int i = 0; i < 8; ++i) {
#pragma unroll
            for (int j = 0; j < 8; ++j) {
                if (j == kl + 1)
                    a[i][j] = (tc == kb) ? -L[i] * U[j] : fmaf(-L[i], U[j], a[i][j]);
                else
                    a[i][j] = fmaf(-L[i], U[j], a[i][j]);
            }
        }
        if (tr == kb && tc == kb) a[kl + 1][kl + 1] += 1.f;
    }
    __syncthreads();
#pragma unroll
    for (int i = 0; i < 8; ++i)
#pragma unroll
        for (int j = 0; j < 8; ++j) Sp[(8 * tr + i) * kSp + 8 * tc + j] = a[i][j];
    return ok;
}

// The A part of the L-tile epilogue's chunk E (S's columns 32E..32E+31, held
// by the threads of half E / 2) as TF32 hi and lo parts into the chunk's stage.
template <int E>
__device__ __forceinline__ void write_a(unsigned char *sm, int g, int row, int half,
                                        const float (&v)[64]) {
    if (half != (E >> 1)) return;
    unsigned char *dst = sm + (size_t)((g + E) % kStages) * kStageBytes;
    constexpr int c0 = 32 * (E & 1);
#pragma unroll
    for (int q = 0; q < 8; ++q) {
        float hi[4], lo[4];
#pragma unroll
        for (int w = 0; w < 4; ++w) {
            const float x = v[c0 + 4 * q + w];
            hi[w] = coop::tc::to_tf32(x);
            lo[w] = coop::tc::to_tf32(x - hi[w]);
        }
        const uint32_t o = poff(row, 4 * q);
        *reinterpret_cast<float4 *>(dst + o) = make_float4(hi[0], hi[1], hi[2], hi[3]);
        *reinterpret_cast<float4 *>(dst + 16384 + o) = make_float4(lo[0], lo[1], lo[2], lo[3]);
    }
}

// The B part of chunk E from registers: the threads holding rows 32E..32E+31
// of B (row = k) write their 64 columns (n = 64 half + t) as TF32 hi and lo
// parts.
template <int E>
__device__ __forceinline__ void write_b(unsigned char *sm, int g, int row, int half,
                                        const float (&v)[64]) {
    if ((row >> 5) != E) return;
    unsigned char *dst = sm + (size_t)((g + E) % kStages) * kStageBytes + 32768;
    const int k = row & 31;
#pragma unroll
    for (int t = 0; t < 64; ++t) {
        const float x = v[t];
        const float hi = coop::tc::to_tf32(x);
        const uint32_t o = poff(64 * half + t, k);
        *reinterpret_cast<float *>(dst + o) = hi;
        *reinterpret_cast<float *>(dst + 16384 + o) = coop::tc::to_tf32(x - hi);
    }
}

// The tensor cores' product of two 128 x 128 tiles into TMEM columns
// tmem..tmem+127 through four 32-wide K chunks of the ring (the fourth reuses
// the first one's stage once its MMAs are done).  A: each thread's row-half
// va (row `row`, columns 64 half..), written chunk by chunk.  B: copied from
// the operand slot bslot (kSlot; after its flag when `flag` is not null), or
// written from each thread's row-half vb (row = k).  Returns with every MMA
// complete; g and naccb advance.
template <bool kSlot>
__device__ __forceinline__ void ring_mma4(const Args &a, unsigned char *sm, uint32_t ring,
                                          uint64_t *full, uint64_t *empty, uint64_t *accb,
                                          int &g, int &naccb, uint32_t tmem, int row, int half,
                                          const float (&va)[64], const float (&vb)[64],
                                          const unsigned char *bslot, const int *flag) {
    const int tid = threadIdx.x;
    const uint32_t bbytes = kSlot ? 32768u : 0u;
    for (int e = 0; e < kStages; ++e) {
        const int gc = g + e;
        if (gc >= kStages && !bulk::wait(&empty[gc % kStages], ((gc - kStages) / kStages) & 1))
            gave_up(a.flags);
    }
    if (kSlot && tid == 0) {
        if (flag && !wait_flag(flag, a.epoch, a.flags)) gave_up(a.flags);
        fence_async_global();
        for (int e = 0; e < kStages; ++e) {
            const int s = (g + e) % kStages;
            unsigned char *dst = sm + (size_t)s * kStageBytes;
            bulk::arrive_expect_tx(&full[s], bbytes);
            bulk::g2s(dst + 32768, bslot + e * kChunkBytes, kChunkBytes, &full[s]);
            bulk::g2s(dst + 49152, bslot + kPartBytes + e * kChunkBytes, kChunkBytes, &full[s]);
        }
    }
    write_a<0>(sm, g, row, half, va);
    write_a<1>(sm, g, row, half, va);
    write_a<2>(sm, g, row, half, va);
    if (!kSlot) {
        write_b<0>(sm, g, row, half, vb);
        write_b<1>(sm, g, row, half, vb);
        write_b<2>(sm, g, row, half, vb);
    }
    fence_async_shared();
    coop::tc::fence_before();
    __syncthreads();
    if (tid == 0) {
        for (int e = 0; e < kStages; ++e) {
            const int gc = g + e, s = gc % kStages;
            if (kSlot) {
                if (!bulk::wait(&full[s], (gc / kStages) & 1)) gave_up(a.flags);
            } else {
                bulk::arrive(&full[s]);  // keeps the stage's phase count
                if (!bulk::wait(&full[s], (gc / kStages) & 1)) gave_up(a.flags);
            }
            coop::tc::fence_after();
            mma_chunk(tmem, ring + s * kStageBytes, e == 0);
            coop::tc::commit(bulk::smem_u32(&empty[s]));
        }
    }
    // chunk 3 reuses chunk 0's stage once its MMAs are done
    {
        const int gc = g + 3, s = gc % kStages;
        if (!bulk::wait(&empty[s], ((gc - kStages) / kStages) & 1)) gave_up(a.flags);
        if (kSlot && tid == 0) {
            unsigned char *dst = sm + (size_t)s * kStageBytes;
            bulk::arrive_expect_tx(&full[s], bbytes);
            bulk::g2s(dst + 32768, bslot + 3 * kChunkBytes, kChunkBytes, &full[s]);
            bulk::g2s(dst + 49152, bslot + kPartBytes + 3 * kChunkBytes, kChunkBytes, &full[s]);
        }
        write_a<3>(sm, g, row, half, va);
        if (!kSlot) write_b<3>(sm, g, row, half, vb);
        fence_async_shared();
        __syncthreads();
        if (tid == 0) {
            if (!kSlot) bulk::arrive(&full[s]);
            if (!bulk::wait(&full[s], (gc / kStages) & 1)) gave_up(a.flags);
            coop::tc::fence_after();
            mma_chunk(tmem, ring + s * kStageBytes, false);
            coop::tc::commit(bulk::smem_u32(&empty[s]));
            coop::tc::commit(bulk::smem_u32(accb));
        }
    }
    g += 4;
    if (!bulk::wait(accb, naccb & 1)) gave_up(a.flags);
    ++naccb;
    coop::tc::fence_after();
}

__global__ void __launch_bounds__(kThreads, 1) k_blu32(Args a) {
    extern __shared__ __align__(1024) unsigned char sm[];
    uint64_t *full = reinterpret_cast<uint64_t *>(sm + kBarOff);
    uint64_t *empty = full + kStages;
    uint64_t *accb = empty + kStages;
    uint32_t *tslot = reinterpret_cast<uint32_t *>(sm + kBarOff + 128);
    int *task_s = reinterpret_cast<int *>(sm + kBarOff + 192);
    float *Sp = reinterpret_cast<float *>(sm);
    float *cbuf = Sp + kB * kSp;
    float *rbuf = cbuf + 4 * kB;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int n = a.n, T = a.T;
    const uint32_t ring = bulk::smem_u32(sm);

    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], 256;" ::"r"(
                         bulk::smem_u32(tslot))
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    if (tid == 0) {
        for (int s = 0; s < kStages; ++s) {
            bulk::init(&full[s], 1);
            bulk::init(&empty[s], 1);
        }
        bulk::init(accb, 1);
        bulk::fence_init();
    }
    coop::tc::fence_before();
    __syncthreads();
    coop::tc::fence_after();
    const uint32_t tmem = *tslot;
    const uint32_t lane_base = (uint32_t)(32 * (warp & 3)) << 16;
    const int row = 32 * (warp & 3) + lane, half = warp >> 2;

    int g = 0;       // chunks filled so far (ring position), same in every thread
    int naccb = 0;   // completions of accb so far
    for (;;) {
        fence_async_shared();
        __syncthreads();
        if (tid == 0) {
            const int t = atomicAdd(a.ticket, 1);
            *task_s = (t < T * T && !ld_acq(&a.flags[kFlagBarrierTimeout])) ? a.tasks[t] : -1;
        }
        __syncthreads();
        const int task = *task_s;
        if (task < 0) break;
        const int i = task >> 16, j = task & 0xffff, m = min(i, j);
        // the tile's entries of A, loaded while the accumulation runs
        float av[64];
        {
            const int gr = i * kB + row;
#pragma unroll
            for (int t = 0; t < 64; ++t) {
                const int gc = j * kB + 64 * half + t;
                av[t] = (gr < n && gc < n) ? a.A[(size_t)gr + (size_t)gc * n] : (gr == gc ? 1.f : 0.f);
            }
        }
        // ------------------------------------------------ accumulation over k < m
        if (m > 0) {
            if (warp == 0) {
                if (lane == 0) {
                    const int total = 4 * m;
                    auto fill = [&](int c) {
                        const int gc = g + c, s = gc % kStages;
                        if (gc >= kStages && !bulk::wait(&empty[s], ((gc - kStages) / kStages) & 1))
                            gave_up(a.flags);
                        const int k = c >> 2, q = c & 3;
                        if (q == 0) {
                            if (!wait_flag(&a.ready[i * T + k], a.epoch, a.flags)) gave_up(a.flags);
                            if (!wait_flag(&a.ready[k * T + j], a.epoch, a.flags)) gave_up(a.flags);
                            fence_async_global();
                        }
                        const unsigned char *L = a.op + (size_t)(i * T + k) * kSlotBytes + q * kChunkBytes;
                        const unsigned char *U = a.op + (size_t)(k * T + j) * kSlotBytes + q * kChunkBytes;
                        unsigned char *dst = sm + (size_t)s * kStageBytes;
                        bulk::arrive_expect_tx(&full[s], kStageBytes);
                        bulk::g2s(dst, L, kChunkBytes, &full[s]);
                        bulk::g2s(dst + 16384, L + kPartBytes, kChunkBytes, &full[s]);
                        bulk::g2s(dst + 32768, U, kChunkBytes, &full[s]);
                        bulk::g2s(dst + 49152, U + kPartBytes, kChunkBytes, &full[s]);
                    };
                    fill(0);
                    if (total > 1) fill(1);
                    for (int c = 0; c < total; ++c) {
                        const int gc = g + c, s = gc % kStages;
                        if (!bulk::wait(&full[s], (gc / kStages) & 1)) gave_up(a.flags);
                        coop::tc::fence_after();
                        mma_chunk(tmem, ring + s * kStageBytes, c == 0);
                        coop::tc::commit(bulk::smem_u32(&empty[s]));
                        if (c + 2 < total) fill(c + 2);
                    }
                    coop::tc::commit(bulk::smem_u32(accb));
                }
                __syncwarp();
            }
            g += 4 * m;
            if (!bulk::wait(accb, naccb & 1)) gave_up(a.flags);
            ++naccb;
            coop::tc::fence_after();
        }
        // ------------------------------------------------ S = A_ij - acc (rows `row`, half `half`)
        float v[64];
        if (m > 0) {
            ld64(tmem + lane_base + 64 * half, v);
        } else {
#pragma unroll
            for (int t = 0; t < 64; ++t) v[t] = 0.f;
        }
#pragma unroll
        for (int t = 0; t < 64; ++t) v[t] = av[t] - v[t];
        unsigned char *slot = a.op + (size_t)(i * T + j) * kSlotBytes;
        if (i < j) {
            // U_ij = S
#pragma unroll
            for (int t = 0; t < 64; ++t) Sp[row * kSp + 64 * half + t] = v[t];
            __syncthreads();
            store_tile(a, Sp, i, j, true, slot);
        } else if (i == j) {
#pragma unroll
            for (int t = 0; t < 64; ++t) Sp[row * kSp + 64 * half + t] = v[t];
            __syncthreads();
            const bool ok = gauss_jordan(Sp, cbuf, rbuf);
            if (tid == 0 && !ok) atomicOr(&a.flags[kFlagSingular], 1);
            __syncthreads();
            // One Newton-Schulz step D' = D + D (I - S D), both products on
            // the tensor cores: Gauss-Jordan without pivoting loses accuracy on
            // ill-conditioned tiles (close pairs), and the step brings D to the
            // accuracy of the products.  Measured on stiff N=4096 Jacobians:
            // the refinement's first residual 1e-1 -> 5e-5, and solves that
            // stagnated or diverged converge in 3 to 4 sweeps.
            float dv[64];
            float ssum = 0.f, dsum = 0.f;
#pragma unroll
            for (int t = 0; t < 64; ++t) {
                dv[t] = Sp[row * kSp + 64 * half + t];
                ssum += fabsf(v[t]);
                dsum += fabsf(dv[t]);
            }
            bool refine = a.refine == 1;
            if (a.refine == 2) {
                // ||S||_inf ||D||_inf: the two halves of each row, then the
                // largest row (the GJ buffers are free now)
                cbuf[128 * half + row] = ssum;
                rbuf[128 * half + row] = dsum;
                __syncthreads();
                float sm_ = 0.f, dm_ = 0.f;
                for (int r = lane; r < kB; r += 32) {
                    sm_ = fmaxf(sm_, cbuf[r] + cbuf[128 + r]);
                    dm_ = fmaxf(dm_, rbuf[r] + rbuf[128 + r]);
                }
                for (int o = 16; o > 0; o >>= 1) {
                    sm_ = fmaxf(sm_, __shfl_xor_sync(0xffffffffu, sm_, o));
                    dm_ = fmaxf(dm_, __shfl_xor_sync(0xffffffffu, dm_, o));
                }
                // every warp computed the same maxima; a non-finite estimate
                // refines too
                refine = !(sm_ * dm_ <= kRefineKappa);
            }
            store_tile(a, Sp, i, j, true, slot);  // D as the B operand of S D
            if (refine) {
            fence_async_global();
            fence_async_shared();
            __syncthreads();
            ring_mma4<true>(a, sm, ring, full, empty, accb, g, naccb, tmem + 128, row, half, v, v,
                            slot, nullptr);
            ld64(tmem + lane_base + 128 + 64 * half, v);  // S D
#pragma unroll
            for (int t = 0; t < 64; ++t) v[t] = (row == 64 * half + t ? 1.f : 0.f) - v[t];
            coop::tc::fence_before();
            __syncthreads();
            coop::tc::fence_after();
            ring_mma4<false>(a, sm, ring, full, empty, accb, g, naccb, tmem + 128, row, half, dv,
                             v, nullptr, nullptr);
            ld64(tmem + lane_base + 128 + 64 * half, v);  // D (I - S D)
#pragma unroll
            for (int t = 0; t < 64; ++t) Sp[row * kSp + 64 * half + t] = dv[t] + v[t];
            __syncthreads();
            store_tile(a, Sp, i, j, true, slot);
            }
        } else {
            // L_ij = S D_j: four K chunks, A part (S as hi/lo) written by the
            // threads holding those columns, B part (D_j) copied from its slot
            const unsigned char *D = a.op + (size_t)(j * T + j) * kSlotBytes;
            for (int e = 0; e < kStages; ++e) {
                const int gc = g + e;
                if (gc >= kStages && !bulk::wait(&empty[gc % kStages], ((gc - kStages) / kStages) & 1))
                    gave_up(a.flags);
            }
            if (tid == 0) {
                if (!wait_flag(&a.ready[j * T + j], a.epoch, a.flags)) gave_up(a.flags);
                fence_async_global();
                for (int e = 0; e < kStages; ++e) {
                    const int s = (g + e) % kStages;
                    unsigned char *dst = sm + (size_t)s * kStageBytes;
                    bulk::arrive_expect_tx(&full[s], 32768);
                    bulk::g2s(dst + 32768, D + e * kChunkBytes, kChunkBytes, &full[s]);
                    bulk::g2s(dst + 49152, D + kPartBytes + e * kChunkBytes, kChunkBytes, &full[s]);
                }
            }
            write_a<0>(sm, g, row, half, v);
            write_a<1>(sm, g, row, half, v);
            write_a<2>(sm, g, row, half, v);
            fence_async_shared();
            __syncthreads();
            if (tid == 0) {
                for (int e = 0; e < kStages; ++e) {
                    const int gc = g + e, s = gc % kStages;
                    if (!bulk::wait(&full[s], (gc / kStages) & 1)) gave_up(a.flags);
                    coop::tc::fence_after();
                    mma_chunk(tmem + 128, ring + s * kStageBytes, e == 0);
                    coop::tc::commit(bulk::smem_u32(&empty[s]));
                }
            }
            // chunk 3 reuses chunk 0's stage once its MMAs are done
            {
                const int gc = g + 3, s = gc % kStages;
                if (!bulk::wait(&empty[s], ((gc - kStages) / kStages) & 1)) gave_up(a.flags);
                if (tid == 0) {
                    unsigned char *dst = sm + (size_t)s * kStageBytes;
                    bulk::arrive_expect_tx(&full[s], 32768);
                    bulk::g2s(dst + 32768, D + 3 * kChunkBytes, kChunkBytes, &full[s]);
                    bulk::g2s(dst + 49152, D + kPartBytes + 3 * kChunkBytes, kChunkBytes, &full[s]);
                }
                write_a<3>(sm, g, row, half, v);
                fence_async_shared();
                __syncthreads();
                if (tid == 0) {
                    if (!bulk::wait(&full[s], (gc / kStages) & 1)) gave_up(a.flags);
                    coop::tc::fence_after();
                    mma_chunk(tmem + 128, ring + s * kStageBytes, false);
                    coop::tc::commit(bulk::smem_u32(&empty[s]));
                    coop::tc::commit(bulk::smem_u32(accb));
                }
            }
            g += 4;
            if (!bulk::wait(accb, naccb & 1)) gave_up(a.flags);
            ++naccb;
            coop::tc::fence_after();
            ld64(tmem + lane_base + 128 + 64 * half, v);
            // the ring's stages 0-2 may be read by no MMA now: every MMA of this
            // tile is complete (accb), so the plain tile may overwrite them
#pragma unroll
            for (int t = 0; t < 64; ++t) Sp[row * kSp + 64 * half + t] = v[t];
            __syncthreads();
            store_tile(a, Sp, i, j, false, slot);
        }
        // publish the tile, then its plain entries (Sp stays intact until the
        // next task's barrier)
        fence_async_global();
        __threadfence();
        __syncthreads();
        if (tid == 0) st_rel(&a.ready[i * T + j], a.epoch);
        store_plain(a, Sp, i, j);
    }
    coop::tc::fence_before();
    __syncthreads();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, 256;" ::"r"(tmem)
                     : "memory");
}

// ---------------------------------------------------------------------------
// Block triangular solves with the factors in LU (FP32): forward
// y_i = b_i - sum_{k<i} L_ik y_k, then backward x_i = D_i (y_i - sum_{j>i} U_ij x_j),
// one CTA per 128-row block, blocks taken from a ticket counter in the order
// of the dependency chain (forward: i = 0, 1, ...; backward: i = T-1, ...), so
// no CTA waits for one that has not started.  Thread t keeps rows 2(t%64),
// 2(t%64)+1 and columns 32(t/64).. of each tile; the next tile's slice is
// loaded before the wait for the values it multiplies.
//
// Hand-off: a finished block publishes its 128 values as 64-bit words
// (epoch << 32) | float bits, one relaxed store each, with no fence and no
// separate flag.  A waiting warp polls the 32 words its column group needs
// (lane l word l, 256 B per warp) until every lane sees this launch's epoch,
// then spreads the values by shuffle: one L2 round trip per hand-off.
struct SolveArgs {
    int n, T;
    const float *LU;
    const double *b;   // right-hand side (n)
    unsigned long long *yt, *xt;  // T*128 each: tagged forward and backward values
    float *x;          // T*128: the solution
    int *ticket;       // ticket counter (0 at the launch; the CTA taking the last ticket resets it)
    int epoch;
    int *flags;        // kFlagBarrierTimeout
    const int *perm;   // rows of P (the block LU factorised P A); null: identity
    const unsigned long long *conv;  // refinement: max|g|, then max|r| after each sweep
    int it;            // refinement sweep of this solve
};

__device__ __forceinline__ unsigned long long ld_relaxed_u64(const unsigned long long *p) {
    unsigned long long v;
    asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ void st_tagged(unsigned long long *p, float v, int epoch) {
    const unsigned long long t =
        ((unsigned long long)(unsigned)epoch << 32) | (unsigned long long)__float_as_uint(v);
    asm volatile("st.relaxed.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(t) : "memory");
}

// Warp-wide: lane l's value of the tagged word p[l] once all 32 words carry
// `epoch` (bounded: after kSpin polls the wait records the timeout and the
// values are used as they are).
__device__ __forceinline__ float ld_tagged(const unsigned long long *p, int epoch, int *flags) {
    const int lane = threadIdx.x & 31;
    long long spins = 0;
    for (;;) {
        const unsigned long long t = ld_relaxed_u64(p + lane);
        if (__all_sync(0xffffffffu, (unsigned)(t >> 32) == (unsigned)epoch))
            return __uint_as_float((unsigned)t);
        __nanosleep(32);
        if (++spins > kSpin) {
            if (lane == 0) gave_up(flags);
            return __uint_as_float((unsigned)t);
        }
    }
}

__device__ __forceinline__ void load_slice(const SolveArgs &s, int ti, int tj, int r2, int cg,
                                           float2 (&w)[32]) {
    const int n = s.n;
    const int gr = ti * kB + 2 * r2;
#pragma unroll
    for (int cc = 0; cc < 32; ++cc) {
        const int gc = tj * kB + 32 * cg + cc;
        float2 t = make_float2(0.f, 0.f);
        if (gc < n && gr < n) t = *reinterpret_cast<const float2 *>(s.LU + (size_t)gr + (size_t)gc * n);
        w[cc] = t;
    }
}

// One row block of the forward (kFwd) or backward pass.
template <bool kFwd>
__device__ __forceinline__ void solve_block(const SolveArgs &s, int i, float (*red)[kB],
                                            float *zs) {
    const int tid = threadIdx.x, r2 = tid & 63, cg = tid >> 6;
    const int T = s.T;
    const unsigned long long *src = kFwd ? s.yt : s.xt;  // values of the other blocks
    float acc0 = 0.f, acc1 = 0.f;
    float2 w[32];
    const int k_first = kFwd ? 0 : T - 1, k_step = kFwd ? 1 : -1;
    const int count = kFwd ? i : T - 1 - i;
    for (int q = 0; q < count; ++q) {
        const int k = k_first + q * k_step;
        load_slice(s, i, k, r2, cg, w);
        // the warp's 32 values of block k (its column group), by shuffle
        const float mine = ld_tagged(src + k * kB + 32 * cg, s.epoch, s.flags);
#pragma unroll
        for (int cc = 0; cc < 32; ++cc) {
            const float yy = __shfl_sync(0xffffffffu, mine, cc);
            acc0 = fmaf(w[cc].x, yy, acc0);
            acc1 = fmaf(w[cc].y, yy, acc1);
        }
    }
    float base = 0.f;
    if (!kFwd) {
        load_slice(s, i, i, r2, cg, w);  // D_i, before the reduction
        // y_i comes from the forward pass of this launch
        if (tid < kB) base = ld_tagged(s.yt + i * kB + (tid & ~31), s.epoch, s.flags);
    }
    red[cg][2 * r2] = acc0;
    red[cg][2 * r2 + 1] = acc1;
    __syncthreads();
    if (tid < kB) {
        const int gr = i * kB + tid;
        if (kFwd) base = gr < s.n ? (float)s.b[s.perm ? s.perm[gr] : gr] : 0.f;
        const float z = base - ((red[0][tid] + red[1][tid]) + (red[2][tid] + red[3][tid]));
        if (kFwd)
            st_tagged(s.yt + gr, z, s.epoch);
        else
            zs[tid] = z;
    }
    if (!kFwd) {
        __syncthreads();
        acc0 = acc1 = 0.f;
#pragma unroll
        for (int cc = 0; cc < 32; ++cc) {
            const float zz = zs[32 * cg + cc];
            acc0 = fmaf(w[cc].x, zz, acc0);
            acc1 = fmaf(w[cc].y, zz, acc1);
        }
        __syncthreads();
        red[cg][2 * r2] = acc0;
        red[cg][2 * r2 + 1] = acc1;
        __syncthreads();
        if (tid < kB) {
            const float xv = (red[0][tid] + red[1][tid]) + (red[2][tid] + red[3][tid]);
            s.x[i * kB + tid] = xv;
            st_tagged(s.xt + i * kB + tid, xv, s.epoch);
        }
    }
}

// Both passes in one launch of 2T CTAs: tickets 0..T-1 are the forward pass's
// blocks 0..T-1, tickets T..2T-1 the backward pass's blocks T-1..0, so every
// wait (forward: lower blocks; backward: higher blocks and its own forward
// block) is on a lower ticket, held by a CTA that is already running.
__global__ void __launch_bounds__(kThreads) k_bsolve32(SolveArgs s) {
    __shared__ int tk_s;
    __shared__ float red[4][kB];
    __shared__ float zs[kB];
    const int T = s.T;
    if (threadIdx.x == 0) {
        const int t = atomicAdd(&s.ticket[0], 1);
        if (t == 2 * T - 1) atomicExch(&s.ticket[0], 0);  // the last ticket: ready for the next launch
        tk_s = t;
    }
    __syncthreads();
    const int t = tk_s;
    if (s.it > 0) {
        // the previous refinement sweep already met its tolerance: nothing to do
        const double g = __longlong_as_double((long long)__ldcg(s.conv));
        const double r = __longlong_as_double((long long)__ldcg(s.conv + s.it));
        if (r <= kIrStop * g) return;
    }
    if (t < T)
        solve_block<true>(s, t, red, zs);
    else if (t < 2 * T)
        solve_block<false>(s, 2 * T - 1 - t, red, zs);
}

// Self-test of the bounded waits: the cooperative LU's grid barrier with a CTA
// that never arrives (which = 0), and the block LU's tile-flag wait on a flag
// that nothing sets (which = 1).  Both give up after their normal poll limits
// and record kFlagBarrierTimeout.
__global__ void k_wait_selftest(int which, unsigned *bar, int *flags, int *flag) {
    __shared__ int dead_s;
    if (threadIdx.x == 0) dead_s = 0;
    __syncthreads();
    if (which == 0) {
        if (blockIdx.x != 0) return;  // the CTA that never arrives
        unsigned gen = 0;
        coop::grid_barrier(bar, flags, gen, &dead_s);
    } else if (threadIdx.x == 0) {
        wait_flag(flag, 1, flags);
    }
}

}  // namespace blu

// ---------------------------------------------------------------------------
// Host side.

int blu_tiles(int n) { return (n + blu::kB - 1) / blu::kB; }

size_t blu_op_bytes(int n) {
    const size_t T = (size_t)blu_tiles(n);
    return T * T * blu::kSlotBytes;
}

// The schedule: ring m = min(i, j) ascending; in a ring the diagonal tile, then
// (m+d, m) and (m, m+d) for d = 1, 2, ...
std::vector<int> blu_schedule(int n) {
    const int T = blu_tiles(n);
    std::vector<int> t;
    t.reserve((size_t)T * T);
    for (int m = 0; m < T; ++m) {
        t.push_back((m << 16) | m);
        for (int d = 1; m + d < T; ++d) {
            t.push_back(((m + d) << 16) | m);
            t.push_back((m << 16) | (m + d));
        }
    }
    return t;
}

void blu_alloc(BluBufs &B, int n, const int *tasks, BluState *state) {
    const int T = blu_tiles(n);
    D4_CUDA_OK(d4::dmalloc((void **)&B.op, blu_op_bytes(n)));
    D4_CUDA_OK(d4::dmalloc((void **)&B.ticket, sizeof(int) * 4));
    D4_CUDA_OK(d4::dmalloc((void **)&B.ready, sizeof(int) * (size_t)T * T));
    D4_CUDA_OK(d4::dmalloc((void **)&B.yt, sizeof(unsigned long long) * (size_t)T * blu::kB));
    D4_CUDA_OK(d4::dmalloc((void **)&B.xt, sizeof(unsigned long long) * (size_t)T * blu::kB));
    D4_CUDA_OK(d4::dmalloc((void **)&B.xs, sizeof(float) * (size_t)T * blu::kB));
    // ticket[0]: the factorisation's (zeroed before each launch); ticket[1]: the
    // solves' (zero here, then reset by the CTA that takes a launch's last one)
    D4_CUDA_OK(cudaMemset(B.ticket, 0, sizeof(int) * 4));
    D4_CUDA_OK(cudaMemset(B.ready, 0, sizeof(int) * (size_t)T * T));
    // tag 0 never matches a launch's epoch (>= 1)
    D4_CUDA_OK(cudaMemset(B.yt, 0, sizeof(unsigned long long) * (size_t)T * blu::kB));
    D4_CUDA_OK(cudaMemset(B.xt, 0, sizeof(unsigned long long) * (size_t)T * blu::kB));
    D4_CUDA_OK(cudaMemset(B.xs, 0, sizeof(float) * (size_t)T * blu::kB));
    B.tasks = tasks;
    B.state = state;
}

void blu_free(BluBufs &B) {
    void *p[] = {B.op, B.ticket, B.ready, B.yt, B.xt, B.xs};
    for (void *q : p)
        if (q) cudaFree(q);
    B = BluBufs();
}

static bool g_blu_attr = false;

void blu_factor_async(const BluBufs &B, int n, const float *A, float *LU, int *flags, int grid,
                      cudaStream_t st) {
    if (!g_blu_attr) {
        D4_CUDA_OK(cudaFuncSetAttribute(blu::k_blu32, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        (int)blu::kSmemBytes));
        g_blu_attr = true;
    }
    const int T = blu_tiles(n);
    blu::Args a;
    a.n = n;
    a.T = T;
    a.A = A;
    a.LU = LU;
    a.op = B.op;
    a.tasks = B.tasks;
    a.ticket = B.ticket;
    a.ready = B.ready;
    a.epoch = ++B.state->lu_epoch;
    a.flags = flags;
    a.refine = 2;
    D4_CUDA_OK(cudaMemsetAsync(B.ticket, 0, sizeof(int), st));
    const int g = std::max(1, std::min(grid, T * T));
    blu::k_blu32<<<g, blu::kThreads, blu::kSmemBytes, st>>>(a);
    check_launch("k_blu32");
}

void blu_solve_async(const BluBufs &B, int n, const float *LU, const double *b, const int *perm,
                     const unsigned long long *conv, int it, int *flags, cudaStream_t st) {
    const int T = blu_tiles(n);
    blu::SolveArgs s;
    s.n = n;
    s.T = T;
    s.LU = LU;
    s.b = b;
    s.yt = B.yt;
    s.xt = B.xt;
    s.x = B.xs;
    s.ticket = B.ticket + 1;
    s.epoch = ++B.state->solve_epoch;
    s.flags = flags;
    s.perm = perm;
    s.conv = conv;
    s.it = it;
    blu::k_bsolve32<<<2 * T, blu::kThreads, 0, st>>>(s);
    check_launch("k_bsolve32");
}

int wait_selftest(int which) {
    unsigned *bar = nullptr;
    int *flags = nullptr;
    D4_CUDA_OK(dmalloc(&bar, sizeof(unsigned) * 64));
    D4_CUDA_OK(dmalloc(&flags, sizeof(int) * (kFlagCount + 1)));
    D4_CUDA_OK(cudaMemset(bar, 0, sizeof(unsigned) * 64));
    D4_CUDA_OK(cudaMemset(flags, 0, sizeof(int) * (kFlagCount + 1)));
    blu::k_wait_selftest<<<which == 0 ? 2 : 1, 32>>>(which, bar, flags, flags + kFlagCount);
    check_launch("k_wait_selftest");
    int h[kFlagCount];
    const cudaError_t e = cudaMemcpy(h, flags, sizeof(h), cudaMemcpyDeviceToHost);
    cudaFree(bar);
    cudaFree(flags);
    D4_CUDA_OK(e);
    return h[kFlagBarrierTimeout] ? D4_ERR_STATE : D4_OK;
}

}  // namespace d4
