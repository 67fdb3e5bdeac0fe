// d4_mixed.cu: the mixed-precision form of the implicit step.
//
// The speeds, the Jacobian A = I + D J, the residuals g, the position updates
// and the error ratio are the FP64 form's (its exact-order sweeps, d4_fp64.cu):
// the quantities that decide where the dislocations go stay FP64.  What runs
// in lower precision is the linear algebra that dominates the step: A is
// rounded to FP32 and factorised by the block LU on the tensor cores
// (d4_blu32.cu, 3xTF32 products; or the pivoted cooperative LU), and each
// solve is refined in FP64 against the FP64 matrix:
//     dx = 0, r = g;  repeat: c = LU32^-1 r (FP32);  dx += c;  r = g - A dx (FP64)
// until max|r| <= kIrStop max|g| (checked on the device: later sweeps return
// at once) or kIrMax sweeps.  The refined dx is the solution of A dx = g to
// that residual, so positions follow the FP64 form's Newton iterations.  A
// Jacobian taken from the FP32 field instead (about 1e-6 relative) moved
// positions 1.7e-8 from the FP64 form within 10 steps at N=4096 and 1e-6
// within 20: the two-iteration scheme of src/simulation.cpp:100-150 passes the
// matrix's error on to the positions, so the matrix the residual multiplies
// must be the FP64 one.
//
// Static pivoting: the block LU factorises P A, with P the row permutation of
// the context's last pivoted (exact partial pivoting) factorisation, identity
// until one ran; an attempt whose block factorisation fails (a bad pivot in a
// diagonal tile, or a residual left above kRefineLimit) is redone with the
// pivoted LU, whose permutation the next block LUs then use.
#include <cstdint>
#include <utility>

#include "d4_field64.cuh"
#include "d4_lu_coop.cuh"
#include "d4_trsv.cuh"

namespace d4 {
namespace {

// FP64 matrix -> FP32, rows gathered through perm (null: identity):
// A32[r + c n] = A[perm[r] + c n].
__global__ void k_to32(int n, const double *__restrict__ A, const int *__restrict__ perm,
                       float *__restrict__ A32) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    const int c = blockIdx.y;
    if (r >= n) return;
    const int src = perm ? perm[r] : r;
    A32[(size_t)r + (size_t)c * n] = (float)A[(size_t)src + (size_t)c * n];
}

__device__ __forceinline__ unsigned long long obits(double v) {
    return (unsigned long long)__double_as_longlong(v);  // ordered for v >= 0
}

// max of two non-negative values where a NaN wins (fmax would drop it): a NaN
// residual must fail the convergence and fallback checks.
__device__ __forceinline__ double nanmax(double a, double b) { return (b > a || b != b) ? b : a; }

// max over the block of v (>= 0 or NaN) into *out by atomicMax on the bit
// pattern (a NaN's bits exceed every finite value's).
__device__ void block_absmax(double v, unsigned long long *out) {
    __shared__ double wm[8];
    for (int o = 16; o > 0; o >>= 1) v = nanmax(v, __shfl_down_sync(0xffffffffu, v, o));
    if ((threadIdx.x & 31) == 0) wm[threadIdx.x >> 5] = v;
    __syncthreads();
    if (threadIdx.x == 0) {
        double m = 0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) m = nanmax(m, wm[w]);
        atomicMax(out, obits(fabs(m)));
    }
}

// g of the stage (as the FP64 form), r = g, dx = 0, max|g| into conv[0]
// (conv zeroed before the launch).
__global__ void __launch_bounds__(256) k_ir_init(int n, trsv::GArgs ga, double *g, double *r,
                                                 double *dx, unsigned long long *conv) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    double a = 0;
    if (i < n) {
        const double gi = trsv::g_of(ga, i);
        g[i] = gi;
        r[i] = gi;
        dx[i] = 0;
        a = fabs(gi);
    }
    block_absmax(a, conv);
}

__device__ __forceinline__ bool converged(const unsigned long long *conv, int done) {
    // after `done` sweeps (done >= 1): max|r| of the last one against max|g|
    if (done < 1) return false;
    const double g = __longlong_as_double((long long)__ldcg(conv));
    const double r = __longlong_as_double((long long)__ldcg(conv + done));
    return r <= kIrStop * g;
}

// One refinement sweep's update in one launch: dx_out = dx + c and
// r = g - A dx_out with the FP64 matrix.  Block (x, y) multiplies rows 256x..
// by column chunk y (FP64, column order, the chunk's corrected dx staged in
// shared memory; the blocks of row block 0 also store it to dx_out, a buffer
// no block reads) into part[y][i]; the last block of each row block to finish
// (a counter per row block, reset by that block) subtracts the chunk sums from
// g in chunk order and adds its rows' max|r| to conv[it + 1].  The order of
// every sum is fixed, so the residual is the same on every run.  When the
// previous sweep already converged the launch only carries dx over.
__global__ void __launch_bounds__(256) k_resid_fused(int n, const double *__restrict__ A,
                                                     const double *__restrict__ dx,
                                                     const float *__restrict__ corr,
                                                     double *dx_out, const double *g,
                                                     double *part, int chunk, int nch,
                                                     unsigned *cnt, double *r,
                                                     unsigned long long *conv, int it) {
    __shared__ double sdx[256];
    __shared__ int last;
    const int c0 = blockIdx.y * chunk, c1 = min(n, c0 + chunk);
    if (converged(conv, it)) {
        if (blockIdx.x == 0)
            for (int t = threadIdx.x; t < c1 - c0; t += blockDim.x) dx_out[c0 + t] = dx[c0 + t];
        if (blockIdx.x == 0 && blockIdx.y == 0 && threadIdx.x == 0)
            atomicMax(conv + it + 1, __ldcg(conv + it));
        return;
    }
    for (int t = threadIdx.x; t < c1 - c0; t += blockDim.x) {
        const double v = dx[c0 + t] + (double)corr[c0 + t];
        sdx[t] = v;
        if (blockIdx.x == 0) dx_out[c0 + t] = v;
    }
    __syncthreads();
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) {
        // four interleaved sums (column c into sum c % 4), combined in a fixed
        // order: independent FMA chains, and 16 loads issued together
        const double *Ai = A + (size_t)i + (size_t)c0 * n;
        const int w = c1 - c0;
        double s0 = 0, s1 = 0, s2 = 0, s3 = 0;
        int c = 0;
        for (; c + 16 <= w; c += 16) {
            double av[16];
#pragma unroll
            for (int u = 0; u < 16; ++u) av[u] = __ldg(Ai + (size_t)(c + u) * n);
#pragma unroll
            for (int u = 0; u < 16; u += 4) {
                s0 += av[u] * sdx[c + u];
                s1 += av[u + 1] * sdx[c + u + 1];
                s2 += av[u + 2] * sdx[c + u + 2];
                s3 += av[u + 3] * sdx[c + u + 3];
            }
        }
        for (; c < w; ++c) {
            const double v = __ldg(Ai + (size_t)c * n) * sdx[c];
            const int m = c & 3;
            if (m == 0)
                s0 += v;
            else if (m == 1)
                s1 += v;
            else if (m == 2)
                s2 += v;
            else
                s3 += v;
        }
        part[(size_t)blockIdx.y * n + i] = (s0 + s1) + (s2 + s3);
    }
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) last = atomicAdd(&cnt[blockIdx.x], 1u) == (unsigned)(nch - 1);
    __syncthreads();
    if (!last) return;
    __threadfence();
    double a = 0;
    if (i < n) {
        double v = g[i];
        for (int q = 0; q < nch; ++q) v = v - __ldcg(part + (size_t)q * n + i);
        r[i] = v;
        a = fabs(v);
    }
    if (threadIdx.x == 0) cnt[blockIdx.x] = 0;
    block_absmax(a, conv + it + 1);
}

// max |r| and max |g| into out[0], out[1] (as ordered bits of non-negatives).
__global__ void k_absmax2(int n, const double *r, const double *g, unsigned long long *out) {
    double m1 = 0, m2 = 0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        m1 = nanmax(m1, fabs(r[i]));
        m2 = nanmax(m2, fabs(g[i]));
    }
    for (int o = 16; o > 0; o >>= 1) {
        m1 = nanmax(m1, __shfl_down_sync(0xffffffffu, m1, o));
        m2 = nanmax(m2, __shfl_down_sync(0xffffffffu, m2, o));
    }
    if ((threadIdx.x & 31) == 0) {
        atomicMax(out, obits(fabs(m1)));
        atomicMax(out + 1, obits(fabs(m2)));
    }
}

// dx -> out = base - dx, with the singular-matrix fix of src/simulation.cpp:646-658.
__global__ void k_ir_apply(int n, const double *dx, const int *flags, const double *base,
                           double *out, double *dx_out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double d = dx[i];
    if (flags[kFlagSingular] && !((-1 < d) && (d < 1))) d = 0;
    if (dx_out) dx_out[i] = d;
    out[i] = base[i] - d;
}

inline int nb(long long n, int t) { return (int)((n + t - 1) / t); }

}  // namespace

Mix32Bufs primary_mix32(Ctx &c) {
    Mix32Bufs B;
    B.A64 = c.A;
    B.A32 = c.A32;
    B.LU32 = c.LU32;
    B.P0 = c.lu32_p0;
    B.Q = c.lu32_q;
    B.mask = c.lu_mask;
    B.bar = c.lu_bar;
    B.flags = c.flags;
    B.perm = c.perm;
    B.piv = c.piv;
    B.g = c.m_g;
    B.r = c.m_r;
    B.dx = c.m_dx;
    B.dx2 = c.m_dx2;
    B.cnt = c.m_cnt;
    B.conv = c.m_conv;
    B.part = c.m_part;
    B.c32 = c.m_c32;
    B.w1 = c.m_w1;
    B.resid = c.m_resid;
    B.resid_count = &c.m_resid_count;
    B.blu = c.blu;
    B.blk = &c.m_blk;
    return B;
}

// Factorisation of the FP64 matrix A (column-major n x n) into B: with
// copy_matrix, A is first copied into B.A64 (stage I's own FP64 matrix, which
// its refinement multiplies while stage II rescales A) and `after_copy` (may
// be null) is recorded once that copy is taken.  The block LU factorises the
// FP32 rounding of P A (P: the static pivots c.spiv); the pivoted cooperative
// LU that of A.  Queued on `st` without waiting.
void factor32_async(Ctx &c, const Mix32Bufs &B, const double *A, bool copy_matrix, int grid,
                    cudaStream_t st, cudaEvent_t after_copy) {
    const int n = c.n;
    const size_t nn = (size_t)n * n;
    const double *src = A;
    if (copy_matrix) {
        D4_CUDA_OK(cudaMemcpyAsync(B.A64, A, sizeof(double) * nn, cudaMemcpyDeviceToDevice, st));
        src = B.A64;
    }
    if (after_copy) D4_CUDA_OK(cudaEventRecord(after_copy, st));
    D4_CUDA_OK(cudaMemsetAsync(B.flags, 0, sizeof(int) * kFlagCount, st));
    *B.blk = c.m_fast;
    if (c.m_fast) {
        // block LU (d4_blu32.cu) of the row-permuted FP32 matrix
        k_to32<<<dim3(nb(n, 256), n), 256, 0, st>>>(n, src, c.spiv, B.A32);
        check_launch("k_to32");
        blu_factor_async(B.blu, n, B.A32, B.LU32, B.flags, grid, st);
        ++c.m_blocklu;
        return;
    }
    k_to32<<<dim3(nb(n, 256), n), 256, 0, st>>>(n, src, nullptr, B.LU32);
    check_launch("k_to32");
    D4_CUDA_OK(cudaMemsetAsync(B.bar, 0, sizeof(unsigned) * 64, st));
    D4_CUDA_OK(cudaMemsetAsync(B.mask, 0, sizeof(unsigned) * c.lu_mask_words, st));
    coop::CoopArgs<float> a;
    a.n = n;
    a.A = B.LU32;
    a.P0 = B.P0;
    a.Q = B.Q;
    a.mask = B.mask;
    a.piv = B.piv;
    a.flags = B.flags;
    a.bar = B.bar;
    a.perm = B.perm;
    a.sched = nullptr;  // the FP32 form has no look-ahead
    a.dg = nullptr;
    void *args[] = {(void *)&a};
    const void *kern = (const void *)coop::k_lu_coop<float>;
    D4_CUDA_OK(cudaLaunchCooperativeKernel(kern, dim3(grid), dim3(coop::kThreads), args,
                                           coop::kRowBufBytes<float>(), st));
    check_launch("k_lu_coop<float>");
}

// After a pivoted factorisation into the primary buffers: its row permutation
// becomes the block LU's static pivots.
void adopt_pivots(Ctx &c) {
    D4_CUDA_OK(cudaMemcpyAsync(c.spiv, c.perm, sizeof(int) * c.n, cudaMemcpyDeviceToDevice,
                               c.stream));
}

int factor32(Ctx &c) {
    factor32_async(c, primary_mix32(c), c.A, false, c.lu32_grid, c.stream, nullptr);
    D4_CUDA_OK(cudaMemcpyAsync(c.h_flags, c.flags, sizeof(int) * kFlagCount,
                               cudaMemcpyDeviceToHost, c.stream));
    D4_CUDA_OK(cudaStreamSynchronize(c.stream));
    if (c.h_flags[kFlagBarrierTimeout]) throw StateError("LU grid barrier timed out");
    if (c.m_blk && c.h_flags[kFlagSingular]) {
        // a diagonal tile met a zero or non-finite pivot: the pivoted LU instead
        ++c.m_fallbacks;
        c.m_fast = 0;
        try {
            factor32_async(c, primary_mix32(c), c.A, false, c.lu32_grid, c.stream, nullptr);
        } catch (...) {
            c.m_fast = 1;
            throw;
        }
        c.m_fast = 1;
        adopt_pivots(c);
        D4_CUDA_OK(cudaMemcpyAsync(c.h_flags, c.flags, sizeof(int) * kFlagCount,
                                   cudaMemcpyDeviceToHost, c.stream));
        D4_CUDA_OK(cudaStreamSynchronize(c.stream));
        if (c.h_flags[kFlagBarrierTimeout]) throw StateError("LU grid barrier timed out");
    }
    count_lu(c, c.h_flags);
    c.factor_singular = c.h_flags[kFlagSingular] != 0;
    c.factor_pivoted = 0;
    return c.factor_singular ? D4_WARN_SINGULAR : D4_OK;
}

int coop_grid_size32(int n) {
    int dev = 0, sms = 0, per_sm = 0;
    D4_CUDA_OK(cudaGetDevice(&dev));
    D4_CUDA_OK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    D4_CUDA_OK(cudaFuncSetAttribute(coop::k_lu_coop<float>,
                                    cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (int)coop::kRowBufBytes<float>()));
    D4_CUDA_OK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(
        &per_sm, coop::k_lu_coop<float>, coop::kThreads, coop::kRowBufBytes<float>()));
    const int g = sms * (per_sm < 1 ? 1 : per_sm);
    return g < (n + coop::kThreads - 1) / coop::kThreads ? -1 : g;
}

// FP32 solve with B's factors: LU32^-1 r (r FP64 in, result FP32), by the
// block solves of the block LU (rows of r through the static pivots), or by
// the cluster solve of the pivoted LU.  Sweep `it` of the refinement: the
// block solve returns at once when sweep it - 1 converged.  Returns the
// result's buffer.
static const float *solve32_once(Ctx &c, const Mix32Bufs &B, cudaStream_t st, const double *r,
                                 int it) {
    if (*B.blk) {
        blu_solve_async(B.blu, c.n, B.LU32, r, c.spiv, B.conv, it, B.flags, st);
        return B.blu.xs;
    }
    trsv::GArgs g{};
    g.gmode = -1;
    g.g_in = r;
    trsv::launch_cluster_solve<float>(c.n, B.LU32, B.perm, B.flags, g, B.w1, B.c32, c.wave_err,
                                      st);
    return B.c32;
}

// The refinement sweeps (k_ir_init has set dx = 0, r = g, conv[0] = max|g|):
// c = LU32^-1 r, dx += c, r = g - A dx, until converged or kIrMax sweeps; dx
// alternates between B.dx and B.dx2, and a converged sweep only carries it
// over, so after kIrMax launches the buffer is known on the host.  Returns it.
static const double *refine(Ctx &c, const Mix32Bufs &B, cudaStream_t st) {
    const int n = c.n, chunk = 256;
    double *dxa = B.dx, *dxb = B.dx2;
    for (int it = 0; it < kIrMax; ++it) {
        const float *corr = solve32_once(c, B, st, B.r, it);
        k_resid_fused<<<dim3(nb(n, 256), nb(n, chunk)), 256, 0, st>>>(
            n, B.A64, dxa, corr, dxb, B.g, B.part, chunk, nb(n, chunk), B.cnt, B.r, B.conv, it);
        check_launch("k_resid_fused");
        std::swap(dxa, dxb);
    }
    return dxa;
}

static void ir_start(Ctx &c, const Mix32Bufs &B, cudaStream_t st, const trsv::GArgs &ga) {
    const int n = c.n;
    D4_CUDA_OK(cudaMemsetAsync(B.conv, 0, sizeof(unsigned long long) * (kIrMax + 1), st));
    k_ir_init<<<nb(n, 256), 256, 0, st>>>(n, ga, B.g, B.r, B.dx, B.conv);
    check_launch("k_ir_init");
}

void solve_update32_with(Ctx &c, const Mix32Bufs &B, const double *dvec, double *dx_out,
                         cudaStream_t st, int gmode, double hval, const double *s_end,
                         const double *s_init, const double *x_new, const double *x_old,
                         const double *base, double *out) {
    const int n = c.n;
    trsv::GArgs ga{};
    ga.gmode = gmode;
    ga.hval = hval;
    ga.dvec = dvec;
    ga.s_end = s_end;
    ga.s_init = s_init;
    ga.x_new = x_new;
    ga.x_old = x_old;
    ir_start(c, B, st, ga);
    const double *dx = refine(c, B, st);
    k_absmax2<<<64, 256, 0, st>>>(n, B.r, B.g, B.resid + 2 * *B.resid_count);
    check_launch("k_absmax2");
    *B.resid_count = (*B.resid_count + 1) % 8;
    k_ir_apply<<<nb(n, 256), 256, 0, st>>>(n, dx, B.flags, base, out, dx_out);
    check_launch("k_ir_apply");
}

void solve_plain32(Ctx &c, const double *g) {
    const int n = c.n;
    Mix32Bufs B = primary_mix32(c);
    trsv::GArgs ga{};
    ga.gmode = -1;
    ga.g_in = g;
    ir_start(c, B, c.stream, ga);
    const double *dx = refine(c, B, c.stream);
    k_absmax2<<<64, 256, 0, c.stream>>>(n, B.r, B.g, B.resid + 2 * *B.resid_count);
    check_launch("k_absmax2");
    *B.resid_count = (*B.resid_count + 1) % 8;
    D4_CUDA_OK(cudaMemcpyAsync(c.dx, dx, sizeof(double) * n, cudaMemcpyDeviceToDevice,
                               c.stream));
}

void solve_update32(Ctx &c, int gmode, double hval, const double *s_end, const double *s_init,
                    const double *x_new, const double *x_old, const double *base, double *out) {
    solve_update32_with(c, primary_mix32(c), c.dvec, c.dx, c.stream, gmode, hval, s_end, s_init,
                        x_new, x_old, base, out);
}

}  // namespace d4
