// d4_sparse.cu: the distant-pair cutoff path, the cutoff-sparse Jacobian solved
// by Jacobi-preconditioned restarted GMRES in FP64.
//
// Under the cutoff (src/simulation.cpp:461-478) the Jacobian keeps only pairs
// closer than the cutoff range (Heaviside, or the Gaussian tail out to 7 cutoff
// radii), about pi r^2 N entries per row, and the reference hands it to UMFPACK
// as a CSC matrix (src/simulation.cpp:635-659).  Here the matrix is still
// assembled densely by the pair kernels, so the row sums d_i and the row
// scaling keep the reference's order, and is then compressed to CSR:
//   k_csr_count  nonzeros per (row, 256-column chunk), one thread per row and chunk
//   k_csr_rows   per-row chunk offsets and the row-pointer scan (one CTA)
//   k_csr_fill   column indices and values in ascending column order
// Every solve of the step then runs GMRES(40) with right Jacobi preconditioning,
// classical Gram-Schmidt with one reorthogonalisation and Givens rotations, to a
// relative residual of 1e-13, as one cooperative kernel: each CTA owns a
// contiguous range of rows, the SpMV is one warp per row (fixed lane split and
// butterfly, so results do not depend on timing), and each reduction goes
// through per-CTA partials (double-buffered) and a bounded grid barrier, three
// barriers per Krylov vector.  A solve that does not converge within the restart
// budget is reported to the host, which redoes it with the dense LU.
#include <algorithm>
#include <cstdint>

#include "d4_internal.h"
#include "d4_trsv.cuh"

namespace d4 {
namespace sp {

constexpr int kM = 40;            // Krylov dimension per restart
constexpr int kRestarts = 6;
constexpr int kThreads = 256;
constexpr int kWarps = kThreads / 32;
constexpr int kStride = kM + 2;   // partials per CTA
constexpr int kChunk = 256;       // columns per counting chunk
constexpr int kGenWord = 32;
constexpr long long kSpinLimit = 1ll << 24;  // polls of >= 64 ns: > 1 s
constexpr double kTol = 1e-13;

struct GmresArgs {
    int n;
    const int *rp, *ci;
    const double *val, *dinv;
    const double *g;  // right-hand side
    double *x;        // solution (starts at 0)
    double *V;        // (kM + 1) x n Krylov basis
    double *z;        // n: preconditioned vector fed to the SpMV
    double *w;        // n scratch
    double *part;     // 2 x G x kStride partial sums
    unsigned *bar;    // barrier words
    int *flags;       // [0] barrier timeout, [1] not converged, [2] iterations
};

__device__ __forceinline__ unsigned ld_acq(const unsigned *p) {
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

// Generation barrier over all CTAs.  The wait gives up after kSpinLimit polls
// (or when another CTA gave up), sets flags[0] and marks the CTA dead, after
// which it no longer waits; the host turns flags[0] into an error.
__device__ void grid_barrier(unsigned *bar, int *flags, unsigned &gen, int *dead) {
    __syncthreads();
    if (threadIdx.x == 0) {
        const unsigned target = gen + 1;
        __threadfence();
        if (atomicAdd(bar, 1u) + 1 == gridDim.x) {
            atomicExch(bar, 0u);
            __threadfence();
            atomicExch(bar + kGenWord, target);
        } else if (!*dead) {
            long long spins = 0;
            while (ld_acq(bar + kGenWord) != target) {
                __nanosleep(64);
                if ((++spins & 255) == 0 &&
                    (spins > kSpinLimit || ld_acq((const unsigned *)&flags[0]))) {
                    atomicOr(&flags[0], 1);
                    *dead = 1;
                    break;
                }
            }
        }
        gen = target;
    }
    __syncthreads();
}

// dst[i] = scale * sum_q val[q] * src[ci[q]] for the CTA's rows, one warp per row.
__device__ __forceinline__ void spmv_rows(const GmresArgs &a, int r0, int r1, const double *src,
                                          double scale, double *dst) {
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    for (int i = r0 + wid; i < r1; i += kWarps) {
        const int q0 = a.rp[i], q1 = a.rp[i + 1];
        double s = 0;
        for (int q = q0 + lane; q < q1; q += 32) s += a.val[q] * __ldcg(src + a.ci[q]);
        for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
        if (lane == 0) dst[i] = s * scale;
    }
    __syncthreads();
}

__global__ void __launch_bounds__(kThreads, 1) k_gmres(GmresArgs a) {
    __shared__ double red[kWarps][kStride];
    __shared__ double H[kM + 1][kM];
    __shared__ double tot[kStride], cs[kM], sn[kM], s[kM + 1], y[kM];
    __shared__ int dead, stop;
    const int n = a.n, tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
    const int rows_per = (n + gridDim.x - 1) / gridDim.x;
    const int r0 = min(n, (int)blockIdx.x * rows_per), r1 = min(n, r0 + rows_per);
    unsigned gen = 0;
    int parity = 0;
    if (tid == 0) {
        dead = 0;
        stop = 0;
    }
    __syncthreads();
    double loc[kStride];
    // Sum over all rows of loc[0..cnt) into tot[0..cnt): warp shuffles, per-warp
    // rows in shared memory, one partial per CTA, grid barrier, then every CTA
    // adds the partials in CTA order (identical totals everywhere).
    auto reduce = [&](int cnt) {
        double *P = a.part + (size_t)parity * gridDim.x * kStride;
        for (int k = 0; k < cnt; ++k) {
            double v = loc[k];
            for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
            if (lane == 0) red[wid][k] = v;
        }
        __syncthreads();
        for (int k = tid; k < cnt; k += kThreads) {
            double v = 0;
            for (int q = 0; q < kWarps; ++q) v += red[q][k];
            P[blockIdx.x * kStride + k] = v;
        }
        grid_barrier(a.bar, a.flags, gen, &dead);
        for (int k = tid; k < cnt; k += kThreads) {
            double v = 0;
            for (int b = 0; b < (int)gridDim.x; ++b) v += __ldcg(P + b * kStride + k);
            tot[k] = v;
        }
        __syncthreads();
        parity ^= 1;
    };
    const int i = r0 + tid;  // the thread's row (rows_per <= kThreads)
    const bool own = i < r1;
    loc[0] = own ? a.g[i] * a.g[i] : 0;
    reduce(1);
    const double gnorm = sqrt(tot[0]);
    int iters = 0;
    bool converged = !(gnorm > 0);
    for (int cycle = 0; cycle < kRestarts && !converged && !dead; ++cycle) {
        // r = g - A x -> V_0, beta = ||r||
        spmv_rows(a, r0, r1, a.x, 1.0, a.w);
        double r = 0;
        if (own) {
            r = a.g[i] - a.w[i];
            a.V[i] = r;
        }
        loc[0] = r * r;
        reduce(1);
        const double beta = sqrt(tot[0]);
        if (!(beta > kTol * gnorm)) {
            converged = true;
            break;
        }
        if (own) {
            a.V[i] = r / beta;
            a.z[i] = a.dinv[i] * (r / beta);
        }
        if (tid == 0) {
            for (int k = 0; k <= kM; ++k) s[k] = 0;
            s[0] = beta;
        }
        grid_barrier(a.bar, a.flags, gen, &dead);
        double zscale = 1.0;  // z holds zscale * M^-1 V_j
        int jdone = 0;
        for (int j = 0; j < kM; ++j) {
            // w = A M^-1 V_j; first Gram-Schmidt pass
            spmv_rows(a, r0, r1, a.z, 1.0 / zscale, a.w);
            double w = own ? a.w[i] : 0;
            for (int k = 0; k <= j; ++k) loc[k] = own ? w * a.V[(size_t)k * n + i] : 0;
            reduce(j + 1);
            double hsum[kM];
            for (int k = 0; k <= j; ++k) hsum[k] = tot[k];
            if (own)
                for (int k = 0; k <= j; ++k) w -= tot[k] * a.V[(size_t)k * n + i];
            // reorthogonalisation
            for (int k = 0; k <= j; ++k) loc[k] = own ? w * a.V[(size_t)k * n + i] : 0;
            reduce(j + 1);
            if (own)
                for (int k = 0; k <= j; ++k) w -= tot[k] * a.V[(size_t)k * n + i];
            for (int k = 0; k <= j; ++k) hsum[k] += tot[k];
            // ||w|| and the next (unnormalised) preconditioned vector share a barrier
            if (own) a.z[i] = a.dinv[i] * w;
            loc[0] = w * w;
            reduce(1);
            const double nrm = sqrt(tot[0]);
            zscale = nrm > 0 ? nrm : 1.0;
            if (own) a.V[(size_t)(j + 1) * n + i] = nrm > 0 ? w / nrm : 0;
            if (tid == 0) {
                for (int k = 0; k <= j; ++k) H[k][j] = hsum[k];
                for (int k = 0; k < j; ++k) {
                    const double t = cs[k] * H[k][j] + sn[k] * H[k + 1][j];
                    H[k + 1][j] = -sn[k] * H[k][j] + cs[k] * H[k + 1][j];
                    H[k][j] = t;
                }
                const double d = sqrt(H[j][j] * H[j][j] + nrm * nrm);
                cs[j] = d > 0 ? H[j][j] / d : 1;
                sn[j] = d > 0 ? nrm / d : 0;
                H[j][j] = d;
                s[j + 1] = -sn[j] * s[j];
                s[j] = cs[j] * s[j];
                stop = (!(fabs(s[j + 1]) > kTol * gnorm) || !(nrm > 0)) ? 1 : 0;
            }
            __syncthreads();
            ++iters;
            jdone = j + 1;
            if (stop || dead) break;
        }
        converged = stop != 0;
        // y = H^-1 s (upper triangular); x += M^-1 V y
        if (tid == 0) {
            for (int k = jdone - 1; k >= 0; --k) {
                double t = s[k];
                for (int q = k + 1; q < jdone; ++q) t -= H[k][q] * y[q];
                y[k] = H[k][k] != 0 ? t / H[k][k] : 0;
            }
        }
        __syncthreads();
        if (own) {
            double u = 0;
            for (int k = 0; k < jdone; ++k) u += y[k] * a.V[(size_t)k * n + i];
            a.x[i] += a.dinv[i] * u;
        }
        grid_barrier(a.bar, a.flags, gen, &dead);
        if (tid == 0) stop = 0;
        __syncthreads();
    }
    if (blockIdx.x == 0 && tid == 0) {
        if (!converged || dead) atomicOr(&a.flags[1], 1);
        a.flags[2] = iters;
    }
}

// Nonzeros of row i in column chunk blockIdx.y (column-major matrix).
template <typename T>
__global__ void k_csr_count(int n, const T *__restrict__ A, int *cnt) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int ch = blockIdx.y;
    if (i >= n) return;
    const int j0 = ch * kChunk, j1 = min(n, j0 + kChunk);
    int c = 0;
    for (int j = j0; j < j1; ++j) c += A[(size_t)i + (size_t)j * n] != T(0);
    cnt[(size_t)ch * n + i] = c;
}

// Per-row chunk offsets off[ch][i] and the row pointer rp[0..n] (one CTA of 1024).
__global__ void __launch_bounds__(1024) k_csr_rows(int n, int nch, const int *cnt, int *off,
                                                   int *rp) {
    __shared__ int part[1024];
    const int tid = threadIdx.x;
    const int per = (n + 1023) / 1024;
    const int b0 = min(n, tid * per), b1 = min(n, b0 + per);
    int sum = 0;
    for (int i = b0; i < b1; ++i) {
        int run = 0;
        for (int ch = 0; ch < nch; ++ch) {
            off[(size_t)ch * n + i] = run;
            run += cnt[(size_t)ch * n + i];
        }
        rp[i] = run;  // row total for now
        sum += run;
    }
    part[tid] = sum;
    __syncthreads();
    for (int o = 1; o < 1024; o <<= 1) {
        const int v = tid >= o ? part[tid - o] : 0;
        __syncthreads();
        part[tid] += v;
        __syncthreads();
    }
    int run = part[tid] - sum;
    for (int i = b0; i < b1; ++i) {
        const int t = rp[i];
        rp[i] = run;
        run += t;
    }
    if (tid == 1023) rp[n] = part[1023];
}

template <typename T>
__global__ void k_csr_fill(int n, const T *__restrict__ A, const int *off, const int *rp, int *ci,
                           double *val, double *dinv) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int ch = blockIdx.y;
    if (i >= n) return;
    const int j0 = ch * kChunk, j1 = min(n, j0 + kChunk);
    int q = rp[i] + off[(size_t)ch * n + i];
    for (int j = j0; j < j1; ++j) {
        const T v = A[(size_t)i + (size_t)j * n];
        if (v != T(0)) {
            ci[q] = j;
            val[q] = (double)v;
            ++q;
        }
    }
    if (i >= j0 && i < j1) {
        const double d = (double)A[(size_t)i + (size_t)i * n];
        dinv[i] = d != 0 ? 1 / d : 1.0;
    }
}

__global__ void k_rhs(int n, trsv::GArgs ga, double *g, double *x) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    g[i] = trsv::g_of(ga, i);
    x[i] = 0;
}

__global__ void k_apply(int n, const double *x, const double *base, double *out, double *dx) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    dx[i] = x[i];
    if (out) out[i] = base[i] - x[i];
}

inline int nb(int n, int t) { return (n + t - 1) / t; }

}  // namespace sp

bool gmres_selected(const Ctx &c) {
    if (c.p.solver == D4_SOLVER_GMRES) return true;
    if (c.p.solver == D4_SOLVER_AUTO) return c.range_sq * c.cutoff_sq < 0.1;
    return false;
}

void sparse_alloc(Ctx &c) {
    const int n = c.n;
    int dev = 0, sms = 0;
    D4_CUDA_OK(cudaGetDevice(&dev));
    D4_CUDA_OK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    // about 128 rows per CTA (one row per thread at most): fewer CTAs, cheaper barriers
    c.sp_grid = std::max(1, std::min(sms, sp::nb(n, 128)));
    if (sp::nb(n, c.sp_grid) > sp::kThreads) throw StateError("n too large for the GMRES grid");
    c.sp_nch = sp::nb(n, sp::kChunk);
    auto ialloc = [](int **p, size_t k) { D4_CUDA_OK(d4::dmalloc((void **)p, sizeof(int) * k)); };
    auto dalloc = [](double **p, size_t k) {
        D4_CUDA_OK(d4::dmalloc((void **)p, sizeof(double) * k));
    };
    ialloc(&c.sp_cnt, (size_t)c.sp_nch * n);
    ialloc(&c.sp_off, (size_t)c.sp_nch * n);
    ialloc(&c.sp_rp, (size_t)n + 1);
    ialloc(&c.sp_flags, 4);
    D4_CUDA_OK(d4::dmalloc((void **)&c.sp_bar, sizeof(unsigned) * 64));
    dalloc(&c.sp_dinv, n);
    dalloc(&c.sp_V, (size_t)(sp::kM + 1) * n);
    dalloc(&c.sp_z, n);
    dalloc(&c.sp_w, n);
    dalloc(&c.sp_g, n);
    dalloc(&c.sp_x, n);
    dalloc(&c.sp_part, (size_t)2 * c.sp_grid * sp::kStride);
    // initial CSR capacity: 64 entries per row, grown on demand
    c.sp_cap = 64 * n;
    ialloc(&c.sp_ci, (size_t)c.sp_cap);
    dalloc(&c.sp_val, (size_t)c.sp_cap);
}

void sparse_free(Ctx &c) {
    void *bufs[] = {c.sp_cnt, c.sp_off, c.sp_rp, c.sp_flags, c.sp_bar, c.sp_dinv, c.sp_V,
                    c.sp_z, c.sp_w, c.sp_g, c.sp_x, c.sp_part, c.sp_ci, c.sp_val};
    for (void *b : bufs)
        if (b) cudaFree(b);
}

// CSR of the current matrix (the FP64 A of either form).  Reads the entry
// count back to size the index and value arrays (one host sync).
void sparse_prepare(Ctx &c) {
    const int n = c.n;
    const dim3 grid(sp::nb(n, 128), c.sp_nch);
    sp::k_csr_count<double><<<grid, 128, 0, c.stream>>>(n, c.A, c.sp_cnt);
    check_launch("k_csr_count");
    sp::k_csr_rows<<<1, 1024, 0, c.stream>>>(n, c.sp_nch, c.sp_cnt, c.sp_off, c.sp_rp);
    check_launch("k_csr_rows");
    D4_CUDA_OK(cudaMemcpyAsync(c.h_flags, c.sp_rp + n, sizeof(int), cudaMemcpyDeviceToHost,
                               c.stream));
    D4_CUDA_OK(cudaStreamSynchronize(c.stream));
    const int nnz = c.h_flags[0];
    if (nnz > c.sp_cap) {
        D4_CUDA_OK(cudaFree(c.sp_ci));
        D4_CUDA_OK(cudaFree(c.sp_val));
        c.sp_ci = nullptr;
        c.sp_val = nullptr;
        c.sp_cap = nnz + nnz / 4 + 1024;
        D4_CUDA_OK(d4::dmalloc((void **)&c.sp_ci, sizeof(int) * (size_t)c.sp_cap));
        D4_CUDA_OK(d4::dmalloc((void **)&c.sp_val, sizeof(double) * (size_t)c.sp_cap));
    }
    c.sp_nnz = nnz;
    sp::k_csr_fill<double><<<grid, 128, 0, c.stream>>>(n, c.A, c.sp_off, c.sp_rp, c.sp_ci,
                                                       c.sp_val, c.sp_dinv);
    check_launch("k_csr_fill");
    c.sp_dense_ready = 0;
}

// One solve of the step by GMRES: g of the stage, x = A^-1 g, out = base - x.
// Returns false when GMRES did not converge (nothing written to out).
bool sparse_solve_update(Ctx &c, int gmode, double hval, const double *s_end,
                         const double *s_init, const double *x_new, const double *x_old,
                         const double *base, double *out) {
    const int n = c.n;
    trsv::GArgs ga{};
    ga.gmode = gmode;
    ga.hval = hval;
    ga.dvec = c.dvec;
    ga.s_end = s_end;
    ga.s_init = s_init;
    ga.x_new = x_new;
    ga.x_old = x_old;
    sp::k_rhs<<<sp::nb(n, 256), 256, 0, c.stream>>>(n, ga, c.sp_g, c.sp_x);
    check_launch("k_rhs");
    D4_CUDA_OK(cudaMemsetAsync(c.sp_bar, 0, sizeof(unsigned) * 64, c.stream));
    D4_CUDA_OK(cudaMemsetAsync(c.sp_flags, 0, sizeof(int) * 4, c.stream));
    sp::GmresArgs a;
    a.n = n;
    a.rp = c.sp_rp;
    a.ci = c.sp_ci;
    a.val = c.sp_val;
    a.dinv = c.sp_dinv;
    a.g = c.sp_g;
    a.x = c.sp_x;
    a.V = c.sp_V;
    a.z = c.sp_z;
    a.w = c.sp_w;
    a.part = c.sp_part;
    a.bar = c.sp_bar;
    a.flags = c.sp_flags;
    void *args[] = {(void *)&a};
    D4_CUDA_OK(cudaLaunchCooperativeKernel((const void *)sp::k_gmres, dim3(c.sp_grid),
                                           dim3(sp::kThreads), args, 0, c.stream));
    check_launch("k_gmres");
    D4_CUDA_OK(cudaMemcpyAsync(c.h_flags, c.sp_flags, sizeof(int) * 4, cudaMemcpyDeviceToHost,
                               c.stream));
    D4_CUDA_OK(cudaStreamSynchronize(c.stream));
    if (c.h_flags[0]) throw StateError("GMRES grid barrier timed out");
    c.sp_solves += 1;
    c.sp_iters += c.h_flags[2];
    if (c.h_flags[1]) {
        c.sp_fallbacks += 1;
        return false;
    }
    sp::k_apply<<<sp::nb(n, 256), 256, 0, c.stream>>>(n, c.sp_x, base, out, c.dx);
    check_launch("k_apply");
    return true;
}

}  // namespace d4
