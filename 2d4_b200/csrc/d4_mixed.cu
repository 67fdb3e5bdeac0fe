// d4_mixed.cu: the mixed-precision form of the implicit step.
//
// Pair stress gradient in FP32 (d4_field32.cuh: compensated image sums,
// cancellation-free central image), each unique pair once per sweep, summed
// into FP64 accumulators.  The pair stress itself, whose sums are the speeds
// that enter the Newton residual g, is the FP64 field: speeds from the FP32
// field (about 1e-6 relative) moved positions by 1.9e-8 from the FP64 form
// within 8 steps at N=4096, while the gradient only shapes the matrix, whose
// error the refined solves remove.  The dense Jacobian A = I + D J is kept in FP32 and
// factorised in FP32 (the cooperative LU of d4_lu_coop.cuh).  FP64 is kept for
// positions, speeds, residuals g, d_i, the position updates and the error ratio;
// each solve is refined in FP64 against the stored FP32 matrix:
//     dx = 0, r = g;  repeat: c = LU32 \ r;  dx += c;  r = g - A32 dx
// so the solution of A32 dx = g is accurate to FP64 rounding times cond(A).
#include <cstdint>
#include <utility>

#include "d4_field32.cuh"
#include "d4_field64.cuh"
#include "d4_lu_coop.cuh"
#include "d4_trsv.cuh"

namespace d4 {
namespace {

__device__ __forceinline__ double bsign(int i, int n) { return i < n / 2 ? 1.0 : -1.0; }

__device__ __forceinline__ void tol_min(double *tol, int idx, double d) {
    atomicMin(reinterpret_cast<unsigned long long *>(tol + idx),
              static_cast<unsigned long long>(__double_as_longlong(d)));
}

__device__ __forceinline__ void tile_of(int t, int T, int &ti, int &tj) {
    int r = 0, rem = t;
    while (rem >= T - r) {
        rem -= T - r;
        ++r;
    }
    ti = r;
    tj = r + rem;
}

struct Pair32Args {
    int n;
    const double *x, *y;
    double *vacc;    // FP64 sum of signed forces per dislocation (k_rowsum32)
    double *subacc;  // FP64 sum of -J_ij per row (k_rowsum32; fused sweep)
    double *part;    // 4 x T x n tile partials: [0] forces as row i, [1] as row j,
                     // [2] -J as row i, [3] -J as row j (slot = the other tile index)
    float *A;        // raw J entries (fused sweep)
    double *tol;
    double min_prec_sq, h, cut_sq, cutoff, range_sq, one_per_cut_sq;
    int heaviside;
};

// Unique pairs in 32x32 tiles (upper triangle); lanes walk i, threadIdx.y
// steps j.  Row sums over the tile's j go through shared memory, column sums
// over i through warp shuffles; each tile stores one partial per row it
// touches (no atomics), and k_rowsum32 adds them in tile order, so the sums
// are the same on every run.
template <bool kJac>
__global__ void __launch_bounds__(256) k_pairs32(Pair32Args a) {
    const int T = (a.n + 31) / 32;
    int ti, tj;
    tile_of(blockIdx.x, T, ti, tj);
    __shared__ double sxi[32], syi[32], sxj[32], syj[32];
    __shared__ double rs[8][33], rj[8][33];
    __shared__ float sv[kJac ? 32 : 1][kJac ? 33 : 1];
    const int tx = threadIdx.x, ty = threadIdx.y;
    const int i0 = ti * 32, j0 = tj * 32;
    if (ty == 0) {
        const int i = i0 + tx, j = j0 + tx;
        sxi[tx] = i < a.n ? a.x[i] : 0;
        syi[tx] = i < a.n ? a.y[i] : 0;
        sxj[tx] = j < a.n ? a.x[j] : 0;
        syj[tx] = j < a.n ? a.y[j] : 0;
    }
    __syncthreads();
    const int i = i0 + tx;
    const double bi = bsign(i, a.n);
    double row_f = 0, row_j = 0, row_min = 1e300;
    for (int lj = ty; lj < 32; lj += 8) {
        const int j = j0 + lj;
        double f = 0, fj = 0;
        float v = 0.f;
        const bool ok = i < a.n && j < a.n && i < j;
        if (ok) {
            const double dx = f64::normalize(sxi[tx] - sxj[lj]);
            const double dy = f64::normalize(syi[tx] - syj[lj]);
            const double dist_sq = dx * dx + dy * dy;
            if (a.tol && dist_sq < a.min_prec_sq) {
                row_min = fmin(row_min, dist_sq);
                tol_min(a.tol, j, dist_sq);
            }
            // the force enters the Newton residual: FP64 field (an FP32 force,
            // ~1e-6 relative, moved positions by ~1e-8 within a few steps)
            const double bj = bsign(j, a.n);
            f = f64::xy(dx, dy, f64::Hyp(f64::exp2pix(dx)), f64::cos2piy(dy)) * bi * bj;
            if (kJac && dist_sq < a.range_sq * a.cut_sq) {
                // the gradient only builds the matrix: FP32, compensated
                float s, sd;
                f32::field<true>((float)dx, (float)dy, s, sd);
                double vv = a.h * bj * bi * (double)sd;
                if (!a.heaviside && dist_sq > a.cut_sq) {
                    const double t = sqrt(dist_sq) - a.cutoff;
                    vv *= exp(-(t * t) * a.one_per_cut_sq);
                }
                v = (float)vv;
                fj = vv;
            }
            if (kJac) a.A[(size_t)i + (size_t)j * a.n] = v;
        }
        if (kJac) sv[tx][lj] = v;
        row_f += f;
        row_j += fj;
        // column sums for row j: -f and -J, reduced over the warp's lanes (i)
        double cf = -f, cj = fj;
        for (int o = 16; o > 0; o >>= 1) {
            cf += __shfl_down_sync(0xffffffffu, cf, o);
            if (kJac) cj += __shfl_down_sync(0xffffffffu, cj, o);
        }
        if (tx == 0 && j < a.n) {
            a.part[((size_t)T + ti) * a.n + j] = cf;
            if (kJac) a.part[((size_t)3 * T + ti) * a.n + j] = -cj;
        }
    }
    if (a.tol && i < a.n && row_min < a.min_prec_sq) tol_min(a.tol, i, row_min);
    rs[ty][tx] = row_f;
    rj[ty][tx] = row_j;
    __syncthreads();
    if (ty == 0 && i < a.n) {
        double sf = 0, sj = 0;
        for (int k = 0; k < 8; ++k) {
            sf += rs[k][tx];
            sj += rj[k][tx];
        }
        a.part[(size_t)tj * a.n + i] = sf;
        if (kJac) a.part[((size_t)2 * T + tj) * a.n + i] = -sj;
    }
    if (kJac) {
        const int j = j0 + tx;
        for (int li = ty; li < 32; li += 8) {
            const int ii = i0 + li;
            if (ii < a.n && j < a.n && ii < j) a.A[(size_t)j + (size_t)ii * a.n] = sv[li][tx];
        }
    }
}

// Row r's partials in tile order: as row j of the tiles (tr, r/32), tr <= r/32,
// then as row i of the tiles (r/32, tj), tj >= r/32.
template <bool kJac>
__global__ void k_rowsum32(int n, const double *part, double *vacc, double *subacc) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= n) return;
    const int T = (n + 31) / 32, R = r / 32;
    double v = 0, w = 0;
    for (int t = 0; t <= R; ++t) {
        v += part[((size_t)T + t) * n + r];
        if (kJac) w += part[((size_t)3 * T + t) * n + r];
    }
    for (int t = R; t < T; ++t) {
        v += part[(size_t)t * n + r];
        if (kJac) w += part[((size_t)2 * T + t) * n + r];
    }
    vacc[r] = v;
    if (kJac) subacc[r] = w;
}

__global__ void k_speed_fin32(int n, const double *vacc, double ext, double *v) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) v[i] = vacc[i] + ext * bsign(i, n);
}

// Row i: speeds at both times, d_i = weight(subSum_i), row scale and diagonal.
__global__ void k_jac_fin32(int n, const double *vacc, const double *subacc, double ext_a,
                            double ext_b, double *v_a, double *v_b, double *dvec, double *sc,
                            float *A, char wfn) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double b = bsign(i, n);
    v_a[i] = vacc[i] + ext_a * b;
    v_b[i] = vacc[i] + ext_b * b;
    const double sub = subacc[i];
    const double d = f64::weight(sub, wfn);
    dvec[i] = d;
    const double s = (1 + d) / 2;
    sc[i] = s;
    A[(size_t)i + (size_t)i * n] = (float)(sub * s + 1);
}

// A_rc *= sc_r off the diagonal (column-major, 2-D grid).
__global__ void k_scale_rows32(int n, float *A, const double *sc) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    const int c = blockIdx.y;
    if (r < n && r != c) A[(size_t)r + (size_t)c * n] = (float)((double)A[(size_t)r + (size_t)c * n] * sc[r]);
}

// Half-step rescale on the FP32 matrix (src/simulation.cpp:584-594).
__global__ void k_half_rescale32(int n, float *A, const double *fac) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    const int c = blockIdx.y;
    if (r >= n) return;
    const double f = fac[r];
    const double e = A[(size_t)r + (size_t)c * n];
    A[(size_t)r + (size_t)c * n] = (float)((r == c) ? 1 + (e - 1) / 2 * f : e / 2 * f);
}

// g of the stage (as the FP64 form), r = g, dx = 0.
__global__ void k_ir_init(int n, trsv::GArgs ga, double *g, double *r, double *dx) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double gi = trsv::g_of(ga, i);
    g[i] = gi;
    r[i] = gi;
    dx[i] = 0;
}

// One refinement update in one launch: dx_out = dx + c and r = g - A32 dx_out.
// Block (x, y) multiplies rows 256x.. by column chunk y (FP64 accumulation in
// column order, the chunk's corrected dx staged in shared memory; the blocks of
// row block 0 also store it to dx_out, a buffer no block reads) into
// part[y][i]; the last block of each row block to finish (a counter per row
// block, reset by that block) subtracts the chunk sums from g in chunk order.
// The arithmetic and its order are those of a separate update, product and
// residual, so the residual is the same on every run.
__global__ void __launch_bounds__(256) k_resid_fused(int n, const float *__restrict__ A,
                                                     const double *__restrict__ dx,
                                                     const float *__restrict__ corr,
                                                     double *dx_out, const double *g,
                                                     double *part, int chunk, int nch,
                                                     unsigned *cnt, double *r) {
    __shared__ double sdx[256];
    __shared__ int last;
    const int c0 = blockIdx.y * chunk, c1 = min(n, c0 + chunk);
    for (int t = threadIdx.x; t < c1 - c0; t += blockDim.x) {
        const double v = dx[c0 + t] + (double)corr[c0 + t];
        sdx[t] = v;
        if (blockIdx.x == 0) dx_out[c0 + t] = v;
    }
    __syncthreads();
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) {
        double s = 0;
        for (int c = c0; c < c1; ++c) s += (double)__ldg(A + (size_t)i + (size_t)c * n) * sdx[c - c0];
        part[(size_t)blockIdx.y * n + i] = s;
    }
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) last = atomicAdd(&cnt[blockIdx.x], 1u) == (unsigned)(nch - 1);
    __syncthreads();
    if (!last) return;
    __threadfence();
    if (i < n) {
        double v = g[i];
        for (int q = 0; q < nch; ++q) v = v - __ldcg(part + (size_t)q * n + i);
        r[i] = v;
    }
    if (threadIdx.x == 0) cnt[blockIdx.x] = 0;
}

// max |r| and max |g| into out[0], out[1] (as ordered bits of non-negatives).
__global__ void k_absmax2(int n, const double *r, const double *g, unsigned long long *out) {
    double m1 = 0, m2 = 0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        m1 = fmax(m1, fabs(r[i]));
        m2 = fmax(m2, fabs(g[i]));
    }
    for (int o = 16; o > 0; o >>= 1) {
        m1 = fmax(m1, __shfl_down_sync(0xffffffffu, m1, o));
        m2 = fmax(m2, __shfl_down_sync(0xffffffffu, m2, o));
    }
    if ((threadIdx.x & 31) == 0) {
        atomicMax(out, (unsigned long long)__double_as_longlong(m1));
        atomicMax(out + 1, (unsigned long long)__double_as_longlong(m2));
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

// The mixed form's field at single points: the FP64 stress its speeds use and
// the FP32 gradient its matrix uses (the same calls as k_pairs32).
__global__ void k_field_mixed(int count, const double *dx, const double *dy, double *xy,
                              double *xyd) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= count) return;
    const double x = dx[k], y = dy[k];
    xy[k] = f64::xy(x, y, f64::Hyp(f64::exp2pix(x)), f64::cos2piy(y));
    float s, sd;
    f32::field<true>((float)x, (float)y, s, sd);
    xyd[k] = (double)sd;
}

inline int nb(long long n, int t) { return (int)((n + t - 1) / t); }

}  // namespace

void field_eval_mixed(Ctx &c, int count, const double *dx, const double *dy, double *xy,
                      double *xyd) {
    k_field_mixed<<<nb(count, 128), 128, 0, c.stream>>>(count, dx, dy, xy, xyd);
    check_launch("k_field_mixed");
}

static Pair32Args pair32(Ctx &c, const double *x, const double *y) {
    Pair32Args a;
    a.n = c.n;
    a.x = x;
    a.y = y;
    a.vacc = c.m_vacc;
    a.subacc = c.m_subacc;
    a.part = c.m_pp;
    a.A = c.A32;
    a.tol = c.use_dipole ? c.tol : nullptr;
    a.min_prec_sq = c.min_prec_sq;
    a.h = 0;
    a.cut_sq = c.cutoff_sq;
    a.cutoff = c.cutoff;
    a.range_sq = c.range_sq;
    a.one_per_cut_sq = 1 / c.cutoff_sq;
    a.heaviside = c.p.heaviside_cutoff;
    return a;
}

static int pair_tiles(int n) {
    const int T = (n + 31) / 32;
    return T * (T + 1) / 2;
}

void speeds32_with(Ctx &c, double *vacc, double *part, cudaStream_t st, const double *x,
                   const double *y, double ext, double *v) {
    Pair32Args a = pair32(c, x, y);
    a.vacc = vacc;
    a.part = part;
    k_pairs32<false><<<pair_tiles(c.n), dim3(32, 8), 0, st>>>(a);
    check_launch("k_pairs32<speeds>");
    k_rowsum32<false><<<nb(c.n, 256), 256, 0, st>>>(c.n, part, vacc, nullptr);
    check_launch("k_rowsum32<speeds>");
    k_speed_fin32<<<nb(c.n, 256), 256, 0, st>>>(c.n, vacc, ext, v);
    check_launch("k_speed_fin32");
}

void speeds32(Ctx &c, const double *x, const double *y, double ext, double *v) {
    speeds32_with(c, c.m_vacc, c.m_pp, c.stream, x, y, ext, v);
}

void jacobian32(Ctx &c, const double *x, const double *y, double h, double ext_a, double ext_b,
                double *v_a, double *v_b) {
    Pair32Args a = pair32(c, x, y);
    a.h = h;
    k_pairs32<true><<<pair_tiles(c.n), dim3(32, 8), 0, c.stream>>>(a);
    check_launch("k_pairs32<jacobian>");
    k_rowsum32<true><<<nb(c.n, 256), 256, 0, c.stream>>>(c.n, c.m_pp, c.m_vacc, c.m_subacc);
    check_launch("k_rowsum32<jacobian>");
    k_jac_fin32<<<nb(c.n, 256), 256, 0, c.stream>>>(c.n, c.m_vacc, c.m_subacc, ext_a, ext_b,
                                                     v_a, v_b, c.dvec, c.fac, c.A32,
                                                     c.p.weight_function);
    check_launch("k_jac_fin32");
    k_scale_rows32<<<dim3(nb(c.n, 256), c.n), 256, 0, c.stream>>>(c.n, c.A32, c.fac);
    check_launch("k_scale_rows32");
}

void jacobian_from_prev32(Ctx &c, double factor) {
    half_weights64(c, factor);  // dvec_new, fac
    k_half_rescale32<<<dim3(nb(c.n, 256), c.n), 256, 0, c.stream>>>(c.n, c.A32, c.fac);
    check_launch("k_half_rescale32");
    D4_CUDA_OK(cudaMemcpyAsync(c.dvec, c.dvec_new, sizeof(double) * c.n, cudaMemcpyDeviceToDevice,
                               c.stream));
}

Mix32Bufs primary_mix32(Ctx &c) {
    Mix32Bufs B;
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
    B.part = c.m_part;
    B.c32 = c.m_c32;
    B.w1 = c.m_w1;
    B.resid = c.m_resid;
    B.resid_count = &c.m_resid_count;
    B.blu = c.blu;
    B.blk = &c.m_blk;
    return B;
}

void factor32_async(Ctx &c, const Mix32Bufs &B, const float *A, bool copy_matrix, int grid,
                    cudaStream_t st, cudaEvent_t after_copy) {
    const int n = c.n;
    const size_t bytes = sizeof(float) * (size_t)n * n;
    *B.blk = c.m_fast;
    if (c.m_fast) {
        // block LU (d4_blu32.cu): reads the matrix, writes the factors and operands
        D4_CUDA_OK(cudaMemsetAsync(B.flags, 0, sizeof(int) * kFlagCount, st));
        if (copy_matrix) D4_CUDA_OK(cudaMemcpyAsync(B.A32, A, bytes, cudaMemcpyDeviceToDevice, st));
        if (after_copy) D4_CUDA_OK(cudaEventRecord(after_copy, st));
        blu_factor_async(B.blu, n, copy_matrix ? B.A32 : A, B.LU32, B.flags, grid, st);
        ++c.m_blocklu;
        return;
    }
    D4_CUDA_OK(cudaMemsetAsync(B.flags, 0, sizeof(int) * kFlagCount, st));
    D4_CUDA_OK(cudaMemsetAsync(B.bar, 0, sizeof(unsigned) * 64, st));
    D4_CUDA_OK(cudaMemsetAsync(B.mask, 0, sizeof(unsigned) * c.lu_mask_words, st));
    D4_CUDA_OK(cudaMemcpyAsync(B.LU32, A, bytes, cudaMemcpyDeviceToDevice, st));
    if (copy_matrix) D4_CUDA_OK(cudaMemcpyAsync(B.A32, A, bytes, cudaMemcpyDeviceToDevice, st));
    if (after_copy) D4_CUDA_OK(cudaEventRecord(after_copy, st));
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
    void *args[] = {(void *)&a};
    const void *kern = (const void *)coop::k_lu_coop<float>;
    D4_CUDA_OK(cudaLaunchCooperativeKernel(kern, dim3(grid), dim3(coop::kThreads), args,
                                           coop::kRowBufBytes<float>(), st));
    check_launch("k_lu_coop<float>");
}

int factor32(Ctx &c) {
    factor32_async(c, primary_mix32(c), c.A32, false, c.lu32_grid, c.stream, nullptr);
    D4_CUDA_OK(cudaMemcpyAsync(c.h_flags, c.flags, sizeof(int) * kFlagCount,
                               cudaMemcpyDeviceToHost, c.stream));
    D4_CUDA_OK(cudaStreamSynchronize(c.stream));
    if (c.h_flags[kFlagBarrierTimeout]) throw StateError("LU grid barrier timed out");
    if (c.m_blk && c.h_flags[kFlagSingular]) {
        // a diagonal tile met a zero or non-finite pivot: the pivoted LU instead
        ++c.m_fallbacks;
        c.m_fast = 0;
        try {
            factor32_async(c, primary_mix32(c), c.A32, false, c.lu32_grid, c.stream, nullptr);
        } catch (...) {
            c.m_fast = 1;
            throw;
        }
        c.m_fast = 1;
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
// block solves of the block LU, or by the cluster solve of the pivoted LU.
// Returns the result's buffer.
static const float *solve32_once(Ctx &c, const Mix32Bufs &B, cudaStream_t st, const double *r) {
    if (*B.blk) {
        blu_solve_async(B.blu, c.n, B.LU32, r, B.flags, st);
        return B.blu.xs;
    }
    trsv::GArgs g{};
    g.gmode = -1;
    g.g_in = r;
    trsv::launch_cluster_solve<float>(c.n, B.LU32, B.perm, B.flags, g, B.w1, B.c32, c.wave_err,
                                      st);
    return B.c32;
}

// The refinement loop: c = LU32^-1 r, dx += c, r = g - A32 dx, c.ir_iters
// times from dx = 0, r = g (k_ir_init); dx alternates between B.dx and B.dx2.
// Returns the buffer holding the final dx.
static const double *refine(Ctx &c, const Mix32Bufs &B, cudaStream_t st) {
    const int n = c.n, chunk = 256;
    double *dxa = B.dx, *dxb = B.dx2;
    for (int it = 0; it < c.ir_iters; ++it) {
        const float *corr = solve32_once(c, B, st, B.r);
        k_resid_fused<<<dim3(nb(n, 256), nb(n, chunk)), 256, 0, st>>>(
            n, B.A32, dxa, corr, dxb, B.g, B.part, chunk, nb(n, chunk), B.cnt, B.r);
        check_launch("k_resid_fused");
        std::swap(dxa, dxb);
    }
    return dxa;
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
    k_ir_init<<<nb(n, 256), 256, 0, st>>>(n, ga, B.g, B.r, B.dx);
    check_launch("k_ir_init");
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
    k_ir_init<<<nb(n, 256), 256, 0, c.stream>>>(n, ga, B.g, B.r, B.dx);
    check_launch("k_ir_init");
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
