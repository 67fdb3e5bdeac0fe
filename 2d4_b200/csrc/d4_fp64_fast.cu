// d4_fp64_fast.cu: the mixed form's FP64 sweeps.  The pair tiles of
// d4_sweep64.cuh with the field of d4_field64_fast.cuh (one reciprocal per
// image, shared by the field and its derivative), compiled with product-add
// contraction, and row sums by column chunks instead of the ordered row
// pipeline; the row scaling and everything after it are the plain form's
// (d4_fp64.cu).
#include "d4_field64_fast.cuh"
#define D4_PAIR_FIELD f64fast
#include "d4_sweep64.cuh"

namespace d4 {
namespace {

// Row sums of the mixed form's sweeps, in place of the ordered row pipeline:
// thread = row (coalesced column loads), a CTA sums `chunk` columns with 16
// loads in flight and four interleaved sums, and the last CTA of each row
// block combines the chunks' partials in chunk order (deterministic).  The
// outputs are row_block's: speeds at ext_a (and ext_b), and for the Jacobian
// d = weight(-sum of the row's raw entries), rowsub and the row scale.
template <bool kJac>
__global__ void __launch_bounds__(256) k_rows_fast(RowArgs a, double *part, unsigned *cnt,
                                                   int chunk, int nch) {
    __shared__ int last;
    const int n = a.n;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int c0 = blockIdx.y * chunk, c1 = min(n, c0 + chunk);
    if (i < n) {
        double f[4] = {0, 0, 0, 0}, g[4] = {0, 0, 0, 0};
        const double *Fi = a.F + i;
        const double *Ai = a.A + i;
        int c = c0;
        for (; c + 16 <= c1; c += 16) {
            double fv[16], av[16];
#pragma unroll
            for (int u = 0; u < 16; ++u) {
                fv[u] = __ldg(Fi + (size_t)(c + u) * n);
                if (kJac) av[u] = __ldg(Ai + (size_t)(c + u) * n);
            }
#pragma unroll
            for (int u = 0; u < 16; ++u)
                if (c + u != i) {
                    f[u & 3] += fv[u];
                    if (kJac) g[u & 3] += av[u];
                }
        }
        for (; c < c1; ++c)  // the chunk's last columns (n not a multiple of 16) into sum 0
            if (c != i) {
                f[0] += __ldg(Fi + (size_t)c * n);
                if (kJac) g[0] += __ldg(Ai + (size_t)c * n);
            }
        part[(size_t)blockIdx.y * n + i] = (f[0] + f[1]) + (f[2] + f[3]);
        if (kJac) part[(size_t)(nch + blockIdx.y) * n + i] = (g[0] + g[1]) + (g[2] + g[3]);
    }
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) last = atomicAdd(&cnt[blockIdx.x], 1u) == (unsigned)(nch - 1);
    __syncthreads();
    if (!last) return;
    __threadfence();
    if (i < n) {
        double sum = 0, acc = 0;
        for (int q = 0; q < nch; ++q) {
            sum += __ldcg(part + (size_t)q * n + i);
            if (kJac) acc += __ldcg(part + (size_t)(nch + q) * n + i);
        }
        const double b = bsign(i, n);
        if (kJac) {
            const double sub = -acc;
            a.v_b[i] = sum + a.ext_b * b;
            a.v_a[i] = sum + a.ext_a * b;
            const double d = f64::weight(sub, a.wfn);
            a.dvec[i] = d;
            a.rowsub[i] = sub;
            a.rowsc[i] = (1 + d) / 2;
        } else {
            a.v_a[i] = sum + a.ext_a * b;
        }
    }
    if (threadIdx.x == 0) cnt[blockIdx.x] = 0;
}

}  // namespace

void rows64_fast(Ctx &c, bool jac, const double *F, double ext_a, double ext_b, double *v_a,
                 double *v_b, cudaStream_t st) {
    const int n = c.n, chunk = 256, nch = (n + chunk - 1) / chunk;
    const int set = (F == c.F_b) ? 1 : 0;  // stage I's sweeps run on their own stream
    RowArgs r{};
    r.n = n;
    r.F = F;
    r.A = c.A;
    r.ext_a = ext_a;
    r.ext_b = ext_b;
    r.v_a = v_a;
    r.v_b = v_b;
    r.dvec = c.dvec;
    r.rowsub = c.rowsub;
    r.rowsc = c.rowsc;
    r.wfn = c.p.weight_function;
    const dim3 grid((n + 255) / 256, nch);
    if (jac)
        k_rows_fast<true><<<grid, 256, 0, st>>>(r, c.fr_part[set], c.fr_cnt[set], chunk, nch);
    else
        k_rows_fast<false><<<grid, 256, 0, st>>>(r, c.fr_part[set], c.fr_cnt[set], chunk, nch);
    check_launch(jac ? "k_rows_fast<jacobian>" : "k_rows_fast<speeds>");
}

void pairs64_fast(Ctx &c, bool jac, const double *x, const double *y, double *F, double h,
                  cudaStream_t st) {
    PairArgs a = pair_args(c, x, y);
    a.F = F;
    a.h = h;
    if (jac)
        k_pairs64<true><<<pair_blocks(c.n), dim3(kTile, c.pair_ty), 0, st>>>(a);
    else
        k_pairs64<false><<<pair_blocks(c.n), dim3(kTile, c.pair_ty), 0, st>>>(a);
    check_launch(jac ? "k_pairs64<jacobian, fast>" : "k_pairs64<speeds, fast>");
}

}  // namespace d4
