// d4_fp64.cu: FP64 pair sweeps and small kernels of the plain form (compiled
// with --fmad=false).  The pair tiles and the ordered row sums live in
// d4_sweep64.cuh.
#include <cstdint>
#include <map>
#include <mutex>
#include <tuple>

#include "d4_sweep64.cuh"

namespace d4 {
namespace {

// Ordered row sums of the stress sweep, v_i = sum_j F[i, j] + ext * b_i, one
// thread per row (the allocation-free sweep; the engine uses the pipelined
// row_block of d4_sweep64.cuh).  Loads are issued 8 at a time ahead of the
// sequential, ordered additions.
__global__ void k_rows_speed64(int n, const double *__restrict__ F, double ext, double *v) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double s = 0;
    const double *col = F + i;
    int j = 0;
    for (; j + 8 <= n; j += 8) {
        double t[8];
#pragma unroll
        for (int u = 0; u < 8; ++u) t[u] = __ldg(col + (size_t)(j + u) * n);
#pragma unroll
        for (int u = 0; u < 8; ++u)
            if (j + u != i) s += t[u];
    }
    for (; j < n; ++j)
        if (j != i) s += col[(size_t)j * n];
    v[i] = s + ext * bsign(i, n);
}

// calcJacobianAndSpeedsFromPrev weights (src/simulation.cpp:552-582).
__global__ void k_half_weights64(int n, const double *dvec, double factor, char wfn,
                                 double *dnew, double *fac) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double old = dvec[i];
    double w = 0.;
    if (old != 0) w = f64::weight(f64::weight_inv(old, wfn) * factor, wfn);
    dnew[i] = w;
    fac[i] = (1 + w) / (1 + old);
}

// Elementwise rescale (src/simulation.cpp:584-594): factor of the row.
__global__ void k_half_rescale64(int n, double *A, const double *fac) {
    const size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    const size_t total = (size_t)n * n;
    if (idx >= total) return;
    const int r = (int)(idx % n), c = (int)(idx / n);
    const double f = fac[r];
    double e = A[idx];
    A[idx] = (r == c) ? 1 + (e - 1) / 2 * f : e / 2 * f;
}

__global__ void k_shift_speed64(int n, double *v, double dif) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) v[i] += dif * bsign(i, n);
}

__global__ void k_fill64(int n, double *v, double val) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) v[i] = val;
}

__global__ void __launch_bounds__(1024) k_error_ratio64(int n, const double *xb, const double *x2,
                                                        const double *tol, double min_prec_sq,
                                                        int use_dipole, double *out) {
    error_ratio_block(n, xb, x2, tol, min_prec_sq, use_dipole, out);
}

__global__ void k_normalize64(int n, double *dst, const double *src) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) dst[i] = f64::normalize(src[i]);
}

// calculateStrainIncrement (src/simulation.cpp:713-720), sequential order.
__global__ void k_strain64(int n, const double *old, const double *nw, double *out) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    double r = 0;
    for (int i = 0; i < n; ++i) r += bsign(i, n) * (nw[i] - old[i]);
    *out = r;
}

// The tabulated field at given points.
__global__ void k_field_tab64(tab::Table tb, int count, const double *dx, const double *dy,
                              double *xy, double *xyd) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= count) return;
    const double2 t = tab::eval<true>(tb, dx[k], dy[k]);
    xy[k] = t.x;
    xyd[k] = t.y;
}

// Field::xy (2-arg, exp2) and Field::xy_diff_x (2-arg, exp) at given points.
__global__ void k_field64(int count, const double *dx, const double *dy, double *xy,
                          double *xyd) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= count) return;
    const double x = dx[k], y = dy[k];
    const double c = f64::cos2piy(y);
    f64::Hyp h2(f64::exp2pix(x));
    xy[k] = f64::xy(x, y, h2, c);
    f64::Hyp he(exp(f64::kPi * 2 * x));
    xyd[k] = f64::xy_diff_x(x, y, he, c);
}

inline int blocks(long long n, int t) { return (int)((n + t - 1) / t); }

}  // namespace

template <bool kJac>
static void launch_rows(Ctx &c, const RowArgs &r, cudaStream_t st) {
    constexpr int bytes = row_smem_bytes<kJac>();
    D4_CUDA_OK(cudaFuncSetAttribute(k_rows64<kJac>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    bytes));
    k_rows64<kJac><<<(c.n + kRowRows - 1) / kRowRows, 64, bytes, st>>>(r);
    check_launch(kJac ? "k_rows64<jacobian>" : "k_rows64<speeds>");
}


void speeds64_with(Ctx &c, double *F, cudaStream_t st, const double *x, const double *y,
                   double ext, double *v) {
    if (c.fast_pairs) {
        pairs64_fast(c, false, x, y, F, 0, st);
        rows64_fast(c, false, F, ext, 0, v, nullptr, st);
        return;
    }
    PairArgs a = pair_args(c, x, y);
    a.F = F;
    if (c.tab)
        k_pairs64<false, true><<<pair_blocks(c.n), dim3(kTile, c.pair_ty), 0, st>>>(a);
    else
        k_pairs64<false><<<pair_blocks(c.n), dim3(kTile, c.pair_ty), 0, st>>>(a);
    check_launch("k_pairs64<speeds>");
    RowArgs r{};
    r.n = c.n;
    r.F = F;
    r.ext_a = ext;
    r.v_a = v;
    r.err = c.wave_err + kWaveErrRows;
    launch_rows<false>(c, r, st);
}

void speeds64(Ctx &c, const double *x, const double *y, double ext, double *v) {
    speeds64_with(c, c.F, c.stream, x, y, ext, v);
}

void jacobian64(Ctx &c, const double *x, const double *y, double h, double ext_a, double ext_b,
                double *v_a, double *v_b) {
    if (c.fast_pairs) {
        pairs64_fast(c, true, x, y, c.F, h, c.stream);
        rows64_fast(c, true, c.F, ext_a, ext_b, v_a, v_b, c.stream);
        k_scale_rows64<<<blocks((long long)c.n * c.n, 256), 256, 0, c.stream>>>(c.n, c.A, c.rowsub,
                                                                               c.rowsc);
        check_launch("k_scale_rows64");
        return;
    }
    PairArgs a = pair_args(c, x, y);
    a.h = h;
    if (c.tab)
        k_pairs64<true, true><<<pair_blocks(c.n), dim3(kTile, c.pair_ty), 0, c.stream>>>(a);
    else
        k_pairs64<true><<<pair_blocks(c.n), dim3(kTile, c.pair_ty), 0, c.stream>>>(a);
    check_launch("k_pairs64<jacobian>");
    RowArgs r{};
    r.n = c.n;
    r.F = c.F;
    r.A = c.A;
    r.ext_a = ext_a;
    r.ext_b = ext_b;
    r.v_a = v_a;
    r.v_b = v_b;
    r.dvec = c.dvec;
    r.rowsub = c.rowsub;
    r.rowsc = c.rowsc;
    r.wfn = c.p.weight_function;
    r.err = c.wave_err + kWaveErrRows;
    launch_rows<true>(c, r, c.stream);
    k_scale_rows64<<<blocks((long long)c.n * c.n, 256), 256, 0, c.stream>>>(c.n, c.A, c.rowsub,
                                                                           c.rowsc);
    check_launch("k_scale_rows64");
}

namespace {
std::mutex g_tune_mu;
std::map<std::tuple<int, int, int>, int> g_tune_cache;  // (device, n, table) -> threads y
}  // namespace

// Each candidate runs the stress and the fused pair kernels (tolerances off,
// writing only the context's scratch F and A) once untimed and three times
// timed with CUDA events on the context's stream; the fastest total wins.
void autotune_pairs(Ctx &c) {
    if (c.pair_tuned) return;
    int dev = 0;
    D4_CUDA_OK(cudaGetDevice(&dev));
    const auto key = std::make_tuple(dev, c.n, c.tab ? c.tab_T : 0);
    {
        std::lock_guard<std::mutex> lk(g_tune_mu);
        auto it = g_tune_cache.find(key);
        if (it != g_tune_cache.end()) {
            c.pair_ty = it->second;
            c.pair_tuned = true;
            return;
        }
    }
    PairArgs a = pair_args(c, c.x0, c.y);
    a.tol = nullptr;
    a.F = c.F;
    a.A = c.A;
    a.h = c.step_size;
    float best = 1e30f;
    int best_ty = 8;
    for (int ty : kPairTyCandidates) {
        float total = 0;
        for (int rep = 0; rep < 4; ++rep) {
            D4_CUDA_OK(cudaEventRecord(c.ev0, c.stream));
            if (c.tab) {
                k_pairs64<false, true><<<pair_blocks(c.n), dim3(kTile, ty), 0, c.stream>>>(a);
                k_pairs64<true, true><<<pair_blocks(c.n), dim3(kTile, ty), 0, c.stream>>>(a);
            } else {
                k_pairs64<false><<<pair_blocks(c.n), dim3(kTile, ty), 0, c.stream>>>(a);
                k_pairs64<true><<<pair_blocks(c.n), dim3(kTile, ty), 0, c.stream>>>(a);
            }
            check_launch("k_pairs64<tune>");
            D4_CUDA_OK(cudaEventRecord(c.ev1, c.stream));
            D4_CUDA_OK(cudaEventSynchronize(c.ev1));
            float ms = 0;
            D4_CUDA_OK(cudaEventElapsedTime(&ms, c.ev0, c.ev1));
            if (rep > 0) total += ms;
        }
        if (total < best) {
            best = total;
            best_ty = ty;
        }
    }
    c.pair_ty = best_ty;
    c.pair_tuned = true;
    std::lock_guard<std::mutex> lk(g_tune_mu);
    g_tune_cache[key] = best_ty;
}

void jacobian_from_prev64(Ctx &c, double factor) {
    k_half_weights64<<<blocks(c.n, 128), 128, 0, c.stream>>>(c.n, c.dvec, factor,
                                                             c.p.weight_function, c.dvec_new,
                                                             c.fac);
    check_launch("k_half_weights64");
    k_half_rescale64<<<blocks((long long)c.n * c.n, 256), 256, 0, c.stream>>>(c.n, c.A, c.fac);
    check_launch("k_half_rescale64");
    D4_CUDA_OK(cudaMemcpyAsync(c.dvec, c.dvec_new, sizeof(double) * c.n, cudaMemcpyDeviceToDevice,
                               c.stream));
}

void half_weights64(Ctx &c, double factor) {
    k_half_weights64<<<blocks(c.n, 128), 128, 0, c.stream>>>(c.n, c.dvec, factor,
                                                             c.p.weight_function, c.dvec_new,
                                                             c.fac);
    check_launch("k_half_weights64");
}

void shift_speed64(Ctx &c, double *v, double dif) {
    k_shift_speed64<<<blocks(c.n, 128), 128, 0, c.stream>>>(c.n, v, dif);
    check_launch("k_shift_speed64");
}

void reset_tol64(Ctx &c) {
    k_fill64<<<blocks(c.n, 128), 128, 0, c.stream>>>(c.n, c.tol, c.min_prec_sq);
    check_launch("k_fill64");
}

void error_ratio64(Ctx &c, const double *xb, const double *x2) {
    k_error_ratio64<<<1, 1024, 0, c.stream>>>(c.n, xb, x2, c.tol, c.min_prec_sq, c.use_dipole,
                                              c.red);
    check_launch("k_error_ratio64");
}

void normalize64(Ctx &c, double *dst, const double *src) {
    k_normalize64<<<blocks(c.n, 128), 128, 0, c.stream>>>(c.n, dst, src);
    check_launch("k_normalize64");
}

void strain_increment64(Ctx &c, const double *x_old, const double *x_new, double *out) {
    k_strain64<<<1, 32, 0, c.stream>>>(c.n, x_old, x_new, out);
    check_launch("k_strain64");
}

void field_eval64(Ctx &c, int count, const double *dx, const double *dy, double *xy,
                  double *xyd) {
    if (c.tab) {
        PairArgs a = pair_args(c, nullptr, nullptr);
        k_field_tab64<<<blocks(count, 128), 128, 0, c.stream>>>(a.tb, count, dx, dy, xy, xyd);
        check_launch("k_field_tab64");
        return;
    }
    k_field64<<<blocks(count, 128), 128, 0, c.stream>>>(count, dx, dy, xy, xyd);
    check_launch("k_field64");
}

}  // namespace d4

// ---------------------------------------------------------------------------
// Allocation-free stress sweep.
//
// Some callers cannot allocate device memory at all: code that runs while a
// stream is being captured into a CUDA graph (an allocation there breaks the
// capture), real-time stepping loops that must not block on the allocator,
// and hosts whose device memory is owned by another framework's allocator
// that this library must not bypass.  For them, d4_speeds_noalloc runs the
// FP64 stress sweep with its n x n pair-force scratch in the file-scope device
// array below instead of a context buffer.  The caller passes device pointers
// for the inputs and outputs; the function calls no cudaMalloc/cudaFree and no
// allocating library routine.
//
// Limit: n <= D4_NOALLOC_MAX_N (1024), i.e. 8 MiB of scratch, held on every
// GPU that loads the library until the process exits.  Every call shares the
// array and it keeps the last call's contents; every entry a call reads is
// written by the same call first, so nothing needs clearing, but calls that
// overlap on the GPU (different streams, or different host threads) race on
// it and must be serialised by the caller.  The first call on a device looks
// up the array's device address (cudaGetSymbolAddress) with that device
// current; make that first call before any stream capture begins.  The
// address is cached per device together with the device's current CUDA
// context: after a device reset (a new primary context, in which the module
// is loaded again and the array may move) the next call looks it up again,
// so that call, too, must come before any capture.
static __device__ __align__(256) double g_noalloc_pair_force[D4_NOALLOC_MAX_N * D4_NOALLOC_MAX_N];

namespace {
constexpr int kMaxDevices = 64;
std::mutex g_noalloc_mu;
double *g_noalloc_addr[kMaxDevices] = {};
void *g_noalloc_ctx[kMaxDevices] = {};

// The calling thread's current CUDA context (the driver's cuCtxGetCurrent,
// reached through the runtime's entry-point query, so the library needs no
// link against the driver library); null when it cannot be queried.
void *current_context() {
    using Fn = int (*)(void **);
    static Fn fn = [] {
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &p, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess)
            return (Fn) nullptr;
        return reinterpret_cast<Fn>(p);
    }();
    void *ctx = nullptr;
    if (!fn || fn(&ctx) != 0) return nullptr;
    return ctx;
}
}  // namespace

extern "C" int d4_speeds_noalloc(int n, const double *x, const double *y, double ext_stress,
                                 double *v, double *tol, double min_prec_sq, void *stream) {
    if (n < 2 || n % 2 != 0 || !x || !y || !v) return D4_ERR_ARG;
    if (n > D4_NOALLOC_MAX_N) return D4_ERR_ARG;  // scratch holds at most 1024 x 1024 forces
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return D4_ERR_CUDA;
    double *scratch = nullptr;
    {
        std::lock_guard<std::mutex> lk(g_noalloc_mu);
        void *ctx = current_context();
        if (!g_noalloc_addr[dev] || ctx != g_noalloc_ctx[dev]) {
            void *p = nullptr;
            if (cudaGetSymbolAddress(&p, g_noalloc_pair_force) != cudaSuccess || !p)
                return D4_ERR_CUDA;
            g_noalloc_addr[dev] = static_cast<double *>(p);
            g_noalloc_ctx[dev] = ctx;
        }
        scratch = g_noalloc_addr[dev];
    }
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    using namespace d4;
    PairArgs a;
    a.n = n;
    a.x = x;
    a.y = y;
    a.F = scratch;
    a.A = nullptr;
    a.tol = tol;
    a.min_prec_sq = min_prec_sq;
    a.h = 0;
    a.cut_sq = a.cutoff = a.range_sq = a.one_per_cut_sq = 0;
    a.heaviside = 0;
    k_pairs64<false><<<pair_blocks(n), dim3(kTile, 8), 0, st>>>(a);
    g_launches.fetch_add(1, std::memory_order_relaxed);
    if (cudaGetLastError() != cudaSuccess) return D4_ERR_CUDA;
    k_rows_speed64<<<blocks(n, 128), 128, 0, st>>>(n, scratch, ext_stress, v);
    g_launches.fetch_add(1, std::memory_order_relaxed);
    if (cudaGetLastError() != cudaSuccess) return D4_ERR_CUDA;
    return D4_OK;
}
