// d4_xpattern.cu: the direct-Fourier pattern analysis of a dislocation
// configuration (the reference's xpattern tool, method df,
// xpattern/xpattern.cpp:393-423).
//
// With K = res/2 + 1 and the four densities m = rho_t (weight 1), kappa
// (weight b), rho_p (b = +1 only) and rho_n (b = -1 only),
//     F_m(kx, ky) = sum_i w_m(b_i) exp(-2 pi i (kx x_i + ky y_i)),
//     S_m(kx)    += sum_ky |F_m(kx, ky)|^2     (over ky ascending).
// F is a complex matrix product, F = Ey^T diag(w) Ex with Ex[i][k] =
// exp(-2 pi i k x_i): k_xp_tables builds Ex and Ey (sincospi of 2 k x, so
// large k x keep their accuracy), k_xp_gemm accumulates F_p and F_n in FP64
// registers over 32 x 32 output tiles (rho_t = F_p + F_n, kappa = F_p - F_n)
// and stores the four |F|^2, and k_xp_colsum adds them over ky in ascending
// order into the caller's running sums.  No atomics: the result repeats bit
// for bit.
#include <cuda_runtime.h>

#include <algorithm>
#include <vector>

#include "d4_internal.h"

namespace d4 {
namespace {

constexpr int kXpTile = 32;  // output tile edge (ky, kx)
constexpr int kXpChunk = 16; // dislocations staged per step

// tab[i * K + k] = exp(-2 pi i k v_i) as (re, im)
__global__ void k_xp_tables(int n, int K, const double *v, double2 *tab) {
    const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= (long long)n * K) return;
    const int i = (int)(idx / K), k = (int)(idx % K);
    double s, c;
    sincospi(2.0 * v[i] * (double)k, &s, &c);
    tab[idx] = make_double2(c, -s);
}

__device__ __forceinline__ void cmac(double2 &acc, double2 a, double2 b) {
    acc.x = fma(a.x, b.x, fma(-a.y, b.y, acc.x));
    acc.y = fma(a.x, b.y, fma(a.y, b.x, acc.y));
}

// Tile (ky0, kx0): 16 x 16 threads, 2 x 2 outputs each.  Dislocations
// [0, npos) are the positive ones, [npos, n) the negative ones.
__global__ void __launch_bounds__(256) k_xp_gemm(int n, int npos, int K, const double2 *Ex,
                                                 const double2 *Ey, double *nrm) {
    __shared__ double2 sx[kXpChunk][kXpTile], sy[kXpChunk][kXpTile];
    const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
    const int kx0 = blockIdx.x * kXpTile, ky0 = blockIdx.y * kXpTile;
    double2 fp[2][2], fn[2][2];
    for (int part = 0; part < 2; ++part) {
        double2 acc[2][2];
#pragma unroll
        for (int a = 0; a < 2; ++a)
#pragma unroll
            for (int b = 0; b < 2; ++b) acc[a][b] = make_double2(0, 0);
        const int i_beg = part == 0 ? 0 : npos, i_end = part == 0 ? npos : n;
        for (int c0 = i_beg; c0 < i_end; c0 += kXpChunk) {
            __syncthreads();
            for (int t = threadIdx.x; t < kXpChunk * kXpTile; t += 256) {
                const int r = t / kXpTile, col = t % kXpTile;
                const int i = c0 + r;
                const bool ok = i < i_end;
                sx[r][col] = (ok && kx0 + col < K) ? Ex[(size_t)i * K + kx0 + col]
                                                   : make_double2(0, 0);
                sy[r][col] = (ok && ky0 + col < K) ? Ey[(size_t)i * K + ky0 + col]
                                                   : make_double2(0, 0);
            }
            __syncthreads();
            const int m = min(kXpChunk, i_end - c0);
            for (int r = 0; r < m; ++r) {
                const double2 x0 = sx[r][tx], x1 = sx[r][tx + 16];
                const double2 y0 = sy[r][ty], y1 = sy[r][ty + 16];
                cmac(acc[0][0], y0, x0);
                cmac(acc[0][1], y0, x1);
                cmac(acc[1][0], y1, x0);
                cmac(acc[1][1], y1, x1);
            }
        }
#pragma unroll
        for (int a = 0; a < 2; ++a)
#pragma unroll
            for (int b = 0; b < 2; ++b) (part == 0 ? fp : fn)[a][b] = acc[a][b];
    }
    const size_t KK = (size_t)K * K;
#pragma unroll
    for (int a = 0; a < 2; ++a)
#pragma unroll
        for (int b = 0; b < 2; ++b) {
            const int ky = ky0 + ty + 16 * a, kx = kx0 + tx + 16 * b;
            if (ky >= K || kx >= K) continue;
            const double2 p = fp[a][b], q = fn[a][b];
            const double tr = p.x + q.x, ti = p.y + q.y;  // rho_t
            const double kr = p.x - q.x, ki = p.y - q.y;  // kappa
            const size_t o = (size_t)ky * K + kx;
            nrm[o] = tr * tr + ti * ti;
            nrm[KK + o] = kr * kr + ki * ki;
            nrm[2 * KK + o] = p.x * p.x + p.y * p.y;
            nrm[3 * KK + o] = q.x * q.x + q.y * q.y;
        }
}

// acc[m][kx] += |F_m(kx, ky)|^2 for ky = 0, 1, ... in order.
__global__ void k_xp_colsum(int K, const double *nrm, double *acc) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= 4 * K) return;
    const int m = t / K, kx = t % K;
    const double *p = nrm + (size_t)m * K * K + kx;
    double v = acc[t];
    for (int ky = 0; ky < K; ++ky) v = v + p[(size_t)ky * K];
    acc[t] = v;
}

}  // namespace
}  // namespace d4

extern "C" int d4_xpattern_df(int n, const double *x, const double *y, const int *b, int res,
                              double *acc) {
    using namespace d4;
    if (n < 0 || res < 2 || res > 65536 || (n > 0 && (!x || !y || !b)) || !acc) return D4_ERR_ARG;
    const int K = res / 2 + 1;
    if ((long long)K * K * 4 * 8 > (8ll << 30)) return D4_ERR_ARG;
    // positives first (stable), so each density's sum runs over one range
    std::vector<double> hx, hy;
    hx.reserve(n);
    hy.reserve(n);
    for (int pass = 0; pass < 2; ++pass)
        for (int i = 0; i < n; ++i)
            if ((b[i] == 1) == (pass == 0)) {
                hx.push_back(x[i]);
                hy.push_back(y[i]);
            }
    int npos = 0;
    for (int i = 0; i < n; ++i) npos += b[i] == 1;
    double *dv = nullptr, *dnrm = nullptr, *dacc = nullptr;
    double2 *ex = nullptr, *ey = nullptr;
    int st = D4_OK;
    auto ok = [&](cudaError_t e) {
        if (e != cudaSuccess && st == D4_OK) st = D4_ERR_CUDA;
        return e == cudaSuccess;
    };
    const size_t tab = (size_t)std::max(n, 1) * K;
    if (ok(d4::dmalloc(&dv, sizeof(double) * 2 * std::max(n, 1))) &&
        ok(d4::dmalloc(&ex, sizeof(double2) * tab)) && ok(d4::dmalloc(&ey, sizeof(double2) * tab)) &&
        ok(d4::dmalloc(&dnrm, sizeof(double) * 4 * (size_t)K * K)) &&
        ok(d4::dmalloc(&dacc, sizeof(double) * 4 * K))) {
        if (n > 0) {
            ok(cudaMemcpy(dv, hx.data(), sizeof(double) * n, cudaMemcpyHostToDevice));
            ok(cudaMemcpy(dv + n, hy.data(), sizeof(double) * n, cudaMemcpyHostToDevice));
        }
        ok(cudaMemcpy(dacc, acc, sizeof(double) * 4 * K, cudaMemcpyHostToDevice));
        if (st == D4_OK) {
            const long long cells = (long long)n * K;
            if (cells > 0) {
                const int gb = (int)((cells + 255) / 256);
                k_xp_tables<<<gb, 256>>>(n, K, dv, ex);
                k_xp_tables<<<gb, 256>>>(n, K, dv + n, ey);
                g_launches.fetch_add(2, std::memory_order_relaxed);
            }
            const int tiles = (K + kXpTile - 1) / kXpTile;
            k_xp_gemm<<<dim3(tiles, tiles), 256>>>(n, npos, K, ex, ey, dnrm);
            k_xp_colsum<<<(4 * K + 255) / 256, 256>>>(K, dnrm, dacc);
            g_launches.fetch_add(2, std::memory_order_relaxed);
            ok(cudaGetLastError());
            ok(cudaMemcpy(acc, dacc, sizeof(double) * 4 * K, cudaMemcpyDeviceToHost));
        }
    }
    cudaFree(dv);
    cudaFree(ex);
    cudaFree(ey);
    cudaFree(dnrm);
    cudaFree(dacc);
    return st;
}
