// d4_adjoint.cu: differentiation of a fixed sequence of accepted implicit steps.
//
// The forward map is the replay of accepted steps (t0_k, h_k): for each step
// the stages II and III of Simulation::run's attempt (src/simulation.cpp:
// 115-150) with the engine's FP64 kernels, so x2 is identical to d4_attempt's,
// then normalize (src/sim_utils.cpp:6-13, derivative 1).  Stage I only decides
// acceptance and is skipped.  Step sizes are constants (the adaptive control is
// not differentiated).  The loss is the accumulated strain sum_i b_i (x2 - x0)
// per step (src/simulation.cpp:713-720).
//
// Both stages are the same map S(z) with hh = h/2 and the stage's weights
// d = weight(-hh g(z)) with g = diag Jt, D = diag((1+d)/2), Dm = diag((1-d)/2),
// A = I - hh D Jt(z) (Jt: the engine's Jacobian, built from xy_diff_x):
//   x1 = z  - A^-1 q,  q = -hh [D v(z; tau_b) + Dm v(z; tau_a)]
//   x  = x1 - A^-1 r,  r = x1 - z - hh [D v(x1; tau_b) + Dm v(z; tau_a)]
// where Jv is the velocities' Jacobian (built from d xy / dx).  The derivative
// is exact for this discrete map: it includes the dependence of A and d on z,
// which needs d xy_diff_x / dx (d4_field_dual.cuh).  d4_tangent propagates a direction forward
// (tangent-linear); d4_adjoint runs the forward with positions checkpointed
// every K steps, then for each segment recomputes its steps storing the stage
// quantities and the transposed LU factors, and sweeps back with transposed
// solves A^T mu = lambda through those factors (P A = L U:
// A^T = U^T L^T P), run by the cluster solve of d4_trsv.cuh.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <functional>
#include <vector>

#include "d4_field_dual.cuh"
#include "d4_internal.h"
#include "d4_trsv.cuh"

namespace d4 {
namespace adj {

__device__ __forceinline__ double bsg(int i, int n) { return i < n / 2 ? 1.0 : -1.0; }

inline int nb(long long n, int t) { return (int)((n + t - 1) / t); }

// ---- pair reductions with the field's first and second x-derivatives ----
//
// Two Jacobians enter.  Jv, the velocities' Jacobian, uses sp = d xy / dx
// (even in the pair's orientation).  Jt, the engine's implicit-step matrix
// A = I - hh D Jt and its diagonal g (the weights' argument), uses
// st = xy_diff_x evaluated as the engine does, at x_p - x_q with p < q, and its
// position derivative tt = +-d xy_diff_x / dx at that orientation (sign + for
// row p), so Jt is exactly symmetric and tt exactly antisymmetric in (i, j):
//   (Jv u)_i = sum_j b_i b_j sp_ij (u_i - u_j),  (Jt u)_i = sum_j b_i b_j st_ij (u_i - u_j)
//   d g_i = sum_j b_i b_j tt_ij (dz_i - dz_j),
//   (dJt[dz] w)_i = sum_j b_i b_j tt_ij (dz_i - dz_j)(w_i - w_j).
enum { kModeJv = 0, kModeJt = 1, kModeJvp = 2, kModeVjp = 3 };
constexpr int kPT = 128;

struct DerivArgs {
    int n;
    const double *x, *y;
    const double *a, *c;          // first-order inputs
    const double *p, *q, *r, *s;  // second-order pair inputs
    const double *u;              // second-order sum input
    double *o[6];
};

// kModeJv:  o0 = Jv a, o1 = Jv c (c may be null)
// kModeJt:  o0 = Jt a, o1 = Jt c (c may be null)
// kModeJvp: o0 = Jv a, o1 = sum bb tt (a_i - a_j), o2 = sum bb tt (a_i - a_j)(q_i - q_j),
//           o3 = sum bb tt (a_i - a_j)(r_i - r_j), o4 = Jt q, o5 = Jt r
// kModeVjp: o0 = sum bb [sp (a_i - a_j) + tt ((p_i - p_j)(q_i - q_j)
//                         + (r_i - r_j)(s_i - s_j) + (u_i + u_j))]
// Grid: (row tiles, column tiles) of kPT x kPT pairs; block (bx, by) sums the
// pairs of its rows with the columns of tile by and writes the partial sums to
// part[(out * tiles + by) * n + i]; k_deriv_sum then adds the tiles in order
// (deterministic results).
template <int kMode>
__global__ void __launch_bounds__(kPT) k_deriv(DerivArgs A, double *part) {
    __shared__ double sx[kPT], sy[kPT], s1[kPT], s2[kPT], s3[kPT], s4[kPT], s5[kPT], s6[kPT];
    const int n = A.n;
    const int i = blockIdx.x * kPT + threadIdx.x;
    const bool own = i < n;
    const double xi = own ? A.x[i] : 0, yi = own ? A.y[i] : 0, bi = bsg(i, n);
    double ai = 0, ci = 0, pi = 0, qi = 0, ri = 0, si = 0, ui = 0;
    if (own) {
        ai = A.a ? A.a[i] : 0;
        if (kMode == kModeJv || kMode == kModeJt) ci = A.c ? A.c[i] : 0;
        if (kMode == kModeJvp) {
            qi = A.q[i];
            ri = A.r[i];
        }
        if (kMode == kModeVjp) {
            pi = A.p[i];
            qi = A.q[i];
            ri = A.r[i];
            si = A.s[i];
            ui = A.u[i];
        }
    }
    double o[6] = {0, 0, 0, 0, 0, 0};
    {
        const int j0 = blockIdx.y * kPT;
        const int j = j0 + threadIdx.x;
        if (j < n) {
            sx[threadIdx.x] = A.x[j];
            sy[threadIdx.x] = A.y[j];
            s1[threadIdx.x] = A.a ? A.a[j] : 0;
            if (kMode == kModeJv || kMode == kModeJt) s2[threadIdx.x] = A.c ? A.c[j] : 0;
            if (kMode == kModeJvp) {
                s2[threadIdx.x] = A.q[j];
                s3[threadIdx.x] = A.r[j];
            }
            if (kMode == kModeVjp) {
                s2[threadIdx.x] = A.p[j];
                s3[threadIdx.x] = A.q[j];
                s4[threadIdx.x] = A.r[j];
                s5[threadIdx.x] = A.s[j];
                s6[threadIdx.x] = A.u[j];
            }
        }
        __syncthreads();
        const int jn = own ? min(kPT, n - j0) : 0;
        for (int t = 0; t < jn; ++t) {
            const int jj = j0 + t;
            if (jj == i) continue;
            const double bb = bi * bsg(jj, n);
            const double dx = f64::normalize(xi - sx[t]);
            const double dy = f64::normalize(yi - sy[t]);
            // the engine's orientation of the pair (lower index first)
            const bool lo = i < jj;
            const double dxo = lo ? dx : f64::normalize(sx[t] - xi);
            const double dyo = lo ? dy : f64::normalize(sy[t] - yi);
            if (kMode == kModeJv) {
                const double sp = dual::xy(dx, dy).d * bb;
                o[0] += sp * (ai - s1[t]);
                o[1] += sp * (ci - s2[t]);
            } else if (kMode == kModeJt) {
                const f64::Hyp h(f64::exp2pix(dxo));
                const double st = f64::xy_diff_x(dxo, dyo, h, f64::cos2piy(dyo)) * bb;
                o[0] += st * (ai - s1[t]);
                o[1] += st * (ci - s2[t]);
            } else {
                const dual::D ft = dual::xy_diff_x(dxo, dyo);
                const double st = ft.v * bb, tt = (lo ? ft.d : -ft.d) * bb;
                if (kMode == kModeJvp) {
                    const double sp = dual::xy(dx, dy).d * bb;
                    const double da = ai - s1[t];
                    o[0] += sp * da;
                    o[1] += tt * da;
                    o[2] += tt * da * (qi - s2[t]);
                    o[3] += tt * da * (ri - s3[t]);
                    o[4] += st * (qi - s2[t]);
                    o[5] += st * (ri - s3[t]);
                } else {
                    const double sp = dual::xy(dx, dy).d * bb;
                    o[0] += sp * (ai - s1[t]) +
                            tt * ((pi - s2[t]) * (qi - s3[t]) + (ri - s4[t]) * (si - s5[t]) +
                                  (ui + s6[t]));
                }
            }
        }
    }
    if (!own) return;
    const int nout = (kMode == kModeJv || kMode == kModeJt) ? (A.o[1] ? 2 : 1)
                     : kMode == kModeJvp                   ? 6
                                                           : 1;
    for (int k = 0; k < nout; ++k) part[((size_t)k * gridDim.y + blockIdx.y) * n + i] = o[k];
}

__global__ void k_deriv_sum(int n, int tiles, int nout, const double *part, DerivArgs A) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    for (int k = 0; k < nout; ++k) {
        double v = 0;
        for (int t = 0; t < tiles; ++t) v += part[((size_t)k * tiles + t) * n + i];
        A.o[k][i] = v;
    }
}

// Launches k_deriv<kMode> over all pair tiles and the in-order tile sum.
template <int kMode>
void run_deriv(Ctx &c, DerivArgs &A, double *part) {
    const int tiles = nb(c.n, kPT);
    const int nout = (kMode == kModeJv || kMode == kModeJt) ? (A.o[1] ? 2 : 1)
                     : kMode == kModeJvp                   ? 6
                                                           : 1;
    k_deriv<kMode><<<dim3(tiles, tiles), kPT, 0, c.stream>>>(A, part);
    check_launch("k_deriv");
    k_deriv_sum<<<nb(c.n, 256), 256, 0, c.stream>>>(c.n, tiles, nout, part, A);
    check_launch("k_deriv_sum");
}

// Transposed solve A^T mu = lam with the factors stored transposed (Lt) and
// perm (P A = L U), by the cluster solve in its transposed mode.
void trsv_t(Ctx &c, const double *Lt, const int *perm, const double *lam, double *mu,
            double *scratch) {
    trsv::GArgs g{};
    g.gmode = -1;
    g.g_in = lam;
    trsv::launch_cluster_solve<double, true>(c.n, Lt, perm, c.flags, g, scratch, mu, c.wave_err,
                                             c.stream);
}

__global__ void k_transpose(int n, const double *__restrict__ a, double *__restrict__ t) {
    __shared__ double tile[32][33];
    const int bx = blockIdx.x * 32, by = blockIdx.y * 32;
    for (int k = threadIdx.y; k < 32; k += 8) {
        const int r = bx + threadIdx.x, c = by + k;
        if (r < n && c < n) tile[k][threadIdx.x] = a[(size_t)r + (size_t)c * n];
    }
    __syncthreads();
    for (int k = threadIdx.y; k < 32; k += 8) {
        const int r = by + threadIdx.x, c = bx + k;
        if (r < n && c < n) t[(size_t)r + (size_t)c * n] = tile[threadIdx.x][k];
    }
}

// d weight / d s at s = weightInv(d) (src/sim_utils.cpp:36-75); 0 where d = 0.
__device__ __forceinline__ double wprime(double d, char t) {
    if (!(d > 0)) return 0;
    const double s = f64::weight_inv(d, t);
    if (t == 'c') return 2 * s / ((s + 1) * (s + 1) * (s + 1));
    if (t == 'p') return 1 / ((s + 1) * (s + 1));
    const double c = 0.412073, u = s + c * s * s, den = u + 1.5;
    return 1.5 * (1 + 2 * c * s) / (den * den);
}

struct StageCoef {
    double hh, rho_a, rho_b;  // hh = h/2; d tau / d tau0 at the stage's two times
    char wfn;
};

// Adjoint, after mu2 = A^-T lam_out and w1 = Jv(x1) (D mu2):
// lam_x1 = lam_out - mu2 + hh w1.
__global__ void k_adj_x1(int n, StageCoef k, const double *lam_out, const double *mu2,
                         const double *w1, double *lam_x1) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) lam_x1[i] = lam_out[i] - mu2[i] + k.hh * w1[i];
}

__global__ void k_scale_d(int n, const double *d, const double *v, double *out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] = (1 + d[i]) / 2 * v[i];
}

// Adjoint, after mu1 = A^-T lam_x1 and Jv(z) D1, Jv(z) D2: the inputs of the
// z-pair sweep (a, q = -hh D mu2, s = -hh D mu1, u = -hh w' c_d) and the
// stage's d L / d tau0 (one CTA; added to *gtau).
__global__ void __launch_bounds__(1024) k_adj_z(int n, StageCoef k, const double *d,
                                                const double *mu1, const double *mu2,
                                                const double *va, const double *vb,
                                                const double *v1b, const double *jd1,
                                                const double *jd2, double *a, double *q,
                                                double *s, double *u, double *gtau) {
    __shared__ double red[32];
    double acc = 0;
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        const double D = (1 + d[i]) / 2, Dm = (1 - d[i]) / 2;
        const double m1 = mu1[i], m2 = mu2[i];
        const double cd = k.hh * (m2 / 2 * (v1b[i] - va[i]) - m2 / 2 * jd2[i] +
                                  m1 / 2 * (vb[i] - va[i]) - m1 / 2 * jd1[i]);
        a[i] = k.hh * (Dm * m2 + m1);
        q[i] = -k.hh * D * m2;
        s[i] = -k.hh * D * m1;
        u[i] = -k.hh * wprime(d[i], k.wfn) * cd;
        acc += k.hh * bsg(i, n) * (k.rho_b * D + k.rho_a * Dm) * (m1 + m2);
    }
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += red[w];
        *gtau += t;
    }
}

// lam_z = mu2 + lam_x1 + o (the z-pair sweep's output).
__global__ void k_adj_out(int n, const double *mu2, const double *lam_x1, const double *o,
                          double *lam_z) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) lam_z[i] = mu2[i] + lam_x1[i] + o[i];
}

// lam = b + lam_next (the strain's d/dx2 plus the later steps').
__global__ void k_adj_seed(int n, const double *lam_next, double *lam) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) lam[i] = bsg(i, n) + lam_next[i];
}

// lam_next = lam_x0 - b (the strain's d/dx0).
__global__ void k_adj_step_end(int n, const double *lam_x0, double *lam_next) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) lam_next[i] = lam_x0[i] - bsg(i, n);
}

// Tangent-linear, first solve's right-hand side: dq - dA D1 with
// dd = w' (-hh dg).  o: the z-pair sweep (Jv dz, dg, H[dz] D1, H[dz] D2, Jv D1, Jv D2).
__global__ void k_tl_rhs1(int n, StageCoef k, double dtau, const double *d, const double *va,
                          const double *vb, const double *o0, const double *o1,
                          const double *o2, const double *o4, double *dd, double *rhs) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double D = (1 + d[i]) / 2, Dm = (1 - d[i]) / 2, b = bsg(i, n);
    const double ddi = wprime(d[i], k.wfn) * (-k.hh * o1[i]);
    dd[i] = ddi;
    const double dq =
        -k.hh * (ddi / 2 * (vb[i] - va[i]) + o0[i] + dtau * (k.rho_b * D + k.rho_a * Dm) * b);
    const double dAD1 = -k.hh * (ddi / 2 * o4[i] + D * o2[i]);
    rhs[i] = dq - dAD1;
}

// Tangent-linear, second solve's right-hand side: dr - dA D2.
__global__ void k_tl_rhs2(int n, StageCoef k, double dtau, const double *d, const double *va,
                          const double *v1b, const double *dz, const double *dx1,
                          const double *jx1, const double *o0, const double *o3,
                          const double *o5, const double *dd, double *rhs) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double D = (1 + d[i]) / 2, Dm = (1 - d[i]) / 2, b = bsg(i, n);
    const double dr = dx1[i] - dz[i] -
                      k.hh * (dd[i] / 2 * (v1b[i] - va[i]) + D * jx1[i] + Dm * o0[i] +
                              dtau * (k.rho_b * D + k.rho_a * Dm) * b);
    const double dAD2 = -k.hh * (dd[i] / 2 * o5[i] + D * o3[i]);
    rhs[i] = dr - dAD2;
}

__global__ void k_sub(int n, const double *a, const double *b, double *out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] = a[i] - b[i];
}

// out = sum_i b_i (x_i - y_i), one CTA.
__global__ void __launch_bounds__(1024) k_bdot(int n, const double *x, const double *y,
                                               double *out) {
    __shared__ double red[32];
    double acc = 0;
    for (int i = threadIdx.x; i < n; i += blockDim.x) acc += bsg(i, n) * (x[i] - y[i]);
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += red[w];
        *out += t;
    }
}

// Device pointers of one stage, valid during the stage hook.
struct Stage {
    const double *z, *x1, *d1, *d2, *d, *va, *vb, *v1b;
    StageCoef k;
};

// Work space of the differentiation calls (freed on destruction).
struct Work {
    std::vector<void *> bufs;
    double *alloc(size_t count) {
        void *p = nullptr;
        D4_CUDA_OK(d4::dmalloc(&p, sizeof(double) * (count ? count : 1)));
        bufs.push_back(p);
        return static_cast<double *>(p);
    }
    int *ialloc(size_t count) {
        void *p = nullptr;
        D4_CUDA_OK(d4::dmalloc(&p, sizeof(int) * (count ? count : 1)));
        bufs.push_back(p);
        return static_cast<int *>(p);
    }
    ~Work() {
        for (void *p : bufs) cudaFree(p);
    }
};

// d tau_ext(t) / d tau0 of the protocol (src/stress_protocol.cpp:13-73).
double dtau_dtau0(const d4_protocol &p, double t) {
    switch (p.kind) {
    case D4_STRESS_FIXED_RATE:
        return 1;
    case D4_STRESS_CYCLIC:
    case D4_STRESS_INC_CYCLIC: {
        const double periodic = t - std::floor((t / p.period + 1. / 4)) * p.period;
        const double r = periodic > p.period / 4 ? 0.0 : 1.0;  // tau0 cancels on the way down
        return p.kind == D4_STRESS_INC_CYCLIC ? r * p.amplitude_rate * t : r;
    }
    default:
        return 0;
    }
}

// One accepted step replayed from c.x0 (stages II and III as attempt() runs
// them), x0 <- normalize(x2); strain increments added to *strain_dev.  The hook
// sees each stage after its second solve, while c.LU holds its factors.
struct Replay {
    Ctx &c;
    const d4_protocol &pr;
    double *sX1, *sD1, *sD2, *sVB, *sV1B;
    explicit Replay(Ctx &cc, const d4_protocol &p, Work &w) : c(cc), pr(p) {
        sX1 = w.alloc(c.n);
        sD1 = w.alloc(c.n);
        sD2 = w.alloc(c.n);
        sVB = w.alloc(c.n);
        sV1B = w.alloc(c.n);
    }
    void copy(double *dst, const double *src) {
        D4_CUDA_OK(cudaMemcpyAsync(dst, src, sizeof(double) * c.n, cudaMemcpyDeviceToDevice,
                                   c.stream));
    }
    void step(double t0, double h, double *strain_dev,
              const std::function<void(int, const Stage &)> &hook) {
        const double t1 = t0 + h, th = t0 + h / 2;
        const double e0 = ext_stress_host(pr, t0), e1 = ext_stress_host(pr, t1),
                     eh = ext_stress_host(pr, th);
        const char wfn = c.p.weight_function;
        // stage II
        jacobian64(c, c.x0, c.y, h, e0, e1, c.v_init, c.speed);
        jacobian_from_prev64(c, (th - t0) / (t1 - t0));
        factor64(c);
        shift_speed64(c, c.speed, eh - e1);
        solve_update64(c, kGHalf, h, c.speed, c.v_init, nullptr, nullptr, c.x0, c.xh);
        copy(sX1, c.xh);
        copy(sD1, c.dx);
        speeds64(c, c.xh, c.y, eh, c.speed2);
        copy(sV1B, c.speed2);
        solve_update64(c, kGNewton, h / 2, c.speed2, c.v_init, c.xh, c.x0, c.xh, c.xh);
        copy(sD2, c.dx);
        if (hook) {
            Stage s{c.x0, sX1, sD1, sD2, c.dvec, c.v_init, c.speed, sV1B,
                    StageCoef{h / 2, dtau_dtau0(pr, t0), dtau_dtau0(pr, th), wfn}};
            hook(0, s);
        }
        // stage III
        jacobian64(c, c.xh, c.y, h / 2, eh, e1, c.v_init2, c.speed2);
        factor64(c);
        copy(sVB, c.speed2);
        solve_update64(c, kGHalf, h, c.speed2, c.v_init2, nullptr, nullptr, c.xh, c.x2);
        copy(sX1, c.x2);
        copy(sD1, c.dx);
        speeds64(c, c.x2, c.y, e1, c.speed2);
        copy(sV1B, c.speed2);
        solve_update64(c, kGNewton, h / 2, c.speed2, c.v_init2, c.x2, c.xh, c.x2, c.x2);
        copy(sD2, c.dx);
        if (hook) {
            Stage s{c.xh, sX1, sD1, sD2, c.dvec, c.v_init2, sVB, sV1B,
                    StageCoef{h / 2, dtau_dtau0(pr, th), dtau_dtau0(pr, t1), wfn}};
            hook(1, s);
        }
        if (strain_dev) {
            k_bdot<<<1, 1024, 0, c.stream>>>(c.n, c.xh, c.x0, strain_dev);
            check_launch("k_bdot");
            k_bdot<<<1, 1024, 0, c.stream>>>(c.n, c.x2, c.xh, strain_dev);
            check_launch("k_bdot");
        }
        normalize64(c, c.x0, c.x2);
    }
};

// o0 = J a, o1 = J cc (cc may be null) for J = Jv (velocities) or Jt (matrix).
template <int kMode>
void deriv_j(Ctx &c, double *part, const double *x, const double *a, const double *cc,
             double *o0, double *o1) {
    DerivArgs A{};
    A.n = c.n;
    A.x = x;
    A.y = c.y;
    A.a = a;
    A.c = cc;
    A.o[0] = o0;
    A.o[1] = o1;
    run_deriv<kMode>(c, A, part);
}

// Validates the context for differentiation: FP64 analytic field with every
// pair inside the Jacobian's range (no cutoff), so Jv is the full Jacobian.
void require_differentiable(const Ctx &c) {
    if (c.p.precision != D4_PREC_FP64 || c.tab || c.use_gmres)
        throw StateError("differentiation needs the FP64 form, analytic field, dense solver");
    if (!(c.range_sq * c.cutoff_sq > 0.5))
        throw StateError("differentiation needs no distant-pair cutoff");
}

// Saves and restores the context's positions and tolerances around a call.
struct Keep {
    Ctx &c;
    double *x0, *tol;
    Keep(Ctx &cc, Work &w) : c(cc) {
        x0 = w.alloc(c.n);
        tol = w.alloc(c.n);
        D4_CUDA_OK(cudaMemcpyAsync(x0, c.x0, sizeof(double) * c.n, cudaMemcpyDeviceToDevice,
                                   c.stream));
        D4_CUDA_OK(cudaMemcpyAsync(tol, c.tol, sizeof(double) * c.n, cudaMemcpyDeviceToDevice,
                                   c.stream));
    }
    ~Keep() {
        cudaMemcpyAsync(c.x0, x0, sizeof(double) * c.n, cudaMemcpyDeviceToDevice, c.stream);
        cudaMemcpyAsync(c.tol, tol, sizeof(double) * c.n, cudaMemcpyDeviceToDevice, c.stream);
        cudaStreamSynchronize(c.stream);
    }
};

}  // namespace adj
}  // namespace d4

namespace {

using d4::Ctx;
using namespace d4::adj;

int guard(Ctx *c, const std::function<int()> &f) {
    try {
        return f();
    } catch (const d4::CudaError &e) {
        c->err = e.what;
        return D4_ERR_CUDA;
    } catch (const d4::StateError &e) {
        c->err = e.what;
        return D4_ERR_STATE;
    } catch (const std::bad_alloc &) {
        c->err = "host allocation failed";
        return D4_ERR_NOMEM;
    }
}

}  // namespace

extern "C" {

int d4_replay(void *ctx, long long steps, const double *t0s, const double *hs,
              const d4_protocol *proto, const double *x0, double *x_end, double *strain) {
    Ctx *c = (Ctx *)ctx;
    if (!c || steps < 0 || (steps > 0 && (!t0s || !hs)) || !x0) return D4_ERR_ARG;
    return guard(c, [&]() {
        require_differentiable(*c);
        const d4_protocol &pr = proto ? *proto : c->p.protocol;
        Work w;
        Keep keep(*c, w);
        double *sd = w.alloc(1);
        D4_CUDA_OK(cudaMemsetAsync(sd, 0, sizeof(double), c->stream));
        D4_CUDA_OK(cudaMemcpyAsync(c->x0, x0, sizeof(double) * c->n, cudaMemcpyHostToDevice,
                                   c->stream));
        Replay rp(*c, pr, w);
        for (long long k = 0; k < steps; ++k) rp.step(t0s[k], hs[k], sd, nullptr);
        if (x_end)
            D4_CUDA_OK(cudaMemcpyAsync(x_end, c->x0, sizeof(double) * c->n,
                                       cudaMemcpyDeviceToHost, c->stream));
        double s = 0;
        D4_CUDA_OK(cudaMemcpyAsync(&s, sd, sizeof(double), cudaMemcpyDeviceToHost, c->stream));
        D4_CUDA_OK(cudaStreamSynchronize(c->stream));
        if (strain) *strain = s;
        return D4_OK;
    });
}

int d4_tangent(void *ctx, long long steps, const double *t0s, const double *hs,
               const d4_protocol *proto, const double *x0, const double *dx0, double dtau0,
               double *strain, double *dstrain) {
    Ctx *c = (Ctx *)ctx;
    if (!c || steps < 0 || (steps > 0 && (!t0s || !hs)) || !x0 || !dx0 || !dstrain)
        return D4_ERR_ARG;
    return guard(c, [&]() {
        require_differentiable(*c);
        const d4_protocol &pr = proto ? *proto : c->p.protocol;
        const int n = c->n;
        Work w;
        Keep keep(*c, w);
        double *sd = w.alloc(2);  // [0] strain, [1] its derivative
        D4_CUDA_OK(cudaMemsetAsync(sd, 0, 2 * sizeof(double), c->stream));
        D4_CUDA_OK(cudaMemcpyAsync(c->x0, x0, sizeof(double) * n, cudaMemcpyHostToDevice,
                                   c->stream));
        double *dz = w.alloc(n), *dzs = w.alloc(n), *dx1 = w.alloc(n), *dd = w.alloc(n),
               *rhs = w.alloc(n), *jx1 = w.alloc(n);
        double *part = w.alloc((size_t)6 * nb(n, kPT) * n);
        double *o[6];
        for (double *&p : o) p = w.alloc(n);
        D4_CUDA_OK(cudaMemcpyAsync(dz, dx0, sizeof(double) * n, cudaMemcpyHostToDevice,
                                   c->stream));
        Replay rp(*c, pr, w);
        auto hook = [&](int stage, const Stage &s) {
            if (stage == 0)  // start of the step: keep dx0 for the strain
                D4_CUDA_OK(cudaMemcpyAsync(dzs, dz, sizeof(double) * n,
                                           cudaMemcpyDeviceToDevice, c->stream));
            DerivArgs A{};
            A.n = n;
            A.x = s.z;
            A.y = c->y;
            A.a = dz;
            A.q = s.d1;
            A.r = s.d2;
            for (int k = 0; k < 6; ++k) A.o[k] = o[k];
            run_deriv<kModeJvp>(*c, A, part);
            k_tl_rhs1<<<nb(n, 256), 256, 0, c->stream>>>(n, s.k, dtau0, s.d, s.va, s.vb, o[0],
                                                          o[1], o[2], o[4], dd, rhs);
            d4::check_launch("k_tl_rhs1");
            d4::solve_plain64(*c, rhs);
            k_sub<<<nb(n, 256), 256, 0, c->stream>>>(n, dz, c->dx, dx1);
            d4::check_launch("k_sub");
            deriv_j<kModeJv>(*c, part, s.x1, dx1, nullptr, jx1, nullptr);
            k_tl_rhs2<<<nb(n, 256), 256, 0, c->stream>>>(n, s.k, dtau0, s.d, s.va, s.v1b, dz,
                                                          dx1, jx1, o[0], o[3], o[5], dd, rhs);
            d4::check_launch("k_tl_rhs2");
            d4::solve_plain64(*c, rhs);
            k_sub<<<nb(n, 256), 256, 0, c->stream>>>(n, dx1, c->dx, dz);
            d4::check_launch("k_sub");
            if (stage == 1) {
                k_bdot<<<1, 1024, 0, c->stream>>>(n, dz, dzs, sd + 1);
                d4::check_launch("k_bdot");
            }
        };
        for (long long k = 0; k < steps; ++k) rp.step(t0s[k], hs[k], sd, hook);
        double r[2];
        D4_CUDA_OK(cudaMemcpyAsync(r, sd, sizeof(r), cudaMemcpyDeviceToHost, c->stream));
        D4_CUDA_OK(cudaStreamSynchronize(c->stream));
        if (strain) *strain = r[0];
        *dstrain = r[1];
        return D4_OK;
    });
}

int d4_adjoint(void *ctx, long long steps, const double *t0s, const double *hs,
               const d4_protocol *proto, int checkpoint_every, const double *x0, double *strain,
               double *grad_x0, double *grad_tau0) {
    Ctx *c = (Ctx *)ctx;
    if (!c || steps < 0 || (steps > 0 && (!t0s || !hs)) || !x0 || !grad_x0 ||
        checkpoint_every <= 0)
        return D4_ERR_ARG;
    return guard(c, [&]() {
        require_differentiable(*c);
        const d4_protocol &pr = proto ? *proto : c->p.protocol;
        const int n = c->n;
        const size_t nn = (size_t)n * n;
        const int K = (int)std::min<long long>(checkpoint_every, std::max<long long>(steps, 1));
        const long long nseg = (steps + K - 1) / K;
        Work w;
        Keep keep(*c, w);
        double *sd = w.alloc(2);  // [0] strain, [1] d strain / d tau0
        D4_CUDA_OK(cudaMemsetAsync(sd, 0, 2 * sizeof(double), c->stream));
        D4_CUDA_OK(cudaMemcpyAsync(c->x0, x0, sizeof(double) * n, cudaMemcpyHostToDevice,
                                   c->stream));
        double *ckpt = w.alloc((size_t)std::max<long long>(nseg, 1) * n);
        // tape: per step and stage 8 vectors, the transposed LU factors, perm
        enum { tZ, tX1, tD1, tD2, tD, tVA, tVB, tV1B, tNum };
        double *tvec = w.alloc((size_t)K * 2 * tNum * n);
        double *tlu = w.alloc((size_t)K * 2 * nn);
        int *tperm = w.ialloc((size_t)K * 2 * n);
        std::vector<StageCoef> tk((size_t)K * 2);
        Replay rp(*c, pr, w);
        // forward with checkpoints
        for (long long k = 0; k < steps; ++k) {
            if (k % K == 0)
                D4_CUDA_OK(cudaMemcpyAsync(ckpt + (size_t)(k / K) * n, c->x0,
                                           sizeof(double) * n, cudaMemcpyDeviceToDevice,
                                           c->stream));
            rp.step(t0s[k], hs[k], sd, nullptr);
        }
        // backward, segment by segment
        double *lam_next = w.alloc(n), *lam = w.alloc(n), *mu1 = w.alloc(n), *mu2 = w.alloc(n),
               *dmu = w.alloc(n), *w1 = w.alloc(n), *lx1 = w.alloc(n), *jd1 = w.alloc(n),
               *jd2 = w.alloc(n), *ea = w.alloc(n), *eq = w.alloc(n), *es = w.alloc(n),
               *eu = w.alloc(n), *oz = w.alloc(n);
        double *part = w.alloc((size_t)6 * nb(n, kPT) * n);
        D4_CUDA_OK(cudaMemsetAsync(lam_next, 0, sizeof(double) * n, c->stream));
        double *tsc = w.alloc(n);  // forward-pass result of the transposed solves
        for (long long seg = nseg - 1; seg >= 0; --seg) {
            const long long k0 = seg * K, k1 = std::min<long long>(steps, k0 + K);
            D4_CUDA_OK(cudaMemcpyAsync(c->x0, ckpt + (size_t)seg * n, sizeof(double) * n,
                                       cudaMemcpyDeviceToDevice, c->stream));
            for (long long k = k0; k < k1; ++k) {
                const size_t slot0 = (size_t)(k - k0) * 2;
                auto hook = [&](int stage, const Stage &s) {
                    const size_t slot = slot0 + stage;
                    double *v = tvec + slot * tNum * n;
                    const double *src[tNum] = {s.z, s.x1, s.d1, s.d2, s.d, s.va, s.vb, s.v1b};
                    for (int q = 0; q < tNum; ++q) rp.copy(v + (size_t)q * n, src[q]);
                    k_transpose<<<dim3(nb(n, 32), nb(n, 32)), dim3(32, 8), 0, c->stream>>>(
                        n, c->LU, tlu + slot * nn);
                    d4::check_launch("k_transpose");
                    D4_CUDA_OK(cudaMemcpyAsync(tperm + slot * n, c->perm, sizeof(int) * n,
                                               cudaMemcpyDeviceToDevice, c->stream));
                    tk[slot] = s.k;
                };
                rp.step(t0s[k], hs[k], nullptr, hook);
            }
            for (long long k = k1 - 1; k >= k0; --k) {
                k_adj_seed<<<nb(n, 256), 256, 0, c->stream>>>(n, lam_next, lam);
                d4::check_launch("k_adj_seed");
                for (int stage = 1; stage >= 0; --stage) {
                    const size_t slot = (size_t)(k - k0) * 2 + stage;
                    const double *v = tvec + slot * tNum * n;
                    const double *Z = v + tZ * n, *X1 = v + tX1 * n, *D1 = v + tD1 * n,
                                 *D2 = v + tD2 * n, *Dv = v + tD * n, *VA = v + tVA * n,
                                 *VB = v + tVB * n, *V1B = v + tV1B * n;
                    const double *Lt = tlu + slot * nn;
                    const int *pm = tperm + slot * n;
                    const StageCoef &kc = tk[slot];
                    // mu2 = A^-T lam; lam_x1 = lam - mu2 + hh Jv(x1) (D mu2)
                    trsv_t(*c, Lt, pm, lam, mu2, tsc);
                    k_scale_d<<<nb(n, 256), 256, 0, c->stream>>>(n, Dv, mu2, dmu);
                    d4::check_launch("k_scale_d");
                    deriv_j<kModeJv>(*c, part, X1, dmu, nullptr, w1, nullptr);
                    k_adj_x1<<<nb(n, 256), 256, 0, c->stream>>>(n, kc, lam, mu2, w1, lx1);
                    d4::check_launch("k_adj_x1");
                    // mu1 = A^-T lam_x1
                    trsv_t(*c, Lt, pm, lx1, mu1, tsc);
                    // z sweep
                    deriv_j<kModeJt>(*c, part, Z, D1, D2, jd1, jd2);
                    k_adj_z<<<1, 1024, 0, c->stream>>>(n, kc, Dv, mu1, mu2, VA, VB, V1B, jd1,
                                                       jd2, ea, eq, es, eu, sd + 1);
                    d4::check_launch("k_adj_z");
                    DerivArgs A{};
                    A.n = n;
                    A.x = Z;
                    A.y = c->y;
                    A.a = ea;
                    A.p = D2;
                    A.q = eq;
                    A.r = D1;
                    A.s = es;
                    A.u = eu;
                    A.o[0] = oz;
                    run_deriv<kModeVjp>(*c, A, part);
                    k_adj_out<<<nb(n, 256), 256, 0, c->stream>>>(n, mu2, lx1, oz, lam);
                    d4::check_launch("k_adj_out");
                }
                k_adj_step_end<<<nb(n, 256), 256, 0, c->stream>>>(n, lam, lam_next);
                d4::check_launch("k_adj_step_end");
            }
        }
        double r[2];
        D4_CUDA_OK(cudaMemcpyAsync(grad_x0, lam_next, sizeof(double) * n, cudaMemcpyDeviceToHost,
                                   c->stream));
        D4_CUDA_OK(cudaMemcpyAsync(r, sd, sizeof(r), cudaMemcpyDeviceToHost, c->stream));
        D4_CUDA_OK(cudaStreamSynchronize(c->stream));
        if (strain) *strain = r[0];
        if (grad_tau0) *grad_tau0 = r[1];
        return D4_OK;
    });
}

}  // extern "C"
