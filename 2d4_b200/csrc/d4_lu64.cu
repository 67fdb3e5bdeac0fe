// d4_lu64.cu: FP64 solves with the LU factors of the plain form (--fmad=false).
//
// Replaces umfpack_di_solve (src/simulation.cpp:643-659) for the dense
// Jacobian, with the residual of each stage (src/simulation.cpp:101,123,142,621)
// built in the prologue and the position update x_new = x - dx in the epilogue.
// The factors come from d4_lu_coop64.cu.  The oracle's forward and backward
// substitution give every entry its updates one k at a time (forward: k
// ascending; backward: k descending, then the division), product and difference
// rounded separately; the wavefront below keeps that per-entry sequence, so the
// solution is bit-identical.
#include <cstdint>

#include "d4_trsv.cuh"

namespace d4 {
using trsv::GArgs;
using trsv::kWaveThreads;

static void launch_solve(Ctx &c, const GArgs &ga) {
    const int nblk = (c.n + 31) / 32;
    unsigned e1 = ++c.wave_epoch;
    unsigned e2 = ++c.wave_epoch;
    GArgs g = ga;
    const double *xin_null = nullptr;
    void *args1[] = {(void *)&c.n, (void *)&c.LU, (void *)&c.perm, (void *)&c.flags, (void *)&g,
                     (void *)&c.xw1, (void *)&xin_null, (void *)&c.wave_done, (void *)&e1,
                     (void *)&c.wave_err};
    const void *fwd = (const void *)trsv::k_trsv_wave<true, double>;
    const void *bwd = (const void *)trsv::k_trsv_wave<false, double>;
    D4_CUDA_OK(cudaLaunchCooperativeKernel(fwd, dim3(nblk), dim3(kWaveThreads), args1, 0, c.stream));
    check_launch("k_trsv_wave<fwd>");
    void *args2[] = {(void *)&c.n, (void *)&c.LU, (void *)&c.perm, (void *)&c.flags, (void *)&g,
                     (void *)&c.xw2, (void *)&c.xw1, (void *)&c.wave_done2, (void *)&e2,
                     (void *)&c.wave_err};
    D4_CUDA_OK(cudaLaunchCooperativeKernel(bwd, dim3(nblk), dim3(kWaveThreads), args2, 0, c.stream));
    check_launch("k_trsv_wave<bwd>");
}

void solve_update64(Ctx &c, int gmode, double hval, const double *s_end, const double *s_init,
                    const double *x_new, const double *x_old, const double *base, double *out) {
    GArgs ga{};
    ga.gmode = gmode;
    ga.hval = hval;
    ga.dvec = c.dvec;
    ga.s_end = s_end;
    ga.s_init = s_init;
    ga.x_new = x_new;
    ga.x_old = x_old;
    ga.base = base;
    ga.out = out;
    ga.dx_out = c.dx;
    ga.fix_singular = 1;
    launch_solve(c, ga);
}

void solve_plain64(Ctx &c, const double *g) {
    GArgs ga{};
    ga.gmode = -1;
    ga.g_in = g;
    ga.dx_out = c.dx;
    launch_solve(c, ga);
}

}  // namespace d4
