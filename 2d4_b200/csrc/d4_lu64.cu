// d4_lu64.cu: FP64 solves with the LU factors of the plain form (--fmad=false).
//
// Replaces umfpack_di_solve (src/simulation.cpp:643-659) for the dense
// Jacobian, with the residual of each stage (src/simulation.cpp:101,123,142,621)
// built in the prologue and the position update x_new = x - dx in the epilogue.
// The factors come from d4_lu_coop64.cu.  The oracle's forward and backward
// substitution give every entry its updates one k at a time (forward: k
// ascending; backward: k descending, then the division), product and difference
// rounded separately; the cluster solve of d4_trsv.cuh keeps that per-entry
// sequence, so the solution is bit-identical.
#include <cstdint>

#include "d4_trsv.cuh"

namespace d4 {
using trsv::GArgs;

static void launch_solve(Ctx &c, const GArgs &ga) {
    trsv::launch_cluster_solve<double>(c.n, c.LU, c.perm, c.flags, ga, c.xw1, c.xw2, c.wave_err,
                                       c.stream);
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

void solve_update64_with(Ctx &c, const LuBufs &L, const SolveBufs &S, cudaStream_t st, int gmode,
                         double hval, const double *s_end, const double *s_init,
                         const double *x_new, const double *x_old, const double *base,
                         double *out) {
    GArgs ga{};
    ga.gmode = gmode;
    ga.hval = hval;
    ga.dvec = S.dvec;
    ga.s_end = s_end;
    ga.s_init = s_init;
    ga.x_new = x_new;
    ga.x_old = x_old;
    ga.base = base;
    ga.out = out;
    ga.dx_out = S.dx;
    ga.fix_singular = 1;
    trsv::launch_cluster_solve<double>(c.n, L.LU, L.perm, L.flags, ga, S.xw1, S.xw2, c.wave_err,
                                       st);
}

void solve_plain64(Ctx &c, const double *g) {
    GArgs ga{};
    ga.gmode = -1;
    ga.g_in = g;
    ga.dx_out = c.dx;
    launch_solve(c, ga);
}

}  // namespace d4
