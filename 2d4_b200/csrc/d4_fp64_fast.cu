// d4_fp64_fast.cu: the mixed form's FP64 pair tiles.  The pair tiles of
// d4_sweep64.cuh with the field of d4_field64_fast.cuh (one reciprocal per
// image, shared by the field and its derivative), compiled with product-add
// contraction; the row sums, row scaling and everything after them are the
// plain form's (d4_fp64.cu).
#include "d4_field64_fast.cuh"
#define D4_PAIR_FIELD f64fast
#include "d4_sweep64.cuh"

namespace d4 {

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
