// d4_lu_coop64.cu: FP64 LU with partial pivoting as one persistent kernel
// (compiled with --fmad=false).
//
// Same result, bit for bit, as the oracle's right-looking Gaussian elimination
// with partial pivoting (first index of the largest |a_ik| wins; an exact zero
// pivot skips its column and marks the matrix singular), which stands in for
// umfpack_di_numeric (src/simulation.cpp:635-640).  Every entry keeps its
// update sequence: a_ij -= l_ik * u_kj for k ascending, product and difference
// rounded separately.
//
// Schedule.  The matrix is processed in 32-column blocks by all CTAs of a
// cooperative launch:
//   pass   every CTA eliminates the block's 32 columns for its rows below the
//          diagonal block, WITHOUT pivoting, starting from a saved copy P0 of
//          the block's columns with the swaps found so far applied.  The 32x32
//          diagonal block of a block's first pass was eliminated and published
//          by the previous update's look-ahead; for block 0 and for passes
//          after a swap every CTA eliminates it redundantly in shared memory.
//          Pre-division values go to Q; a 32-bit mask records the columns
//          where partial pivoting would have swapped (some |a_ik| > |a_kk|) or
//          met a zero pivot.  A grid barrier ends the pass.
//   decide every CTA reads the mask.  Empty: the pass is exact, go on.
//          Otherwise the first flagged column k* gets its exact pivot from Q
//          (first max), the swap (or the singular skip) is appended to the
//          block's list and the pass repeats.  A row swap at column k commutes
//          with the updates of earlier columns, so applying the list to P0 up
//          front is exact.
//   finish CTAs write their rows' multipliers, apply the block's swaps to the
//          other columns and solve U12 = L11^-1 A12 (warp per column), keeping
//          the next diagonal block's entries (after the swaps) aside; grid
//          barrier.
//   update trailing A22 -= L21 U12 in 64x64 tiles on every CTA but the last,
//          the next tile's operands loaded while the current one computes;
//          tiles that hold the next block's columns also refresh P0 and are
//          counted.  The last CTA forms the next diagonal block from the kept
//          entries, L21 and U12 (the same operations in the same order as the
//          tile that owns it), eliminates it and publishes it.  The oracle
//          skips an update whose u_kj is exactly 0; here it is applied
//          (x - l*0 == x for finite l, and the multipliers of an accepted pass
//          are finite: |l| <= 1), so the factors agree bit for bit for every
//          finite matrix.
// The next block's first pass waits for the publication and the P0 tiles
// only, so the update needs no grid barrier of its own and the diagonal block
// leaves the critical path while the update runs.  A block without swaps
// costs one pass and two grid barriers.  Every wait is bounded: after
// kSpinLimit polls a CTA records an error and stops waiting, so a launch
// always ends.
#include "d4_lu_coop.cuh"

namespace d4 {

int coop_grid_size(int n) {
    int dev = 0, sms = 0, per_sm = 0;
    D4_CUDA_OK(cudaGetDevice(&dev));
    D4_CUDA_OK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    D4_CUDA_OK(cudaFuncSetAttribute(coop::k_lu_coop<double>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (int)coop::kRowBufBytes<double>()));
    D4_CUDA_OK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, coop::k_lu_coop<double>, coop::kThreads,
                                                             coop::kRowBufBytes<double>()));
    int g = sms * (per_sm < 1 ? 1 : per_sm);
    // enough threads for one row below the diagonal block per thread
    const int need = (n + coop::kThreads - 1) / coop::kThreads;
    if (g < need) return -1;
    return g;
}

// Factorises A into L.LU on `st` with `grid` CTAs, without waiting: flags
// (L.flags) are read by the caller later.  `after_copy` (may be null) is
// recorded once A has been copied, after which A may change.
void factor64_async(Ctx &c, const LuBufs &L, const double *A, int grid, cudaStream_t st,
                    cudaEvent_t after_copy) {
    const int n = c.n;
    const size_t bytes = sizeof(double) * (size_t)n * n;
    D4_CUDA_OK(cudaMemsetAsync(L.flags, 0, sizeof(int) * kFlagCount, st));
    D4_CUDA_OK(cudaMemsetAsync(L.bar, 0, sizeof(unsigned) * 64, st));
    D4_CUDA_OK(cudaMemsetAsync(L.mask, 0, sizeof(unsigned) * c.lu_mask_words, st));
    D4_CUDA_OK(cudaMemcpyAsync(L.LU, A, bytes, cudaMemcpyDeviceToDevice, st));
    if (after_copy) D4_CUDA_OK(cudaEventRecord(after_copy, st));
    coop::CoopArgs<double> a;
    a.n = n;
    a.A = L.LU;
    a.P0 = L.P0;
    a.Q = L.Q;
    a.mask = L.mask;
    a.piv = L.piv;
    a.flags = L.flags;
    a.bar = L.bar;
    a.perm = L.perm;
    a.sched = L.mask + lu_pass_words((n + kLuNb - 1) / kLuNb);
    a.dg = L.Q + (size_t)n * 64;
    void *args[] = {(void *)&a};
    D4_CUDA_OK(cudaLaunchCooperativeKernel((const void *)coop::k_lu_coop<double>, dim3(grid),
                                           dim3(coop::kThreads), args,
                                           coop::kRowBufBytes<double>(), st));
    check_launch("k_lu_coop<double>");
}

LuBufs primary_lu(Ctx &c) {
    LuBufs L;
    L.LU = c.LU;
    L.P0 = c.lu_p0;
    L.Q = c.lu_q;
    L.mask = c.lu_mask;
    L.bar = c.lu_bar;
    L.flags = c.flags;
    L.perm = c.perm;
    L.piv = c.piv;
    return L;
}

int factor64(Ctx &c) {
    factor64_async(c, primary_lu(c), c.A, c.lu_grid, c.stream, nullptr);
    D4_CUDA_OK(cudaMemcpyAsync(c.h_flags, c.flags, sizeof(int) * kFlagCount,
                               cudaMemcpyDeviceToHost, c.stream));
    D4_CUDA_OK(cudaStreamSynchronize(c.stream));
    if (c.h_flags[kFlagBarrierTimeout]) throw StateError("LU grid barrier timed out");
    count_lu(c, c.h_flags);
    c.factor_singular = c.h_flags[kFlagSingular] != 0;
    c.factor_pivoted = 0;
    return c.factor_singular ? D4_WARN_SINGULAR : D4_OK;
}

}  // namespace d4
