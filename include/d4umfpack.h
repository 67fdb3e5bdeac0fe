/*
 * d4umfpack.h: UMFPACK-compatible solver entry points backed by the B200 engine.
 *
 * Library: 2d4_b200/lib/libd4umfpack.so (links libd4core.so).  These are the
 * five functions of SuiteSparse UMFPACK's public "di" API (int indices,
 * double values) that the reference core calls, with the same names,
 * signatures and return codes, so that the unmodified core links against this
 * library instead of UMFPACK and factorises and solves on the GPU:
 *   umfpack_di_symbolic      src/simulation.cpp:637
 *   umfpack_di_numeric       src/simulation.cpp:638
 *   umfpack_di_free_symbolic src/simulation.cpp:639
 *   umfpack_di_solve         src/simulation.cpp:645 (UMFPACK_A only)
 *   umfpack_di_free_numeric  src/simulation.cpp:626
 * The CSC matrix is expanded to a dense column-major matrix (duplicate entries
 * summed) and factorised with d4_factor (partial pivoting, first maximum wins,
 * exact per-entry update order); solves use d4_solve.  Both return
 * UMFPACK_WARNING_singular_matrix on an exact zero pivot and leave the result
 * as computed, as the reference expects (src/simulation.cpp:646-658).  Odd
 * orders are padded with one identity row and column, which changes no pivot
 * and no arithmetic on the original entries.  Control and Info are ignored
 * (the reference passes null Control and never reads Info).  Device contexts
 * are pooled per order and reused across factorisations; the library is safe
 * to call from several threads.
 */
#ifndef D4UMFPACK_H
#define D4UMFPACK_H

#ifdef __cplusplus
extern "C" {
#endif

#define UMFPACK_A 0
#define UMFPACK_OK 0
#define UMFPACK_WARNING_singular_matrix 1
#define UMFPACK_ERROR_out_of_memory (-1)
#define UMFPACK_ERROR_invalid_Numeric_object (-3)
#define UMFPACK_ERROR_invalid_Symbolic_object (-4)
#define UMFPACK_ERROR_argument_missing (-5)
#define UMFPACK_ERROR_n_nonpositive (-6)
#define UMFPACK_ERROR_invalid_system (-13)
#define UMFPACK_ERROR_internal_error (-911)

int umfpack_di_symbolic(int n_row, int n_col, const int Ap[], const int Ai[], const double Ax[],
                        void **Symbolic, const double Control[], double Info[]);

int umfpack_di_numeric(const int Ap[], const int Ai[], const double Ax[], void *Symbolic,
                       void **Numeric, const double Control[], double Info[]);

int umfpack_di_solve(int sys, const int Ap[], const int Ai[], const double Ax[], double X[],
                     const double B[], void *Numeric, const double Control[], double Info[]);

void umfpack_di_free_symbolic(void **Symbolic);

void umfpack_di_free_numeric(void **Numeric);

#ifdef __cplusplus
}
#endif

#endif
