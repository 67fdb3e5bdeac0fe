/*
 * Project-written stand-in for SuiteSparse's <suitesparse/umfpack.h>.
 *
 * TEST INFRASTRUCTURE ONLY: this header exists so that the reference core
 * (src/simulation.cpp of danieltuzes/2D4) can be compiled unmodified as a CPU
 * oracle.  UMFPACK itself is not installed in this image and its version is not
 * pinned by the reference (cmake/FindUmfpack.cmake), so the oracle is
 * "reference core + this shim" and parity at the UMFPACK boundary is unpinned.
 *
 * Only the five entry points and two constants that the reference calls are
 * declared (src/simulation.cpp:626,637-639,645-646).  The signatures are the
 * public UMFPACK "di" API (int indices, double values); they must be alike so
 * that the reference links against the shim without edits.
 */
#ifndef D4_ORACLE_UMFPACK_SHIM_H
#define D4_ORACLE_UMFPACK_SHIM_H

#ifdef __cplusplus
extern "C" {
#endif

#define UMFPACK_A 0                        /* solve A x = b */
#define UMFPACK_OK 0
#define UMFPACK_WARNING_singular_matrix 1  /* exact zero pivot met */
#define UMFPACK_ERROR_out_of_memory (-1)
#define UMFPACK_ERROR_invalid_system (-13)

int umfpack_di_symbolic(int n_row, int n_col, const int Ap[], const int Ai[],
                        const double Ax[], void **Symbolic,
                        const double Control[], double Info[]);

int umfpack_di_numeric(const int Ap[], const int Ai[], const double Ax[],
                       void *Symbolic, void **Numeric,
                       const double Control[], double Info[]);

int umfpack_di_solve(int sys, const int Ap[], const int Ai[], const double Ax[],
                     double X[], const double B[], void *Numeric,
                     const double Control[], double Info[]);

void umfpack_di_free_symbolic(void **Symbolic);

void umfpack_di_free_numeric(void **Numeric);

#ifdef __cplusplus
}
#endif

#endif
