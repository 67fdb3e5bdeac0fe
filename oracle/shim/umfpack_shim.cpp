/*
 * Project-written UMFPACK stand-in used to link the reference core as a CPU
 * oracle.  TEST INFRASTRUCTURE ONLY (see suitesparse/umfpack.h).
 *
 * The reference hands UMFPACK a CSC matrix (Ap, Ai, Ax) that is in practice
 * fully dense (no cutoff) or sparse (cutoff), factorises it three times per
 * attempted step and solves two right-hand sides per factorisation
 * (src/simulation.cpp:618-659).  This shim expands the CSC matrix to a dense
 * column-major array and factorises it with Gaussian elimination with partial
 * pivoting (LAPACK getrf semantics: the first entry of largest magnitude in the
 * column is the pivot).
 *
 * Two backends, chosen at run time:
 *   - native (default): the plain C loops below, deterministic, single thread.
 *     The C restatement in oracle/d4_oracle.c uses the same loop order, so the
 *     two oracles agree bit for bit when built with the same flags.
 *   - OpenBLAS: if D4REF_OPENBLAS names a shared library exporting the LP64
 *     symbols scipy_dgetrf_/scipy_dgetrs_ (the OpenBLAS that ships inside
 *     scipy), it is dlopen'ed and used with D4REF_THREADS threads (default: all
 *     cores).  This is the "UMFPACK + BLAS" stand-in for CPU timing.
 *
 * Return codes mirror UMFPACK: 0 ok, UMFPACK_WARNING_singular_matrix (1) when
 * an exact zero pivot is met (numeric and every later solve report it).
 */
#include "suitesparse/umfpack.h"

#include <dlfcn.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>
#include <unistd.h>

namespace {

struct Symbolic {
    int n;
};

struct Numeric {
    int n;
    int singular;
    double *lu;  // column-major n x n
    int *piv;    // 0-based pivot rows (native) or 1-based (OpenBLAS)
    int blas;    // 1 if factorised by OpenBLAS
};

typedef void (*getrf_t)(const int *, const int *, double *, const int *, int *, int *);
typedef void (*getrs_t)(const char *, const int *, const int *, const double *, const int *,
                        const int *, double *, const int *, int *, size_t);
typedef void (*setthreads_t)(int);

struct Blas {
    int tried;
    getrf_t getrf;
    getrs_t getrs;
};

Blas g_blas = {0, nullptr, nullptr};

void load_blas() {
    if (g_blas.tried) return;
    g_blas.tried = 1;
    const char *path = getenv("D4REF_OPENBLAS");
    if (!path || !*path) return;
    void *h = dlopen(path, RTLD_NOW | RTLD_LOCAL);
    if (!h) return;
    g_blas.getrf = (getrf_t)dlsym(h, "scipy_dgetrf_");
    g_blas.getrs = (getrs_t)dlsym(h, "scipy_dgetrs_");
    setthreads_t st = (setthreads_t)dlsym(h, "scipy_openblas_set_num_threads");
    if (!g_blas.getrf || !g_blas.getrs) {
        g_blas.getrf = nullptr;
        g_blas.getrs = nullptr;
        return;
    }
    if (st) {
        const char *t = getenv("D4REF_THREADS");
        int nt = t ? atoi(t) : (int)sysconf(_SC_NPROCESSORS_ONLN);
        if (nt < 1) nt = 1;
        st(nt);
    }
}

// Native LU: right-looking, column-major, partial pivoting.
int lu_native(int n, double *a, int *piv) {
    int singular = 0;
    for (int k = 0; k < n; ++k) {
        int p = k;
        double amax = fabs(a[k + (size_t)k * n]);
        for (int i = k + 1; i < n; ++i) {
            double v = fabs(a[i + (size_t)k * n]);
            if (v > amax) {
                amax = v;
                p = i;
            }
        }
        piv[k] = p;
        if (a[p + (size_t)k * n] == 0.0) {
            singular = 1;
            continue;
        }
        if (p != k) {
            for (int j = 0; j < n; ++j) {
                double t = a[k + (size_t)j * n];
                a[k + (size_t)j * n] = a[p + (size_t)j * n];
                a[p + (size_t)j * n] = t;
            }
        }
        double d = a[k + (size_t)k * n];
        for (int i = k + 1; i < n; ++i) a[i + (size_t)k * n] /= d;
        for (int j = k + 1; j < n; ++j) {
            double t = a[k + (size_t)j * n];
            if (t != 0.0) {
                double *cj = a + (size_t)j * n;
                const double *ck = a + (size_t)k * n;
                for (int i = k + 1; i < n; ++i) cj[i] -= ck[i] * t;
            }
        }
    }
    return singular;
}

void solve_native(int n, const double *a, const int *piv, double *x) {
    for (int k = 0; k < n; ++k) {
        int p = piv[k];
        if (p != k) {
            double t = x[k];
            x[k] = x[p];
            x[p] = t;
        }
    }
    for (int k = 0; k < n; ++k) {
        double t = x[k];
        if (t != 0.0) {
            const double *ck = a + (size_t)k * n;
            for (int i = k + 1; i < n; ++i) x[i] -= ck[i] * t;
        }
    }
    for (int k = n - 1; k >= 0; --k) {
        x[k] /= a[k + (size_t)k * n];
        double t = x[k];
        if (t != 0.0) {
            const double *ck = a + (size_t)k * n;
            for (int i = 0; i < k; ++i) x[i] -= ck[i] * t;
        }
    }
}

}  // namespace

extern "C" {

int umfpack_di_symbolic(int n_row, int n_col, const int *, const int *, const double *,
                        void **Sym, const double *, double *) {
    if (n_row != n_col || n_row < 0) return UMFPACK_ERROR_invalid_system;
    Symbolic *s = (Symbolic *)malloc(sizeof(Symbolic));
    if (!s) return UMFPACK_ERROR_out_of_memory;
    s->n = n_row;
    *Sym = s;
    return UMFPACK_OK;
}

int umfpack_di_numeric(const int Ap[], const int Ai[], const double Ax[], void *Sym,
                       void **Num, const double *, double *) {
    load_blas();
    const int n = ((Symbolic *)Sym)->n;
    Numeric *f = (Numeric *)calloc(1, sizeof(Numeric));
    if (!f) return UMFPACK_ERROR_out_of_memory;
    f->n = n;
    f->lu = (double *)calloc((size_t)n * n + 1, sizeof(double));
    f->piv = (int *)calloc((size_t)n + 1, sizeof(int));
    if (!f->lu || !f->piv) return UMFPACK_ERROR_out_of_memory;
    for (int j = 0; j < n; ++j)
        for (int p = Ap[j]; p < Ap[j + 1]; ++p) f->lu[Ai[p] + (size_t)j * n] += Ax[p];
    if (g_blas.getrf) {
        int info = 0;
        g_blas.getrf(&n, &n, f->lu, &n, f->piv, &info);
        f->blas = 1;
        f->singular = info > 0;
    } else {
        f->singular = lu_native(n, f->lu, f->piv);
    }
    *Num = f;
    return f->singular ? UMFPACK_WARNING_singular_matrix : UMFPACK_OK;
}

int umfpack_di_solve(int sys, const int *, const int *, const double *, double X[],
                     const double B[], void *Num, const double *, double *) {
    if (sys != UMFPACK_A) return UMFPACK_ERROR_invalid_system;
    Numeric *f = (Numeric *)Num;
    const int n = f->n;
    memcpy(X, B, sizeof(double) * (size_t)n);
    if (f->blas) {
        const int one = 1;
        int info = 0;
        g_blas.getrs("N", &n, &one, f->lu, &n, f->piv, X, &n, &info, 1);
    } else {
        solve_native(n, f->lu, f->piv, X);
    }
    return f->singular ? UMFPACK_WARNING_singular_matrix : UMFPACK_OK;
}

void umfpack_di_free_symbolic(void **Sym) {
    if (Sym && *Sym) {
        free(*Sym);
        *Sym = nullptr;
    }
}

void umfpack_di_free_numeric(void **Num) {
    if (Num && *Num) {
        Numeric *f = (Numeric *)*Num;
        free(f->lu);
        free(f->piv);
        free(f);
        *Num = nullptr;
    }
}

}  // extern "C"
