// d4_umfpack.cpp: UMFPACK-compatible entry points (include/d4umfpack.h) over
// the engine's C ABI, so that the reference core (src/simulation.cpp:626-659)
// factorises and solves on the GPU without source changes.
//
// Symbolic holds the order.  Numeric owns a device context taken from a pool
// keyed by the (padded) order: contexts are expensive to create (n x n device
// buffers), and the reference creates and frees one Numeric per
// factorisation (src/simulation.cpp:626,638), so a freed context returns to
// the pool and the next factorisation of the same order reuses it.
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <new>
#include <vector>

#include "d4core.h"
#include "d4umfpack.h"

namespace {

struct Symbolic {
    int n;
};

struct Numeric {
    int n;       // order of the system
    int m;       // order of the device context (n rounded up to even)
    void *ctx;
    int singular;
};

std::mutex g_mu;
std::multimap<int, void *> g_pool;  // idle contexts by order

void *take_ctx(int m) {
    {
        std::lock_guard<std::mutex> lk(g_mu);
        auto it = g_pool.find(m);
        if (it != g_pool.end()) {
            void *c = it->second;
            g_pool.erase(it);
            return c;
        }
    }
    d4_params p;
    d4_default_params(&p);
    void *c = nullptr;
    if (d4_create(&c, m, &p) != D4_OK) return nullptr;
    return c;
}

void give_ctx(int m, void *c) {
    std::lock_guard<std::mutex> lk(g_mu);
    g_pool.emplace(m, c);
}

}  // namespace

extern "C" {

int umfpack_di_symbolic(int n_row, int n_col, const int *, const int *, const double *,
                        void **Sym, const double *, double *) {
    if (!Sym) return UMFPACK_ERROR_argument_missing;
    if (n_row <= 0 || n_col <= 0) return UMFPACK_ERROR_n_nonpositive;
    if (n_row != n_col) return UMFPACK_ERROR_invalid_system;
    Symbolic *s = new (std::nothrow) Symbolic{n_row};
    if (!s) return UMFPACK_ERROR_out_of_memory;
    *Sym = s;
    return UMFPACK_OK;
}

int umfpack_di_numeric(const int Ap[], const int Ai[], const double Ax[], void *Sym, void **Num,
                       const double *, double *) {
    if (!Ap || !Ai || !Ax || !Num) return UMFPACK_ERROR_argument_missing;
    if (!Sym) return UMFPACK_ERROR_invalid_Symbolic_object;
    const int n = static_cast<Symbolic *>(Sym)->n;
    const int m = n + (n & 1);
    std::vector<double> dense;
    try {
        dense.assign((size_t)m * m, 0.0);
    } catch (const std::bad_alloc &) {
        return UMFPACK_ERROR_out_of_memory;
    }
    for (int j = 0; j < n; ++j)
        for (int q = Ap[j]; q < Ap[j + 1]; ++q) {
            const int i = Ai[q];
            if (i < 0 || i >= n) return UMFPACK_ERROR_internal_error;
            dense[(size_t)i + (size_t)j * m] += Ax[q];
        }
    if (m != n) dense[(size_t)n + (size_t)n * m] = 1.0;  // identity padding
    void *ctx = take_ctx(m);
    if (!ctx) return UMFPACK_ERROR_out_of_memory;
    int st = d4_set_matrix(ctx, dense.data());
    if (st == D4_OK) st = d4_factor(ctx);
    if (st < 0) {
        d4_destroy(ctx);
        return UMFPACK_ERROR_internal_error;
    }
    Numeric *f = new (std::nothrow) Numeric{n, m, ctx, st == D4_WARN_SINGULAR};
    if (!f) {
        give_ctx(m, ctx);
        return UMFPACK_ERROR_out_of_memory;
    }
    *Num = f;
    return f->singular ? UMFPACK_WARNING_singular_matrix : UMFPACK_OK;
}

int umfpack_di_solve(int sys, const int *, const int *, const double *, double X[],
                     const double B[], void *Num, const double *, double *) {
    if (sys != UMFPACK_A) return UMFPACK_ERROR_invalid_system;
    if (!X || !B) return UMFPACK_ERROR_argument_missing;
    if (!Num) return UMFPACK_ERROR_invalid_Numeric_object;
    Numeric *f = static_cast<Numeric *>(Num);
    int st;
    if (f->m == f->n) {
        st = d4_solve(f->ctx, B, X);
    } else {
        std::vector<double> b(B, B + f->n), x(f->m);
        b.push_back(0.0);
        st = d4_solve(f->ctx, b.data(), x.data());
        std::memcpy(X, x.data(), sizeof(double) * (size_t)f->n);
    }
    if (st < 0) return UMFPACK_ERROR_internal_error;
    return f->singular ? UMFPACK_WARNING_singular_matrix : UMFPACK_OK;
}

void umfpack_di_free_symbolic(void **Sym) {
    if (Sym && *Sym) {
        delete static_cast<Symbolic *>(*Sym);
        *Sym = nullptr;
    }
}

void umfpack_di_free_numeric(void **Num) {
    if (Num && *Num) {
        Numeric *f = static_cast<Numeric *>(*Num);
        give_ctx(f->m, f->ctx);
        delete f;
        *Num = nullptr;
    }
}

}  // extern "C"
