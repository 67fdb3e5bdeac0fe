"""The UMFPACK-compatible library (include/d4umfpack.h, libd4umfpack.so).

The reference core calls five UMFPACK "di" functions
(src/simulation.cpp:626,637-639,645).  The library exports them over the
engine's dense LU.  CPU tests: every declared symbol is exported and the
argument checks that need no device.  GPU tests (marked gpu): factorisation
and solve bit-identical to the oracle's partial-pivot LU for even and odd
orders, the singular warning, and the unmodified reference core linked
against the library (oracle/_ref/libd4ref_gpu.so, built from the reference
sources where they are present) reproducing the reference's N=64 run.
"""
import ctypes as C
import os
import re

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB = os.path.join(ROOT, "2d4_b200", "lib", "libd4umfpack.so")
HDR = os.path.join(ROOT, "include", "d4umfpack.h")
_ip = C.POINTER(C.c_int)
_dp = C.POINTER(C.c_double)


def load():
    L = C.CDLL(LIB)
    L.umfpack_di_symbolic.argtypes = [C.c_int, C.c_int, _ip, _ip, _dp, C.POINTER(C.c_void_p),
                                      _dp, _dp]
    L.umfpack_di_numeric.argtypes = [_ip, _ip, _dp, C.c_void_p, C.POINTER(C.c_void_p), _dp, _dp]
    L.umfpack_di_solve.argtypes = [C.c_int, _ip, _ip, _dp, _dp, _dp, C.c_void_p, _dp, _dp]
    L.umfpack_di_free_symbolic.argtypes = [C.POINTER(C.c_void_p)]
    L.umfpack_di_free_numeric.argtypes = [C.POINTER(C.c_void_p)]
    for f in ("umfpack_di_free_symbolic", "umfpack_di_free_numeric"):
        getattr(L, f).restype = None
    return L


def csc(a):
    """CSC arrays of a dense matrix (explicit zeros dropped)."""
    n = a.shape[0]
    ap, ai, ax = [0], [], []
    for j in range(n):
        nz = np.nonzero(a[:, j])[0]
        ai.extend(nz.tolist())
        ax.extend(a[nz, j].tolist())
        ap.append(len(ai))
    return (np.array(ap, dtype=np.int32), np.array(ai, dtype=np.int32),
            np.array(ax, dtype=np.float64))


def ptrs(ap, ai, ax):
    return (ap.ctypes.data_as(_ip), ai.ctypes.data_as(_ip), ax.ctypes.data_as(_dp))


def test_exports_and_host_checks():
    L = load()
    names = re.findall(r"\b(umfpack_di_\w+)\(", open(HDR).read())
    assert len(set(names)) == 5
    for n in names:
        getattr(L, n)
    ap = np.zeros(3, dtype=np.int32)
    sym = C.c_void_p()
    p = ptrs(ap, ap, np.zeros(1))
    assert L.umfpack_di_symbolic(2, 3, *p, C.byref(sym), None, None) == -13
    assert L.umfpack_di_symbolic(0, 0, *p, C.byref(sym), None, None) == -6
    assert L.umfpack_di_symbolic(2, 2, *p, C.byref(sym), None, None) == 0 and sym.value
    L.umfpack_di_free_symbolic(C.byref(sym))
    assert not sym.value
    num = C.c_void_p()
    assert L.umfpack_di_numeric(*p, None, C.byref(num), None, None) == -4
    x = np.zeros(2)
    assert L.umfpack_di_solve(1, *p, x.ctypes.data_as(_dp), x.ctypes.data_as(_dp), None,
                              None, None) == -13


def factor_solve(L, a, g):
    n = a.shape[0]
    ap, ai, ax = csc(a)
    p = ptrs(ap, ai, ax)
    sym, num = C.c_void_p(), C.c_void_p()
    assert L.umfpack_di_symbolic(n, n, *p, C.byref(sym), None, None) == 0
    st_num = L.umfpack_di_numeric(*p, sym, C.byref(num), None, None)
    L.umfpack_di_free_symbolic(C.byref(sym))
    x = np.empty(n)
    st_sol = L.umfpack_di_solve(0, *p, x.ctypes.data_as(_dp), g.ctypes.data_as(_dp), num,
                                None, None)
    L.umfpack_di_free_numeric(C.byref(num))
    assert not num.value
    return x, st_num, st_sol


@pytest.mark.gpu
@pytest.mark.parametrize("n,seed", [(64, 1), (65, 2), (300, 3), (301, 4)])
def test_solve_bit_exact_vs_oracle(restated, n, seed):
    L = load()
    rng = np.random.default_rng(seed)
    a = rng.standard_normal((n, n))
    a[rng.random((n, n)) < 0.5] = 0.0  # sparse pattern, pivoting needed
    a += np.eye(n) * 0.1
    g = rng.standard_normal(n)
    for _ in range(2):  # the second pass reuses the pooled context
        x, s1, s2 = factor_solve(L, a, g)
        xo, sing, _ = restated.lu_solve(a, g)
        assert (s1, s2) == (sing, sing) == (0, 0)
        assert np.array_equal(x, xo)


@pytest.mark.gpu
def test_singular_warning(restated):
    L = load()
    n = 32
    rng = np.random.default_rng(9)
    a = rng.standard_normal((n, n))
    a[:, 5] = 0.0
    g = rng.standard_normal(n)
    x, s1, s2 = factor_solve(L, a, g)
    xo, sing, _ = restated.lu_solve(a, g)
    assert (s1, s2) == (1, 1) and sing == 1
    same = (x == xo) | (np.isnan(x) & np.isnan(xo))
    assert same.all()


@pytest.mark.gpu
def test_reference_core_on_gpu_solver(pkg, golden, tmp_path):
    """The reference core, compiled unmodified from its sources and linked
    against libd4umfpack.so, runs the N=64 configuration (1000 accepted steps,
    P = 1e-8) with every factorisation and solve on the GPU and reproduces the
    reference's own run (CPU solver) bit for bit."""
    import pyoracle
    if not pyoracle.Reference.available("gpu"):
        pytest.skip("oracle/_ref/libd4ref_gpu.so not built (needs the reference sources)")
    ref = pyoracle.Reference("gpu")
    x, y, b = pkg.dconf.generate(64, 1000)
    path = str(tmp_path / "s64.dconf")
    pkg.dconf.write(path, x, y, b, digits=17)
    p = ref.params(position_precision=1e-8, step_count_limit=999)
    xr, yr, res, _ = ref.run(path, p)
    gold = golden["seed64_run_res"]
    assert (res.successful_steps, res.failed_steps) == (int(gold[2]), int(gold[3]))
    assert np.array_equal(xr, golden["seed64_run_x"])
