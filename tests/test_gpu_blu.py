"""GPU checks of the mixed form's block LU and block solves (marked gpu).

The mixed form factorises the FP32 rounding of the Jacobian (rows in the
order of its last pivoted factorisation) by a block LU without row
interchanges between 128 x 128 tiles (tensor-core products, Gauss-Jordan
inverses of the diagonal tiles) and refines every solve in FP64 against the
FP64 matrix until max|g - A dx| <= 1e-12 max|g|.  Checked through
d4_set_matrix / d4_factor / d4_solve against numpy's LAPACK solve of the same
FP64 matrix: the refined solution to 1e-11 relative (the refinement's stopping
residual times these matrices' condition), for orders that are and are not
multiples of the tile, and the fallback to the pivoted LU when a diagonal
tile has a zero pivot, after which the block LU uses its row order.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def mixed_engine(pkg, n):
    x, y, _ = pkg.dconf.generate_internal(n, 5)
    sd = pkg.SimulationData()
    sd.set_positions(x, y)
    sd.precision_mode = pkg._lib.D4_PREC_MIXED
    return pkg.Engine(sd)


def solve_check(e, a, rhs, tol=1e-11):
    e.set_matrix(a)
    st = e.factor()
    assert st == 0
    for g in rhs:
        dx, st = e.solve(g)
        ref = np.linalg.solve(a, g)
        assert np.abs(dx - ref).max() <= tol * np.abs(ref).max()


@pytest.mark.parametrize("n", [2, 64, 128, 200, 384, 1024])
def test_block_lu_random(pkg, n):
    rng = np.random.default_rng(n)
    a = np.eye(n) + 0.3 * rng.standard_normal((n, n)) / np.sqrt(n)
    e = mixed_engine(pkg, n)
    s0 = e.mixed_stats()
    solve_check(e, a, [rng.standard_normal(n), np.ones(n)])
    s1 = e.mixed_stats()
    assert s1["block_factorizations"] == s0["block_factorizations"] + 1
    assert s1["fallbacks"] == s0["fallbacks"]
    e.close()


def test_block_lu_needs_fallback(pkg):
    """A diagonal tile with an exact zero pivot (rows 0 and 1 swapped in an
    otherwise diagonal matrix): the block LU flags it and d4_factor factorises
    with the pivoted LU instead."""
    n = 256
    rng = np.random.default_rng(3)
    a = np.eye(n) + 0.01 * rng.standard_normal((n, n)) / np.sqrt(n)
    a[[0, 1]] = a[[1, 0]]
    a[0, 0] = 0.0
    a[1, 1] = 0.0
    e = mixed_engine(pkg, n)
    s0 = e.mixed_stats()
    solve_check(e, a, [rng.standard_normal(n)])
    assert e.mixed_stats()["fallbacks"] == s0["fallbacks"] + 1
    # the next block LU factorises the rows in the pivoted LU's order: no fallback
    solve_check(e, a, [rng.standard_normal(n)])
    s2 = e.mixed_stats()
    assert s2["fallbacks"] == s0["fallbacks"] + 1
    assert s2["block_factorizations"] == s0["block_factorizations"] + 2
    e.close()


@pytest.mark.parametrize("n,h", [(512, 1e-5), (1024, 1e-4)])
def test_block_lu_jacobian(pkg, n, h):
    """The implicit step's own matrix A = I + D J."""
    x, y, _ = pkg.dconf.generate_internal(n, 1001)
    e = mixed_engine(pkg, n)
    _, _, a, _, _ = e.jacobian(x, y, h, 0.0, h)
    rng = np.random.default_rng(1)
    solve_check(e, a, [rng.standard_normal(n)])
    e.close()


def test_block_lu_switch(pkg):
    """d4_set_block_lu(0): the pivoted FP32 LU; both paths solve the same
    system to the refinement's accuracy."""
    n = 384
    rng = np.random.default_rng(9)
    a = np.eye(n) + 0.3 * rng.standard_normal((n, n)) / np.sqrt(n)
    g = rng.standard_normal(n)
    e = mixed_engine(pkg, n)
    e.set_block_lu(False)
    s0 = e.mixed_stats()
    solve_check(e, a, [g])
    assert e.mixed_stats()["block_factorizations"] == s0["block_factorizations"]
    e.set_block_lu(True)
    solve_check(e, a, [g])
    assert e.mixed_stats()["block_factorizations"] == s0["block_factorizations"] + 1
    e.close()


def test_block_lu_stiff_jacobian(pkg):
    """The Jacobian of a clustered N=4096 state (tests/golden/stiff_4096.npz,
    made by make_stiff.py): its ill-conditioned diagonal tiles get a
    Newton-Schulz step after Gauss-Jordan, and the refined solve reaches
    max|A dx - g| <= 1e-11 max|g| with the block LU, no fallback (with the
    Gauss-Jordan inverses alone the refinement stagnates near 1e-3)."""
    import os
    z = np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden",
                             "stiff_4096.npz"))
    x, y, h = z["x"], z["y"], float(z["h"])
    e = mixed_engine(pkg, len(x))
    _, _, a, _, _ = e.jacobian(x, y, h, 0.0, h)
    s0 = e.mixed_stats()
    e.set_matrix(a)
    assert e.factor() == 0
    g = np.random.default_rng(5).standard_normal(len(x))
    dx, _ = e.solve(g)
    assert np.abs(a @ dx - g).max() <= 1e-11 * np.abs(g).max()
    s1 = e.mixed_stats()
    assert s1["block_factorizations"] == s0["block_factorizations"] + 1
    assert s1["fallbacks"] == s0["fallbacks"]
    e.close()
