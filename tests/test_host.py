"""Host-side logic and the C-ABI library, no GPU needed."""
import ctypes as C
import os
import re
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_functions():
    src = open(os.path.join(ROOT, "include", "d4core.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(d4_[a-z_0-9]+)\s*\(", src)))


def test_library_exports_every_header_symbol(pkg):
    lib = pkg._lib.load()
    names = header_functions()
    assert len(names) >= 15
    for name in names:
        assert hasattr(lib, name), name
    assert set(names) == set(pkg._lib.SIGNATURES), "ctypes table out of sync with the header"
    out = subprocess.run(["nm", "-D", "--defined-only", pkg._lib.LIB_PATH], capture_output=True,
                         text=True).stdout
    exported = set(re.findall(r" T (d4_\w+)", out))
    assert set(names) <= exported


def test_library_has_sm100a_code(pkg):
    out = subprocess.run(["cuobjdump", "--list-elf", pkg._lib.LIB_PATH], capture_output=True,
                         text=True).stdout
    assert "sm_100a" in out


def test_default_params_and_bad_arguments(pkg):
    lib = pkg._lib.load()
    p = pkg._lib.Params()
    lib.d4_default_params(C.byref(p))
    assert p.position_precision == 1e-5 and p.dipole_precision == 0.05
    assert p.cutoff_multiplier == 1e20 and p.weight_function == b"c"
    assert p.initial_stepsize == 1e-6 and p.sub_config_delay == 5
    ctx = C.c_void_p()
    # odd n (unbalanced Burgers vectors) and bad weight function are rejected
    assert lib.d4_create(C.byref(ctx), 63, C.byref(p)) == -1
    p.weight_function = b"x"
    assert lib.d4_create(C.byref(ctx), 64, C.byref(p)) == -1
    assert lib.d4_destroy(None) == -1
    # solver and field selection: defaults, and combinations rejected before any
    # device work (unknown solver, tabulated field in the mixed form, table size)
    lib.d4_default_params(C.byref(p))
    assert p.solver == pkg._lib.D4_SOLVER_DENSE and p.field == pkg._lib.D4_FIELD_ANALYTIC
    assert p.table_size == 1024
    for kw in (dict(solver=7), dict(field=2),
               dict(field=1, precision=pkg._lib.D4_PREC_MIXED),
               dict(field=1, table_size=8), dict(field=1, table_size=8192)):
        lib.d4_default_params(C.byref(p))
        for k, v in kw.items():
            setattr(p, k, v)
        assert lib.d4_create(C.byref(ctx), 64, C.byref(p)) == -1, kw


def test_dconf_roundtrip_and_sort(pkg, golden, tmp_path):
    dconf = pkg.dconf
    x, y, b = dconf.generate(64, 1000)
    assert (b[:32] == 1).all() and (b[32:] == -1).all()
    assert x.min() >= -0.5 and x.max() < 0.5
    path = str(tmp_path / "s.dconf")
    dconf.write(path, x, y, b, digits=17)
    xs, ys, order = dconf.load(path)
    # the reference's own loader gave these (golden: reference outputs)
    assert np.array_equal(xs, golden["seed64_x"])
    assert np.array_equal(ys, golden["seed64_y"])
    assert np.array_equal(order, golden["seed64_order"])
    out = str(tmp_path / "o.dconf")
    dconf.write_internal(out, xs, ys, order)
    x2, y2, b2 = dconf.read(out)
    assert np.allclose(x2, x, rtol=0, atol=1e-13) and np.array_equal(b2, b)


def test_dconf_rejects_bad_files(pkg, tmp_path):
    p = tmp_path / "bad.dconf"
    p.write_text("0.1 0.2 1\n0.3 0.4 1\n")
    with pytest.raises(ValueError):
        pkg.dconf.read(str(p))
    p.write_text("0.1 0.2 0.5\n0.3 0.4 -0.5\n")
    with pytest.raises(ValueError):
        pkg.dconf.read(str(p))
    p.write_text("0.1 0.2 1\n0.3\n")
    with pytest.raises(ValueError):
        pkg.dconf.read(str(p))


def test_conf_compare_metric(pkg):
    cc = pkg.dconf.conf_compare
    x = np.array([0.1, -0.49, 0.3, 0.0])
    y = np.zeros(4)
    assert cc(x, y, x, y)[0] == 0.0
    x2 = x.copy()
    x2[2] = 0.3 + 2e-9
    d, i, avg, _ = cc(x, y, x2, y)
    assert i == 2 and abs(d - 2e-9) < 1e-15 and abs(avg - 0.5e-9) < 1e-15
    # the reference normalises |xa - xb| into [-0.5, 0.5): a difference across
    # the periodic boundary (0.99 here) counts as -0.01 and never as the max
    x3 = x.copy()
    x3[1] = 0.5 - 1e-12
    d, i, avg, _ = cc(x, y, x3, y)
    assert d == 0.0 and avg < 0
    with pytest.raises(ValueError):
        cc(x, y, x, y + 1e-6)


@pytest.mark.parametrize("kind,kw", [(0, dict(init_ext_stress=0.3)),
                                     (1, dict(init_ext_stress=0.1, rate=2.0)),
                                     (2, dict(init_ext_stress=0.1, rate=2.0, period=0.3)),
                                     (3, dict(init_ext_stress=0.1, rate=2.0, period=0.3,
                                              amplitude_rate=1.5))])
def test_stress_protocols_match_oracle(pkg, restated, kind, kw):
    import pyoracle
    cls = [pkg.StressProtocol, pkg.FixedRateProtocol, pkg.CyclicLoadProtocol,
           pkg.IncreasingCyclicLoadProtocol][kind]
    proto = cls(**kw)
    op = pyoracle.OProtocol(kind, kw.get("init_ext_stress", 0), kw.get("rate", 0),
                            kw.get("period", 0), kw.get("amplitude_rate", 0))
    for t in np.linspace(0, 1.3, 57):
        if kind < 2:
            assert proto.ext_stress(t) == restated.L.d4o_ext_stress(C.byref(op), t)
        c = proto.to_c()
        assert (c.kind, c.tau0) == (kind, kw.get("init_ext_stress", 0))


def test_simulation_data_params(pkg, tmp_path):
    x, y, b = pkg.dconf.generate(8, 3)
    p = str(tmp_path / "a.dconf")
    pkg.dconf.write(p, x, y, b, digits=17)
    sd = pkg.SimulationData(p, "")
    assert sd.dislocation_count == 8
    sd.precision = 1e-8
    sd.step_count_limited, sd.step_count_limit = True, 999
    sd.external_stress = pkg.FixedRateProtocol(0.05, 0.0)
    c = sd.to_params()
    assert c.position_precision == 1e-8 and c.step_count_limit == 999
    assert c.protocol.kind == 1 and c.protocol.tau0 == 0.05
    assert c.time_limit < 0 and c.max_stepsize < 0


def test_new_entry_points_reject_bad_arguments(pkg):
    """The overlap switch, the LU counters and the pattern analysis check
    their arguments before any device work (status -1, D4_ERR_ARG)."""
    lib = pkg._lib.load()
    v = C.c_longlong()
    assert lib.d4_set_overlap(None, 1) == -1
    assert lib.d4_lu_stats(None, C.byref(v), C.byref(v), C.byref(v)) == -1
    x = np.zeros(4)
    b = np.array([1, 1, -1, -1], dtype=np.int32)
    acc = np.zeros(4 * 9)
    ip = b.ctypes.data_as(C.POINTER(C.c_int))
    dp = pkg._lib.ptr
    assert lib.d4_xpattern_df(-1, dp(x), dp(x), ip, 16, dp(acc)) == -1   # negative n
    assert lib.d4_xpattern_df(4, dp(x), dp(x), ip, 1, dp(acc)) == -1     # resolution < 2
    assert lib.d4_xpattern_df(4, None, dp(x), ip, 16, dp(acc)) == -1     # missing input
    assert lib.d4_xpattern_df(4, dp(x), dp(x), ip, 16, None) == -1       # missing sums
    assert lib.d4_xpattern_df(4, dp(x), dp(x), ip, 70000, dp(acc)) == -1  # beyond the maximum


def test_size_limits_rejected_before_device_work(pkg):
    """N outside 2..8192 or odd (the largest system whose substitution vector
    fits one CTA's shared memory; balanced Burgers vectors need even N), and
    ensembles with such an instance, a non-FP64 form or the GMRES solver, are
    refused with D4_ERR_ARG before any device call."""
    lib = pkg._lib.load()
    p = pkg._lib.Params()
    ctx = C.c_void_p()
    for n in (0, -2, 1, 8194, 1 << 20):
        lib.d4_default_params(C.byref(p))
        assert lib.d4_create(C.byref(ctx), n, C.byref(p)) == -1, n
    ens = C.c_void_p()
    for sizes in ([64, 8194], [64, 63], [0], [2, -4]):
        lib.d4_default_params(C.byref(p))
        arr = (C.c_int * len(sizes))(*sizes)
        assert lib.d4_ensemble_create(C.byref(ens), len(sizes), arr, C.byref(p)) == -1, sizes
    arr = (C.c_int * 2)(64, 128)
    assert lib.d4_ensemble_create(C.byref(ens), 0, arr, C.byref(p)) == -1
    for kw in (dict(precision=pkg._lib.D4_PREC_MIXED), dict(field=pkg._lib.D4_FIELD_TABULATED),
               dict(solver=pkg._lib.D4_SOLVER_GMRES), dict(weight_function=b"x")):
        lib.d4_default_params(C.byref(p))
        for k, v in kw.items():
            setattr(p, k, v)
        assert lib.d4_ensemble_create(C.byref(ens), 2, arr, C.byref(p)) == -1, kw


def test_position_check(pkg):
    """d4_check_positions (used by d4_set_positions and
    d4_ensemble_set_positions): finite values inside [-0.5, 0.5)^2 only."""
    lib = pkg._lib.load()
    x = np.linspace(-0.5, 0.49, 8)
    y = np.zeros(8)
    assert lib.d4_check_positions(8, pkg._lib.ptr(x), pkg._lib.ptr(y)) == -1
    for bad in (np.nan, np.inf, -np.inf, 0.5, -0.5000001, 3.0):
        for arr in ("x", "y"):
            xx, yy = x.copy(), y.copy()
            (xx if arr == "x" else yy)[5] = bad
            assert lib.d4_check_positions(8, pkg._lib.ptr(xx), pkg._lib.ptr(yy)) == 5
    assert lib.d4_check_positions(0, None, None) == -1
    assert lib.d4_check_positions(-1, None, None) == -2
