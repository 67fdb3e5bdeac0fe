"""Direct-Fourier pattern analysis (the reference's xpattern -m df,
xpattern/xpattern.cpp:393-423).

CPU: the oracle's vectorised form equals the plain-loop transcription of the
tool's sums at tiny sizes; the command line rejects the tool's other methods.
GPU (marked gpu): d4_xpattern_df against the oracle within 1e-11 of the
largest value (FP64 throughout; the exponentials are formed differently:
sincospi of 2 k x on the device, exp(-2 pi i x k) in the oracle, so the
phases differ by ~k x ulp), summed over two configurations as the tool sums
its input files, repeated bit for bit, and the edge cases (no dislocations,
odd resolution); the command line writes the tool's four files.
"""
import importlib
import io

import numpy as np
import pytest

import xpattern_ref

xp = importlib.import_module("2d4_b200.xpattern")


def signs(n):
    return np.where(np.arange(n) < n // 2, 1.0, -1.0)


def test_oracle_vectorised_equals_loops():
    rng = np.random.default_rng(3)
    for n, res in ((6, 8), (9, 7)):
        x, y = rng.uniform(-0.5, 0.5, n), rng.uniform(-0.5, 0.5, n)
        b = np.where(rng.uniform(size=n) < 0.5, 1.0, -1.0)
        a = xpattern_ref.direct_fourier(x, y, b, res)
        c = xpattern_ref.direct_fourier_loops(x, y, b, res)
        assert np.abs(a - c).max() <= 1e-12 * np.abs(c).max()
    # linearity: rho_t and kappa come from rho_p and rho_n field by field, and
    # the sum over ky of |F_p + F_n|^2 + |F_p - F_n|^2 is 2 (|F_p|^2 + |F_n|^2)
    x, y, b = rng.uniform(-0.5, 0.5, 10), rng.uniform(-0.5, 0.5, 10), signs(10)
    a = xpattern_ref.direct_fourier(x, y, b, 16)
    assert np.allclose(a[0] + a[1], 2 * (a[2] + a[3]), rtol=1e-12)


def test_cli_options_and_checks(tmp_path):
    """The tool's option names, defaults and input checks (status, message)."""
    d = tmp_path / "a.dconf"
    d.write_text("0.1 0.2 1\n-0.1 0.3 -1\n")
    def run(argv):
        out, err = io.StringIO(), io.StringIO()
        return xp.main(argv, out, err), out.getvalue() + err.getvalue()
    st, msg = run([])
    assert st == 255 and "input-fname is missing!" in msg
    st, msg = run(["-i", str(d), "--no-such-option"])
    assert st == 255 and "unrecognized" in msg
    st, msg = run(["-i", str(d)])  # the tool's default method is bc, not built here
    assert st == 255 and "bc is not built here" in msg
    st, msg = run(["-i", str(d), "-m", "xx"])
    assert st == 255 and "xx is unknown" in msg
    st, msg = run(["-i", str(d), "-m", "df", "-r", "1"])
    assert st == 255 and "resulution is smaller than 2" in msg
    st, msg = run(["-i", str(d), "-m", "df", "--create-maps"])
    assert st == 255
    st, msg = run(["-i", str(tmp_path / "a.txt"), "-m", "df"])
    assert st == 1 and "is not a valid input filename" in msg
    ini = tmp_path / "l.ini"
    ini.write_text("a.dconf b.txt\n")
    st, msg = run(["-i", str(ini), "-m", "df"])
    assert st == 2 and "contains invalid dislocation configuration filename b.txt" in msg
    ini.write_text("\n")
    st, msg = run(["-i", str(ini), "-m", "df"])
    assert st == 1 and "Not enough input files" in msg
    st, msg = run(["-i", str(tmp_path / "none.ini"), "-m", "df"])
    assert st == 0 and "couldn't open" in msg
    # like every other check's message, the reference writes this one to
    # std::cerr although it returns 0 (xpattern/xpattern.cpp:88-91)
    out, err = io.StringIO(), io.StringIO()
    assert xp.main(["-i", str(tmp_path / "none.ini"), "-m", "df"], out, err) == 0
    assert "couldn't open" in err.getvalue() and out.getvalue() == ""


def test_input_list(tmp_path):
    lst = tmp_path / "files.ini"
    lst.write_text("a.dconf\n\nb.dconf c.dconf\n")
    assert xp.input_files(str(lst), io.StringIO()) == ["a.dconf", "b.dconf", "c.dconf"]
    assert xp.input_files("c.dconf", io.StringIO()) == ["c.dconf"]


@pytest.mark.gpu
@pytest.mark.parametrize("n,res,seed", [(64, 64, 1000), (1000, 256, 7), (257, 129, 8)])
def test_xpattern_vs_oracle(pkg, n, res, seed):
    x, y, _ = pkg.dconf.generate_internal(n + n % 2, seed)
    x, y = x[:n], y[:n]
    b = signs(n)
    got = xp.direct_fourier(x, y, b, res)
    ref = xpattern_ref.direct_fourier(x, y, b, res)
    assert got.shape == ref.shape == (4, res // 2 + 1)
    assert np.abs(got - ref).max() <= 1e-11 * np.abs(ref).max()
    # k = (0, 0) of rho_p: (number of positive dislocations)^2, exactly
    assert got[2, 0] >= (b == 1).sum() ** 2 * (1 - 1e-15)


@pytest.mark.gpu
def test_xpattern_sums_files_and_repeats(pkg):
    x1, y1, _ = pkg.dconf.generate_internal(128, 1)
    x2, y2, _ = pkg.dconf.generate_internal(200, 2)
    acc = xp.direct_fourier(x1, y1, signs(128), 128)
    acc = xp.direct_fourier(x2, y2, signs(200), 128, acc)
    ref = xpattern_ref.direct_fourier(x1, y1, signs(128), 128) + \
        xpattern_ref.direct_fourier(x2, y2, signs(200), 128)
    assert np.abs(acc - ref).max() <= 1e-11 * np.abs(ref).max()
    again = xp.direct_fourier(x2, y2, signs(200), 128,
                              xp.direct_fourier(x1, y1, signs(128), 128))
    assert np.array_equal(acc, again)


@pytest.mark.gpu
def test_xpattern_edges(pkg):
    z = xp.direct_fourier(np.zeros(0), np.zeros(0), np.zeros(0), 16)
    assert z.shape == (4, 9) and not z.any()
    x, y, _ = pkg.dconf.generate_internal(8, 3)
    got = xp.direct_fourier(x, y, signs(8), 3)  # K = 2
    ref = xpattern_ref.direct_fourier(x, y, signs(8), 3)
    assert np.abs(got - ref).max() <= 1e-12 * np.abs(ref).max()
    with pytest.raises(Exception):
        xp.direct_fourier(x, y, signs(8), 1)


@pytest.mark.gpu
def test_xpattern_cli_files(pkg, tmp_path):
    paths = []
    for k, (n, seed) in enumerate(((64, 11), (96, 12))):
        x, y, _ = pkg.dconf.generate_internal(n, seed)
        p = tmp_path / ("c%d.dconf" % k)
        pkg.dconf.write(str(p), x, y, signs(n))
        paths.append(str(p))
    lst = tmp_path / "list.ini"
    lst.write_text("\n".join(paths) + "\n")
    prefix = str(tmp_path / "out_")
    assert xp.main(["-c", "-i", str(lst), "-m", "df", "-r", "64", "-o", prefix, "-s", "4",
                    "-d", "1", "--digits", "17"], io.StringIO()) == 0
    ref = sum(xpattern_ref.direct_fourier(*pkg.dconf.read(p), 64) for p in paths)
    for m, name in enumerate(xp.NAMES):
        lines = open("%sdf_r64_%s_k.txt" % (prefix, name)).read().splitlines()
        assert lines[0].startswith("# This file contains the Fourier components of " + name)
        vals = np.array([float(v) for v in lines[1:]])
        assert vals.shape == (33,)
        assert np.abs(vals - ref[m]).max() <= 1e-11 * np.abs(ref).max()
