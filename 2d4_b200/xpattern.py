"""Direct-Fourier pattern analysis on the GPU (the reference's xpattern tool,
method ``df``: xpattern/xpattern.cpp:393-423, README.md "Direct Fourier").

For each configuration, with K = res/2 + 1,

    F_m(kx, ky) = sum_i w_m(b_i) exp(-2 pi i (kx x_i + ky y_i))

for the densities m = rho_t (w = 1), kappa (w = b), rho_p (b = +1) and rho_n
(b = -1); the tool's output for density m is sum_ky |F_m(kx, ky)|^2 for
kx = 0..K-1, summed over all input configurations.  ``direct_fourier`` runs
one configuration through ``d4_xpattern_df`` (FP64 on the device, no
atomics); ``python -m 2d4_b200.xpattern -i conf.dconf|list.ini -r 1024 -m df
-o prefix`` writes the tool's four files ``<prefix>df_r<res>_<name>_k.txt``.
The tool's other methods (box counting, Gauss smoothing, Wigner-Seitz) are
not part of this engine; asking for them stops with a message.
"""
import argparse
import ctypes as C
import sys

import numpy as np

from . import _lib, dconf

NAMES = ("rho_t", "kappa", "rho_p", "rho_n")


def direct_fourier(x, y, b, res=1024, acc=None):
    """Adds one configuration's sum_ky |F_m|^2 to acc (shape (4, res//2+1),
    zeros if None) and returns it.  b: Burgers signs (+1 / -1)."""
    lib = _lib.load()
    x = np.ascontiguousarray(x, dtype=np.float64)
    y = np.ascontiguousarray(y, dtype=np.float64)
    bi = np.ascontiguousarray(np.rint(b), dtype=np.int32)
    if not (len(x) == len(y) == len(bi)):
        raise ValueError("x, y and b must have the same length")
    K = res // 2 + 1
    out = np.zeros((4, K)) if acc is None else np.ascontiguousarray(acc, dtype=np.float64)
    if out.shape != (4, K):
        raise ValueError("acc must have shape (4, %d)" % K)
    st = lib.d4_xpattern_df(len(x), _lib.ptr(x), _lib.ptr(y),
                            bi.ctypes.data_as(C.POINTER(C.c_int)), res, _lib.ptr(out))
    if st != 0:
        raise _lib.D4Error("d4_xpattern_df failed: %s" % _lib.D4_ERR.get(st, st))
    return out


def input_files(path):
    """A .dconf path, or a file listing one configuration path per line
    (the tool's .ini input)."""
    if path.endswith(".dconf"):
        return [path]
    with open(path) as f:
        return [line.strip() for line in f if line.strip()]


def main(argv=None, out=None):
    out = out or sys.stdout
    p = argparse.ArgumentParser(prog="2d4_b200.xpattern")
    p.add_argument("-i", "--input-path", required=True)
    p.add_argument("-r", "--resolution", type=int, default=1024)
    p.add_argument("-m", "--method", default="df")
    p.add_argument("-o", "--output-foldername", default="")
    p.add_argument("--digits", type=int, default=6,
                   help="significant digits of the written values (the tool writes 6)")
    args = p.parse_args(argv)
    if args.method != "df":
        print("Method %s is not available in this engine; only df (direct Fourier) is."
              % args.method, file=sys.stderr)
        return 255
    res = args.resolution
    acc = None
    for f in input_files(args.input_path):
        x, y, b = dconf.read(f)
        acc = direct_fourier(x, y, b, res, acc)
    if acc is None:
        acc = np.zeros((4, res // 2 + 1))
    extra = "df_r%d" % res
    for m, name in enumerate(NAMES):
        fn = "%s%s_%s_k.txt" % (args.output_foldername, extra, name)
        with open(fn, "w") as fo:
            fo.write("# This file contains the Fourier components of %s for the file %s using "
                     "the direct Fourier method.\n" % (name, args.input_path))
            for v in acc[m]:
                fo.write("%.*g\n" % (args.digits, v))
    print("Done. Program terminates.", file=out)
    return 0


if __name__ == "__main__":
    sys.exit(main())
