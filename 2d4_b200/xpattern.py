"""Direct-Fourier pattern analysis on the GPU (the reference's xpattern tool,
method ``df``: xpattern/xpattern.cpp:393-423, README.md "Direct Fourier").

For each configuration, with K = res/2 + 1,

    F_m(kx, ky) = sum_i w_m(b_i) exp(-2 pi i (kx x_i + ky y_i))

for the densities m = rho_t (w = 1), kappa (w = b), rho_p (b = +1) and rho_n
(b = -1); the tool's output for density m is sum_ky |F_m(kx, ky)|^2 for
kx = 0..K-1, summed over all input configurations.  ``direct_fourier`` runs
one configuration through ``d4_xpattern_df`` (FP64 on the device, no
atomics); ``python -m 2d4_b200.xpattern -i conf.dconf|list.ini -r 1024 -m df
-o prefix`` takes the tool's options and writes its four files
``<prefix>df_r<res>_<name>_k.txt``.
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


class ToolExit(Exception):
    """A stop of the command line: message and exit status.  The reference
    tool writes every one of these messages to std::cerr, the unreadable .ini
    file's too although it then returns 0 (xpattern/xpattern.cpp:76-120), so
    to_stderr defaults to True."""

    def __init__(self, message, status, to_stderr=True):
        super().__init__(message)
        self.message, self.status, self.to_stderr = message, status, to_stderr


def input_files(path, out=None):
    """The tool's input (xpattern/xpattern.cpp:76-120): a path ending in .dconf,
    or a path ending in .ini whose whitespace-separated entries are .dconf
    paths.  Raises ToolExit with the tool's messages and statuses."""
    out = out or sys.stdout
    if path.endswith(".ini"):
        try:
            with open(path) as f:
                toks = f.read().split()
        except OSError:
            raise ToolExit("The program couldn't open %s for reading. Program terminates." % path, 0)
        for t in toks:
            if not t.endswith(".dconf"):
                raise ToolExit("%s contains invalid dislocation configuration filename %s. "
                               "Program termiantes." % (path, t), 2)
        print("%s as input path contained %d number of files to read." % (path, len(toks)),
              file=out)
        if not toks:
            raise ToolExit("Not enough input files. Program terminates.", 1)
        return toks
    if path.endswith(".dconf"):
        print("%s will be used to read dislocation configuration" % path, file=out)
        return [path]
    raise ToolExit("%s is not a valid input filename. Program terminates." % path, 1)


def main(argv=None, out=None, err=None):
    """The tool's command line (option table xpattern/xpattern.cpp:26-48):
    -i/--input-fname, -r/--resolution (1024), -m/--method (default bc, as in
    the tool; only df is built here), -o/--output-fnameprefix, and the
    options that do not act on df (-s/--sub-sampling, -w/--half-width,
    -d/--debug-level) are accepted.  --create-maps is not built.  An unknown
    method stops with a message (the tool would write all-zero files).
    --digits (not in the tool): significant digits of the values, 6 as the
    tool writes them."""
    out, err = out or sys.stdout, err or sys.stderr

    class _Parser(argparse.ArgumentParser):
        def error(self, message):  # as Boost's parse errors: message, exit(-1)
            raise ToolExit(message, 255)

    p = _Parser(prog="2d4_b200.xpattern", add_help=False)
    p.add_argument("-i", "--input-fname")
    p.add_argument("-r", "--resolution", type=int, default=1024)
    p.add_argument("-m", "--method", default="bc")
    p.add_argument("-s", "--sub-sampling", type=int, default=1)
    p.add_argument("-w", "--half-width", type=float)
    p.add_argument("--create-maps", action="store_true")
    p.add_argument("-o", "--output-fnameprefix", default="")
    p.add_argument("-d", "--debug-level", type=int, default=0)
    p.add_argument("--help", action="store_true")
    p.add_argument("-c", "--hide-copyright", action="store_true")
    p.add_argument("--digits", type=int, default=6)
    try:
        args = p.parse_args(argv)
        if args.help:
            print(p.format_help(), file=out)
            return 0
        if not args.input_fname:
            raise ToolExit("input-fname is missing! Program terminates.", 255)
        files = input_files(args.input_fname, out)
        print("output-fnameprefix = \t%s" % args.output_fnameprefix, file=out)
        res = args.resolution
        if res < 2:
            raise ToolExit("Error: resulution is smaller than 2. Program terminates.", 255)
        if args.method != "df":
            known = args.method in ("bc", "gs", "wspn", "wsts")
            raise ToolExit("Method %s is %s; this engine builds only df (direct Fourier). "
                           "Program terminates." % (args.method, "not built here" if known
                                                     else "unknown"), 255)
        if args.create_maps:
            raise ToolExit("--create-maps is not built here (only the k spectra of df). "
                           "Program terminates.", 255)
    except ToolExit as e:
        print(e.message, file=err if e.to_stderr else out)
        return e.status
    acc = None
    for f in files:
        x, y, b = dconf.read(f)
        acc = direct_fourier(x, y, b, res, acc)
    extra = "df_r%d" % res
    for m, name in enumerate(NAMES):
        fn = "%s%s_%s_k.txt" % (args.output_fnameprefix, extra, name)
        with open(fn, "w") as fo:
            fo.write("# This file contains the Fourier components of %s for the file %s using "
                     "the direct Fourier method.\n" % (name, args.input_fname))
            for v in acc[m]:
                fo.write("%.*g\n" % (args.digits, v))
    print("Done. Program terminates.", file=out)
    return 0


if __name__ == "__main__":
    sys.exit(main())
