"""CPU restatement of the reference's direct-Fourier pattern analysis.
TEST INFRASTRUCTURE ONLY: only tests/ use it, as the checker of
d4_xpattern_df.

Parity unpinned: the reference tool (xpattern/) needs FFTW and
Boost.program_options, which are absent here, and its repository ships no
output files for this method (xpattern/example_with_64_dislocations holds no
data).  The restatement follows xpattern/xpattern.cpp:393-423 term for term:

- exp_f_x[k] = exp(-2 pi i x k), exp_f_y[k] = exp(-2 pi i y k), k = 0..res/2
  (:400-404);
- cmaps[0] += e_x e_y for every dislocation (rho_t), cmaps[1] += b e_x e_y
  (kappa), cmaps[2] for b == 1 (rho_p), cmaps[3] otherwise (rho_n) (:406-415);
- F_absValSqs[m][kx] += |cmaps[m][ky][kx]|^2 over ky (:419-422), summed over
  the input files.

``direct_fourier`` is the vectorised form; ``direct_fourier_loops`` the same
sums as plain loops, used to check it at tiny sizes.
"""
import cmath
import math

import numpy as np


def direct_fourier(x, y, b, res):
    x = np.asarray(x, dtype=np.float64)
    y = np.asarray(y, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    K = res // 2 + 1
    k = np.arange(K, dtype=np.float64)
    ex = np.exp(-2j * np.pi * np.outer(x, k))  # (n, K): [i][kx]
    ey = np.exp(-2j * np.pi * np.outer(y, k))  # (n, K): [i][ky]
    weights = (np.ones_like(b), b, (b == 1).astype(np.float64), (b != 1).astype(np.float64))
    out = np.zeros((4, K))
    for m, w in enumerate(weights):
        F = (ey * w[:, None]).T @ ex  # F[ky][kx]
        out[m] = (np.abs(F) ** 2).sum(axis=0)
    return out


def direct_fourier_loops(x, y, b, res):
    K = res // 2 + 1
    cm = [[[0j] * K for _ in range(K)] for _ in range(4)]
    for xi, yi, bi in zip(x, y, b):
        exf = [cmath.exp(-2 * math.pi * xi * k * 1j) for k in range(K)]
        eyf = [cmath.exp(-2 * math.pi * yi * k * 1j) for k in range(K)]
        for ky in range(K):
            for kx in range(K):
                t = exf[kx] * eyf[ky]
                cm[0][ky][kx] += t
                cm[1][ky][kx] += bi * t
                cm[2 if bi == 1 else 3][ky][kx] += t
    out = np.zeros((4, K))
    for m in range(4):
        for kx in range(K):
            for ky in range(K):
                out[m][kx] += abs(cm[m][ky][kx]) ** 2
    return out
