"""Dislocation configuration files (.dconf) and the seeded synthetic generator.

Format (src/simulation_data.cpp:76-154,177-191): whitespace-separated triplets
``x y b`` per line, b = +-1, sum(b) = 0.  On load the reference sorts the
dislocations by y + b descending (src/simulation_data.cpp:116), so all b = +1
come first and the Burgers vector of internal index i is +1 for i < n/2; the
output is written back in the original order with 14 significant digits.
"""
import numpy as np


def read(path):
    """Returns (x, y, b) in file order; raises ValueError like the reference
    exits (src/simulation_data.cpp:89-113)."""
    vals = []
    with open(path) as f:
        for tok in f.read().split():
            vals.append(float(tok))
    if len(vals) % 3 != 0:
        raise ValueError("%s: cannot read y and b for the last x" % path)
    a = np.array(vals, dtype=np.float64).reshape(-1, 3)
    x, y, b = a[:, 0].copy(), a[:, 1].copy(), a[:, 2].copy()
    if np.any(np.abs(b - np.rint(b)) > 1e-5):
        raise ValueError("%s: Burgers vector must be an integer" % path)
    if b.sum() != 0:
        raise ValueError("%s: sum of Burgers vectors is %g, not 0" % (path, b.sum()))
    return x, y, b


def sort_internal(x, y, b):
    """Internal order of the reference: key y + b descending.  Returns
    (xs, ys, order) with order[original] = internal index
    (src/simulation_data.cpp:116-123).  Ties keep the original order."""
    key = y + b
    idx = sorted(range(len(x)), key=lambda i: (-key[i], i))
    idx = np.array(idx, dtype=np.int64)
    order = np.empty(len(x), dtype=np.uint32)
    order[idx] = np.arange(len(x), dtype=np.uint32)
    return x[idx].copy(), y[idx].copy(), order


def load(path):
    x, y, b = read(path)
    return sort_internal(x, y, b)


def write(path, x, y, b, digits=14):
    with open(path, "w") as f:
        for xi, yi, bi in zip(x, y, b):
            f.write("%.*g\t%.*g\t%d\n" % (digits, xi, digits, yi, int(bi)))


def write_internal(path, xs, ys, order, digits=14):
    """Writes internal-order positions back in the original order
    (writeDislocationDataToFile, src/simulation_data.cpp:177-191)."""
    n = len(xs)
    with open(path, "w") as f:
        for k in range(n):
            i = int(order[k])
            f.write("%.*g\t%.*g\t%d\n" % (digits, xs[i], digits, ys[i], 1 if i < n // 2 else -1))


def generate(n, seed):
    """Seeded synthetic configuration: x, y iid U[-0.5, 0.5), b = +1 for the
    first n/2 and -1 for the rest.  Returns (x, y, b) in file order."""
    if n % 2:
        raise ValueError("n must be even (balanced Burgers vectors)")
    rng = np.random.default_rng(seed)
    x = rng.uniform(-0.5, 0.5, n)
    y = rng.uniform(-0.5, 0.5, n)
    b = np.where(np.arange(n) < n // 2, 1.0, -1.0)
    return x, y, b


def generate_internal(n, seed):
    x, y, b = generate(n, seed)
    return sort_internal(x, y, b)


def _normalize(v):
    while v < -0.5:
        v += 1
    while v >= 0.5:
        v -= 1
    return v


def conf_compare(xa, ya, xb, yb, ind_tol=1e-8):
    """The conf_compare metric (conf_compare/conf_compare.cpp:180-237) on two
    configurations in the same order: returns (max_diff, max_id, avg_abs,
    avg_sq); raises ValueError if a y coordinate differs by more than ind_tol.
    The per-dislocation difference is normalize(|xa - xb|) as there."""
    n = len(xa)
    max_diff, max_id, s, s2 = 0.0, 0, 0.0, 0.0
    for i in range(n):
        yd = _normalize(abs(ya[i] - yb[i]))
        if yd > ind_tol:
            raise ValueError("y values differ for dislocation %d" % i)
        d = _normalize(abs(xa[i] - xb[i]))
        s += d
        s2 += d * d
        if d > max_diff:
            max_diff, max_id = d, i
    return max_diff, max_id, s / n, s2 / n
