"""Generates the golden fixtures of tests/golden/ from the reference itself.

Run here (where the reference tree and oracle/_ref are present):
    make -C oracle ref && python tests/golden/make_golden.py

Every array in golden.npz is an output of the reference core
(oracle/_ref/libd4ref_exact.so: src/*.cpp of danieltuzes/2D4 compiled
unmodified, -O2 -ffp-contract=off, with the project's UMFPACK shim), on:
  - the reference's own input fixture init_config_gen/README_files/1000_64.dconf
    (N=64, its positions are stored here too, as read and sorted by the
    reference's loader);
  - seeded synthetic configurations from 2d4_b200.dconf.generate.
The tests pin the C restatement (oracle/d4_oracle.c) to these arrays bit for
bit, and the GPU path to the restatement.
"""
import importlib
import os
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))
import pyoracle  # noqa: E402

dconf = importlib.import_module("2d4_b200.dconf")


def reference_root():
    """The reference tree: $D4_REFERENCE_ROOT, else the oracle recipe's default."""
    import subprocess
    env = os.environ.get("D4_REFERENCE_ROOT")
    if env:
        return env
    r = subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle"), "ref-root"],
                       capture_output=True, text=True, check=True)
    return r.stdout.strip()


REF_FIXTURE = os.path.join(reference_root(), "init_config_gen", "README_files", "1000_64.dconf")


def parse_log(path):
    rows = []
    with open(path) as f:
        for line in f:
            if line.startswith("#"):
                continue
            t = line.split("\t")
            rows.append([float(t[0]), float(t[1]), float(t[2]), float(t[3]), float(t[4]),
                         float(t[14])])
    return np.array(rows[1:])  # first row is the t=0 line


def main():
    ref = pyoracle.Reference("exact")
    out = {}
    tmp = tempfile.mkdtemp()
    # field known-answer grid: the sandbox's lattice (sandbox/ieee_hyperbolic/
    # ieee_hyperbolic.cpp:527-607: x, y from 1/107183 in steps of 1/300),
    # subsampled, folded into [-0.5, 0.5), plus near-field (Taylor branch) points
    g = 1.0 / 107183 + np.arange(0, 300, 7) / 300.0
    gx, gy = np.meshgrid(g - 0.5, g - 0.5, indexing="ij")
    rng = np.random.default_rng(7)
    near = rng.uniform(-6e-4, 6e-4, (400, 2))
    fx = np.concatenate([gx.ravel(), near[:, 0], rng.uniform(-0.5, 0.5, 600)])
    fy = np.concatenate([gy.ravel(), near[:, 1], rng.uniform(-0.5, 0.5, 600)])
    out["field_dx"], out["field_dy"] = fx, fy
    out["field_xy"] = np.array([ref.L.d4ref_xy(a, b) for a, b in zip(fx, fy)])
    out["field_xyd"] = np.array([ref.L.d4ref_xy_diff_x(a, b) for a, b in zip(fx, fy)])

    cases = {"fix64": REF_FIXTURE}
    x, y, b = dconf.generate(64, 1000)
    p = os.path.join(tmp, "s64.dconf")
    dconf.write(p, x, y, b, digits=17)
    cases["seed64"] = p
    x, y, b = dconf.generate(256, 1005)
    p = os.path.join(tmp, "s256.dconf")
    dconf.write(p, x, y, b, digits=17)
    cases["seed256"] = p

    for name, path in cases.items():
        xs, ys, order = ref.load(path)
        out[name + "_x"], out[name + "_y"], out[name + "_order"] = xs, ys, order
        prm = ref.params(position_precision=1e-8)
        v, tol = ref.speeds(path, prm, xs, ys, 0.0)
        out[name + "_v"], out[name + "_tol"] = v, tol
        if len(xs) > 64:
            continue
        va, vb, a, d, tol2, nnz = ref.jacobian(path, prm, xs, ys, 1e-3, 0.0, 1e-3)
        out[name + "_jac_va"], out[name + "_jac_vb"] = va, vb
        out[name + "_jac_a"], out[name + "_jac_d"], out[name + "_jac_tol"] = a, d, tol2
        # cutoff variants (N=64): Gaussian-tail cutoff u = 0.5 (c = 1/16) and
        # heaviside u = 1 (c = 1/8)
        for tag, kw in (("cutg", dict(cutoff_multiplier=0.5)),
                        ("cuth", dict(cutoff_multiplier=1.0, heaviside_cutoff=1)),
                        ("wp", dict(weight_function="p")), ("wm", dict(weight_function="m"))):
            pr = ref.params(position_precision=1e-8, **kw)
            va, vb, a, d, tol2, nnz = ref.jacobian(path, pr, xs, ys, 2e-3, 0.0, 2e-3)
            out["%s_%s_a" % (name, tag)], out["%s_%s_d" % (name, tag)] = a, d
            out["%s_%s_nnz" % (name, tag)] = np.array(nnz)
        # C1 run: 1000 accepted steps at P = 1e-8 (-C 999), tau = 0
        log = os.path.join(tmp, name + ".log")
        pr = ref.params(position_precision=1e-8, step_count_limit=999)
        xr, yr, res, _ = ref.run(path, pr, log_path=log)
        out[name + "_run_x"] = xr
        out[name + "_run_res"] = np.array([res.sim_time, res.step_size, res.successful_steps,
                                           res.failed_steps])
        out[name + "_run_log"] = parse_log(log)
        # constant stress (FixedRateProtocol(0.1, 0), i.e. -s 0.1 -r 0), P = 1e-6,
        # strain on, 200 steps
        log = os.path.join(tmp, name + "_tau.log")
        pr = ref.params(position_precision=1e-6, step_count_limit=199, const_external_stress=0.1,
                        has_rate=1, rate=0.0, calculate_strain=1)
        xr, yr, res, _ = ref.run(path, pr, log_path=log)
        out[name + "_tau_x"] = xr
        out[name + "_tau_res"] = np.array([res.sim_time, res.step_size, res.successful_steps,
                                           res.failed_steps, res.strain])
        # cyclic load with dipole criterion off, 150 steps
        pr = ref.params(position_precision=1e-6, dipole_precision=0.0, step_count_limit=149,
                        const_external_stress=0.0, has_rate=1, rate=5.0, has_cyclic=1,
                        cyclic_period=0.01)
        xr, yr, res, _ = ref.run(path, pr)
        out[name + "_cyc_x"] = xr
        out[name + "_cyc_res"] = np.array([res.sim_time, res.step_size, res.successful_steps,
                                           res.failed_steps])
    np.savez_compressed(os.path.join(HERE, "golden.npz"), **out)
    print("wrote", os.path.join(HERE, "golden.npz"), sum(v.nbytes for v in out.values()), "bytes")


if __name__ == "__main__":
    main()
