"""Generates tests/golden/golden_runs.npz from the reference itself.

Run here (where the reference tree and oracle/_ref are present):
    make -C oracle ref && python tests/golden/make_golden_runs.py [case ...]

Every array is an output of the reference core built from its own sources
(oracle/_ref/libd4ref_exact.so: src/*.cpp of danieltuzes/2D4 compiled
unmodified, -O2 -ffp-contract=off, with the project's UMFPACK shim):
  c2_*   the headline workload's own step sequence: 100 accepted steps
         (-C 99) at constant stress 0.05 (FixedRateProtocol(0.05, 0)),
         default precision, from the relaxed N=1024 state of
         c2_relaxed_1024.npz; final positions and the accepted/failed counts;
  c3_*   N=4096 (seed 1002, iid uniform, balanced signs), dense Jacobian, 20
         accepted steps at tau = 0.1; the shim's LU is backed by OpenBLAS
         dgetrf/dgetrs here (the single-threaded shim would take hours), so
         these positions carry OpenBLAS's rounding of the solves;
  log_*  the reference's input fixture 1000_64.dconf, tau = 0.1, P = 1e-6,
         strain and order parameter on, 100 accepted steps, with its 15-column
         log (src/simulation.cpp:52-83,184-209; '-' stored as NaN) and the
         sub-configuration dumps (-o prefix, -N 5, -T 2e-4 -b a:
         src/simulation.cpp:232-247, simulation_data.cpp:231-246) by file name;
  aval_* the same fixture at zero stress, P = 1e-8, stopped by the avalanche
         detection limit 0 with speed threshold 0.05 (src/simulation.cpp:215-230,
         722-750): final positions, counts and simulation time;
  ieee_* the IEEE variant of the field (src/Fields/Field.cpp:26-168) on the
         field grid of golden.npz, from the reference's own IEEE evaluator
         (sandbox/ieee_hyperbolic/ieee_hyperbolic.cpp:103-140, built in place
         as oracle/_ref/libd4ref_ieee.so).
Each case runs in its own process (the shim picks its LU backend at load).
"""
import glob
import importlib
import os
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))
OUT = os.path.join(HERE, "golden_runs.npz")


def reference_root():
    env = os.environ.get("D4_REFERENCE_ROOT")
    if env:
        return env
    r = subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle"), "ref-root"],
                       capture_output=True, text=True, check=True)
    return r.stdout.strip()


def parse_full_log(path):
    rows = []
    with open(path) as f:
        for line in f:
            if line.startswith("#"):
                continue
            t = line.rstrip("\n").split("\t")
            rows.append([np.nan if v.strip() == "-" else float(v) for v in t[:15]])
    return np.array(rows)


def write_dconf(dconf, path, x, y):
    b = np.where(np.arange(len(x)) < len(x) // 2, 1, -1)
    dconf.write(path, x, y, b, digits=17)


def case(name):
    import pyoracle
    dconf = importlib.import_module("2d4_b200.dconf")
    tmp = tempfile.mkdtemp()
    out = {}
    if name == "c2":
        z = np.load(os.path.join(HERE, "c2_relaxed_1024.npz"))
        path = os.path.join(tmp, "c2.dconf")
        write_dconf(dconf, path, z["x"], z["y"])
        ref = pyoracle.Reference("exact")
        p = ref.params(step_count_limit=99, const_external_stress=0.05, has_rate=1, rate=0.0)
        xr, yr, res, wall = ref.run(path, p)
    elif name == "c3":
        import scipy
        libs = glob.glob(os.path.join(os.path.dirname(scipy.__file__), "..", "scipy.libs",
                                      "libscipy_openblas-*.so"))
        os.environ["D4REF_OPENBLAS"] = libs[0]
        os.environ.setdefault("D4REF_THREADS", str(os.cpu_count() or 1))
        x, y, b = dconf.generate(4096, 1002)
        path = os.path.join(tmp, "c3.dconf")
        dconf.write(path, x, y, b, digits=17)
        ref = pyoracle.Reference("exact")
        p = ref.params(step_count_limit=19, const_external_stress=0.1, has_rate=1, rate=0.0)
        xr, yr, res, wall = ref.run(path, p)
    elif name == "log":
        path = os.path.join(reference_root(), "init_config_gen", "README_files", "1000_64.dconf")
        ref = pyoracle.Reference("exact")
        log = os.path.join(tmp, "run.log")
        prefix = os.path.join(tmp, "sub_")
        p = ref.params(position_precision=1e-6, step_count_limit=99, const_external_stress=0.1,
                       has_rate=1, rate=0.0, calculate_strain=1, calculate_order_parameter=1,
                       sub_config_path=prefix, sub_config_delay=5, sub_config_times=2e-4,
                       sub_config_times_type="a")
        xr, yr, res, wall = ref.run(path, p, log_path=log)
        out["log_rows"] = parse_full_log(log)
        names = sorted(os.path.basename(f)[len("sub_"):] for f in glob.glob(prefix + "*"))
        out["log_sub_names"] = np.array(names)
        for k, nm in enumerate(names):
            out["log_sub_%d" % k] = np.loadtxt(prefix + nm, ndmin=2)
    elif name == "ieee":
        import ctypes as C
        L = C.CDLL(os.path.join(ROOT, "oracle", "_ref", "libd4ref_ieee.so"))
        for f in ("d4ref_ieee_xy", "d4ref_ieee_xy_diff_x"):
            getattr(L, f).restype = C.c_double
            getattr(L, f).argtypes = [C.c_double, C.c_double]
        g = np.load(os.path.join(HERE, "golden.npz"))
        fx, fy = g["field_dx"], g["field_dy"]
        out["ieee_xy"] = np.array([L.d4ref_ieee_xy(a, b) for a, b in zip(fx, fy)])
        out["ieee_xyd"] = np.array([L.d4ref_ieee_xy_diff_x(a, b) for a, b in zip(fx, fy)])
        tmpnpz = os.path.join(tmp, name + ".npz")
        np.savez_compressed(tmpnpz, **out)
        return tmpnpz
    elif name == "aval":
        path = os.path.join(reference_root(), "init_config_gen", "README_files", "1000_64.dconf")
        ref = pyoracle.Reference("exact")
        p = ref.params(position_precision=1e-8, avalanche_limit=0, avalanche_speed_threshold=0.05)
        xr, yr, res, wall = ref.run(path, p)
    else:
        raise ValueError(name)
    out[name + "_x"] = xr
    out[name + "_res"] = np.array([res.sim_time, res.step_size, res.successful_steps,
                                   res.failed_steps, res.strain])
    tmpnpz = os.path.join(tmp, name + ".npz")
    np.savez_compressed(tmpnpz, **out)
    print("%s: %d accepted, %d failed, %.1f s" % (name, res.successful_steps, res.failed_steps,
                                                  wall), flush=True)
    return tmpnpz


def main(argv):
    names = argv or ["log", "aval", "ieee", "c2", "c3"]
    merged = dict(np.load(OUT)) if os.path.exists(OUT) else {}
    for name in names:
        r = subprocess.run([sys.executable, os.path.abspath(__file__), "--case", name],
                           capture_output=True, text=True, check=True)
        print(r.stdout.strip())
        part = r.stdout.strip().splitlines()[-1].split("->")[-1].strip()
        merged.update(dict(np.load(part)))
    np.savez_compressed(OUT, **merged)
    print("wrote", OUT)


if __name__ == "__main__":
    if len(sys.argv) > 2 and sys.argv[1] == "--case":
        print("->", case(sys.argv[2]))
    else:
        main(sys.argv[1:])
