"""Relaxed N=1024 starting state of the plain FP64 configuration.

The reference core (oracle/_ref/libd4ref_fast.so, reference flags, UMFPACK shim
backed by OpenBLAS) relaxes the seeded configuration (N=1024, seed 1001, iid
uniform, balanced signs) for 500 accepted steps at zero stress with default
precision (-P 1e-5 -p 0.05), i.e. `-C 499`.  The final positions, in the
reference's internal order and at full precision, go to c2_relaxed_1024.npz;
the bench and the tests then run constant stress 0.05 from this state with
time and step size reset (a new reference run from the written state).

Run here: make -C oracle ref && python tests/golden/make_relaxed.py
"""
import glob
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


def main():
    import scipy
    libs = glob.glob(os.path.join(os.path.dirname(scipy.__file__), "..", "scipy.libs",
                                  "libscipy_openblas-*.so"))
    if libs:
        os.environ["D4REF_OPENBLAS"] = libs[0]
    ref = pyoracle.Reference("fast")
    x, y, b = dconf.generate(1024, 1001)
    path = os.path.join(tempfile.mkdtemp(), "c2.dconf")
    dconf.write(path, x, y, b, digits=17)
    p = ref.params(step_count_limit=499)
    xr, yr, res, wall = ref.run(path, p)
    np.savez_compressed(os.path.join(HERE, "c2_relaxed_1024.npz"), x=xr, y=yr,
                        res=np.array([res.sim_time, res.step_size, res.successful_steps,
                                      res.failed_steps, wall]))
    print("relaxed: %d accepted, %d failed, %.1f s" % (res.successful_steps, res.failed_steps,
                                                      wall))


if __name__ == "__main__":
    main()
