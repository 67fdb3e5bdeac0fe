"""Writes tests/golden/stiff_4096.npz: a state of the N=4096 dense workload
(seed 1002 of dconf.generate_internal, constant stress 0.1) after 157
accepted steps of the plain FP64 form, with the step size the run attempts
next.  Two dislocation clusters have formed by then; the Jacobian's 128 x 128
diagonal tiles are ill-conditioned enough that their Gauss-Jordan inverses
alone leave the mixed form's refined solves stagnating (the block LU's
regression case).  Needs a GPU:  python tests/golden/make_stiff.py [out.npz]
"""
import importlib
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))


def main(out):
    pkg = importlib.import_module("2d4_b200")
    x, y, _ = pkg.dconf.generate_internal(4096, 1002)
    sd = pkg.SimulationData()
    sd.set_positions(x, y)
    sd.external_stress = pkg.FixedRateProtocol(0.1, 0.0)
    e = pkg.Engine(sd)
    e.advance(157)
    r = e.advance(0)
    xs, _ = e.positions()
    e.close()
    np.savez_compressed(out, x=xs, y=y, t=r.sim_time, h=r.step_size)
    print("t = %.6e, h = %.3e" % (r.sim_time, r.step_size))


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else os.path.join(HERE, "stiff_4096.npz"))
