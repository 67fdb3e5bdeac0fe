"""ctypes bindings of the CPU oracles.  TEST AND BASELINE INFRASTRUCTURE ONLY.

Only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline / reference
legs use this module, as the checker or the timed CPU baseline.

- ``restated()``: oracle/lib/libd4oracle.so, the C restatement (d4_oracle.c).
- ``reference(kind)``: oracle/_ref/libd4ref_{exact,fast}.so, the reference core
  built from its own sources (oracle/Makefile); absent where it was not built.
"""
import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
RESTATED = os.path.join(HERE, "lib", "libd4oracle.so")
REF_DIR = os.path.join(HERE, "_ref")

_dp = C.POINTER(C.c_double)


def ptr(a):
    return None if a is None else a.ctypes.data_as(_dp)


class OProtocol(C.Structure):
    _fields_ = [("kind", C.c_int), ("tau0", C.c_double), ("rate", C.c_double),
                ("period", C.c_double), ("amp_rate", C.c_double)]


class OParams(C.Structure):
    _fields_ = [
        ("position_precision", C.c_double), ("dipole_precision", C.c_double),
        ("cutoff_multiplier", C.c_double), ("heaviside_cutoff", C.c_int),
        ("initial_stepsize", C.c_double), ("max_stepsize", C.c_double),
        ("weight_function", C.c_char), ("time_limit", C.c_double),
        ("step_count_limit", C.c_longlong), ("strain_increase_limit", C.c_double),
        ("calculate_strain", C.c_int), ("avalanche_limit", C.c_longlong),
        ("avalanche_speed_threshold", C.c_double), ("save_sub_configs", C.c_int),
        ("sub_config_delay", C.c_uint), ("sub_config_delay_during_avalanche", C.c_uint),
        ("sub_config_times", C.c_double), ("sub_config_times_type", C.c_char),
        ("protocol", OProtocol)]


class OResult(C.Structure):
    _fields_ = [("sim_time", C.c_double), ("step_size", C.c_double), ("strain", C.c_double),
                ("successful_steps", C.c_longlong), ("failed_steps", C.c_longlong),
                ("energy", C.c_double)]


class OAttempt(C.Structure):
    _fields_ = [("sim_time", C.c_double), ("step_size", C.c_double), ("ratio", C.c_double),
                ("max_id", C.c_int), ("accepted", C.c_int)]


class RParams(C.Structure):
    _fields_ = [
        ("position_precision", C.c_double), ("dipole_precision", C.c_double),
        ("cutoff_multiplier", C.c_double), ("heaviside_cutoff", C.c_int),
        ("initial_stepsize", C.c_double), ("max_stepsize", C.c_double),
        ("weight_function", C.c_char), ("time_limit", C.c_double),
        ("step_count_limit", C.c_longlong), ("strain_increase_limit", C.c_double),
        ("calculate_strain", C.c_int), ("calculate_order_parameter", C.c_int),
        ("const_external_stress", C.c_double), ("has_rate", C.c_int), ("rate", C.c_double),
        ("has_cyclic", C.c_int), ("cyclic_period", C.c_double),
        ("has_amplitude_rate", C.c_int), ("amplitude_rate", C.c_double),
        ("sub_config_path", C.c_char_p), ("sub_config_delay", C.c_uint),
        ("sub_config_delay_during_avalanche", C.c_uint), ("sub_config_times", C.c_double),
        ("sub_config_times_type", C.c_char), ("avalanche_limit", C.c_longlong),
        ("avalanche_speed_threshold", C.c_double)]


class RResult(C.Structure):
    _fields_ = [("sim_time", C.c_double), ("step_size", C.c_double), ("strain", C.c_double),
                ("successful_steps", C.c_longlong), ("failed_steps", C.c_longlong),
                ("n", C.c_int)]


class Restated:
    """The C restatement, with numpy-friendly wrappers."""

    def __init__(self, path=RESTATED):
        if not os.path.exists(path):
            raise RuntimeError("oracle not built: make -C oracle restated")
        L = C.CDLL(path)
        for f in ("d4o_xy", "d4o_xy_diff_x", "d4o_xy4", "d4o_xy_diff_x4", "d4o_normalize",
                  "d4o_weight", "d4o_weight_inv", "d4o_ext_stress"):
            getattr(L, f).restype = C.c_double
        for f in ("d4o_ieee_xy", "d4o_ieee_xy_diff_x"):
            getattr(L, f).restype = C.c_double
            getattr(L, f).argtypes = [C.c_double, C.c_double]
        for f in ("d4o_xy", "d4o_xy_diff_x"):
            getattr(L, f).argtypes = [C.c_double, C.c_double]
        for f in ("d4o_xy4", "d4o_xy_diff_x4"):
            getattr(L, f).argtypes = [C.c_double] * 4
        L.d4o_normalize.argtypes = [C.c_double]
        L.d4o_weight.argtypes = [C.c_double, C.c_char]
        L.d4o_weight_inv.argtypes = [C.c_double, C.c_char]
        L.d4o_ext_stress.argtypes = [C.POINTER(OProtocol), C.c_double]
        L.d4o_run.restype = C.c_longlong
        self.L = L

    def params(self, **kw):
        p = OParams()
        self.L.d4o_default_params(C.byref(p))
        proto = kw.pop("protocol", None)
        for k, v in kw.items():
            if k in ("weight_function", "sub_config_times_type"):
                v = v.encode() if isinstance(v, str) else v
            setattr(p, k, v)
        if proto:
            for k, v in proto.items():
                setattr(p.protocol, k, v)
        return p

    @staticmethod
    def derived(p, n):
        """min_prec_sq, use_dipole, cutoff, cutoff_sq as Simulation's ctor and
        SimulationData::updateCutOff compute them."""
        mps = p.position_precision * p.position_precision
        use = p.dipole_precision != 0
        if use:
            mps /= p.dipole_precision * p.dipole_precision
        mult = p.cutoff_multiplier
        if not p.heaviside_cutoff and p.cutoff_multiplier >= np.sqrt(2 * float(n)) / 12:
            mult = 1e20
        cut = mult / np.sqrt(float(n))
        return mps, use, cut, cut * cut

    def speeds(self, x, y, ext, tol=None, min_prec_sq=0.0):
        n = len(x)
        v = np.empty(n)
        self.L.d4o_speeds(n, ptr(x), ptr(y), C.c_double(ext), ptr(v), ptr(tol),
                          C.c_double(min_prec_sq))
        return v

    def jacobian(self, x, y, h, ext_a, ext_b, cut_sq, cut, heaviside=0, wfn="c", tol=None,
                 min_prec_sq=0.0):
        n = len(x)
        va, vb, d = np.empty(n), np.empty(n), np.empty(n)
        a = np.empty((n, n))  # row-major
        self.L.d4o_jacobian(n, ptr(x), ptr(y), C.c_double(h), C.c_double(ext_a),
                            C.c_double(ext_b), C.c_double(cut_sq), C.c_double(cut),
                            int(heaviside), C.c_char(wfn.encode()), ptr(va), ptr(vb), ptr(a),
                            ptr(d), ptr(tol), C.c_double(min_prec_sq))
        return va, vb, a, d

    def jacobian_from_prev(self, a, dvec, factor, wfn="c"):
        a = np.ascontiguousarray(a)
        dvec = dvec.copy()
        self.L.d4o_jacobian_from_prev(len(dvec), ptr(a), ptr(dvec), C.c_double(factor),
                                      C.c_char(wfn.encode()))
        return a, dvec

    def lu_solve(self, a_rowmajor, g):
        n = len(g)
        lu = np.asfortranarray(a_rowmajor).copy(order="F")
        piv = np.zeros(n, dtype=np.int32)
        sing = self.L.d4o_lu(n, lu.ctypes.data_as(_dp), piv.ctypes.data_as(C.POINTER(C.c_int)))
        x = np.ascontiguousarray(g, dtype=np.float64).copy()
        self.L.d4o_lu_solve(n, lu.ctypes.data_as(_dp), piv.ctypes.data_as(C.POINTER(C.c_int)),
                            ptr(x))
        return x, sing, piv

    def attempt(self, x0, y, t0, h, p, tol):
        n = len(x0)
        xb, xh, x2 = np.empty(n), np.empty(n), np.empty(n)
        tol = tol.copy()
        r = C.c_double()
        i = C.c_int()
        self.L.d4o_attempt_step(n, ptr(x0), ptr(y), C.c_double(t0), C.c_double(h), C.byref(p),
                                ptr(xb), ptr(xh), ptr(x2), ptr(tol), C.byref(r), C.byref(i))
        return xb, xh, x2, tol, r.value, i.value

    def run(self, x, y, p, record=0):
        x = x.copy()
        y = y.copy()
        res = OResult()
        rec = (OAttempt * max(record, 1))()
        na = self.L.d4o_run(len(x), ptr(x), ptr(y), C.byref(p), C.byref(res),
                            rec if record else None, C.c_longlong(record))
        recs = [(r.sim_time, r.step_size, r.ratio, r.max_id, r.accepted)
                for r in list(rec)[:min(na, record)]] if record else []
        return x, res, na, recs


class Reference:
    """The reference core built from its sources (oracle/_ref)."""

    def __init__(self, kind="exact"):
        path = os.path.join(REF_DIR, "libd4ref_%s.so" % kind)
        if not os.path.exists(path):
            raise RuntimeError("reference oracle not built: make -C oracle ref")
        L = C.CDLL(path)
        for f in ("d4ref_xy", "d4ref_xy_diff_x"):
            getattr(L, f).restype = C.c_double
            getattr(L, f).argtypes = [C.c_double, C.c_double]
        self.L = L

    @staticmethod
    def available(kind="exact"):
        return os.path.exists(os.path.join(REF_DIR, "libd4ref_%s.so" % kind))

    def params(self, **kw):
        p = RParams()
        self.L.d4ref_default_params(C.byref(p))
        for k, v in kw.items():
            if k in ("weight_function", "sub_config_times_type", "sub_config_path"):
                v = v.encode()
            setattr(p, k, v)
        p._keep = [getattr(p, "sub_config_path")]  # the path's bytes live as long as p
        return p

    def load(self, path, cap=1 << 20):
        n = C.c_int()
        x, y = np.empty(cap), np.empty(cap)
        order = np.empty(cap, dtype=np.uint32)
        self.L.d4ref_load(path.encode(), C.byref(n), ptr(x), ptr(y),
                          order.ctypes.data_as(C.POINTER(C.c_uint)), cap)
        k = n.value
        return x[:k].copy(), y[:k].copy(), order[:k].copy()

    def speeds(self, path, p, x, y, t):
        n = len(x)
        v, tol = np.empty(n), np.empty(n)
        self.L.d4ref_speeds(path.encode(), C.byref(p), ptr(x), ptr(y), C.c_double(t), ptr(v),
                            ptr(tol))
        return v, tol

    def jacobian(self, path, p, x, y, h, ta, tb):
        n = len(x)
        va, vb, d, tol = np.empty(n), np.empty(n), np.empty(n), np.empty(n)
        a = np.empty((n, n))
        nnz = C.c_int()
        self.L.d4ref_jacobian(path.encode(), C.byref(p), ptr(x), ptr(y), C.c_double(h),
                              C.c_double(ta), C.c_double(tb), ptr(va), ptr(vb), ptr(a), ptr(d),
                              ptr(tol), C.byref(nnz))
        return va, vb, a, d, tol, nnz.value

    def run(self, path, p, log_path=None):
        res = RResult()
        n = self.load(path)[0].size
        x, y = np.empty(n), np.empty(n)
        wall = C.c_double()
        self.L.d4ref_run(path.encode(), b"/dev/null", log_path.encode() if log_path else None,
                         C.byref(p), C.byref(res), ptr(x), ptr(y), C.byref(wall))
        return x, y, res, wall.value
