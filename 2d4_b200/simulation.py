"""Host-side mirror of the reference's Simulation / SimulationData API.

Names follow the reference's Python binding (src/bindings.cpp:141-207:
``SimulationData`` fields, ``Simulation.create(sd)``, ``run``, ``step``,
``get_time``) and C++ classes (include/simulation.h:122-240,
include/simulation_data.h:80-332).  Every call goes to libd4core.so through
the C ABI of include/d4core.h; there is no CPU path.
"""
import ctypes as C

import numpy as np

from . import _lib
from . import dconf


class StressProtocol:
    """StressProtocol (src/stress_protocol.cpp:8-16): returns 0 at all times,
    whatever initExtStress is (the reference's -s without -r)."""

    kind = _lib.D4_STRESS_NONE

    def __init__(self, init_ext_stress=0.0):
        self.init_ext_stress = float(init_ext_stress)

    def to_c(self):
        p = _lib.Protocol()
        p.kind = self.kind
        p.tau0 = self.init_ext_stress
        p.rate = getattr(self, "rate", 0.0)
        p.period = getattr(self, "period", 0.0)
        p.amplitude_rate = getattr(self, "amplitude_rate", 0.0)
        return p

    def ext_stress(self, t):
        return 0.0


class FixedRateProtocol(StressProtocol):
    """tau = tau0 + rate * t (src/stress_protocol.cpp:22-33)."""

    kind = _lib.D4_STRESS_FIXED_RATE

    def __init__(self, init_ext_stress=0.0, rate=0.0):
        super().__init__(init_ext_stress)
        self.rate = float(rate)

    def ext_stress(self, t):
        return t * self.rate + self.init_ext_stress


class CyclicLoadProtocol(FixedRateProtocol):
    """Triangle wave (src/stress_protocol.cpp:40-56)."""

    kind = _lib.D4_STRESS_CYCLIC

    def __init__(self, init_ext_stress=0.0, rate=0.0, period=0.0):
        super().__init__(init_ext_stress, rate)
        self.period = float(period)


class IncreasingCyclicLoadProtocol(CyclicLoadProtocol):
    """Triangle wave times amplitude_rate * t (src/stress_protocol.cpp:63-73)."""

    kind = _lib.D4_STRESS_INC_CYCLIC

    def __init__(self, init_ext_stress=0.0, rate=0.0, period=0.0, amplitude_rate=0.0):
        super().__init__(init_ext_stress, rate, period)
        self.amplitude_rate = float(amplitude_rate)


# The reference binding's names for the protocol objects.
StressProtocolObject = StressProtocol
FixedRateStressProtocolObject = FixedRateProtocol


class SimulationData:
    """State and parameters of one simulation (include/simulation_data.h:80-332).

    ``SimulationData(path, "")`` reads and sorts a .dconf like the reference's
    constructor.  The attribute names are those of the reference binding."""

    def __init__(self, dislocation_configuration_path=None, point_defect_path=""):
        if point_defect_path:
            raise NotImplementedError("point defects are disabled in the reference build")
        self.precision = 1e-5                  # prec (-P)
        self.dipole_precision = 0.05           # dipole_prec (-p)
        self.cutoff_multiplier = 1e20          # -u
        self.heaviside_cutoff = False          # -h
        self.step_size = 1e-6                  # stepSize (--initial-stepsize)
        self.initial_step_size = None
        self.max_stepsize_limit = 0.0
        self.max_step_size_limited = False
        self.weight_function = "c"
        self.time_limit = 0.0
        self.time_limited = False
        self.step_count_limit = 0
        self.step_count_limited = False
        self.total_accumulated_strain_increase_limit = 0.0
        self.strain_increase_limted = False     # (sic) the reference binding's name
        self.calculate_strain_during_simulation = False
        self.calculate_order_parameter = False
        self.count_avalanches = False
        self.avalanche_speed_threshold = 1e-3
        self.trigger_limit_for_avalanche_count = 0
        self.save_sub_configs = False
        self.sub_config_path = ""
        self.sub_config_delay = 5
        self.sub_config_delay_during_avalanche = 1
        self.sub_config_times = 0.0
        self.sub_config_times_type = "a"
        self.external_stress = StressProtocol()
        self.final_dislocation_configuration_path = ""
        self.logfile_path = ""
        self.precision_mode = _lib.D4_PREC_FP64
        self.solver = _lib.D4_SOLVER_DENSE
        self.field = _lib.D4_FIELD_ANALYTIC
        self.table_size = 1024
        self.simulation_time = 0.0
        self.successful_steps = 0
        self.failed_steps = 0
        self.total_accumulated_strain_increase = 0.0
        self.x = self.y = None
        self.order = None
        if dislocation_configuration_path:
            self.read_dislocation_data_from_file(dislocation_configuration_path)

    @property
    def dislocation_count(self):
        return 0 if self.x is None else len(self.x)

    def read_dislocation_data_from_file(self, path):
        self.x, self.y, self.order = dconf.load(path)

    def set_positions(self, x, y, order=None):
        """Positions in internal order (b = +1 first)."""
        self.x = np.ascontiguousarray(x, dtype=np.float64)
        self.y = np.ascontiguousarray(y, dtype=np.float64)
        self.order = (np.arange(len(x), dtype=np.uint32) if order is None
                      else np.asarray(order, dtype=np.uint32))

    def write_dislocation_data_to_file(self, path):
        dconf.write_internal(path, self.x, self.y, self.order)

    def to_params(self):
        p = _lib.Params()
        _lib.load().d4_default_params(C.byref(p))
        p.position_precision = self.precision
        p.dipole_precision = self.dipole_precision
        p.cutoff_multiplier = self.cutoff_multiplier
        p.heaviside_cutoff = int(bool(self.heaviside_cutoff))
        p.initial_stepsize = (self.initial_step_size if self.initial_step_size is not None
                              else self.step_size)
        p.max_stepsize = self.max_stepsize_limit if self.max_step_size_limited else -1.0
        p.weight_function = self.weight_function.encode()[:1]
        p.time_limit = self.time_limit if self.time_limited else -1.0
        p.step_count_limit = self.step_count_limit if self.step_count_limited else -1
        p.strain_increase_limit = (self.total_accumulated_strain_increase_limit
                                   if self.strain_increase_limted else -1.0)
        p.calculate_strain = int(bool(self.calculate_strain_during_simulation))
        p.calculate_order_parameter = int(bool(self.calculate_order_parameter))
        p.avalanche_limit = self.trigger_limit_for_avalanche_count if self.count_avalanches else -1
        p.avalanche_speed_threshold = self.avalanche_speed_threshold
        p.save_sub_configs = int(bool(self.save_sub_configs))
        p.sub_config_delay = self.sub_config_delay
        p.sub_config_delay_during_avalanche = self.sub_config_delay_during_avalanche
        p.sub_config_times = self.sub_config_times
        p.sub_config_times_type = self.sub_config_times_type.encode()[:1]
        p.protocol = self.external_stress.to_c()
        p.precision = self.precision_mode
        p.solver = self.solver
        p.field = self.field
        p.table_size = self.table_size
        return p


class Engine:
    """A device context (d4_create) over one configuration."""

    def __init__(self, sd, device=0):
        self.lib = _lib.load()
        self.sd = sd
        p = sd.to_params()
        p.device = device
        self.n = sd.dislocation_count
        ctx = C.c_void_p()
        _lib.check(self.lib, None, self.lib.d4_create(C.byref(ctx), self.n, C.byref(p)),
                   "d4_create")
        self.ctx = ctx
        self._call("d4_set_positions", _lib.ptr(sd.x), _lib.ptr(sd.y))
        self._call("d4_set_time", C.c_double(sd.simulation_time), C.c_double(sd.step_size))

    def _call(self, name, *args):
        return _lib.check(self.lib, self.ctx, getattr(self.lib, name)(self.ctx, *args), name)

    def close(self):
        if getattr(self, "ctx", None):
            self.lib.d4_destroy(self.ctx)
            self.ctx = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # building blocks (Simulation's private sweeps)
    def speeds(self, x, y, t):
        v = np.empty(self.n)
        tol = np.empty(self.n)
        x = np.ascontiguousarray(x, dtype=np.float64)
        y = np.ascontiguousarray(y, dtype=np.float64)
        self._call("d4_speeds", _lib.ptr(x), _lib.ptr(y), C.c_double(t), _lib.ptr(v),
                   _lib.ptr(tol))
        return v, tol

    def jacobian(self, x, y, h, t_a, t_b, want_matrix=True):
        n = self.n
        va, vb, d, tol = (np.empty(n) for _ in range(4))
        a = np.empty((n, n), order="F") if want_matrix else None
        x = np.ascontiguousarray(x, dtype=np.float64)
        y = np.ascontiguousarray(y, dtype=np.float64)
        self._call("d4_jacobian", _lib.ptr(x), _lib.ptr(y), C.c_double(h), C.c_double(t_a),
                   C.c_double(t_b), _lib.ptr(va), _lib.ptr(vb),
                   a.ctypes.data_as(C.POINTER(C.c_double)) if a is not None else None,
                   _lib.ptr(d), _lib.ptr(tol))
        return va, vb, a, d, tol

    def jacobian_from_prev(self, factor, want_matrix=True):
        n = self.n
        d = np.empty(n)
        a = np.empty((n, n), order="F") if want_matrix else None
        self._call("d4_jacobian_from_prev", C.c_double(factor),
                   a.ctypes.data_as(C.POINTER(C.c_double)) if a is not None else None,
                   _lib.ptr(d))
        return a, d

    def set_matrix(self, a):
        a = np.asfortranarray(a, dtype=np.float64)
        self._call("d4_set_matrix", a.ctypes.data_as(C.POINTER(C.c_double)))

    def factor(self):
        return self._call("d4_factor")

    def solve(self, g):
        g = np.ascontiguousarray(g, dtype=np.float64)
        dx = np.empty(self.n)
        st = self._call("d4_solve", _lib.ptr(g), _lib.ptr(dx))
        return dx, st

    def reset_tolerance(self):
        self._call("d4_reset_tolerance")

    def tolerance(self):
        """The per-dislocation tolerances (squared distances)."""
        t = np.empty(self.n)
        self._call("d4_get_tolerance", _lib.ptr(t))
        return t

    def restore(self, x, y, sim_time, step_size, tol):
        """Restarts the stepping loop from a saved state: positions, time,
        step size and tolerances (the state carried between accepted steps)."""
        x, y, tol = (np.ascontiguousarray(v, dtype=np.float64) for v in (x, y, tol))
        self._call("d4_set_positions", _lib.ptr(x), _lib.ptr(y))
        self._call("d4_set_time", C.c_double(sim_time), C.c_double(step_size))
        self._call("d4_set_tolerance", _lib.ptr(tol))

    def attempt(self, t0, h):
        r = _lib.AttemptResult()
        self._call("d4_attempt", C.c_double(t0), C.c_double(h), C.byref(r))
        xb, xh, x2 = (np.empty(self.n) for _ in range(3))
        self._call("d4_get_attempt", _lib.ptr(xb), _lib.ptr(xh), _lib.ptr(x2))
        return r, xb, xh, x2

    def advance(self, accepted_steps):
        """Continues the stepping loop for exactly `accepted_steps` accepted steps."""
        r = _lib.RunResult()
        self._call("d4_advance", C.c_longlong(accepted_steps), C.byref(r))
        return r

    def set_overlap(self, enable=True):
        """Stage I on a second stream, concurrent with stages II-III (default),
        or all stages in sequence (d4_set_overlap); identical results."""
        self._call("d4_set_overlap", int(bool(enable)))

    # accepted-step recording and the differentiation of a replayed step sequence
    def record_steps(self, enable=True):
        self._call("d4_record_steps", int(bool(enable)))

    def recorded_steps(self):
        """(t0s, hs) of the accepted steps recorded since record_steps(True)."""
        m = self.lib.d4_recorded_count(self.ctx)
        t0s, hs = np.empty(max(m, 0)), np.empty(max(m, 0))
        self._call("d4_recorded_steps", C.c_longlong(m), _lib.ptr(t0s), _lib.ptr(hs))
        return t0s, hs

    @staticmethod
    def _steps(t0s, hs):
        t0s = np.ascontiguousarray(t0s, dtype=np.float64)
        hs = np.ascontiguousarray(hs, dtype=np.float64)
        assert t0s.shape == hs.shape
        return t0s, hs

    def _proto(self, tau0):
        p = self.sd.external_stress.to_c()
        if tau0 is not None:
            p.tau0 = float(tau0)
        return p

    def replay(self, x0, t0s, hs, tau0=None):
        """Strain and final positions of the fixed-step replay (d4_replay)."""
        t0s, hs = self._steps(t0s, hs)
        x0 = np.ascontiguousarray(x0, dtype=np.float64)
        x_end, strain = np.empty(self.n), C.c_double()
        p = self._proto(tau0)
        self._call("d4_replay", C.c_longlong(len(t0s)), _lib.ptr(t0s), _lib.ptr(hs), C.byref(p),
                   _lib.ptr(x0), _lib.ptr(x_end), C.byref(strain))
        return strain.value, x_end

    def tangent(self, x0, t0s, hs, dx0, dtau0=0.0, tau0=None):
        """(strain, directional derivative along (dx0, dtau0)) (d4_tangent)."""
        t0s, hs = self._steps(t0s, hs)
        x0 = np.ascontiguousarray(x0, dtype=np.float64)
        dx0 = np.ascontiguousarray(dx0, dtype=np.float64)
        strain, ds = C.c_double(), C.c_double()
        p = self._proto(tau0)
        self._call("d4_tangent", C.c_longlong(len(t0s)), _lib.ptr(t0s), _lib.ptr(hs),
                   C.byref(p), _lib.ptr(x0), _lib.ptr(dx0), C.c_double(dtau0), C.byref(strain),
                   C.byref(ds))
        return strain.value, ds.value

    def adjoint(self, x0, t0s, hs, checkpoint_every=20, tau0=None):
        """(strain, d strain / d x0, d strain / d tau0) (d4_adjoint)."""
        t0s, hs = self._steps(t0s, hs)
        x0 = np.ascontiguousarray(x0, dtype=np.float64)
        g, strain, gt = np.empty(self.n), C.c_double(), C.c_double()
        p = self._proto(tau0)
        self._call("d4_adjoint", C.c_longlong(len(t0s)), _lib.ptr(t0s), _lib.ptr(hs),
                   C.byref(p), int(checkpoint_every), _lib.ptr(x0), C.byref(strain), _lib.ptr(g),
                   C.byref(gt))
        return strain.value, g, gt.value

    def profile(self, enable=True):
        self._call("d4_profile", int(bool(enable)))

    def profile_read(self):
        ms = np.zeros(len(_lib.CATEGORIES))
        calls = np.zeros(len(_lib.CATEGORIES), dtype=np.int64)
        self._call("d4_profile_read", _lib.ptr(ms),
                   calls.ctypes.data_as(C.POINTER(C.c_longlong)))
        return {k: (float(ms[i]), int(calls[i])) for i, k in enumerate(_lib.CATEGORIES)}

    def solver_stats(self):
        """Counters of the cutoff sparse solver (d4_solver_stats)."""
        v = [C.c_longlong() for _ in range(4)]
        self._call("d4_solver_stats", *[C.byref(t) for t in v])
        return dict(zip(("solves", "iterations", "fallbacks", "nnz"), [t.value for t in v]))

    def lu_stats(self):
        """Counters of the dense cooperative LU (d4_lu_stats): factorisations,
        passes over their 32-column blocks, row swaps."""
        v = [C.c_longlong() for _ in range(3)]
        self._call("d4_lu_stats", *[C.byref(t) for t in v])
        return dict(zip(("factorizations", "passes", "swaps"), [t.value for t in v]))

    def mixed_stats(self):
        """Mixed form's factorisations (d4_mixed_stats): block LUs run, block-LU
        attempts that failed, attempts run with the pivoted FP32 LU, attempts on
        the FP64 path, worst refined residual of the FP32 attempts that stood."""
        b, f, p, a, w = (C.c_longlong(), C.c_longlong(), C.c_longlong(), C.c_longlong(),
                         C.c_double())
        self._call("d4_mixed_stats", C.byref(b), C.byref(f), C.byref(p), C.byref(a), C.byref(w))
        return {"block_factorizations": b.value, "fallbacks": f.value,
                "pivoted_fp32_attempts": p.value, "fp64_attempts": a.value,
                "worst_refined_residual": w.value}

    def set_block_lu(self, enable=True):
        """Mixed form: block LU with per-attempt fallback (default), or every
        attempt on the FP64 form's factorisations and solves (d4_set_block_lu)."""
        self._call("d4_set_block_lu", int(bool(enable)))

    def positions(self):
        x = np.empty(self.n)
        y = np.empty(self.n)
        self._call("d4_get_positions", _lib.ptr(x), _lib.ptr(y))
        return x, y

    def run(self, log_path=None, sub_config_prefix=None, end_config_path=None,
            max_attempts=0):
        io = _lib.RunIO()
        io.log_path = log_path.encode() if log_path else None
        io.sub_config_prefix = sub_config_prefix.encode() if sub_config_prefix else None
        io.end_config_path = end_config_path.encode() if end_config_path else None
        order = np.ascontiguousarray(self.sd.order, dtype=np.uint32)
        io.order = order.ctypes.data_as(C.POINTER(C.c_uint))
        io.max_attempts = max_attempts
        r = _lib.RunResult()
        self._call("d4_run", C.byref(io), C.byref(r))
        return r


class Simulation:
    """Simulation (include/simulation.h:122-130): ``Simulation(sd)`` or
    ``Simulation.create(sd)``, then ``run()``."""

    def __init__(self, sd, device=0):
        self.sd = sd
        self.engine = Engine(sd, device)
        self.last_result = None

    @staticmethod
    def create(sd):
        return Simulation(sd)

    def run(self, max_attempts=0):
        sd = self.sd
        r = self.engine.run(log_path=sd.logfile_path or None,
                            sub_config_prefix=sd.sub_config_path if sd.save_sub_configs else None,
                            end_config_path=sd.final_dislocation_configuration_path or None,
                            max_attempts=max_attempts)
        sd.x, sd.y = self.engine.positions()
        sd.simulation_time = r.sim_time
        sd.step_size = r.step_size
        sd.successful_steps += r.successful_steps
        sd.failed_steps += r.failed_steps
        sd.total_accumulated_strain_increase += r.strain
        self.last_result = r
        return r

    def step(self):
        """One attempted step (accepted or not), through the same loop."""
        return self.run(max_attempts=1)

    def get_time(self):
        return self.sd.simulation_time


class Field:
    """Field::xy / Field::xy_diff_x (src/Fields/Field.cpp:333-346) evaluated on
    the device in FP64; with tabulated=True, the tabulated field
    (PeriodicShearStressELTE's role, table_size intervals per axis)."""

    def __init__(self, device=0, tabulated=False, table_size=1024):
        self.lib = _lib.load()
        p = _lib.Params()
        self.lib.d4_default_params(C.byref(p))
        p.device = device
        if tabulated:
            p.field = _lib.D4_FIELD_TABULATED
            p.table_size = table_size
        ctx = C.c_void_p()
        _lib.check(self.lib, None, self.lib.d4_create(C.byref(ctx), 2, C.byref(p)), "d4_create")
        self.ctx = ctx

    def eval(self, dx, dy):
        dx = np.ascontiguousarray(dx, dtype=np.float64).ravel()
        dy = np.ascontiguousarray(dy, dtype=np.float64).ravel()
        xy, xyd = np.empty_like(dx), np.empty_like(dx)
        _lib.check(self.lib, self.ctx,
                   self.lib.d4_field_eval(self.ctx, len(dx), _lib.ptr(dx), _lib.ptr(dy),
                                          _lib.ptr(xy), _lib.ptr(xyd)), "d4_field_eval")
        return xy, xyd

    def xy(self, dx, dy):
        return self.eval(np.array([dx]), np.array([dy]))[0][0]

    def xy_diff_x(self, dx, dy):
        return self.eval(np.array([dx]), np.array([dy]))[1][0]

    def __del__(self):
        try:
            if self.ctx:
                self.lib.d4_destroy(self.ctx)
        except Exception:
            pass
