"""ctypes binding of the C ABI in include/d4core.h (libd4core.so).

The library is the product: there is no CPU fallback.  ``load()`` raises if the
shared library is missing or does not export every symbol the header declares.
"""
import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "lib", "libd4core.so")

D4_OK, D4_WARN_SINGULAR = 0, 1
D4_ERR_ARG, D4_ERR_CUDA, D4_ERR_NOMEM, D4_ERR_STATE, D4_ERR_IO = -1, -2, -3, -4, -5
D4_ERR = {-1: "invalid argument", -2: "CUDA error", -3: "out of memory", -4: "bad state",
          -5: "I/O error"}
D4_PREC_FP64, D4_PREC_MIXED = 0, 1
D4_SOLVER_DENSE, D4_SOLVER_GMRES, D4_SOLVER_AUTO = 0, 1, 2
D4_FIELD_ANALYTIC, D4_FIELD_TABULATED = 0, 1
D4_STRESS_NONE, D4_STRESS_FIXED_RATE, D4_STRESS_CYCLIC, D4_STRESS_INC_CYCLIC = 0, 1, 2, 3
CATEGORIES = ["speeds", "jacobian", "factor", "solve", "rescale"]


class Protocol(C.Structure):
    _fields_ = [("kind", C.c_int), ("tau0", C.c_double), ("rate", C.c_double),
                ("period", C.c_double), ("amplitude_rate", C.c_double)]


class Params(C.Structure):
    _fields_ = [
        ("position_precision", C.c_double), ("dipole_precision", C.c_double),
        ("cutoff_multiplier", C.c_double), ("heaviside_cutoff", C.c_int),
        ("initial_stepsize", C.c_double), ("max_stepsize", C.c_double),
        ("weight_function", C.c_char), ("time_limit", C.c_double),
        ("step_count_limit", C.c_longlong), ("strain_increase_limit", C.c_double),
        ("calculate_strain", C.c_int), ("calculate_order_parameter", C.c_int),
        ("avalanche_limit", C.c_longlong), ("avalanche_speed_threshold", C.c_double),
        ("save_sub_configs", C.c_int), ("sub_config_delay", C.c_uint),
        ("sub_config_delay_during_avalanche", C.c_uint), ("sub_config_times", C.c_double),
        ("sub_config_times_type", C.c_char), ("protocol", Protocol), ("precision", C.c_int),
        ("device", C.c_int), ("solver", C.c_int),
        ("field", C.c_int), ("table_size", C.c_int)]


class AttemptResult(C.Structure):
    _fields_ = [("ratio", C.c_double), ("max_id", C.c_int), ("accepted", C.c_int),
                ("singular", C.c_int), ("pivoted", C.c_int), ("refine_residual", C.c_double)]


class RunResult(C.Structure):
    _fields_ = [("sim_time", C.c_double), ("step_size", C.c_double), ("strain", C.c_double),
                ("energy", C.c_double), ("successful_steps", C.c_longlong),
                ("failed_steps", C.c_longlong), ("attempts", C.c_longlong),
                ("pivoted_factorizations", C.c_longlong),
                ("singular_factorizations", C.c_longlong), ("device_seconds", C.c_double)]


class RunIO(C.Structure):
    _fields_ = [("log_path", C.c_char_p), ("sub_config_prefix", C.c_char_p),
                ("end_config_path", C.c_char_p), ("order", C.POINTER(C.c_uint)),
                ("max_attempts", C.c_longlong)]


_dp = C.POINTER(C.c_double)
_vp = C.c_void_p
# name -> (restype, argtypes); every function declared in include/d4core.h
SIGNATURES = {
    "d4_default_params": (None, [C.POINTER(Params)]),
    "d4_create": (C.c_int, [C.POINTER(_vp), C.c_int, C.POINTER(Params)]),
    "d4_destroy": (C.c_int, [_vp]),
    "d4_last_error": (C.c_char_p, [_vp]),
    "d4_set_positions": (C.c_int, [_vp, _dp, _dp]),
    "d4_get_positions": (C.c_int, [_vp, _dp, _dp]),
    "d4_set_time": (C.c_int, [_vp, C.c_double, C.c_double]),
    "d4_speeds": (C.c_int, [_vp, _dp, _dp, C.c_double, _dp, _dp]),
    "d4_jacobian": (C.c_int, [_vp, _dp, _dp, C.c_double, C.c_double, C.c_double, _dp, _dp,
                              _dp, _dp, _dp]),
    "d4_jacobian_from_prev": (C.c_int, [_vp, C.c_double, _dp, _dp]),
    "d4_set_matrix": (C.c_int, [_vp, _dp]),
    "d4_factor": (C.c_int, [_vp]),
    "d4_solve": (C.c_int, [_vp, _dp, _dp]),
    "d4_reset_tolerance": (C.c_int, [_vp]),
    "d4_get_tolerance": (C.c_int, [_vp, _dp]),
    "d4_set_tolerance": (C.c_int, [_vp, _dp]),
    "d4_attempt": (C.c_int, [_vp, C.c_double, C.c_double, C.POINTER(AttemptResult)]),
    "d4_get_attempt": (C.c_int, [_vp, _dp, _dp, _dp]),
    "d4_run": (C.c_int, [_vp, C.POINTER(RunIO), C.POINTER(RunResult)]),
    "d4_field_eval": (C.c_int, [_vp, C.c_int, _dp, _dp, _dp, _dp]),
    "d4_advance": (C.c_int, [_vp, C.c_longlong, C.POINTER(RunResult)]),
    "d4_profile": (C.c_int, [_vp, C.c_int]),
    "d4_profile_read": (C.c_int, [_vp, _dp, C.POINTER(C.c_longlong)]),
    "d4_kernel_launches": (C.c_longlong, []),
    "d4_device_allocations": (C.c_longlong, []),
    "d4_check_positions": (C.c_int, [C.c_int, _dp, _dp]),
    "d4_wait_selftest": (C.c_int, [_vp, C.c_int]),
    "d4_solver_stats": (C.c_int, [_vp] + [C.POINTER(C.c_longlong)] * 4),
    "d4_lu_stats": (C.c_int, [_vp] + [C.POINTER(C.c_longlong)] * 3),
    "d4_mixed_stats": (C.c_int, [_vp] + [C.POINTER(C.c_longlong)] * 4 + [_dp]),
    "d4_set_block_lu": (C.c_int, [_vp, C.c_int]),
    "d4_pair_tile_threads": (C.c_int, [_vp, C.POINTER(C.c_int)]),
    "d4_ensemble_pair_tile_threads": (C.c_int, [_vp, C.POINTER(C.c_int)]),
    "d4_record_steps": (C.c_int, [_vp, C.c_int]),
    "d4_set_overlap": (C.c_int, [_vp, C.c_int]),
    "d4_xpattern_df": (C.c_int, [C.c_int, _dp, _dp, C.POINTER(C.c_int), C.c_int, _dp]),
    "d4_recorded_count": (C.c_longlong, [_vp]),
    "d4_recorded_steps": (C.c_int, [_vp, C.c_longlong, _dp, _dp]),
    "d4_replay": (C.c_int, [_vp, C.c_longlong, _dp, _dp, C.POINTER(Protocol), _dp, _dp, _dp]),
    "d4_tangent": (C.c_int, [_vp, C.c_longlong, _dp, _dp, C.POINTER(Protocol), _dp, _dp,
                             C.c_double, _dp, _dp]),
    "d4_adjoint": (C.c_int, [_vp, C.c_longlong, _dp, _dp, C.POINTER(Protocol), C.c_int, _dp,
                             _dp, _dp, _dp]),
    "d4_ensemble_create": (C.c_int, [C.POINTER(_vp), C.c_int, C.POINTER(C.c_int),
                                     C.POINTER(Params)]),
    "d4_ensemble_destroy": (C.c_int, [_vp]),
    "d4_ensemble_last_error": (C.c_char_p, [_vp]),
    "d4_ensemble_set_positions": (C.c_int, [_vp, C.c_int, _dp, _dp]),
    "d4_ensemble_get_positions": (C.c_int, [_vp, C.c_int, _dp, _dp]),
    "d4_ensemble_run": (C.c_int, [_vp, C.c_longlong, C.POINTER(RunResult)]),
    "d4_speeds_noalloc": (C.c_int, [C.c_int, C.c_void_p, C.c_void_p, C.c_double, C.c_void_p,
                                    C.c_void_p, C.c_double, C.c_void_p]),
}

_LIB = None


def load(path=None):
    """Loads libd4core.so and binds every C-ABI symbol (raises if any is missing)."""
    global _LIB
    if _LIB is not None and path is None:
        return _LIB
    p = path or LIB_PATH
    if not os.path.exists(p):
        raise RuntimeError("libd4core.so not built (%s); run python 2d4_b200/build.py" % p)
    lib = C.CDLL(p)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)  # AttributeError if not exported
        fn.restype = res
        fn.argtypes = args
    if path is None:
        _LIB = lib
    return lib


def ptr(a):
    """Pointer to the data of a C-contiguous float64 numpy array (or None)."""
    if a is None:
        return None
    return a.ctypes.data_as(_dp)


class D4Error(RuntimeError):
    pass


def check(lib, ctx, status, what):
    if status < 0:
        msg = lib.d4_last_error(ctx) if ctx else b""
        raise D4Error("%s failed: %s (%s)" % (what, D4_ERR.get(status, status),
                                               (msg or b"").decode()))
    return status
