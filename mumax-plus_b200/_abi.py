"""ctypes mirror of include/mpx.h (structures, enums and function signatures).

Importing this module needs no GPU: it only describes the C ABI.  `load()`
opens libmpx.so and declares the signatures of every exported entry point.
"""
import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
# MPX_LIBRARY selects another build of the same ABI (the checked build,
# libmpx_checked.so); the default is the in-tree libmpx.so.
LIB_PATH = os.environ.get("MPX_LIBRARY") or os.path.join(HERE, "libmpx.so")

# status codes
MPX_OK = 0
MPX_ERR_INVALID = 1
MPX_ERR_RANGE = 2
MPX_ERR_RUNTIME = 3
MPX_ERR_NOMEM = 4
MPX_ERR_CUDA = 5
MPX_ERR_UNSUPPORTED = 6
MPX_ERR_TIMEOUT = 7
MPX_ERR_NODEVICE = 8

# quantities
MPX_STRAY_FFT = 0
MPX_STRAY_BRUTE = 1
MPX_DFT_FP32 = 0
MPX_DFT_TF32X3 = 1

Q_MAGNETIZATION = 0
Q_EFFECTIVE_FIELD = 1
Q_EXCHANGE_FIELD = 2
Q_DMI_FIELD = 3
Q_ANISOTROPY_FIELD = 4
Q_EXTERNAL_FIELD = 5
Q_DEMAG_FIELD = 6
Q_TORQUE = 7
Q_LLG_TORQUE = 8
Q_DAMPING_TORQUE = 9
Q_EXCHANGE_ENERGY_DENSITY = 10
Q_DMI_ENERGY_DENSITY = 11
Q_ANISOTROPY_ENERGY_DENSITY = 12
Q_ZEEMAN_ENERGY_DENSITY = 13
Q_DEMAG_ENERGY_DENSITY = 14
Q_TOTAL_ENERGY_DENSITY = 15
Q_SPIN_TRANSFER_TORQUE = 16
Q_COUNT = 17

# Runge-Kutta methods, with the names of core/butchertableau.hpp
RK_METHODS = {
    "Heun": 0,
    "BogackiShampine": 1,
    "CashKarp": 2,
    "Fehlberg": 3,
    "DormandPrince": 4,
}
RK_NAMES = {v: k for k, v in RK_METHODS.items()}

DMI_ORDER = ("xxy", "xxz", "xyz", "yxy", "yxz", "yyz", "zxy", "zxz", "zyz")


class Scalar(C.Structure):
    _fields_ = [("uniform", C.c_double), ("cells", C.POINTER(C.c_float))]


class Vector(C.Structure):
    _fields_ = [("uniform", C.c_double * 3), ("cells", C.POINTER(C.c_float))]


class MagnetDesc(C.Structure):
    _fields_ = [
        ("size", C.c_int * 3),
        ("origin", C.c_int * 3),
        ("cellsize", C.c_double * 3),
        ("mastergrid_size", C.c_int * 3),
        ("mastergrid_origin", C.c_int * 3),
        ("pbc_repetitions", C.c_int * 3),
        ("geometry", C.POINTER(C.c_ubyte)),
        ("regions", C.POINTER(C.c_uint)),
        ("msat", Scalar),
        ("aex", Scalar),
        ("alpha", Scalar),
        ("ku1", Scalar),
        ("ku2", Scalar),
        ("frozen_spins", Scalar),
        ("anis_u", Vector),
        ("bias_magnetic_field", Vector),
        ("dmi", Scalar * 9),
        ("lut_regions", C.c_int),
        ("inter_exchange", C.c_double),
        ("inter_exchange_lut", C.POINTER(C.c_float)),
        ("scale_exchange", C.c_double),
        ("scale_exchange_lut", C.POINTER(C.c_float)),
        ("enable_demag", C.c_int),
        ("enable_openbc", C.c_int),
        ("kc1", Scalar),
        ("kc2", Scalar),
        ("kc3", Scalar),
        ("anis_c1", Vector),
        ("anis_c2", Vector),
        ("stray_source_off", C.c_int),
        ("stray_destination_off", C.c_int),
        ("pol", Scalar),
        ("xi", Scalar),
        ("lambda_", Scalar),
        ("epsilon_prime", Scalar),
        ("free_layer_thickness", Scalar),
        ("jcur", Vector),
        ("fixed_layer", Vector),
        ("fixed_layer_below", C.c_int),
        ("zhang_li_off", C.c_int),
        ("slonczewski_off", C.c_int),
        ("temperature", Scalar),
        ("thermal_seed", C.c_uint64),
    ]


class SolverParams(C.Structure):
    _fields_ = [
        ("method", C.c_int),
        ("adaptive", C.c_int),
        ("max_error", C.c_double),
        ("headroom", C.c_double),
        ("lower_bound", C.c_double),
        ("upper_bound", C.c_double),
        ("sensible_factor", C.c_double),
        ("sensible_timestep_default", C.c_double),
    ]


class GroupInfo(C.Structure):
    _fields_ = [
        ("time", C.c_double),
        ("timestep", C.c_double),
        ("steps", C.c_int64),
        ("rejected", C.c_int64),
        ("evaluations", C.c_int64),
        ("status", C.c_int),
        ("last_error", C.c_double),
        ("max_torque", C.c_double),
    ]


E = C.c_void_p  # mpx_engine*
I = C.c_int
P_I = C.POINTER(C.c_int)
P_D = C.POINTER(C.c_double)
P_F = C.POINTER(C.c_float)
P_I64 = C.POINTER(C.c_int64)

SIGNATURES = {
    "mpx_version": (C.c_char_p, []),
    "mpx_last_error": (C.c_char_p, []),
    "mpx_device_count": (I, []),
    "mpx_engine_create": (I, [I, C.POINTER(E)]),
    "mpx_engine_destroy": (I, [E]),
    "mpx_engine_set_stream": (I, [E, C.c_void_p]),
    "mpx_engine_synchronize": (I, [E]),
    "mpx_engine_set_dft": (I, [E, I]),
    "mpx_tc_status": (I, [C.POINTER(C.c_uint)]),
    "mpx_tc_timeout_selftest": (I, [C.POINTER(C.c_uint)]),
    "mpx_engine_set_world_bias": (I, [E, P_D]),
    "mpx_engine_memory": (I, [E, P_I64]),
    "mpx_engine_launch_count": (I, [E, P_I64]),
    "mpx_engine_graph_stats": (I, [E, C.POINTER(C.c_int64), C.POINTER(C.c_int64)]),
    "mpx_group_create": (I, [E, P_I]),
    "mpx_group_destroy": (I, [E, I]),
    "mpx_group_info_get": (I, [E, I, C.POINTER(GroupInfo)]),
    "mpx_group_state_bytes": (I, [E, I, C.POINTER(C.c_int64)]),
    "mpx_group_save": (I, [E, I, C.c_void_p, C.c_int64]),
    "mpx_group_load": (I, [E, I, C.c_void_p, C.c_int64]),
    # descriptions are passed by address so that an identical struct layout
    # declared elsewhere (e.g. by a test harness) is accepted as well
    "mpx_magnet_add": (I, [E, I, C.c_void_p, P_I]),
    "mpx_magnet_add_state": (I, [E, I, C.c_void_p, C.c_void_p, I, P_I]),
    "mpx_magnet_update": (I, [E, I, C.c_void_p]),
    "mpx_magnet_remove": (I, [E, I]),
    "mpx_magnet_bytes": (I, [C.c_void_p, P_I64, P_I64]),
    "mpx_magnet_set_m": (I, [E, I, C.c_void_p, I]),
    "mpx_magnet_get_m": (I, [E, I, C.c_void_p, I]),
    "mpx_eval": (I, [E, I, I, C.c_void_p, I]),
    "mpx_average": (I, [E, I, I, P_D]),
    "mpx_max_norm": (I, [E, I, I, P_D]),
    "mpx_energy": (I, [E, I, I, P_D]),
    "mpx_demag_kernel": (I, [E, I, C.c_void_p, P_I]),
    "mpx_stray_field": (I, [E, I, I, P_I, P_I, I, C.c_void_p, I]),
    "mpx_profile_eval": (I, [E, I, I, P_D]),
    "mpx_profile_attempt": (I, [E, I, I, P_D]),
    "mpx_autotune": (I, [E, I, P_I, P_I]),
    "mpx_solver_set_params": (I, [E, I, C.POINTER(SolverParams)]),
    "mpx_solver_get_params": (I, [E, I, C.POINTER(SolverParams)]),
    "mpx_solver_set_time": (I, [E, I, C.c_double]),
    "mpx_solver_get_time": (I, [E, I, P_D]),
    "mpx_solver_set_timestep": (I, [E, I, C.c_double]),
    "mpx_solver_get_timestep": (I, [E, I, P_D]),
    "mpx_solver_sensible_timestep": (I, [E, I, P_D]),
    "mpx_solver_step": (I, [E, I]),
    "mpx_solver_steps": (I, [E, I, I]),
    "mpx_solver_run": (I, [E, I, C.c_double]),
    "mpx_solver_run_sampled": (I, [E, I, C.POINTER(C.c_double), I, C.POINTER(C.c_double)]),
    "mpx_minimize": (I, [E, I, C.c_double, I]),
    "mpx_relax": (I, [E, I, C.c_double, C.c_double]),
    "mpx_group_start": (I, [E, I, C.c_double, C.c_double]),
    "mpx_advance": (I, [E, I]),
    "mpx_poll": (I, [E, P_I, I, P_I, P_I]),
    "mpx_reduce_noalloc": (I, [C.c_void_p, I, I, C.c_void_p, I, C.c_void_p, P_D]),
    "mpx_bounds_check": (I, [C.POINTER(C.c_ulonglong)]),
}


def header_symbols():
    """Function names declared in include/mpx.h (parsed from the header text)."""
    import re

    path = os.path.join(os.path.dirname(HERE), "include", "mpx.h")
    text = open(path).read()
    return sorted(set(re.findall(r"^\s*(?:mpx_status|const char\*|int)\s+(mpx_\w+)\s*\(", text, re.M)))


_lib = None


def load(path=None):
    """Open libmpx.so (once) and declare the signatures."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    lib = C.CDLL(path or LIB_PATH)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    if path is None:
        _lib = lib
    return lib
