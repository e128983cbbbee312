"""ctypes binding of libpybrown_b200.so (the C ABI in include/pybrown_b200.h).

The library is the product's only compute path: importing this module raises
if it is missing, and there is no CPU fallback.
"""
import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "lib", "libpybrown_b200.so")

# status codes (include/pybrown_b200.h)
PBG_OK = 0
STATUS_NAMES = {
    -1: "PBG_ERR_CUDA", -2: "PBG_ERR_ARG", -3: "PBG_ERR_NOT_SPD", -4: "PBG_ERR_ATTEMPTS",
    -5: "PBG_ERR_NOISE", -6: "PBG_ERR_NOMEM", -7: "PBG_ERR_BARRIER", -8: "PBG_ERR_NAN",
    -9: "PBG_ERR_STATE",
}
PBG_ERR_NOT_SPD = -3
PBG_ERR_ATTEMPTS = -4
PBG_ERR_NOISE = -5
PBG_ERR_BARRIER = -7

HI = {"nohi": 0, "rpy": 1, "rpy_smith": 2, "rpy_lub": 3, "rpy_smith_lub": 4}
PREC = {"fp64": 0, "mixed": 1}
SCHEME = {"ermak": 0, "midpoint": 1}
MAT = {"D": 0, "B": 1, "Mff": 2, "Rff": 3, "R": 4}


class PbgParams(ctypes.Structure):
    _fields_ = [
        ("n_beads", ctypes.c_int),
        ("hydrodynamics", ctypes.c_int),
        ("precision", ctypes.c_int),
        ("propagation_scheme", ctypes.c_int),
        ("box_length", ctypes.c_double),
        ("kBT", ctypes.c_double),
        ("viscosity", ctypes.c_double),
        ("ewald_alpha", ctypes.c_double),
        ("ewald_real", ctypes.c_int),
        ("ewald_imag", ctypes.c_int),
        ("lubrication_cutoff", ctypes.c_double),
        ("cichocki_correction", ctypes.c_int),
        ("check_overlaps", ctypes.c_int),
        ("overlap_treshold", ctypes.c_double),
        ("max_move_attempts", ctypes.c_int),
        ("m_midpoint", ctypes.c_double),
    ]


class PbgStepReport(ctypes.Structure):
    _fields_ = [
        ("draws_consumed", ctypes.c_longlong),
        ("steps_done", ctypes.c_longlong),
        ("last_attempts", ctypes.c_int),
        ("max_attempts", ctypes.c_int),
        ("device_errors", ctypes.c_uint),
        ("status", ctypes.c_int),
    ]


LJ = {(False, False): 0, (True, False): 6, (False, True): 12, (True, True): 612}
ANGLE_DIRECT, ANGLE_P23_DIFF, ANGLE_P12_DIFF = 0, 1, 2


class PbgInteractions(ctypes.Structure):
    _fields_ = [
        ("lennard_jones", ctypes.c_int),
        ("lennard_jones_alpha", ctypes.c_double),
        ("hard_core_radius", ctypes.c_void_p),
        ("epsilon_lj", ctypes.c_void_p),
        ("n_bonds", ctypes.c_int),
        ("bonds", ctypes.c_void_p),
        ("bond_params", ctypes.c_void_p),
        ("n_angles", ctypes.c_int),
        ("angles", ctypes.c_void_p),
        ("angle_params", ctypes.c_void_p),
        ("unit_scale", ctypes.c_double),
    ]


class PbgError(RuntimeError):
    def __init__(self, fn, code, message):
        self.code = code
        super().__init__(f"{fn} -> {STATUS_NAMES.get(code, code)}: {message}")


_dp = ctypes.POINTER(ctypes.c_double)
_ip = ctypes.POINTER(ctypes.c_int)
_vp = ctypes.c_void_p
_i = ctypes.c_int
_d = ctypes.c_double
_ll = ctypes.c_longlong

_SIGNATURES = {
    # tier 1 (reference ABI)
    "RPY_M_matrix": (None, [_dp, _dp, _i, _dp]),
    "RPY_Smith_M_matrix": (None, [_dp, _dp, _d, _d, _i, _i, _i, _dp]),
    "JO_2B_R_matrix": (None, [_d, _d, _d, _d, _d, _dp]),
    "JO_R_lubrication_correction_matrix": (None, [_dp, _dp, _i, _d, _i, _dp]),
    "pointer_pbc_matrix": (None, [_dp, _i, _d, _dp]),
    "pointer_immobile_pbc_matrix": (None, [_dp, _dp, _i, _i, _d, _dp]),
    "check_overlaps": (_i, [_dp, _dp, _i, _d, _d, _ip]),
    # tier 2
    "pbg_last_error": (ctypes.c_char_p, []),
    "pbg_version": (_i, []),
    "pbg_launch_count": (_ll, []),
    "pbg_host_launch_count": (_ll, []),
    "pbg_dev_pointer_matrix": (_i, [_vp, _i, _d, _vp, _vp]),
    "pbg_dev_rpy_matrix": (_i, [_vp, _vp, _i, _d, _d, _vp, _i, _vp]),
    "pbg_dev_smith_matrix": (_i, [_vp, _vp, _i, _d, _d, _i, _i, _d, _i, _vp, _i, _vp]),
    "pbg_dev_smith_matrix_noalloc": (_i, [_vp, _vp, _i, _d, _d, _i, _i, _d, _i, _vp, _i, _vp]),
    "pbg_dev_lubrication_add": (_i, [_vp, _vp, _i, _d, _d, _i, _d, _vp, _i, _vp]),
    "pbg_dev_check_overlaps": (_i, [_vp, _vp, _i, _d, _d, _vp, _vp, _vp]),
    "pbg_dev_cholesky": (_i, [_vp, _i, _i, _i, _vp, _vp]),
    "pbg_dev_spd_inverse": (_i, [_vp, _i, _i, _vp, _vp]),
    "pbg_create": (_i, [ctypes.POINTER(PbgParams), ctypes.POINTER(_vp)]),
    "pbg_destroy": (_i, [_vp]),
    "pbg_set_state": (_i, [_vp, _vp, _vp, _vp, _vp]),
    "pbg_set_force": (_i, [_vp, _vp, _vp]),
    "pbg_set_divergence": (_i, [_vp, _i]),
    "pbg_set_immobile": (_i, [_vp, _i, _vp, _vp, _vp, _vp, _vp]),
    "pbg_set_positions": (_i, [_vp, _vp, _vp]),
    "pbg_set_interactions": (_i, [_vp, ctypes.POINTER(PbgInteractions)]),
    "pbg_get_energy": (_i, [_vp, _dp, _vp]),
    "pbg_get_force": (_i, [_vp, _vp, _vp]),
    "pbg_get_positions": (_i, [_vp, _vp, _vp]),
    "pbg_get_matrix": (_i, [_vp, _i, _vp, _vp]),
    "pbg_set_matrix": (_i, [_vp, _i, _vp, _vp]),
    "pbg_step_begin": (_i, [_vp, _d, _i, _i, _i, _vp]),
    "pbg_step_attempt": (_i, [_vp, _vp, _ip, _vp]),
    "pbg_step_end": (_i, [_vp, _vp]),
    "pbg_step_finish": (_i, [_vp, _vp, _vp]),
    "pbg_run": (_i, [_vp, _ll, _i, _d, _i, _i, _i, _vp, _ll, _vp]),
    "pbg_run_report": (_i, [_vp, ctypes.POINTER(PbgStepReport), _vp]),
    "pbg_batch_create": (_i, [ctypes.POINTER(PbgParams), ctypes.POINTER(_vp)]),
    "pbg_batch_destroy": (_i, [_vp]),
    "pbg_batch_footprint": (_ll, [_i, _i, _i, _i]),
    "pbg_batch_add": (_i, [_vp, ctypes.POINTER(PbgParams), _vp, _vp, _ip]),
    "pbg_batch_remove": (_i, [_vp, _i]),
    "pbg_batch_slots": (_i, [_vp]),
    "pbg_batch_set_positions": (_i, [_vp, _i, _vp]),
    "pbg_batch_get_positions": (_i, [_vp, _i, _vp]),
    "pbg_batch_get_positions_async": (_i, [_vp, _i, _vp, _vp]),
    "pbg_batch_set_force": (_i, [_vp, _i, _vp]),
    "pbg_batch_set_noise": (_i, [_vp, _i, _vp]),
    "pbg_batch_set_seed": (_i, [_vp, _i, ctypes.c_ulonglong, ctypes.c_ulonglong]),
    "pbg_batch_get_draws": (_i, [_vp, _i, ctypes.POINTER(ctypes.c_ulonglong)]),
    "pbg_batch_fill_noise": (_i, [_vp, _vp, _vp]),
    "pbg_batch_step_begin": (_i, [_vp, _d, _i, _i, _vp]),
    "pbg_batch_step_attempt": (_i, [_vp, _vp, _vp, _vp]),
    "pbg_batch_step_end": (_i, [_vp, _vp, _vp]),
    "pbg_batch_step": (_i, [_vp, _d, _i, _i, _vp, _vp, _vp]),
    "pbg_batch_get_matrix": (_i, [_vp, _i, _i, _vp]),
    "pbg_batch_check_factor": (_i, [_vp, _i, _ip, _vp]),
    "pbg_batch_set_schedule": (_i, [_vp, _i, _i]),
    "pbg_batch_autotune": (_i, [_vp, _i, _ip, ctypes.POINTER(ctypes.c_float), _vp]),
    "pbg_batch_graph_state": (_i, [_vp]),
    "pbg_selftest_wait_expiry": (_i, [_ll, _ip, ctypes.POINTER(ctypes.c_uint)]),
}


def _load():
    if not os.path.exists(LIB_PATH):
        raise ImportError(
            f"{LIB_PATH} is missing: build it with `python -m pybrown_b200.build` "
            "(pybrown_b200 has no CPU fallback)")
    lib = ctypes.CDLL(LIB_PATH)
    for name, (res, args) in _SIGNATURES.items():
        fn = getattr(lib, name, None)
        if fn is None:
            continue
        fn.restype = res
        fn.argtypes = args
    return lib


lib = _load()


def last_error():
    msg = lib.pbg_last_error()
    return msg.decode() if msg else ""


def check(fn_name, code):
    """Raise PbgError for a non-zero status returned by `fn_name`."""
    if code != PBG_OK:
        raise PbgError(fn_name, code, last_error())
    return code


def call(fn_name, *args):
    return check(fn_name, getattr(lib, fn_name)(*args))


def dptr(a):
    """ctypes double* of a C-contiguous float64 numpy array."""
    return a.ctypes.data_as(_dp)


def iptr(a):
    return a.ctypes.data_as(_ip)
