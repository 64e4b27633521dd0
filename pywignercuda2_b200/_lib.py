"""ctypes binding of libwigner_b200.so (the sm_100a CUDA library).

The library is built in-tree by ``pywignercuda2_b200.build_lib``.  There is no
fallback: if it is missing or a CUDA device is absent, the classes raise.
"""
import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libwigner_b200.so")

WIG_MAX_FACTORS = 12
WIG4D_NOBS = 11
WIG_RUN_KEEP_NORM = 1
C128, C64 = 0, 1

STATUS = {0: "ok", 1: "invalid argument", 2: "unsupported shape or parameter", 3: "CUDA error",
          4: "device allocation failed", 5: "non-finite value in a reduction",
          6: "component pointers alias", 7: "size above the limit of this call",
          8: "a bounded device wait gave up"}


class WignerError(RuntimeError):
    """A C-ABI call returned a non-zero status."""

    def __init__(self, fn, status, detail=""):
        self.status = status
        msg = "%s failed: %s (%d)" % (fn, STATUS.get(status, "unknown"), status)
        if detail:
            msg += ": " + detail
        super().__init__(msg)


class Factor(ctypes.Structure):
    _fields_ = [("axis_a", ctypes.c_int), ("axis_b", ctypes.c_int),
                ("host_data", ctypes.POINTER(ctypes.c_double))]


class Desc4D(ctypes.Structure):
    _fields_ = [("shape", ctypes.c_int * 4), ("dtype", ctypes.c_int),
                ("d", ctypes.c_double * 4), ("delta", ctypes.c_double * 4),
                ("kin_post_scale", ctypes.c_double), ("pot_post_scale", ctypes.c_double),
                ("n_kin", ctypes.c_int), ("kin", Factor * WIG_MAX_FACTORS),
                ("n_pot", ctypes.c_int), ("pot", Factor * WIG_MAX_FACTORS),
                ("coord", ctypes.POINTER(ctypes.c_double) * 4),
                ("energy_p", ctypes.POINTER(ctypes.c_double)),
                ("energy_x", ctypes.POINTER(ctypes.c_double)),
                ("dv_norm", ctypes.c_double), ("dv_obs", ctypes.c_double),
                ("transform", ctypes.c_int)]


class DescDirac(ctypes.Structure):
    _fields_ = [("shape", ctypes.c_int * 4), ("dtype", ctypes.c_int), ("kvn", ctypes.c_int),
                ("d", ctypes.c_double * 4), ("delta", ctypes.c_double * 4), ("post", ctypes.c_double * 4),
                ("c", ctypes.c_double), ("hbar", ctypes.c_double), ("mass", ctypes.c_double),
                ("dt", ctypes.c_double), ("m_pot", ctypes.c_double),
                ("d_lambda_x", ctypes.c_double), ("d_lambda_y", ctypes.c_double),
                ("coord", ctypes.POINTER(ctypes.c_double) * 4),
                ("acoord", ctypes.POINTER(ctypes.c_double) * 4),
                ("mask_xp", ctypes.POINTER(ctypes.c_double) * 4),
                ("mask_p", ctypes.POINTER(ctypes.c_double) * 4),
                ("n_phase", ctypes.c_int), ("phase", Factor * WIG_MAX_FACTORS),
                ("a_rank", ctypes.c_int), ("a_tabs", ctypes.POINTER(ctypes.c_double)),
                ("obs_xy", ctypes.POINTER(ctypes.c_double)),
                ("dv_norm", ctypes.c_double), ("dv_obs", ctypes.c_double),
                ("a_full", ctypes.POINTER(ctypes.c_double))]


WIGD_NOBS = 19

_lib = None

_P = ctypes.c_void_p
_I = ctypes.c_int
_D = ctypes.c_double
_LL = ctypes.c_longlong
_DP = ctypes.POINTER(ctypes.c_double)
_IP = ctypes.POINTER(ctypes.c_int)

# name -> argtypes (restype int unless listed in _RESTYPE)
SIGNATURES = {
    "wig_status_string": [_I],
    "wig_last_error": [],
    "wig_version": [],
    "wig_faft": [_P, _IP, _I, _I, _D, _D, _D, _P],
    "FAFT64_4D_Z2Z": [_P, _D, _D, _I, _I, _D],
    "IFAFT64_4D_Z2Z": [_P, _D, _D, _I, _I, _D],
    "FAFT128_4D_Z2Z": [_P, _D, _D, _I, _I, _D],
    "FAFT256_4D_Z2Z": [_P, _D, _D, _I, _I, _D],
    "wig_scale": [_P, _LL, _I, _D, _D, _P],
    "wig_divide_by_device_scalar": [_P, _LL, _I, _P, _P],
    "wig_real": [_P, _LL, _I, _P],
    "wig4d_plan_create": [ctypes.POINTER(Desc4D), ctypes.POINTER(_P)],
    "wig4d_plan_destroy": [_P],
    "wig4d_kinetic": [_P, _P, _P, _P],
    "wig4d_potential": [_P, _P, _P],
    "wig4d_apply_factor": [_P, _P, _I, _P],
    "wig4d_reduce": [_P, _P, _P, _P],
    "wig4d_run": [_P, _P, _I, _P, _P],
    "wig4d_run_ex": [_P, _P, _I, _P, _I, _P],
    "wig4d_run_timed": [_P, _P, _I, _P, _P, _DP],
    "wig4d_plan_info": [_P, _IP],
    "wig4d_run_batch": [_P, _P, _I, _I, _P, _P],
    "wig4d_init_ho_ground": [_P, _P, _D, _D, _D, _D, _D, _D, _D, _P],
    "wig4d_init_gaussian": [_P, _P, _D, _D, _D, _D, _D, _D, _D, _D, _P],
    "wig4d_init_cat_xtheta": [_P, _P, _D, _D, _D, _D, _D, _D, _D, _D, _P],
    "wig4d_plan_device_bytes": [_P],
    "wig4d_autotune": [_P, _I, _I, _P, _IP],
    "wig4d_observables_noalloc": [_P, _IP, _I, _P, _P, _P, _P, _P, _P, _D, _D, _P, _P],
    "wigd_plan_create": [ctypes.POINTER(DescDirac), ctypes.POINTER(_P)],
    "wigd_plan_destroy": [_P],
    "wigd_transform": [_P, _P, _I, _I, _P, _P],
    "wigd_mask": [_P, _P, _I, _P],
    "wigd_set_mask": [_P, _I, _P],
    "wigd_real_diag": [_P, _P, _P],
    "wigd_divide": [_P, _P, _P, _P],
    "wigd_reduce": [_P, _P, _P, _I, _P],
    "wigd_norm_ptr": [_P],
    "wigd_kinetic": [_P, _P, _I, _I, _P],
    "wigd_potential": [_P, _P, _P],
    "wigd_init_particle_up": [_P, _P, _D, _D, _D, _D, _D, _D, _P],
    "wigd_init_majorana": [_P, _P, _D, _D, _D, _D, _D, _D, _P],
    "wigd_init_landau": [_P, _P, _D, _D, _D, _P],
    "wigd_run": [_P, _P, _I, _I, _P, _P],
}
_RESTYPE = {"wig_status_string": ctypes.c_char_p, "wig_last_error": ctypes.c_char_p,
            "wig4d_plan_device_bytes": ctypes.c_longlong, "wigd_norm_ptr": ctypes.c_void_p}


def load():
    """Load and type the library once; raise if it is not built."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError("libwigner_b200.so is not built (run pywignercuda2_b200.build_lib.build())")
    lib = ctypes.CDLL(LIB_PATH)
    for name, args in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.argtypes = args
        fn.restype = _RESTYPE.get(name, ctypes.c_int)
    _lib = lib
    return lib


def call(name, *args):
    """Call a status-returning entry point; raise WignerError on failure."""
    lib = load()
    st = getattr(lib, name)(*args)
    if st != 0:
        detail = lib.wig_last_error().decode() if st == 3 else ""
        raise WignerError(name, st, detail)
    return st


def dptr(arr):
    """ctypes double* to a contiguous float64 NumPy array."""
    return arr.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
