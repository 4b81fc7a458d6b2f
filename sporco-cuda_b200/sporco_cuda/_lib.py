"""ctypes binding of libsporco_b200.so (the C ABI in include/sporco_b200.h).

The library is built in place by ``sporco-cuda_b200/build.py``.  There is no
fallback: if the library is missing or cannot be loaded, importing this
module raises ImportError.
"""

from __future__ import annotations

import ctypes as C
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libsporco_b200.so")

if not os.path.exists(LIB_PATH):
    raise ImportError(
        "libsporco_b200.so not found at %s: build it with "
        "`python sporco-cuda_b200/build.py`" % LIB_PATH)

lib = C.CDLL(LIB_PATH)

FP = C.POINTER(C.c_float)
IP = C.POINTER(C.c_int)

SC_OK = 0
STATUS_NAMES = {
    0: "SC_OK", 1: "SC_ERR_INVALID", 2: "SC_ERR_UNSUPPORTED", 3: "SC_ERR_WORKSPACE",
    4: "SC_ERR_CUDA", 5: "SC_ERR_NONFINITE", 6: "SC_ERR_OOM", 7: "SC_ERR_CANCELLED",
}
SC_L1_SCALAR, SC_L1_PER_MAP, SC_L1_FULL = 0, 1, 2


class AlgOpt(C.Structure):
    """Field order of AlgOpt (sporco_cuda/src/algopt.h:7-48)."""

    _fields_ = [
        ("MaxMainIter", C.c_int),
        ("rho", C.c_float),
        ("RhoRsdlRatio", C.c_float),
        ("RhoScaling", C.c_float),
        ("RhoRsdlTarget", C.c_float),
        ("RelaxParam", C.c_float),
        ("AbsStopTol", C.c_float),
        ("RelStopTol", C.c_float),
        ("L1Weight", FP),
        ("L1_WEIGHT_M_SIZE", C.c_int),
        ("L1_WEIGHT_ROW_SIZE", C.c_int),
        ("L1_WEIGHT_COL_SIZE", C.c_int),
        ("Weight", IP),
        ("nWeight", C.c_int),
        ("Verbose", C.c_int),
        ("NonNegCoef", C.c_int),
        ("NoBndryCross", C.c_int),
        ("AuxVarObj", C.c_int),
        ("HighMemSolve", C.c_int),
        ("AutoRho", C.c_int),
        ("AutoRhoScaling", C.c_int),
        ("AutoRhoPeriod", C.c_int),
        ("StdResiduals", C.c_int),
        ("IMG_ROW_SIZE", C.c_int),
        ("IMG_COL_SIZE", C.c_int),
        ("DICT_M_SIZE", C.c_int),
        ("DICT_ROW_SIZE", C.c_int),
        ("DICT_COL_SIZE", C.c_int),
        ("GrdWeight", FP),
        ("WEIGHT_SIZE", C.c_int),
        ("device", C.c_int),
    ]


class ScOptions(C.Structure):
    _fields_ = [
        ("max_iter", C.c_int),
        ("relax", C.c_float),
        ("abs_tol", C.c_float),
        ("rel_tol", C.c_float),
        ("auto_rho", C.c_int),
        ("auto_rho_period", C.c_int),
        ("rho_scaling", C.c_float),
        ("rsdl_ratio", C.c_float),
        ("rsdl_target", C.c_float),
        ("auto_scaling", C.c_int),
        ("std_residuals", C.c_int),
        ("record_itstat", C.c_int),
        ("check_every", C.c_int),
        ("profile", C.c_int),
        ("nonneg", C.c_int),
        ("no_bndry_cross", C.c_int),
        ("warm_start", C.c_int),
    ]


class ScProblem(C.Structure):
    _fields_ = [
        ("B", C.c_int), ("H", C.c_int), ("W", C.c_int), ("M", C.c_int),
        ("Kr", C.c_int), ("Kc", C.c_int),
        ("D", C.c_void_p), ("S", C.c_void_p), ("lmbda", C.c_void_p), ("rho0", C.c_void_p),
        ("grd", C.c_int), ("mu", C.c_float), ("wgrd", C.c_void_p),
        ("l1_kind", C.c_int), ("l1_scalar", C.c_float), ("l1w", C.c_void_p),
        ("mask", C.c_void_p), ("Y", C.c_void_p), ("wgrd_uniform", C.c_int),
        ("U0", C.c_void_p), ("U_out", C.c_void_p),
    ]


class ScProfile(C.Structure):
    _fields_ = [("ms", C.c_double * 4), ("count", C.c_int * 4)]


class ScResult(C.Structure):
    _fields_ = [("iterations", C.c_int), ("rho", C.c_double), ("r", C.c_double),
                ("s", C.c_double)]


def _proto(name, res, args):
    f = getattr(lib, name)
    f.restype = res
    f.argtypes = args
    return f


cuda_wrapper_CBPDN = _proto("cuda_wrapper_CBPDN", None, [FP, FP, C.c_float, C.c_void_p, FP])
cuda_wrapper_CBPDN_GR = _proto("cuda_wrapper_CBPDN_GR", None,
                               [FP, FP, C.c_float, C.c_float, C.c_void_p, FP])
clear_opts = _proto("clear_opts", None, [C.c_void_p])
default_opts = _proto("default_opts", None, [C.c_void_p])
check_cuda_req = _proto("check_cuda_req", C.c_int, [C.c_int])
get_device_count = _proto("get_device_count", C.c_int, [])
get_current_device = _proto("get_current_device", C.c_int, [IP])
set_current_device = _proto("set_current_device", C.c_int, [C.c_int])
get_memory_info = _proto("get_memory_info", C.c_int,
                         [C.POINTER(C.c_size_t), C.POINTER(C.c_size_t)])
get_device_name = _proto("get_device_name", C.c_char_p, [C.c_int])
sc_workspace_size = _proto("sc_workspace_size", C.c_size_t,
                           [C.POINTER(ScProblem), C.POINTER(ScOptions)])
sc_options_from_algopt = _proto("sc_options_from_algopt", None,
                                [C.POINTER(AlgOpt), C.POINTER(ScOptions)])
sc_cbpdn_solve = _proto("sc_cbpdn_solve", C.c_int,
                        [C.POINTER(ScProblem), C.POINTER(ScOptions), C.c_void_p, C.c_size_t,
                         C.POINTER(ScResult), C.c_void_p])
sc_cbpdn_solve_batch = _proto("sc_cbpdn_solve_batch", C.c_int,
                              [C.POINTER(ScProblem), C.c_int, C.POINTER(ScOptions),
                               C.POINTER(C.c_void_p), C.POINTER(C.c_size_t),
                               C.POINTER(ScResult), C.POINTER(C.c_void_p)])
sc_read_state = _proto("sc_read_state", C.c_int,
                       [C.POINTER(ScProblem), C.POINTER(ScOptions), C.c_void_p, IP,
                        C.POINTER(C.c_double), C.POINTER(C.c_double), C.c_void_p])
sc_rfft2 = _proto("sc_rfft2", C.c_int,
                  [C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_void_p])
sc_irfft2 = _proto("sc_irfft2", C.c_int,
                   [C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_void_p])
sc_rfft2_noalloc = _proto("sc_rfft2_noalloc", C.c_int,
                          [C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_void_p])
VP = C.c_void_p
PP, PO = C.POINTER(ScProblem), C.POINTER(ScOptions)
sc_unrolled_workspace_size = _proto("sc_unrolled_workspace_size", C.c_size_t, [PP, PO, C.c_int])
sc_unrolled_forward = _proto("sc_unrolled_forward", C.c_int,
                             [PP, PO, C.c_int, VP, C.c_size_t, VP])
sc_unrolled_backward = _proto("sc_unrolled_backward", C.c_int,
                              [PP, PO, C.c_int, VP, C.c_size_t, VP, VP, VP, VP])
sc_last_profile = _proto("sc_last_profile", C.c_int, [C.POINTER(ScProfile)])
sc_cancel = _proto("sc_cancel", None, [])
sc_launch_count = _proto("sc_launch_count", C.c_ulonglong, [])
sc_last_status = _proto("sc_last_status", C.c_int, [])
sc_last_error = _proto("sc_last_error", C.c_char_p, [])
sc_version = _proto("sc_version", C.c_char_p, [])

# Every symbol include/sporco_b200.h declares (checked by the test suite).
EXPORTED = [
    "cuda_wrapper_CBPDN", "cuda_wrapper_CBPDN_GR", "clear_opts", "default_opts",
    "check_cuda_req", "get_device_count", "get_current_device", "set_current_device",
    "get_memory_info", "get_device_name", "sc_workspace_size", "sc_options_from_algopt",
    "sc_cbpdn_solve", "sc_cbpdn_solve_batch", "sc_read_state", "sc_rfft2", "sc_irfft2",
    "sc_rfft2_noalloc", "sc_unrolled_workspace_size", "sc_unrolled_forward",
    "sc_unrolled_backward", "sc_cancel", "sc_last_profile", "sc_launch_count",
    "sc_last_status", "sc_last_error", "sc_version",
]


class SolverError(RuntimeError):
    """A CUDA solver call returned a non-zero status."""

    def __init__(self, status, msg):
        self.status = status
        super().__init__("%s: %s" % (STATUS_NAMES.get(status, status), msg))


def check(status):
    if status != SC_OK:
        raise SolverError(status, (sc_last_error() or b"").decode(errors="replace"))


def check_last():
    check(sc_last_status())
