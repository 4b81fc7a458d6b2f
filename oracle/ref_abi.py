"""ctypes binding of the compiled reference (oracle/_ref/libsporco_cuda_ref.so).

TEST INFRASTRUCTURE ONLY: used to generate golden fixtures from the
reference's own FP32 GPU path.  The library is built from the reference's
sources by ``oracle/Makefile`` (target ``ref``); this module reproduces the
marshalling that ``sporco_cuda/cbpdn.pyx`` performs before calling the C ABI
``cuda_wrapper_CBPDN`` (src/cbpdn.h:10) and ``cuda_wrapper_CBPDN_GR``
(src/cbpdn_grd.h:10-11).  The struct below has the field order of ``AlgOpt``
(src/algopt.h:7-48) because it must match that ABI byte for byte.
"""

from __future__ import annotations

import ctypes as C
import os

import numpy as np

F32 = np.float32
_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "_ref", "libsporco_cuda_ref.so")


class AlgOpt(C.Structure):
    _fields_ = [
        ("MaxMainIter", C.c_int),
        ("rho", C.c_float),
        ("RhoRsdlRatio", C.c_float),
        ("RhoScaling", C.c_float),
        ("RhoRsdlTarget", C.c_float),
        ("RelaxParam", C.c_float),
        ("AbsStopTol", C.c_float),
        ("RelStopTol", C.c_float),
        ("L1Weight", C.POINTER(C.c_float)),
        ("L1_WEIGHT_M_SIZE", C.c_int),
        ("L1_WEIGHT_ROW_SIZE", C.c_int),
        ("L1_WEIGHT_COL_SIZE", C.c_int),
        ("Weight", C.POINTER(C.c_int)),
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
        ("GrdWeight", C.POINTER(C.c_float)),
        ("WEIGHT_SIZE", C.c_int),
        ("device", C.c_int),
    ]


_lib = None


def available() -> bool:
    return os.path.exists(LIB_PATH)


def lib():
    global _lib
    if _lib is None:
        _lib = C.CDLL(LIB_PATH)
        fp = C.POINTER(C.c_float)
        _lib.cuda_wrapper_CBPDN.argtypes = [fp, fp, C.c_float, C.c_void_p, fp]
        _lib.cuda_wrapper_CBPDN.restype = None
        _lib.cuda_wrapper_CBPDN_GR.argtypes = [fp, fp, C.c_float, C.c_float, C.c_void_p, fp]
        _lib.cuda_wrapper_CBPDN_GR.restype = None
        _lib.clear_opts.argtypes = [C.c_void_p]
        _lib.clear_opts.restype = None
    return _lib


def _fptr(a):
    return a.ctypes.data_as(C.POINTER(C.c_float))


def _set_algopt(o: AlgOpt, opt):
    """cbpdn.pyx:57-79 (every key required, as for a plain dict there)."""
    ar = opt["AutoRho"]
    o.Verbose = int(opt["Verbose"])
    o.MaxMainIter = int(opt["MaxMainIter"])
    o.RelaxParam = F32(opt["RelaxParam"])
    o.AbsStopTol = F32(opt["AbsStopTol"])
    o.RelStopTol = F32(opt["RelStopTol"])
    o.AuxVarObj = int(opt["AuxVarObj"])
    o.HighMemSolve = int(opt["HighMemSolve"])
    o.NonNegCoef = int(opt["NonNegCoef"])
    o.NoBndryCross = int(opt["NoBndryCross"])
    o.StdResiduals = int(ar["StdResiduals"])
    o.AutoRho = int(ar["Enabled"])
    o.AutoRhoScaling = int(F32(ar["AutoScaling"]))
    o.AutoRhoPeriod = int(ar["Period"])
    o.RhoRsdlRatio = F32(ar["RsdlRatio"])
    o.RhoScaling = F32(ar["Scaling"])
    o.RhoRsdlTarget = F32(-1.0 if ar["RsdlTarget"] is None else ar["RsdlTarget"])


def _call(D, S, W, lmbda, mu, opt, grd):
    """_cbpdn / _cbpdngrd (cbpdn.pyx:158-201, 297-349); D is (M, Kr, Kc)."""
    D = np.ascontiguousarray(D, dtype=np.float32)
    S = np.ascontiguousarray(S, dtype=np.float32)
    W = np.ascontiguousarray(W, dtype=np.int32)
    X = np.zeros((D.shape[0], S.shape[0], S.shape[1]), dtype=np.float32)
    o = AlgOpt()
    lib().clear_opts(C.byref(o))
    _set_algopt(o, opt)
    o.device = 0
    o.IMG_ROW_SIZE, o.IMG_COL_SIZE = S.shape
    o.DICT_M_SIZE, o.DICT_ROW_SIZE, o.DICT_COL_SIZE = D.shape
    lam = F32(lmbda)
    o.rho = F32(5e1 * float(lam) + 1.0) if opt["rho"] is None else F32(opt["rho"])
    w = opt["L1Weight"]
    if hasattr(w, "ndim"):
        gl1w = np.ascontiguousarray(np.rollaxis(np.asarray(w, dtype=np.float32), 2, 0))
        o.L1_WEIGHT_M_SIZE, o.L1_WEIGHT_ROW_SIZE, o.L1_WEIGHT_COL_SIZE = gl1w.shape
    else:
        gl1w = np.asarray([w], dtype=np.float32).reshape((1, 1, 1))
        o.L1_WEIGHT_M_SIZE = o.L1_WEIGHT_ROW_SIZE = o.L1_WEIGHT_COL_SIZE = 1
    o.L1Weight = _fptr(gl1w)
    if grd:
        g = opt["GradWeight"]
        gw = np.ascontiguousarray(g, dtype=np.float32).ravel() if hasattr(g, "ndim") \
            else np.asarray([g], dtype=np.float32)
        o.WEIGHT_SIZE = gw.shape[0]
        o.GrdWeight = _fptr(gw)
    if W.size > 1:
        o.Weight = W.ctypes.data_as(C.POINTER(C.c_int))
        o.nWeight = W.size
    keep = (D, S, W, gl1w, X)  # noqa: F841  (keep buffers alive across the call)
    if grd:
        lib().cuda_wrapper_CBPDN_GR(_fptr(D), _fptr(S), lam, F32(mu), C.byref(o), _fptr(X))
    else:
        lib().cuda_wrapper_CBPDN(_fptr(D), _fptr(S), lam, C.byref(o), _fptr(X))
    return X


def _ams_prep(D, opt, grd):
    d0 = np.zeros((D.shape[0], D.shape[1], 1), dtype=np.float32)
    d0[0, 0] = 1.0
    Di = np.dstack((d0, D))
    o2 = dict(opt)
    w = opt["L1Weight"]
    if hasattr(w, "ndim"):
        w0 = np.zeros(w.shape[0:-1] + (1,), dtype=np.float32)
        o2["L1Weight"] = np.dstack((w0, w))
    else:
        a = w * np.ones((1, 1, Di.shape[2]), dtype=np.float32)
        a[..., 0] = 0.0
        o2["L1Weight"] = a
    if grd:
        g = opt["GradWeight"]
        if hasattr(g, "ndim"):
            o2["GradWeight"] = np.hstack((np.zeros((1,), dtype=np.float32), g))
        else:
            a = g * np.ones((Di.shape[2],), dtype=np.float32)
            a[..., 0] = 0.0
            o2["GradWeight"] = a
    return Di, o2


def cbpdn(D, S, lmbda, opt):
    W = np.ones((1, 1), dtype=np.int32)
    X = _call(np.rollaxis(D, 2, 0), S, W, lmbda, 0.0, opt, False)
    return np.rollaxis(X, 0, 3)


def cbpdnmsk(D, S, W, lmbda, opt):
    Di, o2 = _ams_prep(D, opt, False)
    X = _call(np.rollaxis(Di, 2, 0), S, W, lmbda, 0.0, o2, False)
    return np.rollaxis(X, 0, 3)[..., 1:]


def cbpdngrd(D, S, lmbda, mu, opt):
    W = np.ones((1, 1), dtype=np.int32)
    X = _call(np.rollaxis(D, 2, 0), S, W, lmbda, mu, opt, True)
    return np.rollaxis(X, 0, 3)


def cbpdngrdmsk(D, S, W, lmbda, mu, opt):
    Di, o2 = _ams_prep(D, opt, True)
    X = _call(np.rollaxis(Di, 2, 0), S, W, lmbda, mu, o2, True)
    return np.rollaxis(X, 0, 3)[..., 1:]
