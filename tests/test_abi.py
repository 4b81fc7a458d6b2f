"""C ABI checks that need no GPU: the library loads, exports every function
that include/sporco_b200.h declares, the AlgOpt layout matches the
reference's, and the host-side option logic behaves like the reference's."""

import ctypes as C
import os
import re
import subprocess

import numpy as np
import pytest

import sporco_cuda
from sporco_cuda import _lib, cbpdn as cb

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "sporco_b200.h")


def _declared_functions():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    names = re.findall(r"\b([A-Za-z_][A-Za-z0-9_]*)\s*\([^;{]*\)\s*;", src)
    return sorted(set(n for n in names if n not in ("sizeof",)))


def test_header_declarations_are_exported():
    decl = _declared_functions()
    assert len(decl) >= 19
    out = subprocess.check_output(["nm", "-D", "--defined-only", _lib.LIB_PATH], text=True)
    exported = set(line.split()[-1] for line in out.splitlines() if line.strip())
    missing = [d for d in decl if d not in exported]
    assert not missing, missing
    assert sorted(_lib.EXPORTED) == decl


def test_every_declared_symbol_resolves_through_ctypes():
    for name in _declared_functions():
        assert hasattr(_lib.lib, name)


def test_algopt_layout_matches_reference():
    # Size and offsets of the reference's AlgOpt (algopt.h:7-48) as gcc lays
    # it out on x86-64 (sizeof and offsetof compiled against that header).
    assert C.sizeof(_lib.AlgOpt) == 144
    assert _lib.AlgOpt.L1Weight.offset == 32
    assert _lib.AlgOpt.Weight.offset == 56
    assert _lib.AlgOpt.GrdWeight.offset == 128
    assert _lib.AlgOpt.device.offset == 140


def test_clear_and_default_opts_match_reference_defaults():
    a = _lib.AlgOpt()
    _lib.clear_opts(C.byref(a))
    assert a.MaxMainIter == -1 and a.rho == -1 and a.AutoRho == -1 and a.nWeight == -1
    _lib.default_opts(C.byref(a))
    # utils.cu:12-64
    assert a.MaxMainIter == 250
    assert abs(a.RelaxParam - 1.8) < 1e-6
    assert a.RhoScaling == 100
    assert abs(a.RelStopTol - 1e-4) < 1e-9
    assert a.AutoRho == 1 and a.AutoRhoPeriod == 1 and a.AutoRhoScaling == 1
    assert abs(a.RhoRsdlRatio - 1.2) < 1e-6
    assert a.device == 0 and a.nWeight == 1 and a.Verbose == 0


def test_options_from_algopt():
    a = _lib.AlgOpt()
    _lib.clear_opts(C.byref(a))
    _lib.default_opts(C.byref(a))
    o = _lib.ScOptions()
    _lib.sc_options_from_algopt(C.byref(a), C.byref(o))
    assert o.max_iter == 250 and o.auto_rho == 1 and o.auto_rho_period == 1
    assert abs(o.relax - 1.8) < 1e-6


def test_workspace_size_and_invalid_sizes():
    p = _lib.ScProblem()
    p.B, p.H, p.W, p.M, p.Kr, p.Kc = 1, 64, 64, 8, 8, 8
    o = _lib.ScOptions()
    o.max_iter = 10
    n = _lib.sc_workspace_size(C.byref(p), C.byref(o))
    Wp = 36  # 64/2+1 = 33 rounded up to a multiple of 4
    assert n >= 4 * 8 * 64 * 64 + 8 * 8 * 64 * Wp * 2
    p.Kr = 100  # filter larger than the image
    assert _lib.sc_workspace_size(C.byref(p), C.byref(o)) == 0
    assert _lib.sc_last_status() == 1
    p.Kr = 8
    p.H = 1 << 20
    assert _lib.sc_workspace_size(C.byref(p), C.byref(o)) == 0
    assert _lib.sc_last_status() == 2


def test_unrolled_workspace_size_and_rejections():
    p = _lib.ScProblem()
    p.B, p.H, p.W, p.M, p.Kr, p.Kc = 2, 64, 64, 8, 8, 8
    o = _lib.ScOptions()
    o.max_iter = 10
    base = _lib.sc_workspace_size(C.byref(p), C.byref(o))
    R, Cs = 2 * 8 * 64 * 64, 2 * 8 * 64 * 36
    n4 = _lib.sc_unrolled_workspace_size(C.byref(p), C.byref(o), 4)
    # checkpoints for 3 segments (Y and U), 4 Y traces, 4 x^ traces, gV, Fb, gD^
    assert n4 >= base + 4 * R * (2 * 3 + 4 + 1) + 8 * Cs * (4 + 2)
    n10 = _lib.sc_unrolled_workspace_size(C.byref(p), C.byref(o), 10)
    assert n10 > n4
    for seg in (0, 11):
        assert _lib.sc_unrolled_workspace_size(C.byref(p), C.byref(o), seg) == 0
        assert _lib.sc_last_status() == 1
    p.grd = 1
    assert _lib.sc_unrolled_workspace_size(C.byref(p), C.byref(o), 4) == 0
    assert _lib.sc_last_status() == 2
    p.grd = 0
    o.max_iter = 0
    assert _lib.sc_unrolled_workspace_size(C.byref(p), C.byref(o), 1) == 0
    assert _lib.sc_last_status() == 1


def test_no_device_paths_fail_cleanly():
    assert sporco_cuda.util.device_count() >= 0
    if sporco_cuda.util.device_count() == 0:
        assert _lib.check_cuda_req(0) == -1


def test_python_argument_checks():
    D = np.zeros((3, 3, 2), np.float32)
    S = np.zeros((8, 8), np.float32)
    with pytest.raises(TypeError):
        cb.cbpdn(None, S, 0.1, {})
    with pytest.raises(ValueError):
        cb.cbpdn(D.astype(np.float64), S, 0.1, {})
    with pytest.raises(ValueError):
        cb.cbpdn(D[..., 0], S, 0.1, {})
    with pytest.raises(TypeError):
        cb.cbpdnmsk(D, S, [[1]], 0.1, {})


def test_resolve_options_like_set_algopt():
    r = cb.resolve_options({"AutoRho": {"Enabled": False}, "rho": None}, 0.1)
    assert r["AutoRho"] == 0
    assert r["rho"] == np.float32(50 * float(np.float32(0.1)) + 1)
    assert r["MaxMainIter"] == 250 and r["RhoRsdlTarget"] == -1
    r = cb.resolve_options({"AutoRho": {"RsdlTarget": 2.5}}, 0.1)
    assert r["RhoRsdlTarget"] == np.float32(2.5)
