"""Drop-in replacement for ``sporco_cuda.cbpdn`` on B200 (sm_100a).

The four solvers keep the reference's signatures and option semantics
(sporco_cuda/cbpdn.pyx:86-349):

    cbpdn(D, S, lmbda, opt, dev=0)
    cbpdnmsk(D, S, W, lmbda, opt, dev=0)
    cbpdngrd(D, S, lmbda, mu, opt, dev=0)
    cbpdngrdmsk(D, S, W, lmbda, mu, opt, dev=0)

``D`` is (Kr, Kc, M), ``S`` is (H, W), the result is (H, W, M) (for the mask
variants the AMS impulse map is dropped, as in the reference).

* numpy inputs take the reference's own route: host buffers marshalled into
  an ``AlgOpt`` struct and passed to ``cuda_wrapper_CBPDN`` /
  ``cuda_wrapper_CBPDN_GR`` (same C ABI as the reference), which copy to the
  device, solve and copy back.  numpy in, numpy out.
* torch CUDA tensors take the device route (``sc_cbpdn_solve``): no host
  copies, the current torch stream, a torch-allocated workspace.  torch in,
  torch out.

Differences from the reference, all deliberate: errors raise
``SolverError`` instead of terminating the process; a plain dict may omit
keys (the reference's C defaults fill them); ``opt`` is never mutated; a
user ``AutoRho.RsdlTarget`` is honoured; the solve coefficients always follow
the current rho (the reference's are stale after a rho change unless
``HighMemSolve``); after a rho change all of U is rescaled; ``NonNegCoef``
and ``NoBndryCross``, which the reference parses but ignores
(cbpdn.pyx:70-71), are applied as sporco's ConvBPDN applies them.
"""

from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib

F32 = np.float32

__all__ = ["cbpdn", "cbpdnmsk", "cbpdngrd", "cbpdngrdmsk", "SolverError",
           "solve_device", "resolve_options", "ConvBPDN", "cbpdn_batched", "cbpdn_multi"]

SolverError = _lib.SolverError

# C-level defaults the reference applies to unset fields (utils.cu:12-64).
_DEFAULTS = {
    "Verbose": False, "MaxMainIter": 250, "RelaxParam": 1.8, "AbsStopTol": 0.0,
    "RelStopTol": 1e-4, "AuxVarObj": False, "HighMemSolve": False, "NonNegCoef": False,
    "NoBndryCross": False, "rho": None, "L1Weight": 1.0, "GradWeight": 1.0,
}
_AR_DEFAULTS = {"Enabled": True, "Period": 1, "Scaling": 100.0, "RsdlRatio": 1.2,
                "RsdlTarget": None, "AutoScaling": True, "StdResiduals": False}


def _opt_get(opt, key):
    try:
        v = opt[key]
    except (KeyError, TypeError):
        return _DEFAULTS[key]
    return v


def _ar_get(opt, key):
    try:
        ar = opt["AutoRho"]
    except (KeyError, TypeError):
        return _AR_DEFAULTS[key]
    try:
        v = ar[key]
    except (KeyError, TypeError):
        return _AR_DEFAULTS[key]
    if v is None and key != "RsdlTarget":
        return _AR_DEFAULTS[key]
    return v


def resolve_options(opt, lmbda):
    """The scalar fields of ``AlgOpt`` as set_algopt (cbpdn.pyx:57-79) and
    the rho default (cbpdn.pyx:179) set them, as a plain dict."""
    lam32 = F32(lmbda)
    rho = _opt_get(opt, "rho")
    tgt = _ar_get(opt, "RsdlTarget")
    return {
        "Verbose": int(bool(_opt_get(opt, "Verbose"))),
        "MaxMainIter": int(_opt_get(opt, "MaxMainIter")),
        "RelaxParam": F32(_opt_get(opt, "RelaxParam")),
        "AbsStopTol": F32(_opt_get(opt, "AbsStopTol")),
        "RelStopTol": F32(_opt_get(opt, "RelStopTol")),
        "AuxVarObj": int(bool(_opt_get(opt, "AuxVarObj"))),
        "HighMemSolve": int(bool(_opt_get(opt, "HighMemSolve"))),
        "NonNegCoef": int(bool(_opt_get(opt, "NonNegCoef"))),
        "NoBndryCross": int(bool(_opt_get(opt, "NoBndryCross"))),
        "StdResiduals": int(bool(_ar_get(opt, "StdResiduals"))),
        "AutoRho": int(bool(_ar_get(opt, "Enabled"))),
        "AutoRhoScaling": int(F32(_ar_get(opt, "AutoScaling"))),
        "AutoRhoPeriod": int(_ar_get(opt, "Period")),
        "RhoRsdlRatio": F32(_ar_get(opt, "RsdlRatio")),
        "RhoScaling": F32(_ar_get(opt, "Scaling")),
        "RhoRsdlTarget": F32(-1.0 if tgt is None else tgt),
        "rho": F32(5e1 * float(lam32) + 1.0) if rho is None else F32(rho),
    }


# ----------------------------------------------------------------- checks --

def _is_torch(x):
    return type(x).__module__.startswith("torch")


def _check_array(x, ndim, name):
    """Cython's typed-buffer checks for ``np.ndarray[DTYPE_t, ndim=n] not None``."""
    if x is None:
        raise TypeError("Argument '%s' must not be None" % name)
    if not isinstance(x, np.ndarray):
        raise TypeError("Argument '%s' has incorrect type (expected numpy.ndarray, got %s)"
                        % (name, type(x).__name__))
    if x.ndim != ndim:
        raise ValueError("Buffer has wrong number of dimensions (expected %d, got %d)"
                         % (ndim, x.ndim))
    if x.dtype != np.float32:
        raise ValueError("Buffer dtype mismatch, expected 'DTYPE_t' but got '%s'" % x.dtype)


# ------------------------------------------------------- AMS preparation --

def _ams_weights(shape_hw, Mi, opt, grd):
    """Weights with a zero entry for the prepended impulse map
    (cbpdn.pyx:120-137, 245-275).  Returns (l1, grad) in the reference's
    (Hw, Ww, M+1) and (M+1,) shapes."""
    w = _opt_get(opt, "L1Weight")
    if hasattr(w, "ndim"):
        w = np.asarray(w, dtype=F32)
        w0 = np.zeros(w.shape[0:-1] + (1,), dtype=F32)
        l1 = np.dstack((w0, w))
    else:
        l1 = F32(w) * np.ones((1, 1, Mi), dtype=F32)
        l1[..., 0] = 0.0
    g = None
    if grd:
        gw = _opt_get(opt, "GradWeight")
        if hasattr(gw, "ndim"):
            g = np.hstack((np.zeros((1,), dtype=F32), np.asarray(gw, dtype=F32).ravel()))
        else:
            g = F32(gw) * np.ones((Mi,), dtype=F32)
            g[..., 0] = 0.0
    return l1, g


def _impulse_dict(D):
    d0 = np.zeros((D.shape[0], D.shape[1], 1), dtype=F32)
    d0[0, 0] = 1.0
    return np.dstack((d0, D))


# ------------------------------------------------------- host (numpy) path --

def _host_solve(Dm, S, Wmask, lmbda, mu, opt, l1, gw, dev, grd):
    """_cbpdn / _cbpdngrd (cbpdn.pyx:158-201, 297-349) over the C ABI.

    Dm: (M, Kr, Kc) C-contiguous float32; returns (M, H, W) float32."""
    M, Kr, Kc = Dm.shape
    H, W = S.shape
    X = np.zeros((M, H, W), dtype=F32)
    r = resolve_options(opt, lmbda)
    a = _lib.AlgOpt()
    _lib.clear_opts(C.byref(a))
    for k in ("Verbose", "MaxMainIter", "RelaxParam", "AbsStopTol", "RelStopTol", "AuxVarObj",
              "HighMemSolve", "NonNegCoef", "NoBndryCross", "StdResiduals", "AutoRho",
              "AutoRhoScaling", "AutoRhoPeriod", "RhoRsdlRatio", "RhoScaling", "RhoRsdlTarget",
              "rho"):
        setattr(a, k, r[k])
    a.device = int(dev)
    a.IMG_ROW_SIZE, a.IMG_COL_SIZE = H, W
    a.DICT_M_SIZE, a.DICT_ROW_SIZE, a.DICT_COL_SIZE = M, Kr, Kc
    if hasattr(l1, "ndim"):
        l1 = np.asarray(l1, dtype=F32)
        if l1.ndim != 3:
            raise ValueError("L1Weight array must have 3 dimensions (Hw, Ww, M)")
        gl1w = np.ascontiguousarray(np.rollaxis(l1, 2, 0))
        a.L1_WEIGHT_M_SIZE, a.L1_WEIGHT_ROW_SIZE, a.L1_WEIGHT_COL_SIZE = gl1w.shape
    else:
        gl1w = np.asarray([l1], dtype=F32).reshape((1, 1, 1))
        a.L1_WEIGHT_M_SIZE = a.L1_WEIGHT_ROW_SIZE = a.L1_WEIGHT_COL_SIZE = 1
    a.L1Weight = gl1w.ctypes.data_as(_lib.FP)
    gwa = None
    if grd:
        if hasattr(gw, "ndim"):
            gwa = np.ascontiguousarray(np.asarray(gw, dtype=F32).ravel())
        else:
            gwa = np.asarray([gw], dtype=F32)
        a.WEIGHT_SIZE = gwa.shape[0]
        a.GrdWeight = gwa.ctypes.data_as(_lib.FP)
    Wi = np.ascontiguousarray(Wmask, dtype=np.int32)
    if Wi.size > 1:
        if Wi.shape != (H, W):
            raise ValueError("mask shape %s differs from the signal shape %s" % (Wi.shape, (H, W)))
        a.Weight = Wi.ctypes.data_as(_lib.IP)
        a.nWeight = Wi.size
    Dc = np.ascontiguousarray(Dm, dtype=F32)
    Sc = np.ascontiguousarray(S, dtype=F32)
    if grd:
        _lib.cuda_wrapper_CBPDN_GR(Dc.ctypes.data_as(_lib.FP), Sc.ctypes.data_as(_lib.FP),
                                   F32(lmbda), F32(mu), C.byref(a), X.ctypes.data_as(_lib.FP))
    else:
        _lib.cuda_wrapper_CBPDN(Dc.ctypes.data_as(_lib.FP), Sc.ctypes.data_as(_lib.FP),
                                F32(lmbda), C.byref(a), X.ctypes.data_as(_lib.FP))
    _lib.check_last()
    return X


# ------------------------------------------------------ device (torch) path --

def _sc_options(r, record_itstat=False, check_every=32, profile=False):
    o = _lib.ScOptions()
    o.max_iter = r["MaxMainIter"]
    o.relax = r["RelaxParam"]
    o.abs_tol = r["AbsStopTol"]
    o.rel_tol = r["RelStopTol"]
    o.auto_rho = r["AutoRho"]
    o.auto_rho_period = max(1, r["AutoRhoPeriod"])
    o.rho_scaling = r["RhoScaling"]
    o.rsdl_ratio = r["RhoRsdlRatio"]
    o.rsdl_target = r["RhoRsdlTarget"]
    o.auto_scaling = r["AutoRhoScaling"]
    o.std_residuals = r["StdResiduals"]
    o.record_itstat = int(bool(record_itstat or r["Verbose"]))
    o.check_every = int(check_every)
    o.profile = int(bool(profile))
    o.nonneg = r["NonNegCoef"]
    o.no_bndry_cross = r["NoBndryCross"]
    return o


# Per-iteration statistics (sc_read_state): r, s, rho, eps_pri, eps_dua,
# functional at Y, its data fidelity term, its L1 sum.
ITSTAT_FIELDS = 8
ITSTAT_NAMES = ("r", "s", "rho", "epri", "edua", "fnc", "dfid", "regl1")


class DeviceSolve:
    """A prepared device solve: problem struct, options and workspace.

    Built by :func:`prepare_device`; :meth:`run` launches the solve on the
    current torch stream and can be called repeatedly (inputs are re-read
    each time).  Used by the torch path of the four solvers, the batched
    solver and the benchmark."""

    def __init__(self, prob, opts, ws, keep):
        self.prob = prob
        self.opts = opts
        self.ws = ws
        self.keep = keep
        self.result = _lib.ScResult()
        self.last_iters = opts.max_iter  # MaxMainIter of the last run (its itstat rows)

    def run(self, stream=None, warm=False, iters=None):
        """Launch the solve on `stream` (default: the current torch stream)
        and return Y (B, M, H, W).

        warm=False starts from Y = U = 0 at rho0 (or from the warm-start
        iterates given to prepare_device).  warm=True continues the state
        the previous run left in the workspace (iterates, rho, iteration
        count, as sporco's solve() continues its own), re-reading D and S
        (so a dictionary changed with :meth:`set_dict` in between is used);
        warm="same" also keeps their spectra (D and S unchanged).  iters:
        iterations of this run (default MaxMainIter)."""
        import torch
        s = stream if stream is not None else torch.cuda.current_stream()
        keep_iters, keep_warm = self.opts.max_iter, self.opts.warm_start
        if iters is not None:
            self.opts.max_iter = int(iters)
        self.opts.warm_start = 2 if warm == "same" else (1 if warm else 0)
        try:
            st = _lib.sc_cbpdn_solve(C.byref(self.prob), C.byref(self.opts),
                                     C.c_void_p(self.ws.data_ptr()), self.ws.numel(),
                                     C.byref(self.result), C.c_void_p(s.cuda_stream))
        finally:
            self.last_iters = self.opts.max_iter
            self.opts.max_iter, self.opts.warm_start = keep_iters, keep_warm
        _lib.check(st)
        return self.keep["Y"]

    def set_dict(self, Dm):
        """Replace the dictionary (M, Kr, Kc) in place (same shape); the next
        run, cold or warm=True, uses it."""
        import torch
        D = self.keep["D"]
        Dm = torch.as_tensor(Dm, device=D.device, dtype=torch.float32)
        if Dm.shape != D.shape:
            raise ValueError("dictionary shape %s differs from %s" % (tuple(Dm.shape),
                                                                     tuple(D.shape)))
        D.copy_(Dm)

    def state(self):
        import torch
        B = self.prob.B
        iters = (C.c_int * B)()
        rho = (C.c_double * B)()
        it = None
        opts = _lib.ScOptions.from_buffer_copy(self.opts)
        opts.max_iter = self.last_iters  # the itstat layout of the last run
        if opts.record_itstat:
            it = np.zeros((B, max(1, opts.max_iter), ITSTAT_FIELDS), dtype=np.float64)
        st = _lib.sc_read_state(C.byref(self.prob), C.byref(opts),
                                C.c_void_p(self.ws.data_ptr()), iters, rho,
                                it.ctypes.data_as(C.POINTER(C.c_double)) if it is not None else None,
                                C.c_void_p(torch.cuda.current_stream().cuda_stream))
        _lib.check(st)
        return {"iterations": list(iters), "rho": list(rho), "itstat": it}

    def profile(self):
        """Per-kernel device time (ms, launches) of the last run with
        profile=True: column pass, row pass, finalize, rho fix-up."""
        p = _lib.ScProfile()
        _lib.check(_lib.sc_last_profile(C.byref(p)))
        names = ("col_kernel", "row_kernel", "finalize_kernel", "fixup_kernel")
        return {n: (p.ms[i], p.count[i]) for i, n in enumerate(names)}


def prepare_device(Dm, S, lmbda, opt, mu=0.0, grd=False, l1=1.0, gw=1.0, mask=None,
                   rho0=None, Y=None, record_itstat=False, check_every=32, profile=False,
                   workspace=True):
    """Prepare a device solve for a batch of equal-sized images.

    Dm: (M, Kr, Kc) float32 CUDA tensor; S: (B, H, W) float32 CUDA tensor;
    lmbda: float or (B,) tensor/array; l1: scalar, (M,) or broadcastable to
    (M, H, W); gw: scalar or (M,); mask: (B, H, W) int32 tensor (map 0 is
    then the AMS impulse) or None.  Returns a DeviceSolve whose ``run``
    writes Y (B, M, H, W); with workspace=False it has no workspace (for
    callers that size their own, e.g. the unrolled solve)."""
    import torch
    dev = S.device
    B, H, W = S.shape
    M, Kr, Kc = Dm.shape
    r = resolve_options(opt, float(np.asarray(lmbda).ravel()[0]) if not torch.is_tensor(lmbda)
                        else float(lmbda.reshape(-1)[0]))
    lam = torch.as_tensor(np.broadcast_to(np.asarray(lmbda, dtype=F32), (B,)).copy()
                          if not torch.is_tensor(lmbda) else lmbda.float().reshape(-1).expand(B),
                          device=dev).contiguous()
    if rho0 is None:
        rho_opt = _opt_get(opt, "rho")
        if rho_opt is None:
            rho0 = (lam.double() * 5e1 + 1.0).float()
        else:
            rho0 = torch.full((B,), float(F32(rho_opt)), device=dev, dtype=torch.float32)
    rho0 = torch.as_tensor(rho0, device=dev, dtype=torch.float32).reshape(-1).expand(B).contiguous()
    prob = _lib.ScProblem()
    prob.B, prob.H, prob.W, prob.M, prob.Kr, prob.Kc = B, H, W, M, Kr, Kc
    keep = {"D": Dm.contiguous().clone(), "S": S.contiguous(), "lam": lam, "rho0": rho0}
    prob.D = keep["D"].data_ptr()
    prob.S = keep["S"].data_ptr()
    prob.lmbda = lam.data_ptr()
    prob.rho0 = rho0.data_ptr()
    prob.grd = int(bool(grd))
    prob.mu = float(F32(mu))
    if grd:
        g = torch.as_tensor(np.asarray(gw, dtype=F32) if not torch.is_tensor(gw) else gw,
                            dtype=torch.float32, device=dev).reshape(-1)
        if g.numel() == 1:
            g = g.expand(M)
        if g.numel() != M:
            raise ValueError("GradWeight must be a scalar or have M entries")
        keep["gw"] = g.contiguous()
        prob.wgrd = keep["gw"].data_ptr()
        prob.wgrd_uniform = int(bool(torch.all(keep["gw"] == keep["gw"][0]).item()))
    l1a = l1.detach().float() if torch.is_tensor(l1) else np.asarray(l1, dtype=F32)
    l1n = l1a.numel() if torch.is_tensor(l1a) else l1a.size
    if l1n == 1:
        prob.l1_kind = _lib.SC_L1_SCALAR
        prob.l1_scalar = float(np.asarray(_np(l1a), dtype=F32).ravel()[0])
    else:
        t = torch.as_tensor(l1a, dtype=torch.float32, device=dev)
        if t.numel() == M and all(d == 1 for d in t.shape[1:]):
            # one weight per map, e.g. (M,) or (M, 1, 1)
            prob.l1_kind = _lib.SC_L1_PER_MAP
            keep["l1"] = t.reshape(M).contiguous()
        else:
            while t.ndim < 3:
                t = t.unsqueeze(0)
            keep["l1"] = t.expand(M, H, W).contiguous()
            prob.l1_kind = _lib.SC_L1_FULL
        prob.l1w = keep["l1"].data_ptr()
    if mask is not None:
        keep["mask"] = torch.as_tensor(mask, device=dev).to(torch.int32).reshape(B, H, W).contiguous()
        prob.mask = keep["mask"].data_ptr()
    if Y is None:
        Y = torch.empty((B, M, H, W), device=dev, dtype=torch.float32)
    keep["Y"] = Y
    prob.Y = Y.data_ptr()
    o = _sc_options(r, record_itstat=record_itstat, check_every=check_every, profile=profile)
    if not workspace:
        return DeviceSolve(prob, o, None, keep)
    nbytes = _lib.sc_workspace_size(C.byref(prob), C.byref(o))
    if nbytes == 0:
        _lib.check_last()
    ws = torch.empty(nbytes, dtype=torch.uint8, device=dev)
    return DeviceSolve(prob, o, ws, keep)


def solve_device(Dm, S, lmbda, opt, **kw):
    """One-shot device solve; returns Y (B, M, H, W)."""
    ds = prepare_device(Dm, S, lmbda, opt, **kw)
    return ds.run()


def _torch_entry(D, S, W, lmbda, mu, opt, grd, ams):
    import torch
    if not (D.is_cuda and S.is_cuda):
        raise ValueError("torch inputs must be CUDA tensors")
    if D.ndim != 3 or S.ndim != 2:
        raise ValueError("D must be (Kr, Kc, M) and S must be (H, W)")
    D = D.float()
    S = S.float()
    l1 = _opt_get(opt, "L1Weight")
    gw = _opt_get(opt, "GradWeight") if grd else 1.0
    mask = None
    if ams:
        d0 = torch.zeros((D.shape[0], D.shape[1], 1), dtype=D.dtype, device=D.device)
        d0[0, 0] = 1.0
        D = torch.cat((d0, D), dim=2)
        l1, gw = _ams_weights(S.shape, D.shape[2], {"L1Weight": _np(l1), "GradWeight": _np(gw)},
                              grd)
        Wi = torch.as_tensor(W, device=D.device).to(torch.int32)
        if Wi.numel() > 1:
            mask = Wi.reshape(1, *S.shape)
    Dm = D.permute(2, 0, 1).contiguous()
    l1m = l1
    if hasattr(l1, "ndim") and np.ndim(l1) == 3:
        l1m = np.ascontiguousarray(np.rollaxis(_np(l1), 2, 0))
    Y = solve_device(Dm, S.reshape(1, *S.shape), lmbda, opt, mu=mu, grd=grd, l1=l1m, gw=gw,
                     mask=mask)
    X = Y[0].permute(1, 2, 0)
    return X[..., 1:] if ams else X


def _np(x):
    if type(x).__module__.startswith("torch"):
        return x.detach().cpu().numpy()
    return x


# ------------------------------------------------------------ entry points --

def cbpdn(D, S, lmbda, opt, dev=0):
    """GPU ConvBPDN (cbpdn.pyx:86-102)."""
    if _is_torch(D):
        return _torch_entry(D, S, None, lmbda, 0.0, opt, False, False)
    _check_array(D, 3, "D")
    _check_array(S, 2, "S")
    W = np.ones((1, 1), dtype=np.int32)
    X = _host_solve(np.ascontiguousarray(np.rollaxis(D, 2, 0)), np.ascontiguousarray(S), W,
                    lmbda, 0.0, opt, _opt_get(opt, "L1Weight"), None, dev, False)
    return np.rollaxis(X, 0, 3)


def cbpdnmsk(D, S, W, lmbda, opt, dev=0):
    """GPU ConvBPDN with an AMS spatial mask (cbpdn.pyx:108-152)."""
    if _is_torch(D):
        return _torch_entry(D, S, W, lmbda, 0.0, opt, False, True)
    _check_array(D, 3, "D")
    _check_array(S, 2, "S")
    if not isinstance(W, np.ndarray):
        raise TypeError("Argument 'W' has incorrect type (expected numpy.ndarray)")
    Di = _impulse_dict(D)
    l1, _ = _ams_weights(S.shape, Di.shape[2], opt, False)
    X = _host_solve(np.ascontiguousarray(np.rollaxis(Di, 2, 0)), np.ascontiguousarray(S),
                    np.ascontiguousarray(W, dtype=np.int32), lmbda, 0.0, opt, l1, None, dev, False)
    return np.rollaxis(X, 0, 3)[..., 1:]


def cbpdngrd(D, S, lmbda, mu, opt, dev=0):
    """GPU ConvBPDNGradReg (cbpdn.pyx:207-223)."""
    if _is_torch(D):
        return _torch_entry(D, S, None, lmbda, mu, opt, True, False)
    _check_array(D, 3, "D")
    _check_array(S, 2, "S")
    W = np.ones((1, 1), dtype=np.int32)
    X = _host_solve(np.ascontiguousarray(np.rollaxis(D, 2, 0)), np.ascontiguousarray(S), W,
                    lmbda, mu, opt, _opt_get(opt, "L1Weight"), _opt_get(opt, "GradWeight"), dev,
                    True)
    return np.rollaxis(X, 0, 3)


def cbpdngrdmsk(D, S, W, lmbda, mu, opt, dev=0):
    """GPU ConvBPDNGradReg with an AMS spatial mask (cbpdn.pyx:229-291)."""
    if _is_torch(D):
        return _torch_entry(D, S, W, lmbda, mu, opt, True, True)
    _check_array(D, 3, "D")
    _check_array(S, 2, "S")
    if not isinstance(W, np.ndarray):
        raise TypeError("Argument 'W' has incorrect type (expected numpy.ndarray)")
    Di = _impulse_dict(D)
    l1, g = _ams_weights(S.shape, Di.shape[2], opt, True)
    X = _host_solve(np.ascontiguousarray(np.rollaxis(Di, 2, 0)), np.ascontiguousarray(S),
                    np.ascontiguousarray(W, dtype=np.int32), lmbda, mu, opt, l1, g, dev, True)
    return np.rollaxis(X, 0, 3)[..., 1:]


# ------------------------------------------------- persistent (warm) solver --

class ConvBPDN:
    """A persistent solver object for the outer loop of dictionary learning.

    No counterpart in the reference, whose functions solve from zero on every
    call; its main external caller, sporco's ConvBPDNDictLearn, alternates a
    few ADMM iterations of the coefficient step with a dictionary update and
    continues the coefficient step's state (iterates, rho, iteration count)
    across them.  This object keeps that state in device memory:

        b = ConvBPDN(D, S, lmbda, opt)      # (Kr, Kc, M), (H, W)
        X = b.solve()                      # MaxMainIter iterations from zero
        b.setdict(D2)                      # new filters, same shape
        X = b.solve()                      # MaxMainIter more, warm
        X = b.getcoef()

    ``mu`` (not None) adds the gradient term of ``cbpdngrd``; a mask ``W``
    gives the AMS problem of ``cbpdnmsk`` / ``cbpdngrdmsk`` (impulse filter
    prepended, its map dropped from the results).  Results are numpy arrays
    for numpy inputs and torch tensors for torch inputs."""

    def __init__(self, D, S, lmbda, opt, mu=None, W=None, dev=0):
        import torch
        self._torch = _is_torch(D)
        device = D.device if self._torch else torch.device("cuda", dev)
        Dt = torch.as_tensor(D, device=device, dtype=torch.float32)
        St = torch.as_tensor(S, device=device, dtype=torch.float32)
        if Dt.ndim != 3 or St.ndim != 2:
            raise ValueError("D must be (Kr, Kc, M) and S must be (H, W)")
        self._grd = mu is not None
        self._ams = W is not None
        l1 = _opt_get(opt, "L1Weight")
        gw = _opt_get(opt, "GradWeight") if self._grd else 1.0
        mask = None
        if self._ams:
            l1, gw = _ams_weights(St.shape, Dt.shape[2] + 1,
                                  {"L1Weight": _np(l1), "GradWeight": _np(gw)}, self._grd)
            mask = torch.as_tensor(W, device=device).to(torch.int32).reshape(1, *St.shape)
        if hasattr(l1, "ndim") and np.ndim(l1) == 3:
            l1 = np.ascontiguousarray(np.rollaxis(_np(l1), 2, 0))
        self._ds = prepare_device(self._dict(Dt), St[None], lmbda, opt,
                                  mu=0.0 if mu is None else mu, grd=self._grd, l1=l1, gw=gw,
                                  mask=mask, record_itstat=bool(_opt_get(opt, "Verbose")))
        self._started = False

    def _dict(self, Dt):
        import torch
        if self._ams:
            d0 = torch.zeros((Dt.shape[0], Dt.shape[1], 1), dtype=Dt.dtype, device=Dt.device)
            d0[0, 0] = 1.0
            Dt = torch.cat((d0, Dt), dim=2)
        return Dt.permute(2, 0, 1).contiguous()

    def solve(self, iters=None):
        """MaxMainIter (or `iters`) ADMM iterations, continuing the state of
        the previous call; returns the coefficient maps (H, W, M)."""
        self._ds.run(warm=self._started, iters=iters)
        self._started = True
        return self.getcoef()

    def setdict(self, D):
        """Replace the filters (Kr, Kc, M) (same shape); the next solve uses
        them and keeps the iterates, rho and the iteration count."""
        import torch
        Dt = torch.as_tensor(D, device=self._ds.keep["D"].device, dtype=torch.float32)
        self._ds.set_dict(self._dict(Dt))

    def getcoef(self):
        X = self._ds.keep["Y"][0].permute(1, 2, 0)
        if self._ams:
            X = X[..., 1:]
        return X if self._torch else X.contiguous().cpu().numpy()

    def getitstat(self):
        """Per-iteration statistics of the last solve (recorded when the
        options ask for Verbose): dict of arrays r, s, rho, epri, edua, fnc,
        dfid, regl1."""
        st = self._ds.state()
        if st["itstat"] is None:
            return None
        k = st["iterations"][0]
        return {n: st["itstat"][0, :k, i].copy() for i, n in enumerate(ITSTAT_NAMES)}

    @property
    def rho(self):
        return self._ds.state()["rho"][0]


# --------------------------------------------- multi-channel / multi-signal --

def cbpdn_multi(D, S, lmbda, opt, W=None, mu=None, dev=0):
    """Multi-channel and multi-signal CBPDN with a single-channel dictionary.

    No counterpart in the reference, which solves one 2-D single-channel
    signal per call (cbpdn.pyx:87); this is sporco's ConvBPDN layout for a
    signal with C channels and K signals and a dictionary without a channel
    axis: ``D`` (Kr, Kc, M), ``S`` (H, W, C) or (H, W, C, K); the result is
    (H, W, C, K, M), every channel of every signal with its own coefficient
    maps (the problem separates over channels and signals).  All C K images
    are solved in one batched device solve (one rho, residual and stopping
    state per image).  ``mu`` (not None) adds the gradient term of
    ``cbpdngrd``; a mask ``W`` of shape (H, W), (H, W, C) or (H, W, C, K)
    gives the AMS problem of ``cbpdnmsk`` / ``cbpdngrdmsk``.  numpy in,
    numpy out; CUDA tensors in, tensors out."""
    import torch
    as_torch = _is_torch(D)
    device = D.device if as_torch else torch.device("cuda", dev)
    Dt = torch.as_tensor(D, device=device, dtype=torch.float32)
    St = torch.as_tensor(S, device=device, dtype=torch.float32)
    if Dt.ndim != 3:
        raise ValueError("D must be (Kr, Kc, M): a single-channel dictionary")
    if St.ndim == 3:
        St = St[..., None]
    if St.ndim != 4:
        raise ValueError("S must be (H, W, C) or (H, W, C, K)")
    H, Wd, C, K = St.shape
    Sb = St.permute(2, 3, 0, 1).reshape(C * K, H, Wd).contiguous()
    grd = mu is not None
    ams = W is not None
    l1 = _opt_get(opt, "L1Weight")
    gw = _opt_get(opt, "GradWeight") if grd else 1.0
    mask = None
    if ams:
        Wt = torch.as_tensor(W, device=device)
        while Wt.ndim < 4:
            Wt = Wt[..., None]
        mask = Wt.expand(H, Wd, C, K).permute(2, 3, 0, 1).reshape(C * K, H, Wd).to(torch.int32)
        d0 = torch.zeros((Dt.shape[0], Dt.shape[1], 1), device=device)
        d0[0, 0] = 1.0
        Dt = torch.cat((d0, Dt), dim=2)
        l1, gw = _ams_weights(None, Dt.shape[2], {"L1Weight": _np(l1), "GradWeight": _np(gw)},
                              grd)
    if hasattr(l1, "ndim") and np.ndim(l1) == 3:
        l1 = np.ascontiguousarray(np.rollaxis(_np(l1), 2, 0))
    Y = solve_device(Dt.permute(2, 0, 1).contiguous(), Sb, lmbda, opt,
                     mu=0.0 if mu is None else mu, grd=grd, l1=l1, gw=gw, mask=mask)
    X = Y.reshape(C, K, Y.shape[1], H, Wd).permute(3, 4, 0, 1, 2)  # (H, W, C, K, M)
    if ams:
        X = X[..., 1:]
    return X if as_torch else X.contiguous().cpu().numpy()


# ------------------------------------------------------------- batched form --

def cbpdn_batched(D, S_list, lmbda, opt, W_list=None, mu=0.0, grd=False, streams=True,
                  return_info=False):
    """Solve many images of possibly different sizes with one dictionary.

    No counterpart in the reference (which solves one image per call).
    ``D``: (Kr, Kc, M) float32 (numpy or CUDA tensor); ``S_list``: sequence of
    (H_i, W_i) float32 images; ``lmbda``: scalar or one value per image;
    ``W_list``: optional per-image AMS masks (then the impulse filter is
    prepended and map 0 dropped, as in ``cbpdnmsk``); ``grd``/``mu``: gradient
    regularisation as in ``cbpdngrd``.  Every image keeps its own rho,
    residuals and stopping state.  Images are grouped into buckets of equal
    (H, W) (no padding: the circular-boundary problem is unchanged); each
    bucket is one batched solve on its own CUDA stream, and the iterations
    of all buckets are launched in turn by one host driver
    (``sc_cbpdn_solve_batch``).  Returns a list of (H_i, W_i, M) results of
    the input's array type (and, with ``return_info``, per-image iteration
    counts)."""
    import torch
    n = len(S_list)
    lam = np.broadcast_to(np.asarray(lmbda, dtype=F32), (n,))
    as_torch = _is_torch(D)
    dev = D.device if as_torch else torch.device("cuda", torch.cuda.current_device())
    Dt = torch.as_tensor(D, device=dev).float()
    ams = W_list is not None
    M = Dt.shape[2]
    if ams:
        d0 = torch.zeros((Dt.shape[0], Dt.shape[1], 1), device=dev)
        d0[0, 0] = 1.0
        Dt = torch.cat((d0, Dt), dim=2)
    Dm = Dt.permute(2, 0, 1).contiguous()
    Mi = Dm.shape[0]
    l1 = _opt_get(opt, "L1Weight")
    gw = _opt_get(opt, "GradWeight") if grd else 1.0
    if ams:
        l1, gw = _ams_weights(None, Mi, {"L1Weight": _np(l1), "GradWeight": _np(gw)}, grd)
    if hasattr(l1, "ndim") and np.ndim(l1) == 3:
        l1 = np.ascontiguousarray(np.rollaxis(_np(l1), 2, 0))
    buckets = {}
    for i, s in enumerate(S_list):
        buckets.setdefault(tuple(s.shape), []).append(i)
    solves, order = [], []
    for shape, idx in buckets.items():
        S = torch.stack([torch.as_tensor(S_list[i], device=dev).float() for i in idx])
        mask = None
        if ams:
            mask = torch.stack([torch.as_tensor(np.asarray(_np(W_list[i])), device=dev)
                                .to(torch.int32) for i in idx])
        ds = prepare_device(Dm, S, lam[idx], opt, mu=mu, grd=grd, l1=l1, gw=gw, mask=mask)
        solves.append(ds)
        order.append(idx)
    k = len(solves)
    probs = (_lib.ScProblem * k)(*[ds.prob for ds in solves])
    wss = (C.c_void_p * k)(*[ds.ws.data_ptr() for ds in solves])
    wsb = (C.c_size_t * k)(*[ds.ws.numel() for ds in solves])
    res = (_lib.ScResult * k)()
    strm = [torch.cuda.Stream(device=dev) if streams else torch.cuda.current_stream(dev)
            for _ in range(k)]
    cur = torch.cuda.current_stream(dev)
    for st in strm:
        st.wait_stream(cur)
    sp = (C.c_void_p * k)(*[st.cuda_stream for st in strm])
    _lib.check(_lib.sc_cbpdn_solve_batch(probs, k, C.byref(solves[0].opts), wss, wsb, res, sp))
    for st in strm:
        cur.wait_stream(st)
    out = [None] * n
    iters = [0] * n
    for ds, idx in zip(solves, order):
        Y = ds.keep["Y"]
        info = ds.state()
        for j, i in enumerate(idx):
            X = Y[j].permute(1, 2, 0)
            if ams:
                X = X[..., 1:]
            out[i] = X if as_torch else X.contiguous().cpu().numpy()
            iters[i] = info["iterations"][j]
    return (out, iters) if return_info else out
