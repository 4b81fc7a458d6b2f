"""FP64 CPU oracle for the sporco-cuda CBPDN ADMM solvers.

TEST INFRASTRUCTURE ONLY.  This module is the checker: only the test suite,
``__graft_entry__.smoke()`` and the CPU-baseline leg of ``bench.py`` may
import it.  The product (the ``sporco_cuda`` package under
``sporco-cuda_b200/``) never imports it and has no CPU fallback.

It restates, in numpy/scipy float64, the algorithm the reference implements
in ``sporco_cuda/src/cbpdn.cu`` and ``sporco_cuda/src/cbpdn_grd.cu`` (host
ADMM loop) and ``sporco_cuda/src/cbpdn_kernels.cu`` (per-element kernels),
behind the Python conventions of ``sporco_cuda/cbpdn.pyx`` (float32 coercion
of the scalar arguments, rho default, AMS impulse prepended, weight shapes,
``(H, W, M)`` output).  Where the reference deviates from the mathematics it
cites (Boyd et al. 2010, Wohlberg 2015/2016) the oracle follows the
mathematics:

* the Sherman-Morrison coefficients are always derived from the current rho
  (the reference leaves them stale after an AutoRho change unless
  ``HighMemSolve`` is set, ``cbpdn.cu:551-558``);
* the absolute stopping tolerance is scaled by sqrt(n), n the number of
  coefficients (the reference uses sqrt(||X||), ``cbpdn.cu:427-428``);
* a user-supplied ``RsdlTarget`` is honoured (the reference always
  overwrites it, ``cbpdn.cu:159-162``);
* all reductions are exact float64 sums (the reference uses float32
  atomics scaled by 1e6, ``cbpdn_kernels.cu:773-782``);
* a zero normaliser max(||X||, ||Y||) is replaced by 1, as for ||U||;
* after a rho change all of U is rescaled (the reference's cublasSgeam call,
  cbpdn.cu:546-549 and cbpdn_grd.cu:584-587, treats U as an (H M) x H matrix,
  so it rescales H*M*H elements instead of H*M*W: only part of U when H < W,
  and past the end of U when H > W).  ``emulate_ref_rescale=True`` reproduces
  the reference's extent, for pinning against its outputs only.

For AutoRho-off problems, and AutoRho problems solved with ``HighMemSolve``,
these differences are at float32 rounding level; the golden fixtures under
``tests/golden`` (outputs of the compiled reference) pin this.
"""

from __future__ import annotations

import math
import os
from dataclasses import dataclass, field

import numpy as np
import scipy.fft as sfft

F32 = np.float32
_WORKERS = int(os.environ.get("ORACLE_FFT_WORKERS", os.cpu_count() or 1))

# Defaults for option fields left unset, as applied by the reference's
# default_opts (sporco_cuda/src/utils.cu:12-64).
REF_DEFAULTS = {
    "Verbose": False,
    "MaxMainIter": 250,
    "RelaxParam": 1.8,
    "AbsStopTol": 0.0,
    "RelStopTol": 1e-4,
    "AuxVarObj": False,
    "HighMemSolve": False,
    "NonNegCoef": False,
    "NoBndryCross": False,
    "rho": None,
    "L1Weight": 1.0,
    "GradWeight": 1.0,
    "AutoRho": {
        "Enabled": True,
        "Period": 1,
        "Scaling": 100.0,
        "RsdlRatio": 1.2,
        "RsdlTarget": None,
        "AutoScaling": True,
        "StdResiduals": False,
    },
}


def _get(opt, key, default):
    try:
        v = opt[key]
    except (KeyError, TypeError):
        return default
    return default if v is None and default is not None and key != "rho" else v


@dataclass
class Resolved:
    """Scalar options as the reference marshals them (cbpdn.pyx:57-79)."""

    MaxMainIter: int
    RelaxParam: float
    AbsStopTol: float
    RelStopTol: float
    AutoRho: bool
    Period: int
    Scaling: float
    RsdlRatio: float
    RsdlTarget: float | None
    AutoScaling: bool
    StdResiduals: bool
    HighMemSolve: bool
    rho0: float
    extra: dict = field(default_factory=dict)


def resolve_options(opt, lmbda) -> Resolved:
    """Mirror of set_algopt (cbpdn.pyx:57-79) + default_opts (utils.cu:12-64).

    Scalars are rounded to float32 exactly where the reference stores them in
    the float fields of ``AlgOpt`` (algopt.h:7-48).  The rho default is
    50*lambda+1 computed from the float32 lambda (cbpdn.pyx:179).
    """
    ar = _get(opt, "AutoRho", {}) or {}
    dar = REF_DEFAULTS["AutoRho"]
    lam32 = F32(lmbda)
    rho = _get(opt, "rho", None)
    rho0 = F32(5e1 * float(lam32) + 1.0) if rho is None else F32(rho)
    tgt = _get(ar, "RsdlTarget", None)
    return Resolved(
        MaxMainIter=int(_get(opt, "MaxMainIter", REF_DEFAULTS["MaxMainIter"])),
        RelaxParam=float(F32(_get(opt, "RelaxParam", REF_DEFAULTS["RelaxParam"]))),
        AbsStopTol=float(F32(_get(opt, "AbsStopTol", 0.0))),
        RelStopTol=float(F32(_get(opt, "RelStopTol", REF_DEFAULTS["RelStopTol"]))),
        AutoRho=bool(int(_get(ar, "Enabled", dar["Enabled"]))),
        Period=int(_get(ar, "Period", dar["Period"])),
        Scaling=float(F32(_get(ar, "Scaling", dar["Scaling"]))),
        RsdlRatio=float(F32(_get(ar, "RsdlRatio", dar["RsdlRatio"]))),
        RsdlTarget=None if tgt is None else float(F32(tgt)),
        AutoScaling=bool(int(F32(_get(ar, "AutoScaling", dar["AutoScaling"])))),
        StdResiduals=bool(int(_get(ar, "StdResiduals", dar["StdResiduals"]))),
        HighMemSolve=bool(int(_get(opt, "HighMemSolve", False))),
        rho0=float(rho0),
    )


def rsdl_target(res: Resolved, lmbda) -> float:
    """xi of the adaptive-rho rule (cbpdn.cu:159-162; Wohlberg 2015 VI.C)."""
    if res.RsdlTarget is not None:
        return res.RsdlTarget
    if res.StdResiduals:
        return 1.0
    lam = float(F32(lmbda))
    return float(1.0 + 18.3 ** (math.log10(lam) + 1.0)) if lam > 0 else 1.0


# --------------------------------------------------------------------------
# FFT helpers (numpy rfft2 convention, unnormalised forward)
# --------------------------------------------------------------------------

def rfft2(x):
    return sfft.rfft2(x, axes=(-2, -1), workers=_WORKERS)


def irfft2(xf, shape):
    return sfft.irfft2(xf, s=shape, axes=(-2, -1), workers=_WORKERS)


def pad_dict_spectrum(Dm, H, W):
    """rfft2 of the dictionary zero-padded at the top-left corner.

    Follows cuda_Pad_Dict (cbpdn_kernels.cu:602-615) + the batch-M R2C plan
    (cbpdn.cu:171-173, 287-289).  Dm has layout (M, Kr, Kc).
    """
    M, Kr, Kc = Dm.shape
    if Kr > H or Kc > W:
        raise ValueError("filters larger than the signal")
    P = np.zeros((M, H, W), dtype=np.float64)
    P[:, :Kr, :Kc] = Dm
    return rfft2(P)


def gradient_spectrum(H, W):
    """|G_r|^2 + |G_c|^2 on the rfft2 grid (cuda_Cal_Gfw, kernels:1167-1187).

    The two gradient filters are [-1, 1] along the columns and along the rows
    (cbpdn_grd.cu:288-311).
    """
    g = np.zeros((H, W))
    g[0, 0] = -1.0
    g[0, 1 % W] += 1.0
    Gr = rfft2(g)
    g = np.zeros((H, W))
    g[0, 0] = -1.0
    g[1 % H, 0] += 1.0
    Gc = rfft2(g)
    return np.abs(Gr) ** 2 + np.abs(Gc) ** 2


# --------------------------------------------------------------------------
# The ADMM iteration
# --------------------------------------------------------------------------

@dataclass
class Problem:
    """One CBPDN instance in the reference's internal layout.

    D: (M, Kr, Kc) float64 (already rolled, AMS impulse already prepended);
    S: (H, W); lmbda, mu: float32-rounded; wl1: array broadcastable to
    (M, H, W); wgrd: (M,) or None (plain cbpdn); mask: (H, W) int32 or None.
    """

    D: np.ndarray
    S: np.ndarray
    lmbda: float
    mu: float
    wl1: np.ndarray
    wgrd: np.ndarray | None
    mask: np.ndarray | None
    nonneg: bool = False              # NonNegCoef
    nobndry: tuple | None = None      # (Kr, Kc) with NoBndryCross, else None


def _finalize(sums, rho, k, n, res: Resolved, xi: float, hist):
    """Residuals, stopping test and adaptive rho of iteration k from the five
    sums of squares (||X||^2, ||Y||^2, ||U||^2, ||X - Y||^2, ||Yold - Y||^2)
    (cbpdn.cu:405-436, 519-559; Boyd et al. 2010 3.3-3.4; Wohlberg 2015).
    Returns (new rho, rsf, stop)."""
    nX, nY, nU = math.sqrt(sums[0]), math.sqrt(sums[1]), math.sqrt(sums[2])
    r = math.sqrt(sums[3])
    s = rho * math.sqrt(sums[4])
    epri = math.sqrt(n) * res.AbsStopTol + max(nX, nY) * res.RelStopTol
    edua = math.sqrt(n) * res.AbsStopTol + rho * nU * res.RelStopTol
    if not res.StdResiduals:
        rn = max(nX, nY)
        rn = 1.0 if rn == 0.0 else rn
        sn = rho * (1.0 if nU == 0.0 else nU)
        r, s, epri, edua = r / rn, s / sn, epri / rn, edua / sn
    if hist is not None:
        hist["r"].append(r)
        hist["s"].append(s)
        hist["rho"].append(rho)
        hist["epri"].append(epri)
        hist["edua"].append(edua)
    rsf = 1.0
    if res.AutoRho and k > 1 and k % res.Period == 0:
        if res.AutoScaling:
            rhomlt = math.sqrt(r / (s * xi)) if s * xi > 0 else math.inf
            if rhomlt < 1.0:
                rhomlt = 1.0 / rhomlt if rhomlt > 0 else math.inf
            rhomlt = min(rhomlt, res.Scaling)
        else:
            rhomlt = res.Scaling
        if r > xi * res.RsdlRatio * s:
            rsf = rhomlt
        if s > (res.RsdlRatio / xi) * r:
            rsf = 1.0 / rhomlt
    return rsf * rho, rsf, (r <= epri and s <= edua)


def y_step(V, prob: Problem, rho, m0, wl1):
    """Y of the iteration from V = X_r + U for maps m0, m0 + 1, ... (V holds
    a run of consecutive maps starting at map m0).

    The soft threshold at lambda w / rho (cuda_Shrink_CalU_*,
    cbpdn_kernels.cu:129-311), then, when requested, sporco's projections,
    which the reference parses (cbpdn.pyx:70-71) but never applies: with
    NonNegCoef negative coefficients are set to zero, with NoBndryCross the
    coefficients whose filter would cross the bottom or right image boundary
    (the last Kr - 1 rows and last Kc - 1 columns of every map) are set to
    zero (sporco ConvBPDN.ystep / GenericConvBPDN.ystep).  Last, on map 0 of
    masked problems the AMS step Y_0 = (1 - W) V_0 replaces all of that
    (cuda_Cal_X_minus_U_W, cbpdn_kernels.cu:1137-1155).
    """
    Yn = np.sign(V) * np.maximum(np.abs(V) - (prob.lmbda / rho) * wl1, 0.0)
    if prob.nonneg:
        Yn[Yn < 0.0] = 0.0
    if prob.nobndry is not None:
        Kr, Kc = prob.nobndry
        if Kr > 1:
            Yn[:, V.shape[1] - (Kr - 1):, :] = 0.0
        if Kc > 1:
            Yn[:, :, V.shape[2] - (Kc - 1):] = 0.0
    if prob.mask is not None and m0 == 0:
        Yn[0] = (1.0 - prob.mask) * V[0]
    return Yn


def admm(prob: Problem, res: Resolved, xi: float, record=True, Y0=None, U0=None,
         emulate_ref_rescale=False, rho_start=None, k_start=0):
    """Run the CBPDN / CBPDN-GradReg ADMM iterations in float64.

    Loop structure: cbpdn.cu:319-567 (grd: cbpdn_grd.cu:358-606).
    Per iteration k = 1, 2, ...:
      b     = conj(Df) Sf + rho rfft2(Y - U)              (CalYU, R2C, solve)
      d_m   = rho  |  mu w_m |G|^2 + rho                  (solvedbd, 1198-1337)
      cb    = sum_m Df_m b_m / d_m / (1 + sum_m |Df_m|^2 / d_m)
      Xf_m  = (b_m - conj(Df_m) cb) / d_m                 (Sherman-Morrison)
      X     = irfft2(Xf)                                   (C2R, 1/N scaling)
      Xr    = a X + (1 - a) Y                              (OverRelax, 657-689)
      Y'    = soft(Xr + U, lambda w / rho); AMS map 0:
              Y'_0 = (1 - W)(Xr_0 + U_0)                   (Shrink 129-311, 1137-1155)
      U'    = U + Xr - Y'
      r = ||X - Y'||, s = rho ||Y - Y'||, norms of X, Y', U'  (695-783)
      stopping test and adaptive rho                       (cbpdn.cu:405-559)

    Y0, U0, rho_start and k_start continue an earlier run (its returned Y,
    U, rho and iteration count), as sporco's solve() continues its state:
    the iteration numbers (which the adaptive-rho period tests) go on from
    k_start, and MaxMainIter more iterations run.
    """
    D, S = prob.D, prob.S
    M = D.shape[0]
    H, W = S.shape
    N = H * W
    n = M * N
    Df = pad_dict_spectrum(D, H, W)
    Sf = rfft2(S.astype(np.float64))
    DSf = np.conj(Df) * Sf[None]
    grd = prob.wgrd is not None
    if grd:
        Gh = gradient_spectrum(H, W)[None]
        wg = np.asarray(prob.wgrd, dtype=np.float64).reshape(M, 1, 1)
    wl1 = np.broadcast_to(np.asarray(prob.wl1, dtype=np.float64), (M, H, W))
    alpha = res.RelaxParam
    rho = res.rho0 if rho_start is None else rho_start
    Y = np.zeros((M, H, W)) if Y0 is None else np.array(Y0, dtype=np.float64)
    U = np.zeros((M, H, W)) if U0 is None else np.array(U0, dtype=np.float64)
    hist = {"r": [], "s": [], "rho": [], "epri": [], "edua": []}
    k = k_start
    for k in range(k_start + 1, k_start + res.MaxMainIter + 1):
        b = DSf + rho * rfft2(Y - U)
        if grd:
            d = prob.mu * wg * Gh + rho
        else:
            d = rho
        num = np.sum(Df * b / d, axis=0)
        sden = np.sum((Df.real ** 2 + Df.imag ** 2) / d, axis=0)
        cb = num / (1.0 + sden)
        Xf = (b - np.conj(Df) * cb[None]) / d
        X = irfft2(Xf, (H, W))
        Xr = alpha * X + (1.0 - alpha) * Y if alpha != 1.0 else X
        V = Xr + U
        Yn = y_step(V, prob, rho, 0, wl1)
        U = V - Yn
        Yold, Y = Y, Yn
        sums = (float(np.sum(X * X)), float(np.sum(Y * Y)), float(np.sum(U * U)),
                float(np.sum((X - Y) ** 2)), float(np.sum((Yold - Y) ** 2)))
        rho, rsf, stop = _finalize(sums, rho, k, n, res, xi, hist if record else None)
        if rsf != 1.0:
            if emulate_ref_rescale:
                Uf = U.reshape(-1).copy()
                Uf[:min(Uf.size, H * M * H)] /= rsf
                U = Uf.reshape(U.shape)
            else:
                U = U / rsf
        if stop:
            break
    info = {"iterations": k, "rho": rho, "hist": hist, "Y": Y, "U": U}
    return Y, info


def admm_lean(prob: Problem, res: Resolved, xi: float, chunk=16, record=True,
              store_dict_bytes=4 << 30):
    """The iterations of :func:`admm` with the maps processed in chunks, for
    problems whose full-size float64 temporaries do not fit in host memory
    (2048 x 2048 with 256 maps: about 9 GB per array).

    Same mathematics and the same per-iteration steps as :func:`admm`
    (cbpdn.cu:319-567); only the summation order of the sums over the maps
    differs.  Per iteration: pass 1 accumulates sum_m Df_m b_m / d_m and
    sum_m |Df_m|^2 / d_m chunk by chunk; pass 2 forms b again, solves, takes
    the inverse transform and does the element-wise steps chunk by chunk.
    Y and U are the only full-size arrays kept (plus the dictionary spectra
    when they take at most ``store_dict_bytes``; otherwise they are
    recomputed per chunk).  No U0 / Y0 and no reference-rescale emulation.
    """
    D, S = prob.D, prob.S
    M = D.shape[0]
    H, W = S.shape
    n = M * H * W
    Wf = W // 2 + 1
    Sf = rfft2(S.astype(np.float64))
    keep = M * H * Wf * 16 <= store_dict_bytes
    Dfull = pad_dict_spectrum(D, H, W) if keep else None
    grd = prob.wgrd is not None
    Gh = gradient_spectrum(H, W)[None] if grd else None
    wl1 = np.asarray(prob.wl1, dtype=np.float64)
    alpha = res.RelaxParam
    rho = res.rho0
    Y = np.zeros((M, H, W))
    U = np.zeros((M, H, W))
    hist = {"r": [], "s": [], "rho": [], "epri": [], "edua": []}
    chunks = [(m0, min(M, m0 + chunk)) for m0 in range(0, M, chunk)]

    def dict_chunk(m0, m1):
        return Dfull[m0:m1] if keep else pad_dict_spectrum(D[m0:m1], H, W)

    def d_chunk(m0, m1):
        if not grd:
            return rho
        wg = np.asarray(prob.wgrd, dtype=np.float64)[m0:m1].reshape(-1, 1, 1)
        return prob.mu * wg * Gh + rho

    def wl1_chunk(m0, m1):
        return wl1[m0:m1] if wl1.shape[0] > 1 else wl1

    k = 0
    for k in range(1, res.MaxMainIter + 1):
        num = np.zeros((H, Wf), dtype=np.complex128)
        sden = np.zeros((H, Wf))
        for m0, m1 in chunks:
            Dc = dict_chunk(m0, m1)
            d = d_chunk(m0, m1)
            b = np.conj(Dc) * Sf[None] + rho * rfft2(Y[m0:m1] - U[m0:m1])
            num += np.sum(Dc * b / d, axis=0)
            sden += np.sum((Dc.real ** 2 + Dc.imag ** 2) / d, axis=0)
        cb = num / (1.0 + sden)
        sums = [0.0] * 5
        for m0, m1 in chunks:
            Dc = dict_chunk(m0, m1)
            d = d_chunk(m0, m1)
            b = np.conj(Dc) * Sf[None] + rho * rfft2(Y[m0:m1] - U[m0:m1])
            X = irfft2((b - np.conj(Dc) * cb[None]) / d, (H, W))
            Yc, Uc = Y[m0:m1], U[m0:m1]
            V = (alpha * X + (1.0 - alpha) * Yc if alpha != 1.0 else X) + Uc
            Yn = y_step(V, prob, rho, m0, wl1_chunk(m0, m1))
            Un = V - Yn
            sums[0] += float(np.sum(X * X))
            sums[1] += float(np.sum(Yn * Yn))
            sums[2] += float(np.sum(Un * Un))
            sums[3] += float(np.sum((X - Yn) ** 2))
            sums[4] += float(np.sum((Yc - Yn) ** 2))
            Y[m0:m1] = Yn
            U[m0:m1] = Un
        rho, rsf, stop = _finalize(sums, rho, k, n, res, xi, hist if record else None)
        if rsf != 1.0:
            U /= rsf
        if stop:
            break
    info = {"iterations": k, "rho": rho, "hist": hist, "Y": Y, "U": U}
    return Y, info


# --------------------------------------------------------------------------
# Objective (Parseval with Hermitian weights; FP64)
# --------------------------------------------------------------------------

def objective(D, S, Y, lmbda, mu=0.0, wl1=1.0, wgrd=None, mask=None):
    """Functional at coefficient maps Y (M, H, W) of dictionary D (M, Kr, Kc).

    0.5 ||W (sum_m d_m * y_m - s)||^2 + lambda ||wl1 y||_1
      [+ mu/2 sum_m wgrd_m (||G_r y_m||^2 + ||G_c y_m||^2)]
    W is the observation mask (1 when absent).  Circular convolution.
    """
    M = D.shape[0]
    H, W = S.shape
    Df = pad_dict_spectrum(D, H, W)
    Yf = rfft2(Y)
    DX = irfft2(np.sum(Df * Yf, axis=0), (H, W))
    e = DX - S
    if mask is not None:
        e = e * mask
    J = 0.5 * float(np.sum(e * e))
    J += float(lmbda) * float(np.sum(np.abs(np.broadcast_to(wl1, Y.shape) * Y)))
    if wgrd is not None and mu != 0.0:
        g = np.asarray(wgrd, dtype=np.float64).reshape(M, 1, 1)
        gr = Y - np.roll(Y, 1, axis=2)
        gc = Y - np.roll(Y, 1, axis=1)
        J += 0.5 * float(mu) * float(np.sum(g * (gr * gr + gc * gc)))
    return J


# --------------------------------------------------------------------------
# The four entry points, with the calling conventions of cbpdn.pyx
# --------------------------------------------------------------------------

def _l1_weight(opt, M):
    """L1Weight as a (M, H|1, W|1) array (cbpdn.pyx:181-193)."""
    w = _get(opt, "L1Weight", 1.0)
    if hasattr(w, "ndim"):
        w = np.asarray(w, dtype=np.float32)
        if w.ndim != 3:
            raise ValueError("L1Weight array must have 3 dimensions (H, W, M)")
        return np.ascontiguousarray(np.moveaxis(w, 2, 0)).astype(np.float64)
    return np.full((1, 1, 1), float(F32(w)))


def _grad_weight(opt, M):
    """GradWeight as (M,) (cbpdn.pyx:334-341)."""
    g = _get(opt, "GradWeight", 1.0)
    if hasattr(g, "ndim"):
        g = np.asarray(g, dtype=np.float32).ravel()
        if g.size == 1:
            return np.full(M, float(g[0]))
        if g.size != M:
            raise ValueError("GradWeight must be a scalar or have M entries")
        return g.astype(np.float64)
    return np.full(M, float(F32(g)))


def _ams(D, opt, grd):
    """Prepend the AMS impulse filter and zero its weights (cbpdn.pyx:116-137,
    237-275).  Returns (Di (Kr,Kc,M+1), l1 weight, grad weight)."""
    d0 = np.zeros(D.shape[0:2] + (1,), dtype=np.float32)
    d0[0, 0] = 1.0
    Di = np.dstack((d0, D))
    w = _get(opt, "L1Weight", 1.0)
    if hasattr(w, "ndim"):
        w0 = np.zeros(w.shape[0:-1] + (1,), dtype=np.float32)
        wl1 = np.dstack((w0, w))
    else:
        wl1 = F32(w) * np.ones((1, 1, Di.shape[2]), dtype=np.float32)
        wl1[..., 0] = 0.0
    g = None
    if grd:
        g = _get(opt, "GradWeight", 1.0)
        if hasattr(g, "ndim"):
            g = np.hstack((np.zeros((1,), dtype=np.float32), np.asarray(g, dtype=np.float32)))
        else:
            g = F32(g) * np.ones((Di.shape[2],), dtype=np.float32)
            g[..., 0] = 0.0
    return Di, wl1, g


def _run(Dk, S, W, lmbda, mu, opt, grd, wl1=None, wg=None, return_info=False,
         emulate_ref_rescale=False, lean_chunk=0, start=None):
    Dk = np.asarray(Dk, dtype=np.float32)
    S = np.asarray(S, dtype=np.float32)
    M = Dk.shape[2]
    res = resolve_options(opt, lmbda)
    lam = float(F32(lmbda))
    wl1a = _l1_weight({"L1Weight": wl1} if wl1 is not None else opt, M)
    wga = None
    if grd:
        wga = _grad_weight({"GradWeight": wg} if wg is not None else opt, M)
    mask = None
    if W is not None:
        Wi = np.ascontiguousarray(W, dtype=np.int32)
        if Wi.size > 1:
            mask = Wi.astype(np.float64)
    prob = Problem(
        D=np.moveaxis(Dk, 2, 0).astype(np.float64),
        S=S.astype(np.float64),
        lmbda=lam,
        mu=float(F32(mu)),
        wl1=wl1a,
        wgrd=wga,
        mask=mask,
        nonneg=bool(_get(opt, "NonNegCoef", False)),
        nobndry=tuple(Dk.shape[0:2]) if _get(opt, "NoBndryCross", False) else None,
    )
    if lean_chunk > 0:
        Y, info = admm_lean(prob, res, rsdl_target(res, lmbda), chunk=lean_chunk)
    else:
        cont = {}
        if start is not None:  # continue the state of an earlier run's info
            cont = dict(Y0=start["Y"], U0=start["U"], rho_start=start["rho"],
                        k_start=start["iterations"])
        Y, info = admm(prob, res, rsdl_target(res, lmbda),
                       emulate_ref_rescale=emulate_ref_rescale, **cont)
    X = np.moveaxis(Y, 0, 2)
    return (X, info) if return_info else X


def cbpdn(D, S, lmbda, opt, dev=0, return_info=False, emulate_ref_rescale=False,
          lean_chunk=0, start=None):
    """Oracle for sporco_cuda.cbpdn.cbpdn (cbpdn.pyx:86-102).  lean_chunk > 0:
    the map-chunked iterations of admm_lean (large problems); start: the
    info of an earlier run to continue (warm start)."""
    return _run(D, S, None, lmbda, 0.0, opt, False, return_info=return_info,
                emulate_ref_rescale=emulate_ref_rescale, lean_chunk=lean_chunk, start=start)


def cbpdnmsk(D, S, W, lmbda, opt, dev=0, return_info=False, emulate_ref_rescale=False,
             lean_chunk=0, start=None):
    """Oracle for sporco_cuda.cbpdn.cbpdnmsk (cbpdn.pyx:108-152)."""
    Di, wl1, _ = _ams(np.asarray(D, dtype=np.float32), opt, False)
    out = _run(Di, S, W, lmbda, 0.0, opt, False, wl1=wl1, return_info=return_info,
               emulate_ref_rescale=emulate_ref_rescale, lean_chunk=lean_chunk, start=start)
    if return_info:
        return out[0][..., 1:], out[1]
    return out[..., 1:]


def cbpdngrd(D, S, lmbda, mu, opt, dev=0, return_info=False, emulate_ref_rescale=False,
             lean_chunk=0, start=None):
    """Oracle for sporco_cuda.cbpdn.cbpdngrd (cbpdn.pyx:207-223)."""
    return _run(D, S, None, lmbda, mu, opt, True, return_info=return_info,
                emulate_ref_rescale=emulate_ref_rescale, lean_chunk=lean_chunk, start=start)


def cbpdngrdmsk(D, S, W, lmbda, mu, opt, dev=0, return_info=False,
                emulate_ref_rescale=False, lean_chunk=0):
    """Oracle for sporco_cuda.cbpdn.cbpdngrdmsk (cbpdn.pyx:229-291)."""
    Di, wl1, g = _ams(np.asarray(D, dtype=np.float32), opt, True)
    out = _run(Di, S, W, lmbda, mu, opt, True, wl1=wl1, wg=g, return_info=return_info,
               emulate_ref_rescale=emulate_ref_rescale, lean_chunk=lean_chunk)
    if return_info:
        return out[0][..., 1:], out[1]
    return out[..., 1:]


def mse(a, b):
    """sporco.metric.mse restated: mean squared difference."""
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    return float(np.mean((a - b) ** 2))
