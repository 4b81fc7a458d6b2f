"""Deterministic parity cases for the CBPDN solvers.

Cases 1-14 follow the reference's own test file
(``sporco_cuda/tests/test_cbpdn.py:19-344``): image 32x31, 5x5x4 dictionary,
``np.random.seed(12345)`` before each case and the same draw order, lambda
0.1, mu 0.01, 50 iterations, AutoRho disabled.  The reference draws its masks
with ``sporco.signal.rndmask``, which is not available here; a seeded
uniform-threshold mask with the same fill fraction stands in.  The option
dicts hold every key the reference's ``set_algopt`` reads
(``cbpdn.pyx:57-79``), with the values a sporco ``ConvBPDN.Options`` object
supplies by default.

Cases 15+ are added by this project: AutoRho on (with ``HighMemSolve`` so
that the compiled reference re-derives its solve coefficients after each rho
change), no relaxation, odd and even image sizes, and a small version of the
256x256 benchmark problem.
"""

from __future__ import annotations

import numpy as np


def full_opt(grd=False, **over):
    """A plain options dict with every key the reference reads."""
    ar = {
        "Enabled": False,
        "Period": 1,
        "Scaling": 1000.0,
        "RsdlRatio": 1.2,
        "RsdlTarget": None,
        "AutoScaling": True,
        "StdResiduals": False,
    }
    ar.update(over.pop("AutoRho", {}))
    opt = {
        "Verbose": False,
        "MaxMainIter": 50,
        "AbsStopTol": 0.0,
        "RelStopTol": 1e-3,
        "RelaxParam": 1.8,
        "rho": None,
        "AuxVarObj": False,
        "HighMemSolve": False,
        "NonNegCoef": False,
        "NoBndryCross": False,
        "L1Weight": 1.0,
        "AutoRho": ar,
    }
    if grd:
        opt["GradWeight"] = 1.0
    opt.update(over)
    return opt


def rndmask(shape, frc):
    """Stand-in for sporco.signal.rndmask: 1 with probability 1 - frc."""
    return (np.random.uniform(0.0, 1.0, shape) >= frc).astype(np.float32)


def _base(Nr=32, Nc=31, Nd=5, M=4):
    D = np.random.randn(Nd, Nd, M).astype(np.float32)
    s = np.random.randn(Nr, Nc).astype(np.float32)
    return D, s


def make_case(i):
    """Return dict(kind, D, S, W, lmbda, mu, opt, tol) for case i."""
    np.random.seed(12345)
    lmbda, mu = 0.1, 1e-2
    W = None
    tol = 1e-8
    M = 4
    if i == 1:
        D, s = _base()
        kind, opt = "cbpdn", full_opt()
    elif i in (2, 3):
        D, s = _base()
        wl1 = np.random.randn(1, 1, M).astype(np.float32)
        if i == 3:
            wl1[0] = 0.0
        kind, opt = "cbpdn", full_opt(L1Weight=wl1)
    elif i == 4:
        D, s = _base()
        wl1 = np.random.randn(32, 31, M).astype(np.float32)
        kind, opt, tol = "cbpdn", full_opt(L1Weight=wl1), 1e-6
    elif i == 5:
        D, s = _base()
        kind, opt = "cbpdngrd", full_opt(grd=True)
    elif i == 6:
        D, s = _base()
        wg = np.random.randn(M).astype(np.float32)
        kind, opt = "cbpdngrd", full_opt(grd=True, GradWeight=wg)
    elif i == 7:
        D, s = _base()
        wl1 = np.random.randn(1, 1, M).astype(np.float32)
        kind, opt = "cbpdngrd", full_opt(grd=True, L1Weight=wl1)
    elif i == 8:
        D, s = _base()
        wl1 = np.random.randn(32, 31, M).astype(np.float32)
        kind, opt = "cbpdngrd", full_opt(grd=True, L1Weight=wl1)
    elif i == 9:
        D, s = _base()
        wl1 = np.random.randn(32, 31, M).astype(np.float32)
        wg = np.random.randn(M).astype(np.float32)
        kind, opt = "cbpdngrd", full_opt(grd=True, L1Weight=wl1, GradWeight=wg)
    elif i in (10, 11):
        D, s = _base()
        W = rndmask(s.shape, 0.5)
        s *= W
        opt = full_opt()
        if i == 11:
            opt["L1Weight"] = np.random.randn(1, 1, M).astype(np.float32)
        kind = "cbpdnmsk"
    elif i in (12, 13, 14):
        D, s = _base()
        W = rndmask(s.shape, 0.5)
        s *= W
        opt = full_opt(grd=True)
        if i == 13:
            opt["L1Weight"] = np.random.randn(1, 1, M).astype(np.float32)
        if i == 14:
            opt["GradWeight"] = np.random.randn(M).astype(np.float32)
        kind = "cbpdngrdmsk"
    elif i == 15:
        D, s = _base()
        kind = "cbpdn"
        opt = full_opt(MaxMainIter=60, HighMemSolve=True, AutoRho={"Enabled": True})
    elif i == 16:
        D, s = _base()
        kind = "cbpdngrd"
        opt = full_opt(grd=True, MaxMainIter=60, HighMemSolve=True, AutoRho={"Enabled": True})
    elif i == 17:
        D, s = _base()
        kind, opt = "cbpdn", full_opt(RelaxParam=1.0)
    elif i == 18:
        D, s = _base(Nr=31, Nc=32)
        kind, opt = "cbpdn", full_opt()
    elif i == 19:
        D, s = _base(Nr=24, Nc=40, Nd=4, M=6)
        W = rndmask(s.shape, 0.3)
        s *= W
        kind = "cbpdngrdmsk"
        opt = full_opt(grd=True, MaxMainIter=40, HighMemSolve=True,
                       AutoRho={"Enabled": True, "Period": 3})
    elif i == 20:
        # small version of the 256x256 benchmark problem: unit-norm filters,
        # sparse synthetic signal, fixed rho, no early stop
        rng = np.random.default_rng(12345)
        K, M2, H = 8, 8, 64
        D = rng.standard_normal((K, K, M2))
        D /= np.sqrt(np.sum(D * D, axis=(0, 1), keepdims=True))
        D = D.astype(np.float32)
        X0 = (rng.random((H, H, M2)) < 0.01) * rng.standard_normal((H, H, M2))
        Df = np.fft.rfft2(D, s=(H, H), axes=(0, 1))
        s = np.fft.irfft2(np.sum(Df * np.fft.rfft2(X0, axes=(0, 1)), axis=2), s=(H, H))
        s = s + 0.01 * rng.standard_normal((H, H))
        s = (s - s.mean()).astype(np.float32)
        lmbda = 0.05
        kind = "cbpdn"
        opt = full_opt(MaxMainIter=100, RelStopTol=0.0,
                       rho=float(np.float32(50 * np.float32(lmbda) + 1)))
    else:
        raise ValueError(i)
    return dict(kind=kind, D=D, S=s, W=W, lmbda=lmbda, mu=mu, opt=opt, tol=tol)


NCASES = 20


def run(mod, c):
    """Call the solver named by the case on module ``mod`` (same signatures
    as sporco_cuda.cbpdn)."""
    k = c["kind"]
    if k == "cbpdn":
        return mod.cbpdn(c["D"], c["S"], c["lmbda"], c["opt"])
    if k == "cbpdnmsk":
        return mod.cbpdnmsk(c["D"], c["S"], c["W"], c["lmbda"], c["opt"])
    if k == "cbpdngrd":
        return mod.cbpdngrd(c["D"], c["S"], c["lmbda"], c["mu"], c["opt"])
    if k == "cbpdngrdmsk":
        return mod.cbpdngrdmsk(c["D"], c["S"], c["W"], c["lmbda"], c["mu"], c["opt"])
    raise ValueError(k)
