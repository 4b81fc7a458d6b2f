"""NonNegCoef and NoBndryCross (parsed but never applied by the reference,
cbpdn.pyx:70-71; here applied as sporco's ConvBPDN y-step applies them)
against the FP64 oracle, through the reference-facing C ABI (numpy) and the
device path (torch), with adaptive rho so that the fix-up and the state
recomputation see the projections too."""

import numpy as np
import pytest

torch = pytest.importorskip("torch")

import sporco_cuda.cbpdn as cb
from oracle import cbpdn_oracle as O

REL_TOL = 1e-4


def _rel(a, b):
    return float(np.linalg.norm(np.asarray(a, np.float64) - b) / max(np.linalg.norm(b), 1e-30))


def _problem(H, W, M, K, seed):
    rng = np.random.default_rng(seed)
    D = rng.standard_normal((K, K, M)).astype(np.float32)
    D /= np.sqrt(np.sum(D * D, axis=(0, 1), keepdims=True))
    S = rng.standard_normal((H, W)).astype(np.float32)
    Wm = (rng.random((H, W)) < 0.7).astype(np.float32)
    return D, S, Wm


# (H, W, M, K): compiled transform lengths with the 16-tap convolution
# column solve; generic lengths with the transform solve
SHAPES = [(96, 64, 6, 12), (40, 36, 4, 5)]
FLAGS = [{"NonNegCoef": True}, {"NoBndryCross": True},
         {"NonNegCoef": True, "NoBndryCross": True}]


@pytest.mark.gpu
@pytest.mark.parametrize("shape", SHAPES)
@pytest.mark.parametrize("flags", FLAGS, ids=["nonneg", "nobndry", "both"])
@pytest.mark.parametrize("variant", ["cbpdn", "cbpdnmsk", "cbpdngrd"])
def test_projections_match_oracle(shape, flags, variant):
    H, W, M, K = shape
    D, S, Wm = _problem(H, W, M, K, 21)
    lam, mu = 0.05, 0.2
    opt = dict({"MaxMainIter": 30, "RelStopTol": 0.0, "RelaxParam": 1.8,
                "AutoRho": {"Enabled": True}}, **flags)
    if variant == "cbpdn":
        args = (D, S, lam, opt)
    elif variant == "cbpdngrd":
        args = (D, S, lam, mu, opt)
    else:
        args = (D, S * Wm, Wm, lam, opt)
    X = getattr(cb, variant)(*args)
    Xo = getattr(O, variant)(*args)
    assert _rel(X, Xo) < REL_TOL
    if flags.get("NonNegCoef"):
        assert X.min() >= 0.0
    if flags.get("NoBndryCross"):
        assert np.abs(X[H - (K - 1):]).max() == 0.0 and np.abs(X[:, W - (K - 1):]).max() == 0.0
    # the device path takes the same options
    targs = list(args)
    targs[0] = torch.tensor(D, device="cuda")
    targs[1] = torch.tensor(args[1], device="cuda")
    Xt = getattr(cb, variant)(*targs).cpu().numpy()
    assert _rel(Xt, X.astype(np.float64)) < 1e-6
