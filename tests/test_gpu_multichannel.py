"""Multi-channel / multi-signal signals with a single-channel dictionary
(sporco's ConvBPDN layout (H, W, C, K) -> (H, W, C, K, M)): one batched
device solve, equal to solving every channel of every signal alone, and to
the FP64 oracle per channel."""

import numpy as np
import pytest

torch = pytest.importorskip("torch")

import sporco_cuda.cbpdn as cb
from oracle import cbpdn_oracle as O


def _rel(a, b):
    return float(np.linalg.norm(np.asarray(a, np.float64) - b) / np.linalg.norm(b))


OPT = {"MaxMainIter": 25, "RelStopTol": 0.0, "AutoRho": {"Enabled": True}}


@pytest.mark.gpu
@pytest.mark.parametrize("variant", ["cbpdn", "cbpdngrd", "cbpdnmsk"])
def test_channels_and_signals_separate(variant):
    rng = np.random.default_rng(61)
    H, W, C, K, M = 48, 40, 3, 2, 5
    D = rng.standard_normal((6, 6, M))
    D = (D / np.sqrt(np.sum(D * D, axis=(0, 1), keepdims=True))).astype(np.float32)
    S = rng.standard_normal((H, W, C, K)).astype(np.float32)
    Wm = (rng.random((H, W, C)) < 0.7).astype(np.float32) if variant == "cbpdnmsk" else None
    mu = 0.2 if variant == "cbpdngrd" else None
    X = cb.cbpdn_multi(D, S, 0.05, OPT, W=Wm, mu=mu)
    assert X.shape == (H, W, C, K, M) and X.dtype == np.float32
    for c in range(C):
        for k in range(K):
            s = S[..., c, k]
            if variant == "cbpdn":
                ref, orc = cb.cbpdn(D, s, 0.05, OPT), O.cbpdn(D, s, 0.05, OPT)
            elif variant == "cbpdngrd":
                ref, orc = cb.cbpdngrd(D, s, 0.05, mu, OPT), O.cbpdngrd(D, s, 0.05, mu, OPT)
            else:
                w = Wm[..., c]
                ref, orc = cb.cbpdnmsk(D, s, w, 0.05, OPT), O.cbpdnmsk(D, s, w, 0.05, OPT)
            assert _rel(X[..., c, k, :], ref.astype(np.float64)) < 1e-6, (c, k)
            assert _rel(X[..., c, k, :], orc) < 1e-4, (c, k)
    # torch in, torch out; a 3-D signal is one signal with C channels
    Xt = cb.cbpdn_multi(torch.tensor(D, device="cuda"), torch.tensor(S[..., 0], device="cuda"),
                        0.05, OPT, W=Wm, mu=mu)
    assert torch.is_tensor(Xt) and Xt.shape == (H, W, C, 1, M)
    assert _rel(Xt[..., 0, :].cpu().numpy(), X[..., 0, :].astype(np.float64)) < 1e-6
