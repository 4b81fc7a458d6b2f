"""Warm starts for the dictionary-learning outer loop (a persistent device
solve that keeps Y, U, rho and the iteration count across calls and takes a
new dictionary between them): against one longer solve bit for bit, and
against the FP64 oracle continuing its own state with the new dictionary."""

import numpy as np
import pytest

torch = pytest.importorskip("torch")

import sporco_cuda.cbpdn as cb
from oracle import cbpdn_oracle as O

REL_TOL = 1e-4


def _rel(a, b):
    return float(np.linalg.norm(np.asarray(a, np.float64) - b) / np.linalg.norm(b))


def _problem(H, W, M, K, seed):
    rng = np.random.default_rng(seed)
    D = rng.standard_normal((K, K, M)).astype(np.float32)
    D /= np.sqrt(np.sum(D * D, axis=(0, 1), keepdims=True))
    S = rng.standard_normal((H, W)).astype(np.float32)
    Wm = (rng.random((H, W)) < 0.7).astype(np.float32)
    return D, S, Wm


OPT = {"MaxMainIter": 30, "RelStopTol": 0.0, "AutoRho": {"Enabled": True, "Period": 2}}


def _prepare(D, S, mask=None, **kw):
    Dm = torch.tensor(np.moveaxis(D, 2, 0).copy(), device="cuda")
    l1 = 1.0
    if mask is not None:
        Dm = torch.cat((torch.zeros((1,) + Dm.shape[1:], device="cuda"), Dm), 0)
        Dm[0, 0, 0] = 1.0
        l1 = np.ones(Dm.shape[0], np.float32)
        l1[0] = 0.0
        mask = torch.tensor(mask, device="cuda").to(torch.int32)[None]
    return cb.prepare_device(Dm, torch.tensor(S, device="cuda")[None], 0.05, OPT, l1=l1,
                             mask=mask, **kw)


@pytest.mark.gpu
@pytest.mark.parametrize("shape", [(96, 64, 6, 12), (40, 36, 4, 5)])
@pytest.mark.parametrize("masked", [False, True])
@pytest.mark.parametrize("warm", [True, "same"])
def test_warm_continuation_equals_one_solve_bitwise(shape, masked, warm):
    """Split after iteration 11 (no adaptive-rho step) and after iteration 12
    (a rho change whose fix-up of the row spectra the continuation runs)."""
    D, S, Wm = _problem(*shape, 31)
    mask = Wm if masked else None
    ref = _prepare(D, S * (Wm if masked else 1), mask)
    Yr = ref.run(iters=30).clone()
    rhos = ref.state()["rho"]
    for first in (11, 12):
        ds = _prepare(D, S * (Wm if masked else 1), mask)
        ds.run(iters=first)
        Y = ds.run(warm=warm, iters=30 - first)
        assert ds.state()["iterations"][0] == 30 - first
        assert torch.equal(Y, Yr), first
        assert ds.state()["rho"] == rhos


@pytest.mark.gpu
@pytest.mark.parametrize("variant", ["cbpdn", "cbpdnmsk", "cbpdngrd"])
def test_dictionary_update_between_warm_solves_matches_oracle(variant):
    """The outer loop: 12 iterations with D1, the dictionary replaced by D2,
    12 more iterations continuing the state; the oracle continues its own
    state the same way."""
    D1, S, Wm = _problem(96, 64, 6, 12, 41)
    D2, _, _ = _problem(96, 64, 6, 12, 42)
    opt = dict(OPT, MaxMainIter=12)
    mu = 0.2 if variant == "cbpdngrd" else None
    W = Wm if variant == "cbpdnmsk" else None
    Sx = S * Wm if W is not None else S
    b = cb.ConvBPDN(D1, Sx, 0.05, opt, mu=mu, W=W)
    b.solve()
    b.setdict(D2)
    X = b.solve()
    f = getattr(O, variant)
    args = (Sx, W, 0.05, opt) if W is not None else ((Sx, 0.05, mu, opt) if mu else (Sx, 0.05, opt))
    _, info = f(D1, *args, return_info=True)
    Xo = f(D2, *args, start=info)
    assert X.shape == Xo.shape
    assert _rel(X, Xo) < REL_TOL
    # one solve from zero with D2 is a different point
    assert _rel(f(D2, *args), Xo) > 10 * REL_TOL


@pytest.mark.gpu
def test_convbpdn_object_torch_inputs_and_statistics():
    D, S, _ = _problem(64, 48, 5, 7, 51)
    opt = dict(OPT, MaxMainIter=8, Verbose=True)
    b = cb.ConvBPDN(torch.tensor(D, device="cuda"), torch.tensor(S, device="cuda"), 0.05, opt)
    X1 = b.solve().clone()
    st1 = b.getitstat()
    X2 = b.solve()
    st2 = b.getitstat()
    assert torch.is_tensor(X2) and X2.shape == (64, 48, 5)
    assert len(st1["rho"]) == 8 and len(st2["rho"]) == 8
    ref = cb.ConvBPDN(torch.tensor(D, device="cuda"), torch.tensor(S, device="cuda"), 0.05,
                      dict(opt, MaxMainIter=16)).solve()
    assert torch.equal(X2, ref)
    assert not torch.equal(X1, X2)
    # and through the reference-facing C ABI, to float32 rounding
    Xn = cb.cbpdn(D, S, 0.05, dict(opt, MaxMainIter=16, Verbose=False))
    assert _rel(Xn, ref.cpu().numpy().astype(np.float64)) < 1e-6
