"""Gradients of the unrolled CBPDN solve (hand-written adjoint) against torch
autograd of an FP64 unrolled reference and FP64 central finite differences."""

import numpy as np
import pytest

torch = pytest.importorskip("torch")

from oracle import adjoint_oracle as A
from oracle import cbpdn_oracle as O

F32 = np.float32


def _problem(B=2, H=24, W=20, M=3, K=5, seed=0):
    rng = np.random.default_rng(seed)
    D = rng.standard_normal((K, K, M))
    D /= np.sqrt(np.sum(D * D, axis=(0, 1), keepdims=True))
    Sc = rng.standard_normal((B, H, W)) * 0.5
    S = Sc + 0.05 * rng.standard_normal((B, H, W))
    return D.astype(F32), S.astype(F32), Sc.astype(F32)


LAM, BETA, ITERS = 0.05, 0.01, 12


def _opt():
    return {"MaxMainIter": ITERS, "RelStopTol": 0.0, "RelaxParam": 1.8, "rho": None,
            "AutoRho": {"Enabled": False}}


def _consts():
    lam = float(F32(LAM))
    return lam, float(F32(50 * lam + 1)), float(F32(1.8))


def test_fp64_reference_gradient_matches_finite_differences():
    D, S, Sc, = _problem()
    lam, rho, alpha = _consts()
    Dt = torch.tensor(D, dtype=torch.float64, requires_grad=True)
    St = torch.tensor(S, dtype=torch.float64, requires_grad=True)
    L = A.loss(Dt, St, torch.tensor(Sc, dtype=torch.float64), lam, rho, alpha, ITERS, BETA)
    L.backward()
    rng = np.random.default_rng(5)
    for G, base, which in ((Dt.grad, D, "D"), (St.grad, S, "S")):
        dirn = rng.standard_normal(base.shape)
        eps = 1e-6

        def f(x):
            d = torch.tensor(D, dtype=torch.float64) if which == "S" else x
            s = torch.tensor(S, dtype=torch.float64) if which == "D" else x
            return float(A.loss(d, s, torch.tensor(Sc, dtype=torch.float64), lam, rho, alpha,
                                ITERS, BETA))
        x0 = torch.tensor(base, dtype=torch.float64)
        dd = torch.tensor(dirn)
        fd = (f(x0 + eps * dd) - f(x0 - eps * dd)) / (2 * eps)
        an = float(torch.sum(G * dd))
        assert abs(fd - an) <= 1e-5 * max(1.0, abs(an)), (which, fd, an)


@pytest.mark.gpu
def test_unrolled_forward_matches_oracle():
    import sporco_cuda.adjoint as adj
    D, S, _ = _problem()
    X = adj.cbpdn_unrolled(torch.tensor(D, device="cuda"), torch.tensor(S, device="cuda"),
                           LAM, _opt())
    for b in range(S.shape[0]):
        Xo = O.cbpdn(D, S[b], LAM, _opt())
        rel = np.linalg.norm(X[b].cpu().numpy() - Xo) / np.linalg.norm(Xo)
        assert rel < 1e-4


# (B, H, W, M, K, iterations): generic-plan sizes with three segments (the
# transform-solve adjoint); a row length that is not a multiple of 4 and a
# short last segment (8-tap convolution adjoint); compile-time plan sizes
# (64 x 64, 8 taps) with one segment per iteration count square; 11 x 11
# filters at 128 x 128 (16 taps) over 200 iterations (15 segments of 14).
SHAPES = [(2, 24, 20, 3, 5, 12), (1, 32, 30, 4, 5, 10), (2, 64, 64, 8, 7, 9),
          (1, 128, 128, 8, 11, 200)]


@pytest.mark.gpu
@pytest.mark.parametrize("form", ["default", "transform"])
@pytest.mark.parametrize("shape", SHAPES)
def test_unrolled_gradients_match_fp64_autograd_and_fd(shape, form, monkeypatch):
    """Against torch FP64 autograd and FP64 central differences; "transform"
    forces the transform-solve adjoint (SPORCO_B200_ADJOINT) where the
    convolution form would run."""
    import sporco_cuda.adjoint as adj
    B, H, W, M, K, iters = shape
    if form == "transform":
        if shape[0:2] == (2, 24):
            pytest.skip("the transform form is the default here")
        monkeypatch.setenv("SPORCO_B200_ADJOINT", "transform")
    D, S, Sc = _problem(B, H, W, M, K)
    lam, rho, alpha = _consts()
    opt = dict(_opt(), MaxMainIter=iters)
    Dg = torch.tensor(D, device="cuda", requires_grad=True)
    Sg = torch.tensor(S, device="cuda", requires_grad=True)
    X = adj.cbpdn_unrolled(Dg, Sg, LAM, opt)
    R = adj.reconstruct(Dg, X)
    L = torch.sum((R - torch.tensor(Sc, device="cuda")) ** 2) + BETA * torch.sum(torch.abs(X))
    L.backward()
    Dt = torch.tensor(D, dtype=torch.float64, requires_grad=True)
    St = torch.tensor(S, dtype=torch.float64, requires_grad=True)
    Lr = A.loss(Dt, St, torch.tensor(Sc, dtype=torch.float64), lam, rho, alpha, iters, BETA)
    Lr.backward()
    assert abs(float(L) - float(Lr)) / float(Lr) < 1e-5
    for g, r in ((Dg.grad, Dt.grad), (Sg.grad, St.grad)):
        g = g.double().cpu()
        rel = float(torch.linalg.norm(g - r) / torch.linalg.norm(r))
        assert rel < 1e-4, rel
    # directional finite differences of the FP64 loss against the GPU gradient.
    # The loss is only piecewise smooth (a coefficient crossing its shrinkage
    # threshold is a kink); a central difference means something only where
    # both one-sided differences agree, so a step of 1e-6 that straddles a
    # kink is shrunk until it does not.
    rng = np.random.default_rng(7)
    for g, base, which in ((Dg.grad, D, "D"), (Sg.grad, S, "S")):
        dd = torch.tensor(rng.standard_normal(base.shape))

        def f(x):
            d = torch.tensor(D, dtype=torch.float64) if which == "S" else x
            s = torch.tensor(S, dtype=torch.float64) if which == "D" else x
            return float(A.loss(d, s, torch.tensor(Sc, dtype=torch.float64), lam, rho, alpha,
                                iters, BETA))
        x0 = torch.tensor(base, dtype=torch.float64)
        f0 = f(x0)
        for eps in (1e-6, 1e-7, 1e-8):
            fp, fm = f(x0 + eps * dd), f(x0 - eps * dd)
            fwd, bwd = (fp - f0) / eps, (f0 - fm) / eps
            if abs(fwd - bwd) <= 1e-3 * max(1.0, abs(fwd)):
                break
        fd = (fp - fm) / (2 * eps)
        an = float(np.sum(g.double().cpu().numpy() * dd.numpy()))
        assert abs(fd - an) <= 1e-4 * max(1.0, abs(fd)), (which, eps, fd, an)
